// C ABI of janc_b200 (declared in include/janc_b200.h): handle lifetime,
// workspace, argument checks and the per-step launch sequence.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>

#include <cmath>

#include "../../include/janc_b200.h"
#include "jb_chem_gen.cuh"
#include "jb_ops.h"

struct jb_handle {
  jb_mech_params mech;
  jb_grid grid;
  int dim;
  int precision;
  const jb::Ops* ops;
  int device;
  // workspace
  double* W[2];        // RK stage states [nv][ncell]
  double* auxw[2];     // stage aux [2][ncell]
  double* cand;        // Halley iterates [6][ncell]
  double* strips;      // ghost strips [4][nv+2][lstrip]
  jb_slots* slots;
  long long ws_bytes;
  // optional per-kernel timing of jb_advance (jb_set_kernel_timing)
  int timing;
  int nev;
  cudaEvent_t ev[2 * JB_TIMED_MAX];
  int ev_cat[JB_TIMED_MAX];
  double acc_ms[JB_KCAT_COUNT];
  long long acc_n[JB_KCAT_COUNT];
  char err[512];
};

namespace {

int set_err(jb_handle* h, int code, const char* fmt, ...) {
  if (h) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(h->err, sizeof(h->err), fmt, ap);
    va_end(ap);
  }
  return code;
}

int check_cuda(jb_handle* h, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return JB_OK;
  return set_err(h, JB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define JB_TRY(expr, what)                          \
  do {                                              \
    int _rc = check_cuda(h, (expr), what);          \
    if (_rc) return _rc;                            \
  } while (0)

// Launch with optional timing events around it (category cat).
#define JB_TIMED(cat, expr, what)                                             \
  do {                                                                        \
    bool _t = h->timing && h->nev < JB_TIMED_MAX;                             \
    if (_t) cudaEventRecord(h->ev[2 * h->nev], st);                           \
    JB_TRY(expr, what);                                                       \
    if (_t) {                                                                 \
      cudaEventRecord(h->ev[2 * h->nev + 1], st);                             \
      h->ev_cat[h->nev++] = cat;                                              \
    }                                                                         \
  } while (0)

bool bc_ok(int k) { return k >= JB_BC_PERIODIC && k <= JB_BC_RDC_INJECTOR; }

}  // namespace

// Derived tables and the structure check against the generated chemistry.
void jb::derive_mech(jb_mech_params& m) {
  int ok = m.ns == JB_GEN_NS && m.nr == JB_GEN_NR && m.nreac == JB_GEN_NREAC;
  for (int i = 0; i < m.nreac; ++i) {
    m.lnA[i] = std::log(m.A[i]);
    if (!(m.A[i] > 0.0)) ok = 0;
    for (int n = 0; n < m.nr; ++n) m.tbinvM[i][n] = m.tb[i][n] / m.M[n];
    if (ok) {
      if ((int)m.is_tb[i] != JB_GEN_ISTB[i] || (int)m.vsum[i] != JB_GEN_VSUM[i]) ok = 0;
      for (int k = 0; k < m.nr; ++k)
        if (m.vf[i][k] != (double)JB_GEN_VF[i][k] || m.vb[i][k] != (double)JB_GEN_VB[i][k]) ok = 0;
      for (int j = 0; j < m.ns; ++j)
        if ((m.tb[i][j] != 0.0) != (JB_GEN_TBNZ[i][j] != 0)) ok = 0;
    }
  }
  m.tcr_uniform = 1;
  for (int k = 1; k < m.ns; ++k)
    if (m.Tcr[k] != m.Tcr[0]) m.tcr_uniform = 0;
  m.lnpref = std::log(m.pref);
  m.lnT0 = std::log(m.T0);
  m.gen_ok = ok;
}


extern "C" {

const char* jb_version(void) { return "janc_b200 0.1 (sm_100a)"; }

int jb_create(const jb_mech_params* mech, int dim, int nx, int ny, double dx, double dy,
              const int bc[4], int precision, jb_handle** out) {
  if (!out || !mech || !bc) return JB_ERR_ARG;
  *out = nullptr;
  if (dim != 1 && dim != 2) return JB_ERR_ARG;
  if (mech->ns != 9 || mech->nr != 8 || mech->nreac != 19) return JB_ERR_UNSUPPORTED;
  if (nx < 4 || (dim == 2 && ny < 4)) return JB_ERR_ARG;
  if (dim == 1) ny = 1;
  if (!(dx > 0.0) || (dim == 2 && !(dy > 0.0))) return JB_ERR_ARG;
  for (int s = 0; s < 2 * dim; ++s)
    if (!bc_ok(bc[s])) return JB_ERR_ARG;
  if (dim == 1 && (bc[0] == JB_BC_RDC_INJECTOR || bc[1] == JB_BC_RDC_INJECTOR)) return JB_ERR_UNSUPPORTED;
  if (precision != JB_PREC_STRICT && precision != JB_PREC_FP64 && precision != JB_PREC_MIXED)
    return JB_ERR_UNSUPPORTED;
  jb_handle* h = new (std::nothrow) jb_handle();
  if (!h) return JB_ERR_ARG;
  std::memset(h, 0, sizeof(*h));
  h->mech = *mech;
  jb::derive_mech(h->mech);
  h->dim = dim;
  h->precision = precision;
  h->ops = precision == JB_PREC_STRICT ? &jb::strict_ops
          : precision == JB_PREC_MIXED  ? &jb::mixed_ops
                                        : &jb::fast_ops;
  jb_grid& g = h->grid;
  g.nx = nx;
  g.ny = ny;
  g.nv = dim == 2 ? 12 : 11;
  g.nY = dim == 2 ? 4 : 3;
  g.ncell = (long long)nx * ny;
  g.dx = dx;
  g.dy = dim == 2 ? dy : 1.0;
  g.idx = 1.0 / g.dx;
  g.idy = 1.0 / g.dy;
  for (int s = 0; s < 4; ++s) g.bc[s] = s < 2 * dim ? bc[s] : JB_BC_PERIODIC;
  g.Pb = 0.0;
  g.Yinj = nullptr;
  g.inj_block_p = 1.0;
  g.lstrip = nx > ny ? nx : ny;
  cudaGetDevice(&h->device);
  const size_t nc = (size_t)g.ncell;
  size_t bytes_W = sizeof(double) * g.nv * nc;
  size_t bytes_aux = sizeof(double) * 2 * nc;
  size_t bytes_cand = sizeof(double) * JB_NCAND * nc;
  size_t bytes_strip = sizeof(double) * 4 * (g.nv + 2) * (size_t)g.lstrip;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMalloc(&h->W[i], bytes_W);
  for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMalloc(&h->auxw[i], bytes_aux);
  if (e == cudaSuccess) e = cudaMalloc(&h->cand, bytes_cand);
  if (e == cudaSuccess) e = cudaMalloc(&h->strips, bytes_strip);
  if (e == cudaSuccess) e = cudaMalloc(&h->slots, sizeof(jb_slots));
  if (e == cudaSuccess) e = cudaMemset(h->strips, 0, bytes_strip);
  if (e == cudaSuccess) e = cudaMemset(h->slots, 0, sizeof(jb_slots));
  if (e != cudaSuccess) {
    jb_destroy(h);
    return JB_ERR_CUDA;
  }
  h->ws_bytes = (long long)(2 * bytes_W + 2 * bytes_aux + bytes_cand + bytes_strip + sizeof(jb_slots));
  *out = h;
  return JB_OK;
}

int jb_destroy(jb_handle* h) {
  if (!h) return JB_OK;
  if (h->timing)
    for (int i = 0; i < 2 * JB_TIMED_MAX; ++i) cudaEventDestroy(h->ev[i]);
  for (int i = 0; i < 2; ++i) {
    if (h->W[i]) cudaFree(h->W[i]);
    if (h->auxw[i]) cudaFree(h->auxw[i]);
  }
  if (h->cand) cudaFree(h->cand);
  if (h->strips) cudaFree(h->strips);
  if (h->slots) cudaFree(h->slots);
  delete h;
  return JB_OK;
}

int jb_set_theta(jb_handle* h, double Pb, const double* Yinj, double inj_block_p) {
  if (!h) return JB_ERR_ARG;
  h->grid.Pb = Pb;
  h->grid.Yinj = Yinj;
  h->grid.inj_block_p = inj_block_p;
  return JB_OK;
}

static int check_theta(jb_handle* h) {
  const jb_grid& g = h->grid;
  for (int s = 0; s < 2 * h->dim; ++s) {
    if (g.bc[s] == JB_BC_RDC_INJECTOR && !g.Yinj)
      return set_err(h, JB_ERR_ARG, "injector boundary needs theta['Yinj'] (jb_set_theta)");
  }
  return JB_OK;
}

int jb_flux_func(jb_handle* h, const double* U, const double* aux, double dt, double* rhs,
                 void* stream) {
  if (!h || !U || !aux || !rhs) return set_err(h, JB_ERR_ARG, "null pointer");
  if (int rc = check_theta(h)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const jb::Ops& o = *h->ops;
  JB_TRY(o.slots_reset(h->slots, st), "slots_reset");
  JB_TRY(o.select(h->dim, false, true, false, h->mech, h->grid, U, aux, nullptr, nullptr, h->strips,
                  h->slots, -1, 3, st),
         "alpha");
  JB_TRY(o.flux(h->dim, 0, h->mech, h->grid, U, aux, nullptr, rhs, nullptr, h->strips, h->slots, 3,
                -1, dt, st),
         "flux");
  return JB_OK;
}

int jb_update_aux(jb_handle* h, const double* U, const double* aux_in, double* aux_out,
                  void* stream) {
  if (!h || !U || !aux_in || !aux_out) return set_err(h, JB_ERR_ARG, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const jb::Ops& o = *h->ops;
  JB_TRY(o.slots_reset(h->slots, st), "slots_reset");
  JB_TRY(o.halley(h->dim, h->mech, h->grid, U, aux_in, h->cand, h->slots, 0, st), "halley");
  JB_TRY(o.select(h->dim, true, false, false, h->mech, h->grid, U, nullptr, h->cand, aux_out,
                  h->strips, h->slots, 0, 0, st),
         "select");
  return JB_OK;
}

int jb_reaction_source_terms(jb_handle* h, const double* U, const double* aux, double dt,
                             double* S, void* stream) {
  if (!h || !U || !aux || !S) return set_err(h, JB_ERR_ARG, "null pointer");
  if (!(dt > 0.0)) return set_err(h, JB_ERR_ARG, "dt must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  JB_TRY(h->ops->chem(h->dim, true, h->mech, h->grid, U, aux, S, nullptr, h->slots, -1, dt, st),
         "chem");
  return JB_OK;
}

static int advance_impl(jb_handle* h, const double* U, const double* aux, double* U_out,
                        double* aux_out, double dt_fixed, double cfl, int nsteps, double* dt_hist,
                        void* stream, bool chemistry) {
  if (!h || !U || !aux || !U_out || !aux_out) return set_err(h, JB_ERR_ARG, "null pointer");
  if (nsteps < 1) return set_err(h, JB_ERR_ARG, "nsteps must be >= 1");
  if (!(cfl > 0.0) && !(dt_fixed > 0.0)) return set_err(h, JB_ERR_ARG, "need cfl > 0 or dt > 0");
  if (U == U_out || aux == aux_out) return set_err(h, JB_ERR_ARG, "outputs must not alias inputs");
  if (int rc = check_theta(h)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const jb::Ops& o = *h->ops;
  const int d = h->dim;
  const bool use_cfl = cfl > 0.0;
  const jb_mech_params& m = h->mech;
  const jb_grid& g = h->grid;
  JB_TIMED(JB_KCAT_OTHER, o.slots_reset(h->slots, st), "slots_reset");
  // alpha (and CFL minimum) of the initial state, ghost strips for stage 1
  JB_TIMED(JB_KCAT_SELECT, o.select(d, false, true, use_cfl, m, g, U, aux, nullptr, nullptr, h->strips, h->slots, -1, 3,
                  st),
         "prep");
  for (int s = 0; s < nsteps; ++s) {
    const double* Un = s == 0 ? U : U_out;
    const double* an = s == 0 ? aux : aux_out;
    JB_TIMED(JB_KCAT_OTHER, o.step_begin(h->slots, use_cfl ? cfl : 0.0, dt_fixed, dt_hist, s, st), "step_begin");
    // stage 1: U1 = U + L(U)
    JB_TIMED(JB_KCAT_FLUX, o.flux(d, 1, m, g, Un, an, Un, h->W[0], h->cand, h->strips, h->slots, 0, 0, 0.0, st), "stage1");
    JB_TIMED(JB_KCAT_SELECT, o.select(d, true, true, false, m, g, h->W[0], nullptr, h->cand, h->auxw[0], h->strips,
                    h->slots, 0, 1, st),
           "select1");
    // stage 2: U2 = 3/4 U + 1/4 (U1 + L(U1))
    JB_TIMED(JB_KCAT_FLUX, o.flux(d, 2, m, g, h->W[0], h->auxw[0], Un, h->W[1], h->cand, h->strips, h->slots, 1, 1,
                  0.0, st),
           "stage2");
    JB_TIMED(JB_KCAT_SELECT, o.select(d, true, true, false, m, g, h->W[1], nullptr, h->cand, h->auxw[1], h->strips,
                    h->slots, 1, 2, st),
           "select2");
    // stage 3: U3 = 1/3 U + 2/3 (U2 + L(U2))
    JB_TIMED(JB_KCAT_FLUX, o.flux(d, 3, m, g, h->W[1], h->auxw[1], Un, h->W[0], h->cand, h->strips, h->slots, 2, 2,
                  0.0, st),
           "stage3");
    if (!chemistry) {
      // advance_flux only (TVD_RK3.py:5-12): U3, aux3 are the result
      const size_t bytes = sizeof(double) * g.nv * (size_t)g.ncell;
      JB_TRY(cudaMemcpyAsync(U_out, h->W[0], bytes, cudaMemcpyDeviceToDevice, st), "copy U3");
      JB_TIMED(JB_KCAT_SELECT, o.select(d, true, true, use_cfl, m, g, U_out, nullptr, h->cand, aux_out,
                                        h->strips, h->slots, 2, 3, st),
               "select3");
      continue;
    }
    JB_TIMED(JB_KCAT_SELECT, o.select(d, true, false, false, m, g, h->W[0], nullptr, h->cand, h->auxw[0], h->strips,
                    h->slots, 2, 0, st),
           "select3");
    // chemistry and the final temperature solve
    JB_TIMED(JB_KCAT_CHEM, o.chem(d, false, m, g, h->W[0], h->auxw[0], U_out, h->cand, h->slots, 3, 0.0, st), "chem");
    JB_TIMED(JB_KCAT_SELECT, o.select(d, true, true, use_cfl, m, g, U_out, nullptr, h->cand, aux_out, h->strips,
                    h->slots, 3, 3, st),
           "select4");
  }
  return JB_OK;
}

int jb_advance(jb_handle* h, const double* U, const double* aux, double* U_out, double* aux_out,
               double dt_fixed, double cfl, int nsteps, double* dt_hist, void* stream) {
  return advance_impl(h, U, aux, U_out, aux_out, dt_fixed, cfl, nsteps, dt_hist, stream, true);
}

int jb_rk3(jb_handle* h, const double* U, const double* aux, double* U_out, double* aux_out,
           double dt, void* stream) {
  return advance_impl(h, U, aux, U_out, aux_out, dt, 0.0, 1, nullptr, stream, false);
}

int jb_u_to_prim(jb_handle* h, const double* U, const double* aux, double* rho, double* u, double* v,
                 double* Y, double* p, double* a, void* stream) {
  if (!h || !U || !aux || !rho || !u || !Y || !p || !a || (h->dim == 2 && !v))
    return set_err(h, JB_ERR_ARG, "null pointer");
  JB_TRY(h->ops->prim(h->dim, h->mech, h->grid, U, aux, rho, u, v, Y, p, a, (cudaStream_t)stream), "prim");
  return JB_OK;
}

int jb_cfl_dt(jb_handle* h, const double* U, const double* aux, double cfl, double* dt_out,
              void* stream) {
  if (!h || !U || !aux || !dt_out) return set_err(h, JB_ERR_ARG, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const jb::Ops& o = *h->ops;
  JB_TRY(o.slots_reset(h->slots, st), "slots_reset");
  JB_TRY(o.select(h->dim, false, false, true, h->mech, h->grid, U, aux, nullptr, nullptr, h->strips,
                  h->slots, -1, 3, st),
         "cfl");
  JB_TRY(o.dt_from_slots(h->slots, cfl, dt_out, st), "dt");
  return JB_OK;
}

int jb_get_thermo(jb_handle* h, long long n, const double* T, const double* Y, double* cp,
                  double* gamma, double* hh, double* R, double* dcp, void* stream) {
  if (!h || !T || !Y || !cp || !gamma || !hh || !R || !dcp) return set_err(h, JB_ERR_ARG, "null pointer");
  if (n <= 0) return JB_OK;
  JB_TRY(h->ops->thermo(h->mech, n, T, Y, cp, gamma, hh, R, dcp, (cudaStream_t)stream), "thermo");
  return JB_OK;
}

int jb_status(jb_handle* h, unsigned* status, void* stream) {
  if (!h || !status) return JB_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned v = 0;
  JB_TRY(cudaMemcpyAsync(&v, &h->slots->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st),
         "status copy");
  JB_TRY(cudaStreamSynchronize(st), "status sync");
  JB_TRY(cudaMemsetAsync(&h->slots->status, 0, sizeof(unsigned), st), "status clear");
  *status = v;
  return JB_OK;
}

long long jb_workspace_bytes(const jb_handle* h) { return h ? h->ws_bytes : 0; }

int jb_set_kernel_timing(jb_handle* h, int enable) {
  if (!h) return JB_ERR_ARG;
  if (enable && !h->timing) {
    for (int i = 0; i < 2 * JB_TIMED_MAX; ++i)
      if (cudaEventCreate(&h->ev[i]) != cudaSuccess) return set_err(h, JB_ERR_CUDA, "event create");
    h->timing = 1;
  }
  h->nev = 0;
  for (int c = 0; c < JB_KCAT_COUNT; ++c) { h->acc_ms[c] = 0.0; h->acc_n[c] = 0; }
  return JB_OK;
}

int jb_kernel_times(jb_handle* h, double* ms, long long* launches) {
  if (!h || !ms || !launches) return JB_ERR_ARG;
  if (h->timing && h->nev > 0) {
    JB_TRY(cudaEventSynchronize(h->ev[2 * h->nev - 1]), "event sync");
    for (int i = 0; i < h->nev; ++i) {
      float t = 0.f;
      JB_TRY(cudaEventElapsedTime(&t, h->ev[2 * i], h->ev[2 * i + 1]), "event time");
      h->acc_ms[h->ev_cat[i]] += t;
      h->acc_n[h->ev_cat[i]] += 1;
    }
    h->nev = 0;
  }
  for (int c = 0; c < JB_KCAT_COUNT; ++c) { ms[c] = h->acc_ms[c]; launches[c] = h->acc_n[c]; }
  return JB_OK;
}

int jb_set_spacing(jb_handle* h, double dx, double dy) {
  if (!h || !(dx > 0.0) || (h->dim == 2 && !(dy > 0.0))) return set_err(h, JB_ERR_ARG, "bad spacing");
  h->grid.dx = dx;
  h->grid.idx = 1.0 / dx;
  if (h->dim == 2) {
    h->grid.dy = dy;
    h->grid.idy = 1.0 / dy;
  }
  return JB_OK;
}

int jb_sizeof_mech_params(void) { return (int)sizeof(jb_mech_params); }
int jb_sizeof_grid(void) { return (int)sizeof(jb_grid); }

const char* jb_last_error(const jb_handle* h) { return h ? h->err : "null handle"; }

}  // extern "C"
