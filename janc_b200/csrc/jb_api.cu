// C ABI of janc_b200 (declared in include/janc_b200.h): handle lifetime,
// workspace, argument checks and the per-step launch sequence.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <cmath>

#include "../../include/janc_b200.h"
#include "jb_adjoint.h"
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
  // adjoint support
  double base_A[JB_NREAC_MAX];  // pre-exponential factors as created (jb_set_log_A_offset)
  int probe[4];                 // x0, y0, wx, wy of the pressure probe (wx*wy = 0: none)
  void* fwork;                  // mixed 2D flux scratch (float32 primitives, x flux differences)
  jb_transport tr;              // laminar transport model (viscous fluxes when grid.visc is set)
  double* vbuf;                 // viscous node planes and node fluxes
  double* vcell;                // viscous rhs of the current stage state (nv x ncell)
  double* adj_ws;               // stage adjoints, primitives, face scratch, reductions
  unsigned char* adj_mult;      // padded-grid multiplicity of each cell (alpha ties)
  double* adj_B1;
  double* adj_B2;
  double* adj_prims;  // rho, u, v, p of the three stage states of a step
  double* adj_scratch;
  double* adj_red;
  // x-slab exchange (jb_set_exchange): caller-owned buffers and transport
  jb_exchange_fn xch;
  void* xch_user;
  double* xsend;  // [2][nv+2][3][ny] edge columns packed for the neighbours
  double* xsendy;   // [2][nv+2][nx][3] edge rows for the bottom / top boundary functions
  long long* xred;  // CFL pair reduced over the ranks
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
    if (!bc_ok(bc[s]) && bc[s] != JB_BC_HALO) return JB_ERR_ARG;
  if (dim == 1 && (bc[0] == JB_BC_RDC_INJECTOR || bc[1] == JB_BC_RDC_INJECTOR)) return JB_ERR_UNSUPPORTED;
  if (precision != JB_PREC_STRICT && precision != JB_PREC_FP64 && precision != JB_PREC_MIXED)
    return JB_ERR_UNSUPPORTED;
  jb_handle* h = new (std::nothrow) jb_handle();
  if (!h) return JB_ERR_ARG;
  std::memset(h, 0, sizeof(*h));
  h->mech = *mech;
  jb::derive_mech(h->mech);
  for (int i = 0; i < JB_NREAC_MAX; ++i) h->base_A[i] = h->mech.A[i];
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
  // mixed 2D: float32 primitives of the stage state and of the state being
  // written (two buffers used in turn), then the x flux differences
  const size_t bytes_fwork = precision == JB_PREC_MIXED && dim == 2 ? sizeof(float) * 18 * nc : 0;
  if (e == cudaSuccess && bytes_fwork) e = cudaMalloc(&h->fwork, bytes_fwork);
  if (e != cudaSuccess) {
    jb_destroy(h);
    return JB_ERR_CUDA;
  }
  h->ws_bytes = (long long)(2 * bytes_W + 2 * bytes_aux + bytes_cand + bytes_strip + sizeof(jb_slots) + bytes_fwork);
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
  if (h->fwork) cudaFree(h->fwork);
  if (h->vbuf) cudaFree(h->vbuf);
  if (h->adj_ws) cudaFree(h->adj_ws);
  if (h->adj_mult) cudaFree(h->adj_mult);
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
    if (g.bc[s] == JB_BC_HALO && !h->xch)
      return set_err(h, JB_ERR_ARG, "a halo side needs an exchange (jb_set_exchange)");
  }
  return JB_OK;
}

// One slab exchange: pack, hand the stream to the transport, unpack.  No-op
// for a handle without an exchange.
static int exchange(jb_handle* h, const double* U, const double* aux, int flags, int aidx, cudaStream_t st) {
  if (!h->xch) return JB_OK;
  if (!h->grid.halo_ring) flags &= ~JB_XCH_DT;  // one domain: its own CFL minimum
  if (!flags) return JB_OK;
  const jb::Ops& o = *h->ops;
  JB_TRY(o.xch_pre(h->dim, h->grid, U, aux, h->xsend, h->xsendy, h->slots, h->xred, flags, st), "exchange pack");
  const int rc = h->xch(h->xch_user, flags, (void*)st);
  if (rc != 0) return set_err(h, JB_ERR_ARG, "exchange transport failed (%d)", rc);
  JB_TRY(o.xch_post(h->dim, h->mech, h->grid, h->slots, h->xred, aidx, flags, st), "exchange unpack");
  return JB_OK;
}

int jb_set_exchange(jb_handle* h, double* send, double* halo, long long* red, jb_exchange_fn fn, void* user) {
  if (!h) return JB_ERR_ARG;
  if (!fn) {
    h->xch = nullptr;
    h->xch_user = nullptr;
    h->xsend = nullptr;
    h->xred = nullptr;
    h->xsendy = nullptr;
    h->grid.halo = nullptr;
    h->grid.haloy = nullptr;
    h->grid.halo_ring = 0;
    return JB_OK;
  }
  if (!send || !halo || !red) return set_err(h, JB_ERR_ARG, "exchange needs send, halo and red buffers");
  if (h->grid.nx < 3) return set_err(h, JB_ERR_ARG, "a slab needs at least 3 columns");
  h->xch = fn;
  h->xch_user = user;
  h->xsend = send;
  h->xred = red;
  h->grid.halo = halo;
  h->grid.halo_ring = 1;
  return JB_OK;
}

int jb_set_ghost_cells(jb_handle* h, double* sendx, double* halox, double* sendy, double* haloy,
                       jb_exchange_fn fn, void* user) {
  if (!h) return JB_ERR_ARG;
  if (!fn) return jb_set_exchange(h, nullptr, nullptr, nullptr, nullptr, nullptr);
  const jb_grid& g = h->grid;
  const bool hx = g.bc[0] == JB_BC_HALO || g.bc[1] == JB_BC_HALO;
  const bool hy = h->dim == 2 && (g.bc[2] == JB_BC_HALO || g.bc[3] == JB_BC_HALO);
  if (hx && (!sendx || !halox)) return set_err(h, JB_ERR_ARG, "x ghost sides need sendx and halox buffers");
  if (hy && (!sendy || !haloy)) return set_err(h, JB_ERR_ARG, "y ghost sides need sendy and haloy buffers");
  if (!hx && !hy) return set_err(h, JB_ERR_ARG, "no side was created with JB_BC_HALO");
  h->xch = fn;
  h->xch_user = user;
  h->xsend = hx ? sendx : nullptr;
  h->xsendy = hy ? sendy : nullptr;
  h->xred = nullptr;
  h->grid.halo = hx ? halox : nullptr;
  h->grid.haloy = hy ? haloy : nullptr;
  h->grid.halo_ring = 0;
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
                  h->slots, -1, 3, nullptr, st),
         "alpha");
  if (int rc = exchange(h, U, aux, JB_XCH_HALO, 3, st)) return rc;
  if (h->grid.visc)
    JB_TRY(o.visc(h->dim, h->mech, h->grid, h->tr, U, aux, h->strips, h->vbuf, h->vcell, st), "viscous");
  JB_TRY(o.flux(h->dim, 0, h->mech, h->grid, U, aux, nullptr, rhs, h->strips, h->slots, 3, jb_fin_cand(nullptr, -1),
                nullptr, nullptr, dt, st),
         "flux");
  return JB_OK;
}

int jb_boundary_conditions(jb_handle* h, const double* U, const double* aux, double* Up, double* auxp,
                           void* stream) {
  if (!h || !U || !aux || !Up || !auxp) return set_err(h, JB_ERR_ARG, "null pointer");
  if (int rc = check_theta(h)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const jb::Ops& o = *h->ops;
  // the ghost strips (outlet / injector states) and ghost layers of (U, aux)
  JB_TRY(o.slots_reset(h->slots, st), "slots_reset");
  JB_TRY(o.select(h->dim, false, true, false, h->mech, h->grid, U, aux, nullptr, nullptr, h->strips, h->slots,
                  -1, 3, nullptr, st),
         "strips");
  if (int rc = exchange(h, U, aux, JB_XCH_HALO, 3, st)) return rc;
  JB_TRY(o.pad(h->dim, h->grid, U, aux, h->strips, Up, auxp, st), "pad");
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
                  h->strips, h->slots, 0, 0, nullptr, st),
         "select");
  return JB_OK;
}

int jb_reaction_source_terms(jb_handle* h, const double* U, const double* aux, double dt,
                             double* S, void* stream) {
  if (!h || !U || !aux || !S) return set_err(h, JB_ERR_ARG, "null pointer");
  if (!(dt > 0.0)) return set_err(h, JB_ERR_ARG, "dt must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  JB_TRY(h->ops->chem(h->dim, true, h->mech, h->grid, U, aux, S, jb_fin_cand(nullptr, -1), h->slots, dt, st),
         "chem");
  return JB_OK;
}

// Record of one step for the adjoint, in doubles from the step's base:
// U, aux, U1, aux1, U2, aux2, U3, aux3 (each nv resp. 2 fields); the next
// step's record (or the final state) follows.
static long long rec_stride(const jb_handle* h) { return 4LL * (h->grid.nv + 2) * h->grid.ncell; }

static int advance_impl(jb_handle* h, const double* U, const double* aux, double* U_out,
                        double* aux_out, double dt_fixed, double cfl, int nsteps, double* dt_hist,
                        void* stream, bool chemistry, double* probe_p = nullptr, double* rec = nullptr,
                        double* rec_slots = nullptr) {
  if (!h || !U || !aux || !U_out || !aux_out) return set_err(h, JB_ERR_ARG, "null pointer");
  if (nsteps < 1) return set_err(h, JB_ERR_ARG, "nsteps must be >= 1");
  if (!(cfl > 0.0) && !(dt_fixed > 0.0)) return set_err(h, JB_ERR_ARG, "need cfl > 0 or dt > 0");
  if (U == U_out || aux == aux_out) return set_err(h, JB_ERR_ARG, "outputs must not alias inputs");
  if (int rc = check_theta(h)) return rc;
  if (probe_p && h->probe[2] * h->probe[3] <= 0)
    return set_err(h, JB_ERR_ARG, "probe pressures need jb_set_probe");
  if (rec && (!rec_slots || !chemistry)) return set_err(h, JB_ERR_ARG, "a record needs rec_slots");
  if (rec && h->xch) return set_err(h, JB_ERR_UNSUPPORTED, "the adjoint record is single-domain");
  if (!chemistry && nsteps != 1) return set_err(h, JB_ERR_ARG, "the flux-only step is one step");
  cudaStream_t st = (cudaStream_t)stream;
  const jb::Ops& o = *h->ops;
  const int d = h->dim;
  const bool use_cfl = cfl > 0.0;
  const jb_mech_params& m = h->mech;
  const jb_grid& g = h->grid;
  const size_t nU = (size_t)g.nv * g.ncell, nA = 2 * (size_t)g.ncell;
  const long long RS = rec ? rec_stride(h) : 0;
  if (rec) {
    JB_TRY(cudaMemcpyAsync(rec, U, sizeof(double) * nU, cudaMemcpyDeviceToDevice, st), "record U0");
    JB_TRY(cudaMemcpyAsync(rec + nU, aux, sizeof(double) * nA, cudaMemcpyDeviceToDevice, st), "record aux0");
  }
  // Per-cell mode (mixed: 2D, and 1D with flux splitting): each stage kernel
  // and the chemistry finish their new state's temperature per cell and
  // reduce its LF alpha (and, after the chemistry, the CFL minimum) in their
  // epilogue, so no select pass runs between them.  Global-stop mode (strict
  // and fp64, and the mixed 1D Godunov path): the kernels write the Halley
  // iterates and a select pass after each picks the reference's iteration
  // count.
  const bool pc = o.per_cell && (d == 2 || g.scheme == JB_FLUX_LF || g.scheme == JB_FLUX_SW);
  // mixed 2D: float32 u, v, p of the current state (pin) and the buffer the
  // next kernel writes (pout), swapped after each writer
  float* pin = h->fwork ? static_cast<float*>(h->fwork) : nullptr;
  float* pout = pin ? pin + 3 * g.ncell : nullptr;
  void* dfx = pin ? static_cast<void*>(pin + 6 * g.ncell) : nullptr;
  auto swap_prims = [&]() {
    float* t = pin;
    pin = pout;
    pout = t;
  };
  JB_TIMED(JB_KCAT_OTHER, o.slots_reset(h->slots, st), "slots_reset");
  // alpha (and CFL minimum) of the initial state, ghost strips for stage 1
  JB_TIMED(JB_KCAT_SELECT, o.select(d, false, true, use_cfl, m, g, U, aux, nullptr, nullptr, h->strips, h->slots, -1, 3,
                  pin, st),
         "prep");
  for (int s = 0; s < nsteps; ++s) {
    double* r = rec ? rec + s * RS : nullptr;
    const double* Un = r ? r : (s == 0 ? U : U_out);
    const double* an = r ? r + nU : (s == 0 ? aux : aux_out);
    double* W1 = r ? r + (nU + nA) : h->W[0];
    double* A1 = r ? W1 + nU : h->auxw[0];
    double* W2 = r ? A1 + nA : h->W[1];
    double* A2 = r ? W2 + nU : h->auxw[1];
    double* W3 = r ? A2 + nA : h->W[0];
    double* A3 = r ? W3 + nU : h->auxw[0];
    double* Uo = r ? r + RS : U_out;
    double* Ao = r ? r + RS + nU : aux_out;
    if (!chemistry) {  // advance_flux only (TVD_RK3.py:5-12): stage 3 writes the result
      W3 = U_out;
      A3 = aux_out;
    }
    // slabs: the CFL minimum over the ranks and the halo of the step's state
    if (int rc = exchange(h, Un, an, (use_cfl ? JB_XCH_DT : 0) | JB_XCH_HALO, 3, st)) return rc;
    JB_TIMED(JB_KCAT_OTHER, o.step_begin(h->slots, use_cfl ? cfl : 0.0, dt_fixed, dt_hist, s, st), "step_begin");
    // stage 1: U1 = U + L(U)
    if (g.visc)
      JB_TIMED(JB_KCAT_FLUX, o.visc(d, m, g, h->tr, Un, an, h->strips, h->vbuf, h->vcell, st), "viscous");
    if (pc) {
      JB_TIMED(JB_KCAT_FLUX, o.flux(d, 1, m, g, Un, an, Un, W1, h->strips, h->slots, 0,
                                    jb_fin_cell(A1, pout, 1, 0), pin, dfx, 0.0, st), "stage1");
      swap_prims();
      JB_TIMED(JB_KCAT_SELECT, o.strips(d, m, g, W1, A1, h->strips, h->slots, 1, st), "strips1");
    } else {
      JB_TIMED(JB_KCAT_FLUX, o.flux(d, 1, m, g, Un, an, Un, W1, h->strips, h->slots, 0, jb_fin_cand(h->cand, 0),
                                    pin, dfx, 0.0, st), "stage1");
      JB_TIMED(JB_KCAT_SELECT, o.select(d, true, true, false, m, g, W1, nullptr, h->cand, A1, h->strips,
                      h->slots, 0, 1, pin, st),
             "select1");
    }
    if (int rc = exchange(h, W1, A1, JB_XCH_HALO, 1, st)) return rc;
    // stage 2: U2 = 3/4 U + 1/4 (U1 + L(U1))
    if (g.visc)
      JB_TIMED(JB_KCAT_FLUX, o.visc(d, m, g, h->tr, W1, A1, h->strips, h->vbuf, h->vcell, st), "viscous");
    if (pc) {
      JB_TIMED(JB_KCAT_FLUX, o.flux(d, 2, m, g, W1, A1, Un, W2, h->strips, h->slots, 1,
                                    jb_fin_cell(A2, pout, 2, 0), pin, dfx, 0.0, st), "stage2");
      swap_prims();
      JB_TIMED(JB_KCAT_SELECT, o.strips(d, m, g, W2, A2, h->strips, h->slots, 2, st), "strips2");
    } else {
      JB_TIMED(JB_KCAT_FLUX, o.flux(d, 2, m, g, W1, A1, Un, W2, h->strips, h->slots, 1, jb_fin_cand(h->cand, 1),
                                    pin, dfx, 0.0, st), "stage2");
      JB_TIMED(JB_KCAT_SELECT, o.select(d, true, true, false, m, g, W2, nullptr, h->cand, A2, h->strips,
                      h->slots, 1, 2, pin, st),
             "select2");
    }
    if (int rc = exchange(h, W2, A2, JB_XCH_HALO, 2, st)) return rc;
    // stage 3: U3 = 1/3 U + 2/3 (U2 + L(U2))
    if (g.visc)
      JB_TIMED(JB_KCAT_FLUX, o.visc(d, m, g, h->tr, W2, A2, h->strips, h->vbuf, h->vcell, st), "viscous");
    if (pc) {
      // without the chemistry this is the step's result: its alpha, CFL
      // minimum and primitives serve the next step
      const jb_fin f3 = chemistry ? jb_fin_cell(A3, nullptr, -1, 0) : jb_fin_cell(A3, pout, 3, use_cfl);
      JB_TIMED(JB_KCAT_FLUX, o.flux(d, 3, m, g, W2, A2, Un, W3, h->strips, h->slots, 2, f3, pin, dfx, 0.0, st),
               "stage3");
      if (!chemistry) {
        swap_prims();
        JB_TIMED(JB_KCAT_SELECT, o.strips(d, m, g, W3, A3, h->strips, h->slots, 3, st), "strips3");
        continue;
      }
    } else {
      JB_TIMED(JB_KCAT_FLUX, o.flux(d, 3, m, g, W2, A2, Un, W3, h->strips, h->slots, 2, jb_fin_cand(h->cand, 2),
                                    pin, dfx, 0.0, st), "stage3");
      if (!chemistry) {
        JB_TIMED(JB_KCAT_SELECT, o.select(d, true, true, use_cfl, m, g, W3, nullptr, h->cand, A3,
                                          h->strips, h->slots, 2, 3, pin, st),
                 "select3");
        continue;
      }
      // the adjoint record keeps aux3; otherwise the stage-3 temperature is
      // taken from the iterates inside the chemistry kernel
      if (rec)
        JB_TIMED(JB_KCAT_SELECT, o.select(d, true, false, false, m, g, W3, nullptr, h->cand, A3, h->strips,
                        h->slots, 2, 0, nullptr, st),
               "select3");
    }
    // chemistry and the final temperature solve
    if (pc) {
      JB_TIMED(JB_KCAT_CHEM, o.chem(d, false, m, g, W3, A3, Uo, jb_fin_cell(Ao, pout, 3, use_cfl), h->slots, 0.0, st),
               "chem");
      swap_prims();
      JB_TIMED(JB_KCAT_SELECT, o.strips(d, m, g, Uo, Ao, h->strips, h->slots, 3, st), "strips4");
    } else {
      JB_TIMED(JB_KCAT_CHEM, o.chem(d, false, m, g, W3, rec ? A3 : nullptr, Uo, jb_fin_cand(h->cand, 3), h->slots,
                                    0.0, st),
               "chem");
      JB_TIMED(JB_KCAT_SELECT, o.select(d, true, true, use_cfl, m, g, Uo, nullptr, h->cand, Ao, h->strips,
                      h->slots, 3, 3, pin, st),
             "select4");
    }
    if (rec)
      JB_TRY(cudaMemcpyAsync(rec_slots + s * (sizeof(jb_slots) / sizeof(double)), h->slots, sizeof(jb_slots),
                             cudaMemcpyDeviceToDevice, st),
             "record slots");
    if (probe_p)
      JB_TRY(jb::adj::probe_mean(d, m, g, Uo, Ao, h->probe[0], h->probe[1], h->probe[2], h->probe[3], probe_p + s, st),
             "probe");
  }
  if (rec) {
    JB_TRY(cudaMemcpyAsync(U_out, rec + nsteps * RS, sizeof(double) * nU, cudaMemcpyDeviceToDevice, st), "U_out");
    JB_TRY(cudaMemcpyAsync(aux_out, rec + nsteps * RS + nU, sizeof(double) * nA, cudaMemcpyDeviceToDevice, st),
           "aux_out");
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
                  h->slots, -1, 3, nullptr, st),
         "cfl");
  if (int rc = exchange(h, U, aux, JB_XCH_DT, 3, st)) return rc;
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

int jb_set_reconstruction(jb_handle* h, int recon) {
  if (!h) return JB_ERR_ARG;
  if (recon != JB_RECON_WENO5 && recon != JB_RECON_MUSCL) return set_err(h, JB_ERR_ARG, "unknown reconstruction");
  h->grid.recon = recon;
  return JB_OK;
}

int jb_set_transport(jb_handle* h, const jb_transport* tr) {
  if (!h) return JB_ERR_ARG;
  if (!tr) {  // Euler fluxes again
    if (h->vbuf) cudaFree(h->vbuf);
    h->vbuf = h->vcell = nullptr;
    h->grid.visc = nullptr;
    return JB_OK;
  }
  const jb_transport& t = *tr;
  auto bad01 = [](int v) { return v != 0 && v != 1; };
  if (bad01(t.viscosity_model) || bad01(t.conductivity_model) || bad01(t.diffusivity_model) ||
      bad01(t.turbulence_model))
    return set_err(h, JB_ERR_ARG, "unknown transport model");
  if (t.turbulence_model && h->dim != 2)
    return set_err(h, JB_ERR_UNSUPPORTED, "the LES sub-grid model (Vreman) is 2D only");
  if (!(t.Pr > 0.0) || !(t.Le > 0.0) || !(t.Pr_t > 0.0) || !(t.Le_t > 0.0) ||
      (t.viscosity_model == 0 && !(t.T_ref > 0.0)))
    return set_err(h, JB_ERR_ARG, "transport parameters must be positive");
  if (!h->vbuf) {
    const long long n = jb::visc_scratch_doubles(h->dim, h->grid) + (long long)h->grid.nv * h->grid.ncell;
    JB_TRY(cudaMalloc(&h->vbuf, sizeof(double) * n), "viscous scratch");
    h->vcell = h->vbuf + jb::visc_scratch_doubles(h->dim, h->grid);
    h->ws_bytes += (long long)sizeof(double) * n;
  }
  h->tr = t;
  h->grid.visc = h->vcell;
  return JB_OK;
}

int jb_set_flux_scheme(jb_handle* h, int scheme) {
  if (!h) return JB_ERR_ARG;
  if (scheme != JB_FLUX_LF && scheme != JB_FLUX_HLLC && scheme != JB_FLUX_AUSMPW && scheme != JB_FLUX_SW)
    return set_err(h, JB_ERR_ARG, "unknown flux scheme");
  h->grid.scheme = scheme;
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

int jb_set_probe(jb_handle* h, int x0, int y0, int wx, int wy) {
  if (!h) return JB_ERR_ARG;
  if (x0 < 0 || y0 < 0 || wx < 0 || wy < 0 || x0 + wx > h->grid.nx || y0 + wy > h->grid.ny || wx * wy > 1024)
    return set_err(h, JB_ERR_ARG, "probe outside the grid (or over 1024 cells)");
  h->probe[0] = x0;
  h->probe[1] = y0;
  h->probe[2] = wx;
  h->probe[3] = wy;
  return JB_OK;
}

int jb_set_log_A_offset(jb_handle* h, const double* offset) {
  if (!h) return JB_ERR_ARG;
  for (int i = 0; i < h->mech.nreac; ++i) h->mech.A[i] = h->base_A[i] * (offset ? std::exp(offset[i]) : 1.0);
  jb::derive_mech(h->mech);
  return JB_OK;
}

long long jb_record_doubles(const jb_handle* h) { return h ? rec_stride(h) : 0; }

int jb_advance_ex(jb_handle* h, const double* U, const double* aux, double* U_out, double* aux_out,
                  double dt_fixed, double cfl, int nsteps, double* dt_hist, double* probe_p, double* rec,
                  double* rec_slots, void* stream) {
  return advance_impl(h, U, aux, U_out, aux_out, dt_fixed, cfl, nsteps, dt_hist, stream, true, probe_p, rec,
                      rec_slots);
}

// Multiplicity of every cell in the reference's padded array (periodic pad
// of both axes, then the four sides; corners keep the periodic wrap; 1D:
// the x axis alone): how many padded entries copy it.  The ghosts of a
// pressure-outlet side are not copies and count as entries of their own (in
// the adjoint kernels).
static void padded_multiplicity(int dim, const jb_grid& g, std::vector<unsigned char>& mult) {
  const int nx = g.nx, ny = g.ny, pad_y = dim == 2 ? 3 : 0;
  mult.assign((size_t)nx * ny, 0);
  auto per = [](int c, int n) { return c < 0 ? n - 1 + c : (c >= n ? c - n + 1 : c); };
  auto side = [](int c, int n, int kind, bool& ok) {
    ok = true;
    const bool lo = c < 0;
    switch (kind) {
      case JB_BC_PERIODIC: return lo ? n - 1 + c : c - n + 1;
      case JB_BC_SLIP_WALL: return lo ? 0 : n - 1;
      case JB_BC_ZERO_GRADIENT:
      case JB_BC_NO_SLIP_WALL: return lo ? -1 - c : 2 * n - 1 - c;
      default: ok = false; return 0;
    }
  };
  for (int x = -3; x < nx + 3; ++x)
    for (int y = -pad_y; y < ny + pad_y; ++y) {
      const bool xin = x >= 0 && x < nx, yin = y >= 0 && y < ny;
      int sx = x, sy = y;
      bool ok = true;
      if (!xin && !yin) {
        sx = per(x, nx);
        sy = per(y, ny);
      } else if (!xin) {
        sx = side(x, nx, g.bc[x < 0 ? 0 : 1], ok);
      } else if (!yin) {
        sy = side(y, ny, g.bc[y < 0 ? 2 : 3], ok);
      }
      if (ok && sx >= 0 && sx < nx && sy >= 0 && sy < ny) mult[(size_t)sx * ny + sy] += 1;
    }
}

// What jb_adjoint_step differentiates; checked when the workspace is reserved
// and again at every step (the flux scheme can change in between).
static int adj_supported(jb_handle* h) {
  if (h->grid.scheme != JB_FLUX_LF || h->grid.visc || h->grid.recon != JB_RECON_WENO5)
    return set_err(h, JB_ERR_UNSUPPORTED, "the adjoint differentiates the inviscid LF / WENO5-JS path");
  if (h->xch || h->grid.bc[0] == JB_BC_HALO || h->grid.bc[1] == JB_BC_HALO)
    return set_err(h, JB_ERR_UNSUPPORTED, "the adjoint is single-domain (no x slabs)");
  for (int s = 0; s < 2 * h->dim; ++s)
    if (h->grid.bc[s] == JB_BC_RDC_INJECTOR && s != 2)
      return set_err(h, JB_ERR_UNSUPPORTED, "the injector side of the adjoint is the bottom side (2D)");
  return JB_OK;
}

int jb_adjoint_reserve(jb_handle* h) {
  if (!h) return JB_ERR_ARG;
  if (h->adj_ws) return JB_OK;
  if (int rc = adj_supported(h)) return rc;
  const jb_grid& g = h->grid;
  const size_t nc = (size_t)g.ncell, nU = (size_t)g.nv * nc;
  const size_t nsc = jb::adj::flux_scratch_doubles(h->dim, g);
  const size_t n = 2 * nU + 12 * nc + nsc + jb::adj::RED_N;
  std::vector<unsigned char> mult;
  padded_multiplicity(h->dim, g, mult);
  cudaError_t e = cudaMalloc(&h->adj_ws, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMalloc(&h->adj_mult, nc);
  if (e == cudaSuccess) e = cudaMemset(h->adj_ws, 0, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMemcpy(h->adj_mult, mult.data(), nc, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (h->adj_ws) cudaFree(h->adj_ws);
    if (h->adj_mult) cudaFree(h->adj_mult);
    h->adj_ws = nullptr;
    h->adj_mult = nullptr;
    return check_cuda(h, e, "adjoint workspace");
  }
  h->adj_B1 = h->adj_ws;
  h->adj_B2 = h->adj_B1 + nU;
  h->adj_prims = h->adj_B2 + nU;
  h->adj_scratch = h->adj_prims + 12 * nc;
  h->adj_red = h->adj_scratch + nsc;
  h->ws_bytes += (long long)(sizeof(double) * n + nc);
  return JB_OK;
}

int jb_adjoint_step(jb_handle* h, const double* rec, const double* rec_slots, double cfl, double* Ubar,
                    double* Abar, const double* dt_bar, const double* pp_bar, double* lnA_bar, void* stream) {
  if (!h || !rec || !rec_slots || !Ubar || !Abar || !lnA_bar) return set_err(h, JB_ERR_ARG, "null pointer");
  if (pp_bar && h->probe[2] * h->probe[3] <= 0) return set_err(h, JB_ERR_ARG, "probe adjoint needs jb_set_probe");
  if (int rc = adj_supported(h)) return rc;
  if (!h->adj_ws) return set_err(h, JB_ERR_ARG, "call jb_adjoint_reserve before jb_adjoint_step");
  cudaStream_t st = (cudaStream_t)stream;
  const jb_mech_params& m = h->mech;
  const jb_grid& g = h->grid;
  const size_t nc = (size_t)g.ncell, nU = (size_t)g.nv * nc, nA = 2 * nc;
  const double* Un = rec;
  const double* An = Un + nU;
  const double* W1 = An + nA;
  const double* A1 = W1 + nU;
  const double* W2 = A1 + nA;
  const double* A2 = W2 + nU;
  const double* W3 = A2 + nA;
  const double* A3 = W3 + nU;
  const double* U4 = rec + rec_stride(h);
  const double* A4 = U4 + nU;
  const double* slots = rec_slots;
  const double* slot_dt = slots + offsetof(jb_slots, dt) / sizeof(double);
  double* red = h->adj_red;
  double *B1 = h->adj_B1, *B2 = h->adj_B2, *P = h->adj_prims, *sc = h->adj_scratch;
  const unsigned char* mult = h->adj_mult;
  const double c_cfl = cfl > 0.0 ? cfl : 0.0;
  JB_TRY(cudaMemsetAsync(red, 0, sizeof(double) * jb::adj::RED_N, st), "reduction clear");
  // loss term of this step, the final temperature solve; primitives and tie
  // counts of the three stage states
  const int d = h->dim;
  JB_TRY(jb::adj::vjp_begin(d, m, g, U4, A4, pp_bar, h->probe, Ubar, Abar, rec, P, mult, slots, c_cfl, red, sc, st),
         "adjoint begin");
  // chemistry (and update_aux of U3): B1 = Ubar3
  JB_TRY(jb::adj::chem_vjp(d, m, g, W3, A3, Ubar, B1, slot_dt, red + jb::adj::RED_DTB, lnA_bar, st), "chemistry");
  // stage 3: U3 = 1/3 U + 2/3 (U2 + dt L(U2, aux2)); B2 = Ubar2, Ubar = 1/3 B1
  JB_TRY(jb::adj::flux_stage(d, m, g, W2, A2, P + 8 * nc, B1, 2.0 / 3.0, slots, 2, 0.0, mult, red, dt_bar, sc, B2, false,
                             nullptr, Ubar, 1.0 / 3.0, false, st),
         "stage 3");
  // stage 2: U2 = 3/4 U + 1/4 (U1 + dt L(U1, aux1)); B1 = Ubar1, Ubar += 3/4 B2
  JB_TRY(jb::adj::flux_stage(d, m, g, W1, A1, P + 4 * nc, B2, 0.25, slots, 1, 0.0, mult, red, dt_bar, sc, B1, false,
                             nullptr, Ubar, 0.75, true, st),
         "stage 2");
  // stage 1: U1 = U + dt L(U, aux), with alpha 1 and the CFL time step
  JB_TRY(jb::adj::flux_stage(d, m, g, Un, An, P, B1, 1.0, slots, 0, c_cfl, mult, red, dt_bar, sc, Ubar, true, Abar,
                             nullptr, 0.0, false, st),
         "stage 1");
  return JB_OK;
}

int jb_state_from_PTY_vjp(jb_handle* h, const double* P, const double* T, const double* Y, const double* Ubar,
                          const double* Abar, double* Tbar, void* stream) {
  if (!h || !P || !T || !Y || !Ubar || !Abar || !Tbar) return set_err(h, JB_ERR_ARG, "null pointer");
  JB_TRY(jb::adj::init_vjp(h->dim, h->mech, h->grid.ncell, P, T, Y, Ubar, Abar, Tbar, (cudaStream_t)stream), "init vjp");
  return JB_OK;
}

static int amr_check(jb_handle* h, int nb, int bx, int by) {
  if (!h) return JB_ERR_ARG;
  if (h->dim != 2) return set_err(h, JB_ERR_ARG, "block AMR is 2D");
  if (h->grid.scheme != JB_FLUX_LF || h->grid.visc)
    return set_err(h, JB_ERR_UNSUPPORTED, "block AMR supports LF flux splitting without viscosity");
  if (nb < 0 || bx < 1 || by < 1) return set_err(h, JB_ERR_ARG, "bad block shape");
  return JB_OK;
}

static bool overlaps(const double* a, const double* b, long long n) {
  return a && b && a < b + n && b < a + n;
}

int jb_amr_stage(jb_handle* h, int nb, int bx, int by, double dx, double dy, int stage, const double* G,
                 const double* U0, double dt, double* out, void* stream) {
  if (int rc = amr_check(h, nb, bx, by)) return rc;
  if (stage < 1 || stage > 3) return set_err(h, JB_ERR_ARG, "stage must be 1, 2 or 3");
  if (!G || !out || (stage > 1 && !U0)) return set_err(h, JB_ERR_ARG, "null pointer");
  if (!(dx > 0.0) || !(dy > 0.0)) return set_err(h, JB_ERR_ARG, "dx and dy must be positive");
  const int nv = h->grid.nv;
  const long long nc = (long long)(bx + 6) * (by + 6), n = (long long)nb * (nv + 2) * nc;
  if (overlaps(out, G, n) || (stage > 1 && overlaps(out, U0, n)))
    return set_err(h, JB_ERR_ARG, "out must not overlap G or U0");
  if (nb == 0) return JB_OK;
  jb::jb_amr_io io;
  io.gU = G;
  io.gA = G + nv * nc;
  io.gsU = io.gsA = (nv + 2) * nc;
  io.u0 = stage > 1 ? U0 : nullptr;
  io.u0s = (nv + 2) * nc;
  io.oU = out;
  io.oA = out + nv * nc;
  io.osU = io.osA = (nv + 2) * nc;
  JB_TRY(h->ops->amr_stage(h->mech, h->grid, nb, bx, by, dx, dy, stage, io, h->slots, dt, (cudaStream_t)stream),
         "amr_stage");
  return JB_OK;
}

int jb_amr_flux(jb_handle* h, int nb, int bx, int by, double dx, double dy, const double* U, const double* aux,
                double dt, double* rhs, void* stream) {
  if (int rc = amr_check(h, nb, bx, by)) return rc;
  if (!U || !aux || !rhs) return set_err(h, JB_ERR_ARG, "null pointer");
  if (!(dx > 0.0) || !(dy > 0.0)) return set_err(h, JB_ERR_ARG, "dx and dy must be positive");
  const int nv = h->grid.nv;
  const long long nc = (long long)(bx + 6) * (by + 6);
  if (overlaps(rhs, U, (long long)nb * nv * nc)) return set_err(h, JB_ERR_ARG, "rhs must not overlap U");
  if (nb == 0) return JB_OK;
  jb::jb_amr_io io;
  io.gU = U;
  io.gA = aux;
  io.gsU = nv * nc;
  io.gsA = 2 * nc;
  io.u0 = nullptr;
  io.u0s = 0;
  io.oU = rhs;
  io.oA = nullptr;
  io.osU = nv * nc;
  io.osA = 0;
  JB_TRY(h->ops->amr_stage(h->mech, h->grid, nb, bx, by, dx, dy, 0, io, h->slots, dt, (cudaStream_t)stream),
         "amr_flux");
  return JB_OK;
}

int jb_amr_update_aux(jb_handle* h, int nb, int nx, int ny, const double* U, const double* aux_in, double* aux_out,
                      void* stream) {
  if (!h) return JB_ERR_ARG;
  if (h->dim != 2) return set_err(h, JB_ERR_ARG, "block AMR is 2D");
  if (nb < 0 || nx < 1 || ny < 1) return set_err(h, JB_ERR_ARG, "bad block shape");
  if (!U || !aux_in || !aux_out) return set_err(h, JB_ERR_ARG, "null pointer");
  const long long nc = (long long)nx * ny;
  if (overlaps(aux_out, aux_in, 2LL * nb * nc)) return set_err(h, JB_ERR_ARG, "aux_out must not overlap aux_in");
  if (nb == 0) return JB_OK;
  JB_TRY(h->ops->amr_update(h->mech, nb, nc, U, aux_in, aux_out, h->slots, (cudaStream_t)stream), "amr_update");
  return JB_OK;
}

int jb_amr_chem(jb_handle* h, int nb, int bx, int by, const double* blk, double dt, double* out, void* stream) {
  if (int rc = amr_check(h, nb, bx, by)) return rc;
  if (!blk || !out) return set_err(h, JB_ERR_ARG, "null pointer");
  if (!(dt > 0.0)) return set_err(h, JB_ERR_ARG, "dt must be positive");
  const long long n = (long long)nb * (h->grid.nv + 2) * bx * by;
  if (out != blk && overlaps(out, blk, n)) return set_err(h, JB_ERR_ARG, "out must equal blk or not overlap it");
  if (nb == 0) return JB_OK;
  JB_TRY(h->ops->amr_chem(h->mech, nb, bx, by, blk, out, h->slots, dt, (cudaStream_t)stream), "amr_chem");
  return JB_OK;
}

int jb_sizeof_mech_params(void) { return (int)sizeof(jb_mech_params); }
int jb_sizeof_grid(void) { return (int)sizeof(jb_grid); }

const char* jb_last_error(const jb_handle* h) { return h ? h->err : "null handle"; }

}  // extern "C"
