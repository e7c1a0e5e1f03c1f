// JANC per-step hot path as sm_100a kernels.
//
// This header is compiled twice: jb_strict.cu (namespace jb::strict, built
// with -fmad=false so every expression rounds exactly as the reference's
// float64 array code does) and jb_fast.cu (namespace jb::fast, FMA
// contraction allowed).  Each function cites the reference file it restates
// (paths inside the JANC repository, src/janc_v2/...).
//
// Data layout (the reference's, C-contiguous float64):
//   U   [nv][nx][ny]   nv = 4 + 8 in 2D (rho, rho u, rho v, rho E, rho Y_1..8)
//                      nv = 3 + 8 in 1D (ny == 1)
//   aux [2][nx][ny]    gamma, T
//   cand[6][nx][ny]    Halley iterates T_0..T_5 of the last temperature solve
//   strips[4][nv+2][L] ghost states of pressure-outlet / injector sides
//                      (L = max(nx, ny)); fields U..., gamma, T
#include <cuda.h>  // CUtensorMap (the tile kernels' TMA descriptors)
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "jb_fin.h"
#include "jb_types.h"

#ifndef JB_NS
#error "define JB_NS before including jb_kernels.cuh"
#endif

namespace jb {
namespace JB_NS {
namespace {  // internal linkage: several translation units include this header

constexpr int NS = 9;
constexpr int NR = 8;
constexpr int NREAC = 19;
constexpr double HALLEY_TOL = 5e-9;  // model/thermo_model.py:18
constexpr int HALLEY_MAX = 5;        // model/thermo_model.py:17

typedef jb_mech_params MP;

typedef jb_grid Grid;
typedef jb_slots Slots;

__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}
__device__ __forceinline__ double bitsd(unsigned long long b) {
  return __longlong_as_double((long long)b);
}

// ---------------------------------------------------------------------------
// block reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ unsigned warp_or(unsigned v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// All threads of the block must call; returns the result in thread 0.
__device__ __forceinline__ void block_reduce_store(double ax, double ay, double dtm,
                                                   unsigned bits, Slots* s, int aidx,
                                                   bool do_alpha, bool do_dt, int midx) {
  __shared__ double rax[32], ray[32], rdt[32];
  __shared__ unsigned rbits[32];
  ax = warp_max(ax);
  ay = warp_max(ay);
  dtm = warp_min(dtm);
  bits = warp_or(bits);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { rax[w] = ax; ray[w] = ay; rdt[w] = dtm; rbits[w] = bits; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int nw = (blockDim.x + 31) >> 5;
    for (int i = 1; i < nw; ++i) {
      ax = fmax(ax, rax[i]); ay = fmax(ay, ray[i]); dtm = fmin(dtm, rdt[i]); bits |= rbits[i];
    }
    if (do_alpha) {
      if (ax > 0.0) atomicMax(&s->ax[aidx], dbits(ax));
      if (ay > 0.0) atomicMax(&s->ay[aidx], dbits(ay));
    }
    if (do_dt) atomicMin(&s->dtmin_next, dbits(dtm));
    if (midx >= 0 && (bits & 0xffffu)) atomicOr(&s->mask[midx], bits & 0xffffu);
    if (bits >> 16) atomicOr(&s->status, bits >> 16);
  }
}

// ---------------------------------------------------------------------------
// NASA7 thermo (model/thermo_model.py:80-133)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double poly4(const double* c, double T) {
  double y = c[0];
  y = y * T + c[1];
  y = y * T + c[2];
  y = y * T + c[3];
  return y;
}
__device__ __forceinline__ double poly5(const double* c, double T) {
  double y = c[0];
  y = y * T + c[1];
  y = y * T + c[2];
  y = y * T + c[3];
  y = y * T + c[4];
  return y;
}
__device__ __forceinline__ double poly6(const double* c, double T) {
  double y = c[0];
  y = y * T + c[1];
  y = y * T + c[2];
  y = y * T + c[3];
  y = y * T + c[4];
  y = y * T + c[5];
  return y;
}

// advective + viscous rhs of field f at cell (NS_flux, solver_2D/flux.py:117-118);
// g.visc holds the viscous part computed for the stage state, or is null.
// The LF stage kernels take VISC as a template flag, so that their inviscid
// instantiations read no viscous pointer: a pointer not known to be free of
// aliasing with the kernel's output keeps the compiler from batching the
// epilogue's loads ahead of its stores.
template <bool VISC>
__device__ __forceinline__ double visc_add(const Grid& g, int f, long long cell, double adv) {
  return VISC ? adv + g.visc[f * g.ncell + cell] : adv;
}

// Runtime form (Godunov stage kernels).
__device__ __forceinline__ double visc_add(const Grid& g, int f, long long cell, double adv) {
  return g.visc ? adv + g.visc[f * g.ncell + cell] : adv;
}

// fill_Y (thermo_model.py:80-82): the last species closes the mass balance.
__device__ __forceinline__ void fill_Y(const double* Y8, double* Yf) {
  double s = Y8[0];
#pragma unroll
  for (int k = 1; k < NR; ++k) s = s + Y8[k];
#pragma unroll
  for (int k = 0; k < NR; ++k) Yf[k] = Y8[k];
  Yf[NR] = 1.0 - s;
}

// get_R (thermo_model.py:87-92): R = sum_k (1/M_k) Y_k
__device__ __forceinline__ double get_R(const MP& m, const double* Yf) {
  double r = m.invM[0] * Yf[0];
#pragma unroll
  for (int k = 1; k < NS; ++k) r = r + m.invM[k] * Yf[k];
  return r;
}

struct Th {
  double cp, h, dcp;
};

// get_thermo_nasa7 mixture sums (thermo_model.py:100-126)
__device__ __forceinline__ Th thermo_mix(const MP& m, double T, const double* Yf) {
  Th t;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const bool lo = T < m.Tcr[k];
    double cpk = lo ? poly5(m.cp_lo[k], T) : poly5(m.cp_hi[k], T);
    double dck = lo ? poly4(m.dcp_lo[k], T) : poly4(m.dcp_hi[k], T);
    double hk = lo ? poly6(m.h_lo[k], T) : poly6(m.h_hi[k], T);
    if (k == 0) {
      t.cp = cpk * Yf[0]; t.h = hk * Yf[0]; t.dcp = dck * Yf[0];
    } else {
      t.cp = t.cp + cpk * Yf[k]; t.h = t.h + hk * Yf[k]; t.dcp = t.dcp + dck * Yf[k];
    }
  }
  return t;
}

__device__ __forceinline__ double cp_mix(const MP& m, double T, const double* Yf) {
  double cp = 0.0;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const bool lo = T < m.Tcr[k];
    double cpk = lo ? poly5(m.cp_lo[k], T) : poly5(m.cp_hi[k], T);
    cp = (k == 0) ? cpk * Yf[0] : cp + cpk * Yf[k];
  }
  return cp;
}

// Halley iterates of the temperature solve (thermo_model.py:135-153).  The
// reference stops all cells together when max|res| <= tol, so every cell
// runs the five iterations, keeps T_0..T_5, and reports per iteration whether
// its residual exceeded tol (bits 0..4) or was NaN (bits 8..12).  The
// iteration count is fixed later from the OR of all cells' masks.
__device__ __forceinline__ unsigned halley_iterates(const MP& m, double e, const double* Yf,
                                                    double R, double T0, double* cand) {
  unsigned bits = 0;
  double T = T0;
  cand[0] = T;
#pragma unroll
  for (int i = 0; i < HALLEY_MAX; ++i) {
    Th t = thermo_mix(m, T, Yf);
    double res = (t.h - R * T) - e;
    double d1 = t.cp - R;
    double d2 = t.dcp;
    if (fabs(res) > HALLEY_TOL) bits |= 1u << i;
    if (res != res) bits |= 1u << (8 + i);
    double dT = ((-2.0 * res) * d1) / ((2.0 * (d1 * d1)) - res * d2);
    T = T + dT;
    cand[i + 1] = T;
  }
  return bits;
}

#if JB_FAST
// Fast-variant Halley iterates.  When every species switches NASA7 ranges at
// the same temperature (m.tcr_uniform), the mixture's cp, dcp/dT and h are
// polynomials in T whose coefficients are the Y-weighted sums of the
// species' coefficients; they are formed once per cell for the range the
// iterate is in, so each iteration costs ~15 FMAs instead of ~140.  The
// rounding differs from the reference's per-species sums at the ulp level.
struct MixPoly {
  double cp[5], dcp[4], h[6];
};

template <bool LO>
__device__ __forceinline__ void mix_poly_range(const MP& m, const double* Yf, MixPoly& P) {
  const auto& cp = LO ? m.cp_lo : m.cp_hi;
  const auto& dcp = LO ? m.dcp_lo : m.dcp_hi;
  const auto& h = LO ? m.h_lo : m.h_hi;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      if (j < 5) a += Yf[k] * cp[k][j];
      if (j < 4) b += Yf[k] * dcp[k][j];
      c += Yf[k] * h[k][j];
    }
    if (j < 5) P.cp[j] = a;
    if (j < 4) P.dcp[j] = b;
    P.h[j] = c;
  }
}

// branch (warp-uniform away from the switch isotherm) so the coefficients are
// read straight from the parameter bank
__device__ __forceinline__ void mix_poly(const MP& m, const double* Yf, bool lo, MixPoly& P) {
  if (lo) mix_poly_range<true>(m, Yf, P);
  else mix_poly_range<false>(m, Yf, P);
}

__device__ __forceinline__ unsigned halley_iterates_fast(const MP& m, double e, const double* Yf, double R,
                                                         double T0, double* cand) {
  unsigned bits = 0;
  double T = T0;
  cand[0] = T;
  const double Tcr = m.Tcr[0];
  bool lo = T < Tcr;
  MixPoly P;
  mix_poly(m, Yf, lo, P);
#pragma unroll 1
  for (int i = 0; i < HALLEY_MAX; ++i) {
    const bool lo_i = T < Tcr;
    if (lo_i != lo) {  // the iterate crossed the range boundary (rare)
      lo = lo_i;
      mix_poly(m, Yf, lo, P);
    }
    const double cp = poly5(P.cp, T), d2 = poly4(P.dcp, T), h = poly6(P.h, T);
    const double res = (h - R * T) - e;
    const double d1 = cp - R;
    if (fabs(res) > HALLEY_TOL) bits |= 1u << i;
    if (res != res) bits |= 1u << (8 + i);
    const double dT = ((-2.0 * res) * d1) / ((2.0 * (d1 * d1)) - res * d2);
    T = T + dT;
    cand[i + 1] = T;
  }
  return bits;
}
#endif

// Halley iterates in the variant's arithmetic (see halley_iterates).
__device__ __forceinline__ unsigned halley_any(const MP& m, double e, const double* Yf, double R, double T0,
                                               double* cand) {
#if JB_FAST
  if (m.tcr_uniform) return halley_iterates_fast(m, e, Yf, R, T0, cand);
#endif
  return halley_iterates(m, e, Yf, R, T0, cand);
}

// Number of Halley iterations the reference's global while-loop performs.
__device__ __forceinline__ int halley_count(unsigned word) {
  for (int i = 0; i < HALLEY_MAX; ++i) {
    bool any_gt = (word >> i) & 1u;
    bool any_nan = (word >> (8 + i)) & 1u;
    if (!any_gt || any_nan) return i;
  }
  return HALLEY_MAX;
}

// ---------------------------------------------------------------------------
// primitive recovery (solver_{1D,2D}/aux_func.py U_to_prim)
// ---------------------------------------------------------------------------
template <int DIM>
struct Prim {
  double rho, u, v, p, a, R;
};

template <int DIM>
__device__ __forceinline__ Prim<DIM> u_to_prim(const MP& m, const double* q, double gamma, double T) {
  Prim<DIM> r;
  constexpr int nY = DIM == 1 ? 3 : 4;
#if JB_FAST
  // one reciprocal; p = T sum_k (rho Y_k)/M_k with rho Y_N2 = rho - sum rho Y_k
  r.rho = q[0];
  const double ri = 1.0 / r.rho;
  r.u = q[1] * ri;
  r.v = DIM == 2 ? q[2] * ri : 0.0;
  double sr = q[nY], pr = m.invM[0] * q[nY];
#pragma unroll
  for (int k = 1; k < NR; ++k) { sr += q[nY + k]; pr += m.invM[k] * q[nY + k]; }
  pr += m.invM[NR] * (r.rho - sr);
  r.R = pr * ri;
  r.p = pr * T;
  r.a = sqrt(gamma * r.p * ri);
  return r;
#endif
  r.rho = q[0];
  r.u = q[1] / r.rho;
  r.v = DIM == 2 ? q[2] / r.rho : 0.0;
  double Y8[NR], Yf[NS];
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = q[nY + k] / r.rho;
  fill_Y(Y8, Yf);
  r.R = get_R(m, Yf);
  r.p = r.rho * r.R * T;
  r.a = sqrt(gamma * r.p / r.rho);
  return r;
}

#if JB_FAST
// Per-cell Halley solve of the fp64 and mixed variants.  The reference
// (thermo_model.py:135-153) iterates all cells until the largest residual is
// within tol, so every cell except the slowest ones takes at least one more
// step after its own residual is within tol, which polishes it to round-off.
// Here each cell iterates until its residual is within tol and then takes
// that one more step (at most HALLEY_MAX steps; a NaN residual stops at once,
// as it stops the reference's loop).  The result equals the global rule's to
// round-off except for the cells that set the global count, which differ by
// at most tol / cv (in SI units ~1e-12 K; in nondimensional units, where e is
// O(1), up to ~1e-9 relative).  Returns T and cp at the last evaluated
// temperature (get_T_nasa7 returns gamma there).
__device__ __forceinline__ bool halley_go(double res, bool& polished) {
  if (fabs(res) > HALLEY_TOL) return true;
  if (polished || res == 0.0 || res != res) return false;  // converged: one more step, none if exact or NaN
  polished = true;
  return true;
}

// Mixture enthalpy polynomial of one NASA7 range (the Y-weighted sum of the
// species' h coefficients).  cp = dh/dT and dcp/dT = d2h/dT2 in real
// arithmetic (the tables' cp and dcp are the same NASA7 coefficients times
// the powers), so the per-cell solve holds six coefficients and takes h, cp
// and dcp from one Horner pass with two derivatives.
template <bool LO>
__device__ __forceinline__ void mix_h_range(const MP& m, const double* Yf, double* H) {
  const auto& h = LO ? m.h_lo : m.h_hi;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double c = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) c += Yf[k] * h[k][j];
    H[j] = c;
  }
}

__device__ __forceinline__ void mix_h(const MP& m, const double* Yf, bool lo, double* H) {
  if (lo) mix_h_range<true>(m, Yf, H);
  else mix_h_range<false>(m, Yf, H);
}

// h(T), cp = h'(T) and dcp = h''(T) of a degree-5 polynomial in the tables' order
__device__ __forceinline__ void poly6_d2(const double* c, double T, double& h, double& cp, double& dcp) {
  double p = c[0], d1 = 0.0, d2 = 0.0;
#pragma unroll
  for (int j = 1; j < 6; ++j) {
    d2 = d2 * T + d1;
    d1 = d1 * T + p;
    p = p * T + c[j];
  }
  h = p;
  cp = d1;
  dcp = 2.0 * d2;
}

__device__ __forceinline__ double halley_cell(const MP& m, double e, const double* Yf, double R, double T0,
                                              double& cp_out) {
  double T = T0;
  bool polished = false;
  if (m.tcr_uniform) {
    const double Tcr = m.Tcr[0];
    bool lo = T < Tcr;
    double H[6], h, cp, d2;
    mix_h(m, Yf, lo, H);
    poly6_d2(H, T, h, cp, d2);
    double res = (h - R * T) - e;
#pragma unroll 1
    for (int i = 0; i < HALLEY_MAX && halley_go(res, polished); ++i) {
      const double d1 = cp - R;
      T = T + ((-2.0 * res) * d1) / ((2.0 * (d1 * d1)) - res * d2);
      const bool lo_i = T < Tcr;
      if (lo_i != lo) {  // the iterate crossed the range boundary (rare)
        lo = lo_i;
        mix_h(m, Yf, lo, H);
      }
      poly6_d2(H, T, h, cp, d2);
      res = (h - R * T) - e;
    }
    cp_out = cp;
    return T;
  }
  Th t = thermo_mix(m, T, Yf);
  double res = (t.h - R * T) - e;
#pragma unroll 1
  for (int i = 0; i < HALLEY_MAX && halley_go(res, polished); ++i) {
    const double d1 = t.cp - R;
    T = T + ((-2.0 * res) * d1) / ((2.0 * (d1 * d1)) - res * t.dcp);
    t = thermo_mix(m, T, Yf);
    res = (t.h - R * T) - e;
  }
  cp_out = t.cp;
  return T;
}
#endif

// The temperature solve of a new state q (nv float64 fields) at cell c with
// initial guess T0 (jb_fin.h).  The mode is fixed at compile time, as the
// host's step sequence chooses it: CELL (per-cell) in the mixed variant's 2D
// kernels, global stop otherwise (the fp64 and strict builds keep the
// reference's global stopping rule exactly).  Global-stop mode: the Halley iterates into
// fin.cand; returns the mask bits.  Per-cell mode: the converged (gamma, T)
// into fin.aux, the float32 u, v, p into fin.prims, and the new state's wave
// speeds and CFL candidate folded into amx, amy, dtm as the select pass does
// (LF.py nanmax(|u| + a), set_simulator.py:420-443); returns status bits
// << 16.
template <int DIM, bool CELL>
__device__ __forceinline__ unsigned finish_state(const MP& m, const Grid& g, const jb_fin& fin, const double* q,
                                                 double T0, long long c, double& amx, double& amy, double& dtm,
                                                 Slots* slots) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  const long long nc = g.ncell;
  const double rho = q[0];
#if JB_FAST
  if constexpr (CELL) {
    // one reciprocal of rho; the primitives of the wave speeds as u_to_prim
    // forms them (p = T sum_k (rho Y_k)/M_k, rho Y_N2 = rho - sum rho Y_k)
    // are taken before the solve so that the state is no longer needed
    const double ri = 1.0 / rho;
    const double u = q[1] * ri, v = DIM == 2 ? q[2] * ri : 0.0;
    const double e = DIM == 2 ? q[3] * ri - 0.5 * (u * u + v * v) : q[2] * ri - 0.5 * (u * u);
    double Y8[NR], Yf[NS];
    double sr = q[nY], prs = m.invM[0] * q[nY];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      Y8[k] = q[nY + k] * ri;
      if (k > 0) {
        sr += q[nY + k];
        prs += m.invM[k] * q[nY + k];
      }
    }
    prs += m.invM[NR] * (rho - sr);
    fill_Y(Y8, Yf);
    const double R = get_R(m, Yf);
    double cp;
    const double T = halley_cell(m, e, Yf, R, T0, cp);
    const double gamma = cp / (cp - R);
    fin.aux[c] = gamma;
    fin.aux[nc + c] = T;
    unsigned st = 0;
    if (fin.aidx >= 0 || fin.cfl || fin.prims) {
      const double p = prs * T;
      const double a = sqrt(gamma * p * ri);
      if (DIM == 2 && fin.prims) {
        fin.prims[c] = (float)u;
        fin.prims[nc + c] = (float)v;
        fin.prims[2 * nc + c] = (float)p;
      }
      const double sx = fabs(u) + a, sy = fabs(v) + a;
      amx = fmax(amx, sx);
      amy = fmax(amy, sy);
      if (!(sx == sx) || !(T == T)) st |= JB_ERR_NONFINITE;
      if (fin.cfl) {
        // the CFL candidate as the select pass forms it (1D: dx / (|u| + a))
        const double d = DIM == 1 ? g.dx / sx : 1.0 / (sx * g.idx + sy * g.idy);
        dtm = fmin(dtm, d);
        if (!(d == d) || !(d > 0.0)) st |= JB_ERR_NONFINITE;
        if (!(d == d)) atomicOr(&slots->dtnan, 1u);  // jnp.min propagates NaN
      }
    } else if (!(T == T)) {
      st |= JB_ERR_NONFINITE;
    }
    return st << 16;
  } else
#endif
  {
    (void)amx; (void)amy; (void)dtm; (void)slots;
    const double u = q[1] / rho, v = DIM == 2 ? q[2] / rho : 0.0;
    const double e = q[nY - 1] / rho - 0.5 * (u * u + v * v);
    double Y8[NR], Yf[NS];
#pragma unroll
    for (int k = 0; k < NR; ++k) Y8[k] = q[nY + k] / rho;
    fill_Y(Y8, Yf);
    const double R = get_R(m, Yf);
    double cnd[JB_NCAND];
    const unsigned bits = halley_any(m, e, Yf, R, T0, cnd);
#pragma unroll
    for (int i = 0; i < JB_NCAND; ++i) fin.cand[i * nc + c] = cnd[i];
    return bits;
  }
}

// Block-level end of finish_state (all threads of the block call it).
__device__ __forceinline__ void finish_reduce(const jb_fin& fin, double amx, double amy, double dtm,
                                              unsigned bits, Slots* slots) {
  const bool cell_mode = fin.aux != nullptr;
  block_reduce_store(amx, amy, dtm, bits, slots, fin.aidx < 0 ? 0 : fin.aidx, cell_mode && fin.aidx >= 0,
                     cell_mode && fin.cfl, cell_mode ? -1 : fin.midx);
}

// ---------------------------------------------------------------------------
// boundary ghost states that are not plain copies
// ---------------------------------------------------------------------------
// pressure_outlet (boundary_conditions_{1D,2D}/pressure_outlet.py:5-22);
// q is the boundary-adjacent cell, out receives U (nv), gamma, T.
template <int DIM>
__device__ void pressure_outlet_state(const MP& m, const double* q, double gamma, double T,
                                      double normal_vel, double Pb, double* out) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  constexpr int nv = nY + NR;
  double rho = q[0];
  double u = q[1] / rho;
  double v = DIM == 2 ? q[2] / rho : 0.0;
  double Y8[NR], Yf[NS];
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = q[nY + k] / rho;
  fill_Y(Y8, Yf);
  double R = get_R(m, Yf);
  double p = rho * (R * T);
  double a = sqrt(gamma * p / rho);
  bool sub = normal_vel / a < 1.0;
  double rho_c = sub ? Pb / (p / rho) : rho;
  double p_c = sub ? Pb * 1.0 : p;
  double T_c = sub ? p_c / (rho_c * R) : T;
  Th t = thermo_mix(m, T_c, Yf);
  double g_c = t.cp / (t.cp - R);
  out[0] = rho_c;
  out[1] = rho_c * u;
  if (DIM == 2) {
    out[2] = rho_c * v;
    out[3] = rho_c * t.h - p_c + 0.5 * rho_c * (u * u + v * v);
  } else {
    out[2] = rho_c * t.h - p_c + 0.5 * rho_c * (u * u);
  }
#pragma unroll
  for (int k = 0; k < NR; ++k) out[nY + k] = rho_c * Y8[k];
  out[nv] = g_c;
  out[nv + 1] = T_c;
}

// Rotating-detonation injector of examples/janc_basic_example2.ipynb
// (bottom_boundary + inj_model, after Fievisohn et al. 2017): bisection on
// the throat Mach number of a choked injector fed at nondimensional total
// pressure 1 and temperature 1; blocked (slip-like) when p_in >= 1.
__device__ void injector_state(const MP& m, const double* q, double gamma, double T,
                               const double* Yinj8, double block_p, double* out) {
  constexpr int nY = 4;
  constexpr int nv = nY + NR;
  double rho = q[0];
  double u = q[1] / rho;
  double v = q[2] / rho;
  double Y8[NR], Yf[NS];
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = q[nY + k] / rho;
  fill_Y(Y8, Yf);
  double R = get_R(m, Yf);
  double p = rho * R * T;
  // inj_model
  double Yi[NS];
  fill_Y(Yinj8, Yi);
  double Ri = get_R(m, Yi);
  const double gam = 1.29;
  const double A1 = 1.0, A3 = 5.0, A2 = 4.0;
  const double C0 = sqrt(gam * Ri * 1.0);
  const double gh = (gam - 1.0) / 2.0;
  const double e1 = -gam / (gam - 1.0);
  const double e2 = -(gam + 1.0) / 2.0 / (gam - 1.0);
  const double gg = gam / (gam - 1.0);
  const double P3 = p;
  double M1 = 0.0, M2 = 1.0, MFC = 0.0, V3 = 0.0;
  for (int it = 0; it < 20; ++it) {
    double M = 0.5 * (M1 + M2);
    double base = 1.0 + gh * (M * M);
    double P1 = 1.0 * pow(base, e1);
    double V1 = M * pow(base, -0.5) * C0;
    MFC = 1.0 * sqrt(gam / Ri) * M * pow(base, e2);
    double B = gg * P3 * A3 / MFC;
    double C = -gam / (gam - 1.0) * Ri * 1.0;
    V3 = (-B + sqrt(B * B - 2.0 * C)) / 1.0;
    double P2 = (MFC * (V3 - V1) - P1 * A1 + P3 * A3) / A2;
    M2 = (P2 >= P1) ? M : M2;
    M1 = (P2 < P1) ? M : M1;
  }
  double rho_i = MFC / V3 / A3;
  double T_i = P3 / (Ri * rho_i);
  Th ti = thermo_mix(m, T_i, Yi);
  double g_i = ti.cp / (ti.cp - Ri);
  double rho_inj = p / (Ri * T_i);
  // bottom_boundary selection
  bool blk = p >= block_p;
  double rho_c = blk ? rho : rho_inj;
  double u_c = blk ? u : 0.0;
  double v_c = blk ? -v : V3;
  double T_c = blk ? T : T_i;
  double h_c;
  if (blk) {
    Th t = thermo_mix(m, T, Yf);
    h_c = t.h;
  } else {
    h_c = ti.h;
  }
  double g_c = blk ? gamma : g_i;
  out[0] = rho_c;
  out[1] = rho_c * u_c;
  out[2] = rho_c * v_c;
  out[3] = rho_c * h_c - p + 0.5 * rho_c * (u_c * u_c + v_c * v_c);
#pragma unroll
  for (int k = 0; k < NR; ++k) out[nY + k] = rho_c * (blk ? Y8[k] : Yinj8[k]);
  out[nv] = g_c;
  out[nv + 1] = T_c;
}

// ---------------------------------------------------------------------------
// WENO5-JS (solver_{1D,2D}/reconstruction/WENO5_JS.py), reference order
// ---------------------------------------------------------------------------
constexpr double W_EPS = 1e-6;
constexpr double W_C1 = 1.0 / 10.0, W_C2 = 3.0 / 5.0, W_C3 = 3.0 / 10.0;
constexpr double W_Q = 1.0 / 4.0, W_D = 13.0 / 12.0;
constexpr double W_13 = 1.0 / 3.0, W_76 = 7.0 / 6.0, W_116 = 11.0 / 6.0;
constexpr double W_m16 = -1.0 / 6.0, W_56 = 5.0 / 6.0, W_16 = 1.0 / 6.0;

#if JB_FAST
// Same weights with one division: alpha_k = C_k / d_k^2 is scaled by
// d_1^2 d_2^2 d_3^2, so w_k = C_k prod_{j!=k} d_j^2 / sum.  (The float64
// range covers the squared products of the smoothness indicators met here.)
__device__ __forceinline__ double weno_combine(double IS1, double IS2, double IS3, double q1, double q2,
                                               double q3) {
  const double e1 = W_EPS + IS1, e2 = W_EPS + IS2, e3 = W_EPS + IS3;
  const double s1 = e1 * e1, s2 = e2 * e2, s3 = e3 * e3;
  const double a1 = W_C1 * (s2 * s3), a2 = W_C2 * (s1 * s3), a3 = W_C3 * (s1 * s2);
  return (a1 * q1 + a2 * q2 + a3 * q3) / (a1 + a2 + a3);
}

__device__ __forceinline__ double weno_L(double fjm2, double fjm1, double fj, double fjp1, double fjp2) {
  double t1 = fjm2 - 4.0 * fjm1 + 3.0 * fj, s1 = fjm2 - 2.0 * fjm1 + fj;
  double t2 = fjm1 - fjp1, s2 = fjm1 - 2.0 * fj + fjp1;
  double t3 = 3.0 * fj - 4.0 * fjp1 + fjp2, s3 = fj - 2.0 * fjp1 + fjp2;
  double IS1 = W_Q * (t1 * t1) + W_D * (s1 * s1);
  double IS2 = W_Q * (t2 * t2) + W_D * (s2 * s2);
  double IS3 = W_Q * (t3 * t3) + W_D * (s3 * s3);
  double q1 = W_13 * fjm2 - W_76 * fjm1 + W_116 * fj;
  double q2 = W_m16 * fjm1 + W_56 * fj + W_13 * fjp1;
  double q3 = W_13 * fj + W_56 * fjp1 - W_16 * fjp2;
  return weno_combine(IS1, IS2, IS3, q1, q2, q3);
}

__device__ __forceinline__ double weno_R(double fjm2, double fjm1, double fj, double fjp1, double fjp2) {
  double t1 = fjp2 - 4.0 * fjp1 + 3.0 * fj, s1 = fjp2 - 2.0 * fjp1 + fj;
  double t2 = fjp1 - fjm1, s2 = fjp1 - 2.0 * fj + fjm1;
  double t3 = 3.0 * fj - 4.0 * fjm1 + fjm2, s3 = fj - 2.0 * fjm1 + fjm2;
  double IS1 = W_Q * (t1 * t1) + W_D * (s1 * s1);
  double IS2 = W_Q * (t2 * t2) + W_D * (s2 * s2);
  double IS3 = W_Q * (t3 * t3) + W_D * (s3 * s3);
  double q1 = W_13 * fjp2 - W_76 * fjp1 + W_116 * fj;
  double q2 = W_m16 * fjp1 + W_56 * fj + W_13 * fjm1;
  double q3 = W_13 * fj + W_56 * fjm1 - W_16 * fjm2;
  return weno_combine(IS1, IS2, IS3, q1, q2, q3);
}
#else
// left-biased value at j+1/2 from cells j-2..j+2 (interface_L_*)
__device__ __forceinline__ double weno_L(double fjm2, double fjm1, double fj, double fjp1, double fjp2) {
  double t1 = fjm2 - 4.0 * fjm1 + 3.0 * fj, s1 = fjm2 - 2.0 * fjm1 + fj;
  double t2 = fjm1 - fjp1, s2 = fjm1 - 2.0 * fj + fjp1;
  double t3 = 3.0 * fj - 4.0 * fjp1 + fjp2, s3 = fj - 2.0 * fjp1 + fjp2;
  double IS1 = W_Q * (t1 * t1) + W_D * (s1 * s1);
  double IS2 = W_Q * (t2 * t2) + W_D * (s2 * s2);
  double IS3 = W_Q * (t3 * t3) + W_D * (s3 * s3);
  double e1 = W_EPS + IS1, e2 = W_EPS + IS2, e3 = W_EPS + IS3;
  double a1 = W_C1 / (e1 * e1), a2 = W_C2 / (e2 * e2), a3 = W_C3 / (e3 * e3);
  double w1 = a1 / (a1 + a2 + a3), w2 = a2 / (a1 + a2 + a3), w3 = a3 / (a1 + a2 + a3);
  double q1 = W_13 * fjm2 - W_76 * fjm1 + W_116 * fj;
  double q2 = W_m16 * fjm1 + W_56 * fj + W_13 * fjp1;
  double q3 = W_13 * fj + W_56 * fjp1 - W_16 * fjp2;
  return w1 * q1 + w2 * q2 + w3 * q3;
}

// right-biased value at j-1/2 from cells j-2..j+2 (interface_R_*)
__device__ __forceinline__ double weno_R(double fjm2, double fjm1, double fj, double fjp1, double fjp2) {
  double t1 = fjp2 - 4.0 * fjp1 + 3.0 * fj, s1 = fjp2 - 2.0 * fjp1 + fj;
  double t2 = fjp1 - fjm1, s2 = fjp1 - 2.0 * fj + fjm1;
  double t3 = 3.0 * fj - 4.0 * fjm1 + fjm2, s3 = fj - 2.0 * fjm1 + fjm2;
  double IS1 = W_Q * (t1 * t1) + W_D * (s1 * s1);
  double IS2 = W_Q * (t2 * t2) + W_D * (s2 * s2);
  double IS3 = W_Q * (t3 * t3) + W_D * (s3 * s3);
  double e1 = W_EPS + IS1, e2 = W_EPS + IS2, e3 = W_EPS + IS3;
  double a1 = W_C1 / (e1 * e1), a2 = W_C2 / (e2 * e2), a3 = W_C3 / (e3 * e3);
  double w1 = a1 / (a1 + a2 + a3), w2 = a2 / (a1 + a2 + a3), w3 = a3 / (a1 + a2 + a3);
  double q1 = W_13 * fjp2 - W_76 * fjp1 + W_116 * fj;
  double q2 = W_m16 * fjp1 + W_56 * fj + W_13 * fjm1;
  double q3 = W_13 * fj + W_56 * fjm1 - W_16 * fjm2;
  return w1 * q1 + w2 * q2 + w3 * q3;
}
#endif

// ---------------------------------------------------------------------------
// ghost-cell source mapping (boundary/boundary.py:120-132,
// boundary/boundary_padding.py:4-45, boundary_conditions_{1D,2D}/*.py)
// ---------------------------------------------------------------------------
// kind: 0 interior copy of (xs, ys) with sign flips, 1 strip value, 2 unused
// kind 1 reads a ghost strip (layer < 0: one state per boundary position,
// shared by the 3 ghost layers) or, on a JB_BC_HALO side, the neighbour's
// column `layer` (0..2, outward order of the padded array) in g.halo.
struct Src {
  int kind, xs, ys, side, pos, flip, layer;
};

// One axis: coordinate c on an axis of length n, lo/hi side kinds.
__device__ __forceinline__ bool map_axis(int c, int n, int kind, bool lo, int& cs, int& flip,
                                         bool& strip, int normal_field, int dim) {
  strip = false;
  flip = 0;
  switch (kind) {
    case JB_BC_PERIODIC:  // node-periodic quirk: ghosts are n-4..n-2 and 1..3
      cs = lo ? n - 1 + c : c - n + 1;
      return true;
    case JB_BC_SLIP_WALL:
      cs = lo ? 0 : n - 1;
      flip = 1 << normal_field;
      return true;
    case JB_BC_ZERO_GRADIENT:
      cs = lo ? -1 - c : 2 * n - 1 - c;
      return true;
    case JB_BC_NO_SLIP_WALL:
      cs = lo ? -1 - c : 2 * n - 1 - c;
      flip = dim == 2 ? 6 : 2;
      return true;
    default:
      strip = true;
      return true;
  }
}

template <int DIM>
__device__ __forceinline__ Src map_cell(const Grid& g, int x, int y) {
  Src s;
  s.kind = 2; s.xs = 0; s.ys = 0; s.side = 0; s.pos = 0; s.flip = 0; s.layer = -1;
  bool xin = x >= 0 && x < g.nx;
  bool yin = DIM == 1 ? true : (y >= 0 && y < g.ny);
  if (xin && yin) {
    s.kind = 0; s.xs = x; s.ys = y;
    return s;
  }
  if (!xin && yin) {
    if (x < -3 || x >= g.nx + 3) return s;
    bool lo = x < 0;
    int side = lo ? 0 : 1;
    int cs, flip;
    bool strip;
    map_axis(x, g.nx, g.bc[side], lo, cs, flip, strip, 1, DIM);
    if (strip) {
      s.kind = 1; s.side = side; s.pos = y;
      if (g.bc[side] == JB_BC_HALO) s.layer = lo ? x + 3 : x - g.nx;
      return s;
    }
    s.kind = 0; s.xs = cs; s.ys = y; s.flip = flip;
    return s;
  }
  if (DIM == 2 && xin && !yin) {
    if (y < -3 || y >= g.ny + 3) return s;
    bool lo = y < 0;
    int side = lo ? 2 : 3;
    int cs, flip;
    bool strip;
    map_axis(y, g.ny, g.bc[side], lo, cs, flip, strip, 2, DIM);
    if (strip) {
      s.kind = 1; s.side = side; s.pos = x;
      if (g.bc[side] == JB_BC_HALO) s.layer = lo ? y + 3 : y - g.ny;
      return s;
    }
    s.kind = 0; s.xs = x; s.ys = cs; s.flip = flip;
    return s;
  }
  return s;  // corner: never read by a stencil
}

__device__ __forceinline__ size_t strip_idx(const Grid& g, int side, int q, int pos) {
  return ((size_t)side * (g.nv + 2) + q) * g.lstrip + pos;
}

// halo[2][nv+2][3][ny]: x side, field (U..., gamma, T), ghost layer, row
__device__ __forceinline__ size_t halo_idx(const Grid& g, int side, int layer, int q, int y) {
  return (((size_t)side * (g.nv + 2) + q) * 3 + layer) * g.ny + y;
}

// haloy[2][nv+2][nx][3]: y side - 2, field, column, ghost layer
__device__ __forceinline__ size_t haloy_idx(const Grid& g, int side, int layer, int q, int x) {
  return (((size_t)(side - 2) * (g.nv + 2) + q) * g.nx + x) * 3 + layer;
}

// Field q (U..., gamma at nv, T at nv + 1) of a kind-1 ghost.
__device__ __forceinline__ double ghost(const Grid& g, const double* strips, const Src& s, int q) {
  if (s.layer < 0) return strips[strip_idx(g, s.side, q, s.pos)];
  return s.side < 2 ? g.halo[halo_idx(g, s.side, s.layer, q, s.pos)] : g.haloy[haloy_idx(g, s.side, s.layer, q, s.pos)];
}

// LF split flux F(f) of one cell in direction dir (0: x, 1: y) as the
// reference assembles it (flux_splitting/LF.py); Y = U_f / rho for species.
template <int DIM>
__device__ __forceinline__ double lf_flux(int f, int dir, double q, double rho, double u, double v,
                                          double p, double E) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  double vn = dir == 0 ? u : v;
  if (f == 0) return rho * vn;
  if (DIM == 1) {
    if (f == 1) return rho * (u * u) + p;
    if (f == 2) return u * (E + p);
  } else {
    if (f == 1) return dir == 0 ? rho * (u * u) + p : rho * u * v;
    if (f == 2) return dir == 0 ? rho * u * v : rho * (v * v) + p;
    if (f == 3) return vn * (E + p);
  }
  (void)nY;
#if JB_FAST
  return vn * q;
#else
  return rho * vn * (q / rho);
#endif
}

// Steger-Warming split fluxes of field f in direction dir (0: x, 1: y)
// (flux_splitting/SW.py): H+- = sum over the eigenvalue groups theta - a,
// theta, theta + a of lambda+- H_k, lambda+- = (lambda +- sqrt(lambda^2 +
// eps^2)) / 2 with eps = 1e-6, H_1,4 = (rho, rho u -+ rho a n, E + p -+ rho a
// theta, rho Y) / (2 gamma), H_2 = (gamma - 1) / gamma (rho, rho u,
// rho |u|^2 / 2, rho Y); expressions in the reference's order.
template <int DIM, class R>
__device__ __forceinline__ void sw_split(int f, int dir, R qf, R rho, R u, R v, R p, R E, R a, R gamma,
                                         R& hp, R& hm) {
  constexpr int nE = DIM == 1 ? 2 : 3;
  const R theta = dir == 0 ? u : v;
  const R ra = rho * a;
  R x1, x2, x4;
  if (f == 0) {
    x1 = x2 = x4 = rho;
  } else if (f == 1 || (DIM == 2 && f == 2)) {
    const R m = f == 1 ? rho * u : rho * v;
    const bool normal = (f == 1) == (dir == 0);
    x1 = normal ? m - ra : m;
    x2 = m;
    x4 = normal ? m + ra : m;
  } else if (f == nE) {
    x1 = (E + p) - ra * theta;
    x2 = DIM == 1 ? (R)0.5 * rho * (u * u) : (R)0.5 * rho * (u * u + v * v);
    x4 = (E + p) + ra * theta;
  } else {
#if JB_FAST
    x1 = x2 = x4 = qf;
#else
    x1 = x2 = x4 = rho * (qf / rho);
#endif
  }
  const R c1 = (R)1 / ((R)2 * gamma), c2 = (gamma - (R)1) / gamma;
  const R h1 = c1 * x1, h2 = c2 * x2, h4 = c1 * x4;
  const R l1 = theta - a, l2 = theta, l4 = theta + a;
  const R e2 = (R)(1e-6 * 1e-6);
  const R s1 = sqrt(l1 * l1 + e2), s2 = sqrt(l2 * l2 + e2), s4 = sqrt(l4 * l4 + e2);
  const R lp1 = (R)0.5 * (l1 + s1), lp2 = (R)0.5 * (l2 + s2), lp4 = (R)0.5 * (l4 + s4);
  const R lm1 = (R)0.5 * (l1 - s1), lm2 = (R)0.5 * (l2 - s2), lm4 = (R)0.5 * (l4 - s4);
  hp = lp1 * h1 + lp2 * h2 + lp4 * h4;
  hm = lm1 * h1 + lm2 * h2 + lm4 * h4;
}

#if JB_FAST
// ---------------------------------------------------------------------------
// float32 flux arithmetic of the mixed-precision variant
// ---------------------------------------------------------------------------
// The reference's epsilon is absolute (1e-6) while SI flux magnitudes reach
// ~1e11, so (eps + IS)^2 overflows float32.  The weights are formed as ratios
// to the smallest (eps + IS_k), alpha_k ~ C_k (min/(eps + IS_k))^2, which is
// the same normalised weight in real arithmetic and cannot overflow.
// One approximate reciprocal (MUFU.RCP, ~1 ulp).  The WENO weights' operands
// are at least eps (smoothness sums eps + IS) or the smallest linear weight
// (weight sums, where one ratio is 1), never denormal or huge, so no range
// fix-up is needed around it.
__device__ __forceinline__ float rcp_fast(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ float weno_combine32(float IS1, float IS2, float IS3, float q1, float q2,
                                                float q3, float eps) {
  const float e1 = eps + IS1, e2 = eps + IS2, e3 = eps + IS3;
  const float mn = fminf(e1, fminf(e2, e3));
  const float r1 = mn * rcp_fast(e1), r2 = mn * rcp_fast(e2), r3 = mn * rcp_fast(e3);
  const float a1 = 0.1f * (r1 * r1), a2 = 0.6f * (r2 * r2), a3 = 0.3f * (r3 * r3);
  return (a1 * q1 + a2 * q2 + a3 * q3) * rcp_fast(a1 + a2 + a3);
}

// Left/right-biased float32 values.  The ratio form of the weights never
// squares (eps + IS), so only IS itself must stay in range: |f| below ~1e18
// (SI fluxes stay below ~1e12).  Tiny fields give IS << eps and the linear
// weights, as the reference's absolute eps does.
__device__ __forceinline__ float weno_L(float fjm2, float fjm1, float fj, float fjp1, float fjp2) {
  const float t1 = fjm2 - 4.f * fjm1 + 3.f * fj, s1 = fjm2 - 2.f * fjm1 + fj;
  const float t2 = fjm1 - fjp1, s2 = fjm1 - 2.f * fj + fjp1;
  const float t3 = 3.f * fj - 4.f * fjp1 + fjp2, s3 = fj - 2.f * fjp1 + fjp2;
  const float IS1 = 0.25f * (t1 * t1) + (13.f / 12.f) * (s1 * s1);
  const float IS2 = 0.25f * (t2 * t2) + (13.f / 12.f) * (s2 * s2);
  const float IS3 = 0.25f * (t3 * t3) + (13.f / 12.f) * (s3 * s3);
  const float q1 = (1.f / 3.f) * fjm2 - (7.f / 6.f) * fjm1 + (11.f / 6.f) * fj;
  const float q2 = (-1.f / 6.f) * fjm1 + (5.f / 6.f) * fj + (1.f / 3.f) * fjp1;
  const float q3 = (1.f / 3.f) * fj + (5.f / 6.f) * fjp1 - (1.f / 6.f) * fjp2;
  return weno_combine32(IS1, IS2, IS3, q1, q2, q3, 1e-6f);
}

__device__ __forceinline__ float weno_R(float fjm2, float fjm1, float fj, float fjp1, float fjp2) {
  const float t1 = fjp2 - 4.f * fjp1 + 3.f * fj, s1 = fjp2 - 2.f * fjp1 + fj;
  const float t2 = fjp1 - fjm1, s2 = fjp1 - 2.f * fj + fjm1;
  const float t3 = 3.f * fj - 4.f * fjm1 + fjm2, s3 = fj - 2.f * fjm1 + fjm2;
  const float IS1 = 0.25f * (t1 * t1) + (13.f / 12.f) * (s1 * s1);
  const float IS2 = 0.25f * (t2 * t2) + (13.f / 12.f) * (s2 * s2);
  const float IS3 = 0.25f * (t3 * t3) + (13.f / 12.f) * (s3 * s3);
  const float q1 = (1.f / 3.f) * fjp2 - (7.f / 6.f) * fjp1 + (11.f / 6.f) * fj;
  const float q2 = (-1.f / 6.f) * fjp1 + (5.f / 6.f) * fj + (1.f / 3.f) * fjm1;
  const float q3 = (1.f / 3.f) * fj + (5.f / 6.f) * fjm1 - (1.f / 6.f) * fjm2;
  return weno_combine32(IS1, IS2, IS3, q1, q2, q3, 1e-6f);
}

template <int DIM>
__device__ __forceinline__ float lf_flux(int f, int dir, float q, float rho, float u, float v, float p,
                                         float E) {
  const float vn = dir == 0 ? u : v;
  if (f == 0) return rho * vn;
  if (DIM == 1) {
    if (f == 1) return rho * (u * u) + p;
    if (f == 2) return u * (E + p);
  } else {
    if (f == 1) return dir == 0 ? rho * (u * u) + p : rho * u * v;
    if (f == 2) return dir == 0 ? rho * u * v : rho * (v * v) + p;
    if (f == 3) return vn * (E + p);
  }
  return vn * q;
}
#endif

// jnp.minimum / jnp.maximum: a NaN operand gives NaN (fmin / fmax drop it)
__device__ __forceinline__ double nan_min(double a, double b) { return (a != a || b != b) ? a + b : fmin(a, b); }
__device__ __forceinline__ double nan_max(double a, double b) { return (a != a || b != b) ? a + b : fmax(a, b); }
__device__ __forceinline__ float nan_min(float a, float b) { return (a != a || b != b) ? a + b : fminf(a, b); }
__device__ __forceinline__ float nan_max(float a, float b) { return (a != a || b != b) ? a + b : fmaxf(a, b); }

// jnp.sign: -1, 0 (signed zero kept), +1, NaN
template <class R>
__device__ __forceinline__ R sign_ref(R x) { return x > R(0) ? R(1) : (x < R(0) ? R(-1) : x); }

// MUSCL (reconstruction/MUSCL.py): min_mod_limiter, kappa = 1/3, beta = 1.
// Arguments as the WENO forms take them (cells j-2 .. j+2); MUSCL reads the
// middle three.  Left: q_j + s_L; right: q_j - s_R.
template <class R>
__device__ __forceinline__ R minmod_ref(R x, R y) {
  const R m1 = nan_min(x * sign_ref(y), y * sign_ref(x));
  return sign_ref(x) * nan_max(R(0), m1);
}
template <class R>
__device__ __forceinline__ R muscl_L(R, R fjm1, R fj, R fjp1, R) {
  const R dm = fj - fjm1, dp = fjp1 - fj;
  const R fw = minmod_ref(dp, R(1) * dm), bw = minmod_ref(dm, R(1) * dp);
  return fj + R(0.25) * (R(1.0 - 1.0 / 3.0) * bw + R(1.0 + 1.0 / 3.0) * fw);
}
template <class R>
__device__ __forceinline__ R muscl_R(R, R fjm1, R fj, R fjp1, R) {
  const R dm = fj - fjm1, dp = fjp1 - fj;
  const R fw = minmod_ref(dp, R(1) * dm), bw = minmod_ref(dm, R(1) * dp);
  return fj - R(0.25) * (R(1.0 - 1.0 / 3.0) * fw + R(1.0 + 1.0 / 3.0) * bw);
}

// the grid's face reconstruction (a warp-uniform choice)
template <class R>
__device__ __forceinline__ R recon_L(const Grid& g, R a, R b, R c, R d, R e) {
  return g.recon == JB_RECON_MUSCL ? muscl_L(a, b, c, d, e) : weno_L(a, b, c, d, e);
}
template <class R>
__device__ __forceinline__ R recon_R(const Grid& g, R a, R b, R c, R d, R e) {
  return g.recon == JB_RECON_MUSCL ? muscl_R(a, b, c, d, e) : weno_R(a, b, c, d, e);
}

// rho, u, v, p of one cell for the flux (U_to_prim; the flux needs no gamma)
template <int DIM>
__device__ __forceinline__ void flux_prims(const MP& m, const double* q, double T, double& rho,
                                           double& u, double& v, double& p) {
  Prim<DIM> pr = u_to_prim<DIM>(m, q, 1.0, T);
  rho = pr.rho;
  u = pr.u;
  v = pr.v;
  p = pr.p;
}

#if JB_FAST
template <int DIM>
__device__ __forceinline__ void flux_prims(const MP& m, const float* q, float T, float& rho, float& u,
                                           float& v, float& p) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  rho = q[0];
  const float ri = __fdividef(1.f, rho);
  u = q[1] * ri;
  v = DIM == 2 ? q[2] * ri : 0.f;
  float sr = q[nY], pr = (float)m.invM[0] * q[nY];
#pragma unroll
  for (int k = 1; k < NR; ++k) {
    sr += q[nY + k];
    pr += (float)m.invM[k] * q[nY + k];
  }
  pr += (float)m.invM[NR] * (rho - sr);
  p = pr * T;
}
#endif

// ---------------------------------------------------------------------------
// stage kernels
// ---------------------------------------------------------------------------
// STAGE 0: flux_func only, out = dt * total_flux(BC(U, aux))
//           (simulation/set_simulator.py:26-29, 44-47)
// STAGE 1..3: SSP-RK3 stage (simulation/time_step/TVD_RK3.py:5-12)
//           out = a U^n + b (U_k + dt L(U_k)), followed by the Halley
//           iterates of update_aux (solver_{1D,2D}/aux_func.py:21-29)
constexpr int TX2 = 15, TY2 = 16, PX2 = TX2 + 6, PY2 = TY2 + 6;
constexpr int NT2 = 256;
constexpr int SM2_Q = PX2 * PY2;                  // padded cells of a tile
constexpr int SM2_HX = PX2 * TY2, SM2_HY = TX2 * PY2;
constexpr int SM2_FX = (TX2 + 1) * TY2, SM2_FY = TX2 * (TY2 + 1);
// Shared-memory layout of the padded tile fields: rows of PYS = 24 cells
// holding padded cells y0 - 4 .. y0 + 19 (the tile's y0 - 3 .. y0 + 18 at
// offsets 1..22), so that a TMA box can start at the even column y0 - 4
// (16-byte aligned for float64) and fill a field as one dense box.
constexpr int PYS = 24, SM2_QF = PX2 * PYS;       // field stride
__host__ __device__ constexpr int tile_ci(int px, int py) { return px * PYS + py + 1; }
// fields of the staged tile: the 12 conserved fields, gamma, T
constexpr int TQ_G = 12, TQ_T = 13, TQ_N = 14;

template <class R>
__host__ __device__ constexpr size_t sw_smem2d_bytes() {
  return sizeof(R) * SM2_QF;  // the sound speed a
}

template <class R>
__host__ __device__ constexpr size_t smem2d_bytes(int) {
  return sizeof(R) * ((size_t)TQ_N * SM2_QF + 4 * SM2_QF + 2 * SM2_HX + 2 * SM2_HY + SM2_FX + SM2_FY);
}

// ---- TMA: bulk tensor loads into shared memory completing on an mbarrier
// (no cluster multicast; the tensor maps cover this GPU's own buffers)
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
// Bounded wait on a TMA mbarrier (phase 0): false after ~1 s of clock cycles.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, 0))
    if (clock64() - t0 > 2000000000LL) return false;
  return true;
}

// R is the arithmetic type of the flux (LF split, WENO, primitives): double
// for the float64 variants, float for the mixed variant.  The RK combination
// and the Halley iterates are float64 in every variant.
template <int STAGE, class R, bool VISC, bool SW = false>
__global__ void __launch_bounds__(NT2, sizeof(R) == 4 ? 3 : 2) k_flux2d(MP m, Grid g, const double* __restrict__ Uk,
                                                 const double* __restrict__ auxk,
                                                 const double* __restrict__ Un,
                                                 double* __restrict__ out,
                                                 const double* __restrict__ strips, Slots* slots,
                                                 int aidx, jb_fin fin, double dt_arg,
                                                 const __grid_constant__ CUtensorMap tmU,
                                                 const __grid_constant__ CUtensorMap tmA, int use_tma) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ __align__(8) unsigned long long tma_bar;
  constexpr int nv = 12;
  constexpr bool EXACT = sizeof(R) == sizeof(double);
  R* sQ = reinterpret_cast<R*>(smraw);   // [TQ_N][PX2][PYS]: U, gamma, T
  R* sP = sQ + (size_t)TQ_N * SM2_QF;    // [4][PX2][PYS]: rho, u, v, p
  R* sHxp = sP + 4 * SM2_QF;             // [PX2][TY2]
  R* sHxm = sHxp + SM2_HX;
  R* sHyp = sHxm + SM2_HX;               // [TX2][PY2]
  R* sHym = sHyp + SM2_HY;
  R* sFx = sHym + SM2_HY;                // [TX2+1][TY2]
  R* sFy = sFx + SM2_FX;                 // [TX2][TY2+1]
  R* sG = sQ + TQ_G * SM2_QF;            // gamma
  // Steger-Warming only (launched with sw_smem2d more bytes): the sound speed
  R* sA = sFy + SM2_FY;                  // [PX2][PYS]
  constexpr bool sw = SW;

  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * TX2, y0 = blockIdx.y * TY2;
  const long long nc = g.ncell;
  const double dt = STAGE == 0 ? dt_arg : slots->dt;
  const R ax = (R)bitsd(slots->ax[aidx]);
  const R ay = (R)bitsd(slots->ay[aidx]);

  // ---- load the padded tile with ghost cells.  float64 tiles: two TMA boxes
  // (the 12 conserved fields, and gamma / T) over padded rows x0-3 .. x0+17
  // and columns y0-4 .. y0+19 in one transaction; the cells outside the
  // domain (filled with zeros by the copy) are then replaced by their ghost
  // values.  Without TMA every padded cell is loaded here.
  const bool tma = EXACT && use_tma;
  if (tma) {
    if (tid == 0) mbar_init(&tma_bar, 1);
    __syncthreads();
    if (tid == 0) {
      mbar_expect_tx(&tma_bar, (unsigned)(sizeof(double) * (TQ_N * SM2_QF)));
      tma_load_3d(sQ, &tmU, y0 - 4, x0 - 3, 0, &tma_bar);
      tma_load_3d(sQ + TQ_G * SM2_QF, &tmA, y0 - 4, x0 - 3, 0, &tma_bar);
    }
    if (!mbar_wait_bounded(&tma_bar)) {
      if (tid == 0) atomicOr(&slots->status, (unsigned)JB_ERR_TIMEOUT);
      mbar_wait_bounded(&tma_bar);  // the copy must not land after the block has left
      return;
    }
  }
  for (int i = tid; i < SM2_Q; i += NT2) {
    const int px = i / PY2, py = i % PY2;
    const int x = x0 + px - 3, y = y0 + py - 3;
    if (tma && x >= 0 && x < g.nx && y >= 0 && y < g.ny) continue;
    const int k = tile_ci(px, py);
    Src s = map_cell<2>(g, x, y);
    if (s.kind == 0) {
      size_t c = (size_t)s.xs * g.ny + s.ys;
      for (int q = 0; q < nv; ++q) {
        double v = Uk[q * nc + c];
        sQ[q * SM2_QF + k] = (R)(((s.flip >> q) & 1) ? -v : v);
      }
      sQ[TQ_T * SM2_QF + k] = (R)auxk[nc + c];
      sG[k] = (R)auxk[c];
    } else if (s.kind == 1) {
      for (int q = 0; q < nv; ++q) sQ[q * SM2_QF + k] = (R)ghost(g, strips, s, q);
      sQ[TQ_T * SM2_QF + k] = (R)ghost(g, strips, s, nv + 1);
      sG[k] = (R)ghost(g, strips, s, nv);
    } else {
      for (int q = 0; q < TQ_N; ++q) sQ[q * SM2_QF + k] = (R)1.0;
    }
  }
  __syncthreads();
  // ---- primitives (aux_func.U_to_prim) on every padded cell
  for (int i = tid; i < SM2_Q; i += NT2) {
    const int k = tile_ci(i / PY2, i % PY2);
    R q[nv];
#pragma unroll
    for (int f = 0; f < nv; ++f) q[f] = sQ[f * SM2_QF + k];
    R rho, u, v, p;
    flux_prims<2>(m, q, sQ[TQ_T * SM2_QF + k], rho, u, v, p);
    sP[k] = rho;
    sP[SM2_QF + k] = u;
    sP[2 * SM2_QF + k] = v;
    sP[3 * SM2_QF + k] = p;
    if (sw) sA[k] = sqrt(sG[k] * p / rho);
  }
  __syncthreads();

  const bool owner = tid < TX2 * TY2;
  const int ix = owner ? tid / TY2 : 0, iy = owner ? tid % TY2 : 0;
  const int gx = x0 + ix, gy = y0 + iy;
  const bool live = owner && gx < g.nx && gy < g.ny;
  const size_t cell = (size_t)gx * g.ny + gy;

#if JB_FAST
  // H-phase work items of this thread (<= 3 of the 666), fixed for all fields
  constexpr int NH2 = (SM2_HX + SM2_HY + NT2 - 1) / NT2;
  int h_src[NH2], h_dst[NH2];
#pragma unroll
  for (int r = 0; r < NH2; ++r) {
    const int i = tid + r * NT2;
    int px = 0, py = 0, dst = -1;
    if (i < SM2_HX) { px = i / TY2; py = i % TY2 + 3; dst = i; }
    else if (i < SM2_HX + SM2_HY) { int j = i - SM2_HX; px = j / PY2 + 3; py = j % PY2; dst = i; }
    h_src[r] = tile_ci(px, py);
    h_dst[r] = dst;
  }
#endif
  for (int f = 0; f < nv; ++f) {
    // ---- split fluxes H+/- = 0.5 (F +/- alpha U)
#if JB_FAST
    // F = vel q + pressure terms (x: p in rho u, u p in rho E; y: p in rho v,
    // v p in rho E), the reference's LF flux regrouped
#pragma unroll
    for (int r = 0; r < NH2; ++r) {
      const int dst = h_dst[r];
      if (dst < 0) continue;
      const int c = h_src[r];
      const bool xdir = dst < SM2_HX;
      const R vel = xdir ? sP[SM2_QF + c] : sP[2 * SM2_QF + c];
      const R qf = sQ[f * SM2_QF + c];
      R F = vel * qf;
      if (f == (xdir ? 1 : 2)) F += sP[3 * SM2_QF + c];
      if (f == 3) F += vel * sP[3 * SM2_QF + c];
      const R al = xdir ? ax : ay;
      R hp = (R)0.5 * (F + al * qf), hm = (R)0.5 * (F - al * qf);
      if (sw)
        sw_split<2, R>(f, xdir ? 0 : 1, qf, sP[c], sP[SM2_QF + c], sP[2 * SM2_QF + c], sP[3 * SM2_QF + c],
                       sQ[3 * SM2_QF + c], sA[c], sG[c], hp, hm);
      if (xdir) { sHxp[dst] = hp; sHxm[dst] = hm; }
      else { sHyp[dst - SM2_HX] = hp; sHym[dst - SM2_HX] = hm; }
    }
#else
    for (int i = tid; i < SM2_HX + SM2_HY; i += NT2) {
      int px, py, dir;
      if (i < SM2_HX) { px = i / TY2; py = i % TY2 + 3; dir = 0; }
      else { int j = i - SM2_HX; px = j / PY2 + 3; py = j % PY2; dir = 1; }
      int c = tile_ci(px, py);
      R rho = sP[c], u = sP[SM2_QF + c], v = sP[2 * SM2_QF + c], p = sP[3 * SM2_QF + c];
      R E = sQ[3 * SM2_QF + c];
      R qf = sQ[f * SM2_QF + c];
      R hp, hm;
      if (sw) {
        sw_split<2, R>(f, dir, qf, rho, u, v, p, E, sA[c], sG[c], hp, hm);
      } else {
        R F = lf_flux<2>(f, dir, qf, rho, u, v, p, E);
        R al = dir == 0 ? ax : ay;
        hp = (R)0.5 * (F + al * qf);
        hm = (R)0.5 * (F - al * qf);
      }
      if (dir == 0) { sHxp[px * TY2 + (py - 3)] = hp; sHxm[px * TY2 + (py - 3)] = hm; }
      else { sHyp[(px - 3) * PY2 + py] = hp; sHym[(px - 3) * PY2 + py] = hm; }
    }
#endif
    __syncthreads();
    // ---- face values: F = L(H+) + R(H-)
    {
      int mxf = tid / TY2, jy = tid % TY2;  // x-faces: 16 x 16 = 256
      const R* hp = sHxp + jy;
      const R* hm = sHxm + jy;
      R L = recon_L(g, hp[(mxf) * TY2], hp[(mxf + 1) * TY2], hp[(mxf + 2) * TY2], hp[(mxf + 3) * TY2],
                        hp[(mxf + 4) * TY2]);
      R Rr = recon_R(g, hm[(mxf + 1) * TY2], hm[(mxf + 2) * TY2], hm[(mxf + 3) * TY2], hm[(mxf + 4) * TY2],
                    hm[(mxf + 5) * TY2]);
      sFx[mxf * TY2 + jy] = L + Rr;
      if (tid < SM2_FY) {
        int jx = tid / (TY2 + 1), myf = tid % (TY2 + 1);
        const R* gp = sHyp + jx * PY2 + myf;
        const R* gm = sHym + jx * PY2 + myf;
        R Lg = recon_L(g, gp[0], gp[1], gp[2], gp[3], gp[4]);
        R Rg = recon_R(g, gm[1], gm[2], gm[3], gm[4], gm[5]);
        sFy[jx * (TY2 + 1) + myf] = Lg + Rg;
      }
    }
    __syncthreads();
    // ---- divergence and the RK combination
    if (live) {
      double dF = (double)(sFx[(ix + 1) * TY2 + iy] - sFx[ix * TY2 + iy]);
      double dG = (double)(sFy[ix * (TY2 + 1) + iy + 1] - sFy[ix * (TY2 + 1) + iy]);
#if JB_FAST
      double rhs = dt * visc_add<VISC>(g, f, cell, -(dF * g.idx + dG * g.idy));
#else
      double rhs = dt * visc_add<VISC>(g, f, cell, -(dF / g.dx + dG / g.dy));
#endif
      // the state itself is float64 in every variant
      double uk = EXACT ? (double)sQ[f * SM2_QF + tile_ci(ix + 3, iy + 3)] : Uk[f * nc + cell];
      double r;
      if (STAGE == 0) r = rhs;
      else if (STAGE == 1) r = uk + rhs;
      else if (STAGE == 2) r = 3.0 / 4.0 * Un[f * nc + cell] + 1.0 / 4.0 * (uk + rhs);
      else r = 1.0 / 3.0 * Un[f * nc + cell] + 2.0 / 3.0 * (uk + rhs);
      out[f * nc + cell] = r;
    }
    __syncthreads();
  }

  if (STAGE == 0) return;
  // ---- update_aux on the new state (Halley iterates, or per cell)
  unsigned bits = 0;
  double amx = 0.0, amy = 0.0, dtm = __longlong_as_double(0x7ff0000000000000LL);
  if (live) {
    double q[12];
    for (int f = 0; f < 12; ++f) q[f] = out[f * nc + cell];
    const double T0 = EXACT ? (double)sQ[TQ_T * SM2_QF + tile_ci(ix + 3, iy + 3)] : auxk[nc + cell];
    bits = finish_state<2, !EXACT>(m, g, fin, q, T0, cell, amx, amy, dtm, slots);
  }
  finish_reduce(fin, amx, amy, dtm, bits, slots);
}

#if JB_FAST
// ---------------------------------------------------------------------------
// mixed-precision 2D RK stage as an x-line sweep plus y runs (STAGE 1..3)
// ---------------------------------------------------------------------------
// float32 LF splitting and WENO5-JS on float32 primitives, float64 RK
// combination and temperature solve:
//   k_sweep_x    one thread per (y line, x segment of seg cells, field
//                pair; seg chosen by the host for whole waves): a register
//                window of the split fluxes walks the
//                segment's faces and writes the x flux difference
//                F_{i+1/2} - F_{i-1/2} of each cell
//   k_flux_y_rk  one block per segment of S cells of a column (S = 32 x
//                warps, up to 256, one cell per thread): split fluxes of all
//                fields on the segment and its 3 + 3 halo cells in shared
//                memory, the S + 1 y faces and the differences, then the
//                RK combination with the x part and the temperature solve
//                of the new state
// Fields are handled in pairs (rho, rho u), (rho v, rho E), (rho Y_1, rho
// Y_2), ... with sm_100's paired float32 instructions (FFMA2 / FADD2 /
// FMUL2), which issue two float32 operations at once.  The x differences are
// stored as float2 pairs: dfx[6][ncell][2].  The stage state's float32 u, v,
// p come from the kernel that wrote that state (prims[3][ncell]).
constexpr int SX_NT = 128;
#ifndef JB_YR_W
#define JB_YR_W 4
#endif
constexpr int YR_W = JB_YR_W, YR_NT = 32 * YR_W;  // most warps of a y-run block
// shared memory of a y-run block of S cells: H+ and H- of the S + 6 window
// cells and the S + 1 face values, six field pairs each
__host__ __device__ constexpr size_t yr_smem(int S) {
  return sizeof(float2) * (2 * 6 * (size_t)(S + 6) + 6 * (size_t)(S + 1));
}

typedef float2 f2;
__device__ __forceinline__ f2 f2s(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 f2add(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 f2mul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 f2fma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }

// WENO5-JS (reconstruction/WENO5_JS.py) of two fields at once: the
// left-biased value at the face between c and d from cells a..e (the
// right-biased value at the face between b and c is weno2(e, d, c, b, a)).
// The inputs are split fluxes without the 1/2 (H' = F +- alpha q = 2 H), so
// the smoothness indicators are formed as t^2 + 13/3 s^2 (16 IS) with eps
// scaled by 16, which leaves every weight exactly as the reference's in real
// arithmetic; the caller halves the face value.  Weights in the ratio form
// to the smallest eps + IS (no float32 overflow for SI fluxes ~1e11), with
// the linear weights C_k folded into the candidate polynomials.
__device__ __forceinline__ f2 weno2(f2 a, f2 b, f2 c, f2 d, f2 e) {
  const f2 t1 = f2fma(c, f2s(3.f), f2fma(b, f2s(-4.f), a));
  const f2 s1 = f2add(f2fma(b, f2s(-2.f), a), c);
  const f2 t2 = f2fma(d, f2s(-1.f), b);
  const f2 s2 = f2add(f2fma(c, f2s(-2.f), b), d);
  const f2 t3 = f2fma(c, f2s(3.f), f2fma(d, f2s(-4.f), e));
  const f2 s3 = f2add(f2fma(d, f2s(-2.f), c), e);
  const f2 e16 = f2s(16e-6f), k13 = f2s(13.f / 3.f);
  const f2 e1 = f2fma(t1, t1, f2fma(f2mul(s1, k13), s1, e16));
  const f2 e2 = f2fma(t2, t2, f2fma(f2mul(s2, k13), s2, e16));
  const f2 e3 = f2fma(t3, t3, f2fma(f2mul(s3, k13), s3, e16));
  const f2 mn = make_float2(fminf(e1.x, fminf(e2.x, e3.x)), fminf(e1.y, fminf(e2.y, e3.y)));
  const f2 r1 = f2mul(mn, make_float2(rcp_fast(e1.x), rcp_fast(e1.y)));
  const f2 r2 = f2mul(mn, make_float2(rcp_fast(e2.x), rcp_fast(e2.y)));
  const f2 r3 = f2mul(mn, make_float2(rcp_fast(e3.x), rcp_fast(e3.y)));
  const f2 w1 = f2mul(r1, r1), w2 = f2mul(r2, r2), w3 = f2mul(r3, r3);
  // C_k times the candidate values (C = 1/10, 6/10, 3/10)
  const f2 q1 = f2fma(c, f2s(11.f / 60.f), f2fma(b, f2s(-7.f / 60.f), f2mul(a, f2s(1.f / 30.f))));
  const f2 q2 = f2fma(d, f2s(0.2f), f2fma(c, f2s(0.5f), f2mul(b, f2s(-0.1f))));
  const f2 q3 = f2fma(e, f2s(-0.05f), f2fma(d, f2s(0.25f), f2mul(c, f2s(0.1f))));
  const f2 num = f2fma(w3, q3, f2fma(w2, q2, f2mul(w1, q1)));
  const f2 den = f2fma(w3, f2s(0.3f), f2fma(w2, f2s(0.6f), f2mul(w1, f2s(0.1f))));
  return f2mul(num, make_float2(rcp_fast(den.x), rcp_fast(den.y)));
}

// Doubled split fluxes of field pair j at one cell for direction dir:
// F = vel q (+ p in the normal momentum, + vel p in rho E), H' = F +- alpha q.
__device__ __forceinline__ void split2(int j, int dir, f2 q, float vel, float p, float al, f2& hp, f2& hm) {
  // pair 0 = (rho, rho u), pair 1 = (rho v, rho E)
  f2 c = make_float2(0.f, 0.f);
  if (j == 0 && dir == 0) c.y = p;
  if (j == 1) {
    if (dir == 1) c.x = p;
    c.y = vel * p;
  }
  const f2 F = f2fma(f2s(vel), q, c);
  hp = f2fma(f2s(al), q, F);
  hm = f2fma(f2s(-al), q, F);
}

// Field pair j (or all 12 fields for DIR 1, as six pairs), the normal
// velocity and the pressure of padded cell (x, y): interior and copied ghosts
// from the state and the primitives, outlet / injector ghosts and ghost
// layers from their buffers.  DIR 0: x sweep; DIR 1, 2: y run (2: one pair).
template <int DIR>
__device__ __forceinline__ void win_load2(const MP& m, const Grid& g, const double* __restrict__ Uk,
                                          const float* __restrict__ prims, const double* __restrict__ strips, int x,
                                          int y, int j, f2* q, float& vel, float& p) {
  constexpr int NP = DIR == 1 ? 6 : 1;
  const long long nc = g.ncell;
  const Src s = map_cell<2>(g, x, y);
  if (s.kind == 0) {
    const long long src = (long long)s.xs * g.ny + s.ys;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const int f = 2 * (DIR == 1 ? i : j);
      const double v0 = Uk[f * nc + src], v1 = Uk[(f + 1) * nc + src];
      q[i] = make_float2((float)(((s.flip >> f) & 1) ? -v0 : v0), (float)(((s.flip >> (f + 1)) & 1) ? -v1 : v1));
    }
    vel = prims[(DIR == 0 ? 0 : nc) + src];
    if (s.flip & (DIR == 0 ? 2 : 4)) vel = -vel;
    p = prims[2 * nc + src];
  } else if (s.kind == 1) {
    float qa[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) qa[i] = (float)ghost(g, strips, s, i);
    float rho, u, v;
    flux_prims<2>(m, qa, (float)ghost(g, strips, s, 13), rho, u, v, p);
    vel = DIR == 0 ? u : v;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const int f = 2 * (DIR == 1 ? i : j);
      q[i] = make_float2(qa[f], qa[f + 1]);
    }
  } else {
#pragma unroll
    for (int i = 0; i < NP; ++i) q[i] = make_float2(1.f, 1.f);
    vel = 1.f;
    p = 1.f;
  }
}

#ifndef JB_SX_MINB
#define JB_SX_MINB 7  // 72 registers: the paired window and WENO still fit without spills
#endif
#ifndef JB_SX_PF
#define JB_SX_PF 1  // cells fetched ahead of the window (a divisor of 6)
#endif
__global__ void __launch_bounds__(SX_NT, JB_SX_MINB) k_sweep_x(MP m, Grid g, const double* __restrict__ Uk,
                                                   const float* __restrict__ prims,
                                                   const double* __restrict__ strips, const Slots* slots, int aidx,
                                                   float2* __restrict__ dfx, int nlb, int seg_len) {
  const int j = blockIdx.x % 6;
  const int rest = blockIdx.x / 6;
  const int y = (rest % nlb) * SX_NT + threadIdx.x, seg = rest / nlb;
  if (y >= g.ny) return;
  const long long nc = g.ncell;
  const double* u0 = Uk + 2 * j * nc;
  const double* u1 = u0 + nc;
  const float al = (float)bitsd(slots->ax[aidx]);
  const int a0 = seg * seg_len, a1 = min(a0 + seg_len, g.nx);  // cells [a0, a1), faces a0 .. a1
  f2 Hp[6], Hm[6];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    f2 q;
    float vel, p;
    win_load2<0>(m, g, Uk, prims, strips, a0 - 3 + k, y, j, &q, vel, p);
    split2(j, 0, q, vel, p, al, Hp[k], Hm[k]);
  }
  // The hi-side ghost cells nx .. nx+2 of the line (the last segment's
  // window reaches them) go to this thread's column of shared memory first,
  // so that the face loop's fetch is a plain load: the ghost mapping stays
  // out of the unrolled loop body.
  __shared__ float gh[3][4][SX_NT];
  if (a1 + 2 >= g.nx) {
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
      f2 q;
      float vel, p;
      win_load2<0>(m, g, Uk, prims, strips, g.nx + k, y, j, &q, vel, p);
      gh[k][0][threadIdx.x] = q.x;
      gh[k][1][threadIdx.x] = q.y;
      gh[k][2][threadIdx.x] = vel;
      gh[k][3][threadIdx.x] = p;
    }
  }
  // the cells about to enter the window, fetched JB_SX_PF faces ahead into
  // buffer (c - a0) % JB_SX_PF and left untouched until then so that their
  // loads overlap the WENO arithmetic (a >= a0 + 2 >= 0 here)
  double n0[JB_SX_PF], n1[JB_SX_PF];
  float nv[JB_SX_PF], np[JB_SX_PF];
  auto fetch = [&](int a, int b) {
    if (a < g.nx) {
      const long long src = (long long)a * g.ny + y;
      n0[b] = u0[src];
      n1[b] = u1[src];
      nv[b] = prims[src];
      np[b] = prims[2 * nc + src];
    } else {
      const int k = a - g.nx;
      n0[b] = gh[k][0][threadIdx.x];
      n1[b] = gh[k][1][threadIdx.x];
      nv[b] = gh[k][2][threadIdx.x];
      np[b] = gh[k][3][threadIdx.x];
    }
  };
#pragma unroll
  for (int k = 0; k < JB_SX_PF; ++k) fetch(a0 + 2 + k, (2 + k) % JB_SX_PF);
  float2* out = dfx + (long long)j * nc + y;
  f2 Fprev = make_float2(0.f, 0.f);
  // cell c lives in window slot (c - a0 + 3) % 6: the face loop is unrolled
  // over the window's period so that the window rotates by renaming
#pragma unroll 1
  for (int fb = a0; fb <= a1; fb += 6) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int fa = fb + r;
      if (fa > a1) break;
      const int bc = (r + 2) % JB_SX_PF;  // buffer of cell fa + 2 ((fb - a0) is a multiple of 6)
      split2(j, 0, make_float2((float)n0[bc], (float)n1[bc]), nv[bc], np[bc], al, Hp[(r + 5) % 6],
             Hm[(r + 5) % 6]);  // cell fa+2
      if (fa + JB_SX_PF <= a1) fetch(fa + 2 + JB_SX_PF, bc);
      // face fa (cells fa-1 | fa): H+ of cells fa-3 .. fa+1, H- of fa-2 .. fa+2
      const f2 F = f2mul(f2s(0.5f), f2add(weno2(Hp[r % 6], Hp[(r + 1) % 6], Hp[(r + 2) % 6], Hp[(r + 3) % 6],
                                                Hp[(r + 4) % 6]),
                                          weno2(Hm[(r + 5) % 6], Hm[(r + 4) % 6], Hm[(r + 3) % 6],
                                                Hm[(r + 2) % 6], Hm[(r + 1) % 6])));
      if (fa > a0) out[(long long)(fa - 1) * g.ny] = f2fma(Fprev, f2s(-1.f), F);
      Fprev = F;
    }
  }
}

#ifndef JB_YR_MINB
#define JB_YR_MINB (32 / JB_YR_W)  // 64 registers (64 B of spills)
#endif
template <int STAGE, bool VISC>
__global__ void __launch_bounds__(YR_NT, JB_YR_MINB) k_flux_y_rk(MP m, Grid g, const double* __restrict__ Uk,
                                                       const double* __restrict__ auxk,
                                                       const double* __restrict__ Un, const float* __restrict__ prims,
                                                       const double* __restrict__ strips,
                                                       const float2* __restrict__ dfx, double* __restrict__ out,
                                                       Slots* slots, int aidx, jb_fin fin, int nsy) {
  extern __shared__ __align__(128) unsigned char smraw[];
  const int S = blockDim.x, t = threadIdx.x;
  const int C = S + 6, NF = S + 1;
  f2* sHp = reinterpret_cast<f2*>(smraw);  // [6][C]: cell y0 - 3 + j in slot j
  f2* sHm = sHp + 6 * C;
  f2* sF = sHm + 6 * C;  // [6][NF]: face y0 + k (cells y0+k-1 | y0+k)
  const long long nc = g.ncell;
  const int x = blockIdx.x / nsy, y0 = (blockIdx.x % nsy) * S;
  const float al = (float)bitsd(slots->ay[aidx]);
  // ---- split fluxes on the window: the segment's own cells one per
  // thread, the 3 + 3 halo cells as 36 (cell, pair) items
  {
    const int jj = t + 3;
    f2 q[6];
    float vel, p;
    if (y0 + t < g.ny) {
      const long long cell = (long long)x * g.ny + y0 + t;
#pragma unroll
      for (int i = 0; i < 6; ++i)
        q[i] = make_float2((float)Uk[2 * i * nc + cell], (float)Uk[(2 * i + 1) * nc + cell]);
      vel = prims[nc + cell];
      p = prims[2 * nc + cell];
    } else {
      win_load2<1>(m, g, Uk, prims, strips, x, y0 + t, 0, q, vel, p);
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) split2(i, 1, q[i], vel, p, al, sHp[i * C + jj], sHm[i * C + jj]);
  }
#pragma unroll 1
  for (int i = t; i < 36; i += S) {
    const int h = i / 6, pr = i % 6;
    const int jj = h < 3 ? h : S + h;
    f2 q;
    float vel, p;
    win_load2<2>(m, g, Uk, prims, strips, x, y0 - 3 + jj, pr, &q, vel, p);
    split2(pr, 1, q, vel, p, al, sHp[pr * C + jj], sHm[pr * C + jj]);
  }
  __syncthreads();
  // ---- faces: face y0 + t of every pair, and face y0 + S by threads 0..5
  // (one pair each)
#pragma unroll 1
  for (int i = 0; i < 6; ++i) {
    const f2* hp = sHp + i * C + t;
    const f2* hm = sHm + i * C + t;
    sF[i * NF + t] = f2mul(f2s(0.5f), f2add(weno2(hp[0], hp[1], hp[2], hp[3], hp[4]),
                                             weno2(hm[5], hm[4], hm[3], hm[2], hm[1])));
  }
  if (t < 6) {
    const f2* hp = sHp + t * C + S;
    const f2* hm = sHm + t * C + S;
    sF[t * NF + S] = f2mul(f2s(0.5f), f2add(weno2(hp[0], hp[1], hp[2], hp[3], hp[4]),
                                             weno2(hm[5], hm[4], hm[3], hm[2], hm[1])));
  }
  __syncthreads();
  // ---- RK combination (float64) and update_aux of the new state
  const int y = y0 + t;
  const bool live = y < g.ny;
  unsigned bits = 0;
  double amx = 0.0, amy = 0.0, dtm = __longlong_as_double(0x7ff0000000000000LL);
  if (live) {
    const long long cell = (long long)x * g.ny + y;
    const double dt = slots->dt;
    double q[12];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const float2 dF = dfx[i * nc + cell];
      const f2 dG = f2fma(sF[i * NF + t], f2s(-1.f), sF[i * NF + t + 1]);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int f = 2 * i + h;
        const double rhs = dt * visc_add<VISC>(g, f, cell, -((double)(h ? dF.y : dF.x) * g.idx +
                                                            (double)(h ? dG.y : dG.x) * g.idy));
        const double uk = Uk[f * nc + cell];  // read again (L1): no registers held across the WENO
        double r;
        if (STAGE == 1) r = uk + rhs;
        else if (STAGE == 2) r = 3.0 / 4.0 * Un[f * nc + cell] + 1.0 / 4.0 * (uk + rhs);
        else r = 1.0 / 3.0 * Un[f * nc + cell] + 2.0 / 3.0 * (uk + rhs);
        out[f * nc + cell] = r;
        q[f] = r;
      }
    }
    bits = finish_state<2, true>(m, g, fin, q, auxk[nc + cell], cell, amx, amy, dtm, slots);
  }
  finish_reduce(fin, amx, amy, dtm, bits, slots);
}
#endif  // JB_FAST

// 1D: a block of NT threads handles a tile of NT-1 cells, so its NT faces
// map one-to-one onto threads.
constexpr int NT1 = 256;

template <class R, int NT = NT1>
__host__ __device__ constexpr size_t sw_smem1d_bytes() {
  return sizeof(R) * 2 * (NT + 5);
}

template <class R, int NT = NT1>
__host__ __device__ constexpr size_t smem1d_bytes(int nq) {
  return sizeof(R) * ((size_t)nq * (NT + 5) + 3 * (NT + 5) + 2 * (NT + 5) + NT);
}

// One tile [x0, x0 + NT - 1) of a 1D stage (see k_flux2d for STAGE and R).
// Every thread of the block must call it.  The new state's temperature is
// finished as fin says: float64 tiles write the Halley iterates and return
// this thread's mask bits; float tiles (the mixed variant) solve per cell
// into fin.aux, fold the new state's wave speed (and, with fin.cfl, the CFL
// candidate) into amx and dtm, and return status bits << 16.  Pointers are
// plain (not restrict) because the persistent ensemble kernel calls it on
// buffers written by other blocks of the same launch.
template <int STAGE, class R, int NT, bool VISC = false, bool SW = false>
__device__ __forceinline__ unsigned flux1d_tile(const MP& m, const Grid& g, const double* Uk,
                                                const double* auxk, const double* Un, double* out,
                                                const jb_fin& fin, const double* strips, double alpha,
                                                double dt, int x0, unsigned char* smraw, double& amx,
                                                double& dtm, Slots* slots) {
  constexpr int TX1 = NT - 1, PX1 = NT + 5;
  constexpr int nv = 11, nq = nv + 1;
  constexpr bool EXACT = sizeof(R) == sizeof(double);
  R* sQ = reinterpret_cast<R*>(smraw);  // [nq][PX1]
  R* sP = sQ + (size_t)nq * PX1;        // [3][PX1]: rho, u, p
  R* sHp = sP + 3 * PX1;
  R* sHm = sHp + PX1;
  R* sF = sHm + PX1;                    // [TX1+1]
  R* sG = sF + NT;                      // Steger-Warming only: gamma, a [PX1] each
  R* sA = sG + PX1;
  constexpr bool sw = SW;
  const int tid = threadIdx.x;
  const long long nc = g.ncell;
  const R ax = (R)alpha;

  for (int i = tid; i < PX1; i += NT) {
    int x = x0 + i - 3;
    Src s = map_cell<1>(g, x, 0);
    if (s.kind == 0) {
      for (int q = 0; q < nv; ++q) {
        double v = Uk[q * nc + s.xs];
        sQ[q * PX1 + i] = (R)(((s.flip >> q) & 1) ? -v : v);
      }
      sQ[nv * PX1 + i] = (R)auxk[nc + s.xs];
      if (sw) sG[i] = (R)auxk[s.xs];
    } else if (s.kind == 1) {
      for (int q = 0; q < nv; ++q) sQ[q * PX1 + i] = (R)ghost(g, strips, s, q);
      sQ[nv * PX1 + i] = (R)ghost(g, strips, s, nv + 1);
      if (sw) sG[i] = (R)ghost(g, strips, s, nv);
    } else {
      for (int q = 0; q < nq; ++q) sQ[q * PX1 + i] = (R)1.0;
      if (sw) sG[i] = (R)1.0;
    }
  }
  __syncthreads();
  for (int i = tid; i < PX1; i += NT) {
    R q[nv];
#pragma unroll
    for (int f = 0; f < nv; ++f) q[f] = sQ[f * PX1 + i];
    R rho, u, v, p;
    flux_prims<1>(m, q, sQ[nv * PX1 + i], rho, u, v, p);
    sP[i] = rho;
    sP[PX1 + i] = u;
    sP[2 * PX1 + i] = p;
    if (sw) sA[i] = sqrt(sG[i] * p / rho);
  }
  __syncthreads();
  const bool live = tid < TX1 && x0 + tid < g.nx;
  const size_t cell = (size_t)(x0 + tid);
  for (int f = 0; f < nv; ++f) {
    for (int i = tid; i < PX1; i += NT) {
#if JB_FAST
      // F = u q + p (rho u) + u p (rho E): the reference's LF flux regrouped
      const R u = sP[PX1 + i], qf = sQ[f * PX1 + i];
      R F = u * qf;
      if (f == 1) F += sP[2 * PX1 + i];
      if (f == 2) F += u * sP[2 * PX1 + i];
#else
      R rho = sP[i], u = sP[PX1 + i], p = sP[2 * PX1 + i];
      R qf = sQ[f * PX1 + i];
      R F = lf_flux<1>(f, 0, qf, rho, u, (R)0, p, sQ[2 * PX1 + i]);
#endif
      if (sw) {
        sw_split<1, R>(f, 0, qf, sP[i], sP[PX1 + i], (R)0, sP[2 * PX1 + i], sQ[2 * PX1 + i], sA[i], sG[i],
                       sHp[i], sHm[i]);
      } else {
        sHp[i] = (R)0.5 * (F + ax * qf);
        sHm[i] = (R)0.5 * (F - ax * qf);
      }
    }
    __syncthreads();
    {
      int mf = tid;  // NT faces
      R L = recon_L(g, sHp[mf], sHp[mf + 1], sHp[mf + 2], sHp[mf + 3], sHp[mf + 4]);
      R Rr = recon_R(g, sHm[mf + 1], sHm[mf + 2], sHm[mf + 3], sHm[mf + 4], sHm[mf + 5]);
      sF[mf] = L + Rr;
    }
    __syncthreads();
    if (live) {
      double dF = (double)(sF[tid + 1] - sF[tid]);
#if JB_FAST
      double rhs = dt * visc_add<VISC>(g, f, cell, -(dF * g.idx));
#else
      double rhs = dt * visc_add<VISC>(g, f, cell, -(dF / g.dx));
#endif
      double uk = EXACT ? (double)sQ[f * PX1 + tid + 3] : Uk[f * nc + cell];
      double r;
      if (STAGE == 0) r = rhs;
      else if (STAGE == 1) r = uk + rhs;
      else if (STAGE == 2) r = 3.0 / 4.0 * Un[f * nc + cell] + 1.0 / 4.0 * (uk + rhs);
      else r = 1.0 / 3.0 * Un[f * nc + cell] + 2.0 / 3.0 * (uk + rhs);
      out[f * nc + cell] = r;
    }
    __syncthreads();
  }
  unsigned bits = 0;
  if (STAGE == 0) return bits;
  if (live) {
    double q[11];
    for (int f = 0; f < 11; ++f) q[f] = out[f * nc + cell];
    const double T0 = EXACT ? (double)sQ[nv * PX1 + tid + 3] : auxk[nc + cell];
    // float tiles (the mixed variant): the temperature solve per cell, with
    // the new state's alpha and CFL candidate; float64 tiles: the Halley
    // iterates of the global stop
    double amy = 0.0;
    bits = finish_state<1, !EXACT>(m, g, fin, q, T0, cell, amx, amy, dtm, slots);
  }
  __syncthreads();  // the tile's shared memory is reused by the next tile
  return bits;
}

template <int STAGE, class R, bool VISC, bool SW = false>
__global__ void __launch_bounds__(NT1) k_flux1d(MP m, Grid g, const double* __restrict__ Uk,
                                                 const double* __restrict__ auxk,
                                                 const double* __restrict__ Un,
                                                 double* __restrict__ out,
                                                 const double* __restrict__ strips, Slots* slots,
                                                 int aidx, jb_fin fin, double dt_arg) {
  extern __shared__ __align__(128) unsigned char smraw[];
  const double dt = STAGE == 0 ? dt_arg : slots->dt;
  // the tile body is shared with the persistent ensemble kernel
  double amx = 0.0, dtm = __longlong_as_double(0x7ff0000000000000LL);
  unsigned bits = flux1d_tile<STAGE, R, NT1, VISC, SW>(m, g, Uk, auxk, Un, out, fin, strips,
                                                       bitsd(slots->ax[aidx]), dt, blockIdx.x * (NT1 - 1), smraw,
                                                       amx, dtm, slots);
  if (STAGE == 0) return;
  finish_reduce(fin, amx, 0.0, dtm, bits, slots);
}

// ---------------------------------------------------------------------------
// Halley iterates for a standalone update_aux (aux_func.update_aux)
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void k_halley(MP m, Grid g, const double* __restrict__ U, const double* __restrict__ aux,
                         double* __restrict__ cand, Slots* slots, int midx) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  const long long nc = g.ncell;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned bits = 0;
  if (c < nc) {
    double rho = U[c];
    double u = U[nc + c] / rho;
    double v = DIM == 2 ? U[2 * nc + c] / rho : 0.0;
    double e = DIM == 2 ? U[3 * nc + c] / rho - 0.5 * (u * u + v * v) : U[2 * nc + c] / rho - 0.5 * (u * u);
    double Y8[NR], Yf[NS];
#pragma unroll
    for (int k = 0; k < NR; ++k) Y8[k] = U[(nY + k) * nc + c] / rho;
    fill_Y(Y8, Yf);
    double R = get_R(m, Yf);
    double cnd[JB_NCAND];
    bits = halley_any(m, e, Yf, R, aux[nc + c], cnd);
#pragma unroll
    for (int i = 0; i < JB_NCAND; ++i) cand[i * nc + c] = cnd[i];
  }
  block_reduce_store(0.0, 0.0, 0.0, bits, slots, 0, false, false, midx);
}

// ---------------------------------------------------------------------------
// select / reduce pass: finishes a temperature solve (SELECT) or takes aux
// as given, then the LF wave-speed maxima over the padded grid (ALPHA:
// flux_splitting/LF.py "nanmax(|u|+a)"), the CFL minimum (CFL:
// set_simulator.py:420-443) and the non-copy ghost strips (STRIPS).
// ---------------------------------------------------------------------------
// One cell of the select pass; folds its wave speeds / CFL candidate into
// amx, amy, dtm and status bits into st.  mask: the Halley mask of the solve
// being finished (SELECT); slots: where a NaN CFL candidate is flagged.
// STRIPS: a boundary cell of a pressure-outlet / injector side also builds
// its ghost state here (k_select leaves that to k_strips).
template <int DIM, bool SELECT, bool ALPHA, bool CFL, bool STRIPS = true>
__device__ __forceinline__ void select_cell(const MP& m, const Grid& g, const double* U, const double* aux_in,
                                            const double* cand, double* aux_out, double* strips,
                                            Slots* slots, unsigned mask, long long c, double& amx,
                                            double& amy, double& dtm, unsigned& st,
                                            float* prims = nullptr) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  constexpr int nv = nY + NR;
  const long long nc = g.ncell;
  {
    double q[nv];
#pragma unroll
    for (int f = 0; f < nv; ++f) q[f] = U[f * nc + c];
    double gamma, T;
    if (SELECT) {
      int n = halley_count(mask);
      T = cand[n * nc + c];
      double Y8[NR], Yf[NS];
#if JB_FAST
      const double ri = 1.0 / q[0];
#pragma unroll
      for (int k = 0; k < NR; ++k) Y8[k] = q[nY + k] * ri;
#else
#pragma unroll
      for (int k = 0; k < NR; ++k) Y8[k] = q[nY + k] / q[0];
#endif
      fill_Y(Y8, Yf);
      double R = get_R(m, Yf);
      double cp = cp_mix(m, T, Yf);
      gamma = cp / (cp - R);
      aux_out[c] = gamma;
      aux_out[nc + c] = T;
    } else {
      gamma = aux_in[c];
      T = aux_in[nc + c];
    }
    if (ALPHA || CFL) {
      Prim<DIM> pr = u_to_prim<DIM>(m, q, gamma, T);
      if (DIM == 2 && prims) {  // float32 primitives for the next mixed-precision flux stage
        prims[c] = (float)pr.u;
        prims[nc + c] = (float)pr.v;
        prims[2 * nc + c] = (float)pr.p;
      }
      double sx = fabs(pr.u) + pr.a;
      double sy = fabs(pr.v) + pr.a;
      amx = fmax(amx, sx);
      amy = fmax(amy, sy);
      if (!(sx == sx) || !(T == T)) st |= JB_ERR_NONFINITE;
      if (CFL) {
#if JB_FAST
        double d = DIM == 1 ? g.dx / sx : 1.0 / (sx * g.idx + sy * g.idy);
#else
        double d = DIM == 1 ? g.dx / sx : 1.0 / (sx / g.dx + sy / g.dy);
#endif
        dtm = fmin(dtm, d);
        if (!(d == d) || !(d > 0.0)) st |= JB_ERR_NONFINITE;
        // jnp.min (set_simulator.py:423,441) returns NaN if any candidate is
        // NaN; the reduction below skips NaN, so record it separately
        if (!(d == d)) atomicOr(&slots->dtnan, 1u);
      }
      if (ALPHA && STRIPS) {
        // ghost states that are not copies of interior cells
        int x = DIM == 1 ? (int)c : (int)(c / g.ny);
        int y = DIM == 1 ? 0 : (int)(c % g.ny);
        for (int side = 0; side < 2 * DIM; ++side) {
          int kind = g.bc[side];
          if (kind != JB_BC_PRESSURE_OUTLET && kind != JB_BC_RDC_INJECTOR) continue;
          bool on = side == 0 ? x == 0 : side == 1 ? x == g.nx - 1 : side == 2 ? y == 0 : y == g.ny - 1;
          if (!on) continue;
          double gs[nv + 2];
          if (kind == JB_BC_PRESSURE_OUTLET) {
            double un = side < 2 ? q[1] / q[0] : q[2] / q[0];
            if (side == 0 || side == 2) un = -un;
            pressure_outlet_state<DIM>(m, q, gamma, T, un, g.Pb, gs);
          } else {
            if (DIM == 2) {
              double Yi[NR];
              for (int k = 0; k < NR; ++k) Yi[k] = g.Yinj[k * g.nx + x];
              injector_state(m, q, gamma, T, Yi, g.inj_block_p, gs);
            }
          }
          int pos = side < 2 ? y : x;
          for (int f = 0; f < nv + 2; ++f) strips[strip_idx(g, side, f, pos)] = gs[f];
          Prim<DIM> pg = u_to_prim<DIM>(m, gs, gs[nv], gs[nv + 1]);
          double gx = fabs(pg.u) + pg.a, gy = fabs(pg.v) + pg.a;
          amx = fmax(amx, gx);
          amy = fmax(amy, gy);
        }
      }
    }
  }
}

template <int DIM, bool SELECT, bool ALPHA, bool CFL>
__global__ void __launch_bounds__(256, 4) k_select(MP m, Grid g, const double* __restrict__ U, const double* __restrict__ aux_in,
                         const double* __restrict__ cand, double* __restrict__ aux_out,
                         double* __restrict__ strips, Slots* slots, int midx, int aidx,
                         float* __restrict__ prims) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double amx = 0.0, amy = 0.0, dtm = __longlong_as_double(0x7ff0000000000000LL);
  unsigned st = 0;
  if (c < g.ncell)
    select_cell<DIM, SELECT, ALPHA, CFL, false>(m, g, U, aux_in, cand, aux_out, strips, slots,
                                                SELECT ? slots->mask[midx] : 0u, c, amx, amy, dtm, st,
                                                ALPHA ? prims : nullptr);
  if (ALPHA || CFL) block_reduce_store(amx, amy, dtm, st << 16, slots, aidx, ALPHA, CFL, -1);
}

// The ghost state of an outlet / injector side at boundary position pos from
// the boundary cell's (U, gamma, T) into the strip, and its wave speeds
// folded into amx, amy (nothing for other sides).
template <int DIM>
__device__ __forceinline__ void strip_one(const MP& m, const Grid& g, const double* U, const double* aux,
                                          double* strips, int side, int pos, double& amx, double& amy) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  constexpr int nv = nY + NR;
  const long long nc = g.ncell;
  const int kind = side >= 0 ? g.bc[side] : JB_BC_PERIODIC;
  if (kind == JB_BC_PRESSURE_OUTLET || kind == JB_BC_RDC_INJECTOR) {
    const int x = side == 0 ? 0 : side == 1 ? g.nx - 1 : pos;
    const int y = DIM == 1 ? 0 : (side == 2 ? 0 : side == 3 ? g.ny - 1 : pos);
    const long long c = DIM == 1 ? (long long)x : (long long)x * g.ny + y;
    double q[nv];
#pragma unroll
    for (int f = 0; f < nv; ++f) q[f] = U[f * nc + c];
    const double gamma = aux[c], T = aux[nc + c];
    double gs[nv + 2];
    if (kind == JB_BC_PRESSURE_OUTLET) {
      double un = side < 2 ? q[1] / q[0] : q[2] / q[0];
      if (side == 0 || side == 2) un = -un;
      pressure_outlet_state<DIM>(m, q, gamma, T, un, g.Pb, gs);
    } else {
      if (DIM == 2) {
        double Yi[NR];
        for (int k = 0; k < NR; ++k) Yi[k] = g.Yinj[k * g.nx + x];
        injector_state(m, q, gamma, T, Yi, g.inj_block_p, gs);
      }
    }
    for (int f = 0; f < nv + 2; ++f) strips[strip_idx(g, side, f, pos)] = gs[f];
    Prim<DIM> pg = u_to_prim<DIM>(m, gs, gs[nv], gs[nv + 1]);
    amx = fmax(amx, fabs(pg.u) + pg.a);
    amy = fmax(amy, fabs(pg.v) + pg.a);
  }
}

// Ghost strips of the pressure-outlet and injector sides (the padded grid's
// entries that are not copies of interior cells) and their wave speeds into
// the alpha maxima: one thread per boundary position, after the pass that
// wrote the boundary cells' (gamma, T) into aux.  Positions: side 0 and 1
// (x = 0, nx-1) ny each, then sides 2 and 3 (y = 0, ny-1) nx each.
template <int DIM>
__global__ void __launch_bounds__(128) k_strips(MP m, Grid g, const double* __restrict__ U,
                                                const double* __restrict__ aux, double* __restrict__ strips,
                                                Slots* slots, int aidx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ns = DIM == 1 ? 1 : g.ny;
  double amx = 0.0, amy = 0.0;
  int side = -1, pos = 0;
  if (t < 2 * ns) { side = t / ns; pos = t % ns; }
  else if (DIM == 2 && t < 2 * ns + 2 * g.nx) { side = 2 + (t - 2 * ns) / g.nx; pos = (t - 2 * ns) % g.nx; }
  strip_one<DIM>(m, g, U, aux, strips, side, pos, amx, amy);
  block_reduce_store(amx, amy, 0.0, 0u, slots, aidx, true, false, -1);
}

}  // namespace
}  // namespace JB_NS
}  // namespace jb

#include "jb_chem_gen.cuh"

namespace jb {
namespace JB_NS {
namespace {

// ---------------------------------------------------------------------------
// point-implicit chemistry (model/reaction_model.py:91-193)
// ---------------------------------------------------------------------------
// (I/dt - M_k J) x = M_k w by LU with partial pivoting (first maximal
// |pivot| as LAPACK idamax), then detailed_reaction's clip and S = rho dY
// (construct_matrix_equation, reaction_model.py:132-159 and :183-193).
// Gaussian elimination of A x = b in registers with partial pivoting (first
// maximal |pivot|, as LAPACK idamax) when PIVOT, else without exchanges;
// every loop has a constant trip count so the matrix stays in registers.
template <bool PIVOT>
__device__ __forceinline__ void lu_solve(double (&J)[NR][NR], double (&b)[NR], double (&x)[NR], unsigned& st) {
#if JB_FAST
  double ipv[NR];
#endif
#pragma unroll
  for (int c = 0; c < NR; ++c) {
    if (PIVOT) {
      int p = c;
      double best = fabs(J[c][c]);
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        if (r > c) {
          double v = fabs(J[r][c]);
          if (v > best) { best = v; p = r; }
        }
      }
      // branch-free row exchange over the columns still active (the
      // eliminated columns are not used again)
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        if (r > c) {
          const bool sw = p == r;
#pragma unroll
          for (int j = 0; j < NR; ++j) {
            if (j >= c) {
              const double x0 = J[c][j], x1 = J[r][j];
              J[c][j] = sw ? x1 : x0;
              J[r][j] = sw ? x0 : x1;
            }
          }
          const double y0 = b[c], y1 = b[r];
          b[c] = sw ? y1 : y0;
          b[r] = sw ? y0 : y1;
        }
      }
    }
    if (J[c][c] == 0.0) st |= JB_ERR_SINGULAR;
#if JB_FAST
    // one reciprocal per pivot (kept for the back substitution)
    ipv[c] = 1.0 / J[c][c];
#endif
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      if (r > c) {
#if JB_FAST
        const double l = J[r][c] * ipv[c];
#else
        const double l = J[r][c] / J[c][c];
#endif
#pragma unroll
        for (int j = 0; j < NR; ++j)
          if (j > c) J[r][j] = J[r][j] - l * J[c][j];
        b[r] = b[r] - l * b[c];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    const int r = NR - 1 - i;
    double s = b[r];
#pragma unroll
    for (int j = 0; j < NR; ++j)
      if (j > r) s = s - J[r][j] * x[j];
#if JB_FAST
    x[r] = s * ipv[r];
#else
    x[r] = s / J[r][r];
#endif
  }
}

// (I/dt - M_k J) x = M_k w by LU with partial pivoting, then
// detailed_reaction's clip and S = rho dY (construct_matrix_equation,
// reaction_model.py:132-159 and :183-193; the reference solves with
// jnp.linalg.solve, a partially pivoted LU).  The fast variants first test
// the matrix for diagonal dominance by columns: partial pivoting then never
// exchanges rows (each diagonal entry is the first maximum of its column, and
// elimination keeps the dominance), so the elimination without the pivot
// search and exchanges computes the same values; the other cells (the hot
// reaction zone, where M_k J outweighs 1/dt) take the pivoted form.
__device__ __forceinline__ void chem_solve(const MP& m, double (&J)[NR][NR], const double* w, double rho,
                                           const double* Y8, double dt, double* S, unsigned& st) {
  double b[NR];
  const double idt = 1.0 / dt;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    b[k] = m.M[k] * w[k];
#pragma unroll
    for (int n = 0; n < NR; ++n) {
      double jk = m.M[k] * J[k][n];
      J[k][n] = (k == n ? idt : 0.0) - jk;  // J now holds A
    }
  }
  double x[NR];
#if JB_FAST
  bool cdd = true;
#pragma unroll
  for (int c = 0; c < NR; ++c) {
    double off = 0.0;
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r != c) off += fabs(J[r][c]);
    cdd = cdd && fabs(J[c][c]) > off;
  }
  if (cdd) lu_solve<false>(J, b, x, st);
  else lu_solve<true>(J, b, x, st);
#else
  lu_solve<true>(J, b, x, st);
#endif
  // detailed_reaction (:183-193): dY = clip(drhoY/rho, -Y, 1-Y); S = rho dY
#if JB_FAST
  const double irho = 1.0 / rho;
#endif
#pragma unroll
  for (int k = 0; k < NR; ++k) {
#if JB_FAST
    double dY = x[k] * irho;
#else
    double dY = x[k] / rho;
#endif
    double lo = -Y8[k], hi = 1.0 - Y8[k];
    dY = dY < lo ? lo : dY;
    dY = dY > hi ? hi : dY;
    S[k] = rho * dY;
  }
}


// Rates, analytic Jacobian d(omega)/d(rho Y) and the solve of
// (I/dt - J) x = omega for one cell.  Returns S_k = rho * clip(x_k/rho).
__device__ void chem_cell(const MP& m, double rho, const double* Y8, double T, double dt,
                          double* S, unsigned& st) {
  double Yf[NS], X[NS], Xc[NS], logX[NR], gk[NR];
  fill_Y(Y8, Yf);
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    X[k] = rho * Yf[k] / m.M[k];
    Xc[k] = X[k] < 1e-50 ? 1e-50 : X[k];
  }
#pragma unroll
  for (int k = 0; k < NR; ++k) logX[k] = log(Xc[k]);
  // get_gibbs (reaction_model.py:78-89): g = s/R - h/(R T)
  const double lT = log(m.T0 * T);
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const bool lo = T < m.Tcr[k];
    double h = lo ? poly6(m.hc_lo[k], T) : poly6(m.hc_hi[k], T);
    double s = lo ? poly5(m.s_lo[k], T) + m.lg_lo[k] * lT : poly5(m.s_hi[k], T) + m.lg_hi[k] * lT;
    gk[k] = s - h / T;
  }
  double w[NR], J[NR][NR], rMX[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    w[k] = 0.0;
    rMX[k] = 1.0 / (m.M[k] * Xc[k]);
#pragma unroll
    for (int n = 0; n < NR; ++n) J[k][n] = 0.0;
  }
  const double rT = m.pref / T;
#pragma unroll 1
  for (int i = 0; i < NREAC; ++i) {
    // reactionConstant_i (reaction_model.py:91-122)
    double kfi = m.A[i] * pow(T, m.B[i]) * exp(-m.EaR[i] / T);
    double Ms = m.tb[i][0] * X[0];
#pragma unroll
    for (int j = 1; j < NS; ++j) Ms = Ms + m.tb[i][j] * X[j];
    double Mi = m.is_tb[i] * Ms + (1.0 - m.is_tb[i]);
    double sf = m.vf[i][0] * logX[0], sb = m.vb[i][0] * logX[0], sg = m.dv[i][0] * gk[0];
#pragma unroll
    for (int k = 1; k < NR; ++k) {
      sf = sf + m.vf[i][k] * logX[k];
      sb = sb + m.vb[i][k] * logX[k];
      sg = sg + m.dv[i][k] * gk[k];
    }
    double kf = kfi * exp(sf);
    double vs = m.vsum[i];
    double pw = vs == 0.0 ? 1.0 : (vs == 1.0 ? rT : (vs == -1.0 ? 1.0 / rT : pow(rT, vs)));
    double kb = kfi / (exp(sg) * pw) * exp(sb);
    double dq = kf - kb;
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const double dv = m.dv[i][k];
      if (dv == 0.0) continue;
      w[k] = w[k] + dv * Mi * dq;
#pragma unroll
      for (int n = 0; n < NR; ++n) {
        const double a = m.tb[i][n];
        const double vfn = m.vf[i][n], vbn = m.vb[i][n];
        const bool t2 = vfn != 0.0 || vbn != 0.0;
        if (a == 0.0 && !t2) continue;
        double term;
        double t1v = dv * dq * (a / m.M[n]);
        if (t2) {
          double t2v = rMX[n] * dv * Mi * (vfn * kf - vbn * kb);
          term = a == 0.0 ? t2v : t1v + t2v;
        } else {
          term = t1v;
        }
        J[k][n] = J[k][n] + term;
      }
    }
  }
  chem_solve(m, J, w, rho, Y8, dt, S, st);
}

#if JB_FAST
constexpr int CHEM_SH = 3 * NREAC;  // per-cell shared doubles of the specialised path

// Specialised chemistry (structure compiled in by gen_chem.py): one
// exponential per reaction and one per species, the concentration and
// equilibrium factors as products (their exponents are small integers),
// FMA-contracted.  sh points at this thread's column of a [CHEM_SH][stride]
// shared array.
__device__ __forceinline__ void chem_cell_gen(const MP& m, double rho, const double* Y8, double T,
                                              double dt, double* S, unsigned& st, double* sh,
                                              int stride) {
  double Yf[NS], X[NS], Xc[NR], E[NR], iE[NR], rMX[NR], w[NR];
  fill_Y(Y8, Yf);
#pragma unroll
  for (int k = 0; k < NS; ++k) X[k] = rho * Yf[k] * m.invM[k];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double xc = X[k] < 1e-50 ? 1e-50 : X[k];
    Xc[k] = xc;
    rMX[k] = m.invM[k] / xc;
  }
  const double lT = log(T), invT = 1.0 / T, lT0T = lT + m.lnT0;
  // get_gibbs (reaction_model.py:78-89): g = s/R - h/(R T); E = exp(g)
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const bool lo = T < m.Tcr[k];
    const double h = lo ? poly6(m.hc_lo[k], T) : poly6(m.hc_hi[k], T);
    const double s = lo ? poly5(m.s_lo[k], T) + m.lg_lo[k] * lT0T : poly5(m.s_hi[k], T) + m.lg_hi[k] * lT0T;
    E[k] = exp(s - h * invT);
    iE[k] = 1.0 / E[k];
  }
  chem_rates_gen(m, lT, invT, T / m.pref, m.pref * invT, X, Xc, E, iE, sh, stride, w);
  double J[NR][NR];
  chem_jac_gen(m, rMX, sh, stride, J);
  chem_solve(m, J, w, rho, Y8, dt, S, st);
}
#endif

// Chemistry of one cell at temperature T.  WRITE_S: reaction_source_terms
// output S (zeros for the flow fields).  Otherwise U_out = U + S followed by
// the final update_aux (set_simulator.py:117-122) started from T, in the
// mode of fin (finish_state; per-cell mode folds the wave speeds and the CFL
// candidate of the new state into amx, amy, dtm).  sh: this thread's column
// of the [CHEM_SH][blockDim] shared array.
template <int DIM, bool WRITE_S, bool GEN, bool CELL = false>
__device__ __forceinline__ void chem_cell_step(const MP& m, const Grid& g, const double* U, double T,
                                               double* out, const jb_fin& fin, long long c, double dt,
                                               double* sh, unsigned& bits, unsigned& st, double& amx,
                                               double& amy, double& dtm, Slots* slots) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  constexpr int nv = nY + NR;
  const long long nc = g.ncell;
  {
    double q[nv];
#if JB_FAST
    // only rho and the species enter the chemistry; the other fields are
    // read after it so that they hold no registers across the solve
    q[0] = U[c];
#pragma unroll
    for (int k = 0; k < NR; ++k) q[nY + k] = U[(nY + k) * nc + c];
#else
#pragma unroll
    for (int f = 0; f < nv; ++f) q[f] = U[f * nc + c];
#endif
    double rho = q[0];
    double Y8[NR], S[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) Y8[k] = q[nY + k] / rho;
#if JB_FAST
    if (GEN) chem_cell_gen(m, rho, Y8, T, dt, S, st, sh, blockDim.x);
    else chem_cell(m, rho, Y8, T, dt, S, st);
#pragma unroll
    for (int f = 1; f < nY; ++f) q[f] = U[f * nc + c];
#else
    (void)sh;
    chem_cell(m, rho, Y8, T, dt, S, st);
#endif
    if (WRITE_S) {
#pragma unroll
      for (int f = 0; f < nY; ++f) out[f * nc + c] = 0.0;
#pragma unroll
      for (int k = 0; k < NR; ++k) out[(nY + k) * nc + c] = S[k];
    } else {
#pragma unroll
      for (int k = 0; k < NR; ++k) q[nY + k] = q[nY + k] + S[k];
#pragma unroll
      for (int f = 0; f < nv; ++f) out[f * nc + c] = q[f];
      bits |= finish_state<DIM, CELL>(m, g, fin, q, T, c, amx, amy, dtm, slots);
    }
  }
}

// CELL: the mixed variant's 2D step (per-cell temperature solve)
template <int DIM, bool WRITE_S, bool GEN, bool CELL>
#ifndef JB_CHEM_NT
#define JB_CHEM_NT 128
#endif
#ifndef JB_CHEM_MINB
#define JB_CHEM_MINB (384 / JB_CHEM_NT)
#endif
__global__ void __launch_bounds__(JB_CHEM_NT, JB_CHEM_MINB) k_chem(MP m, Grid g, const double* __restrict__ U,
                                              const double* __restrict__ aux,
                                              double* __restrict__ out, jb_fin fin,
                                              Slots* slots, double dt_arg) {
  extern __shared__ double shc[];
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = WRITE_S ? dt_arg : slots->dt;
  unsigned bits = 0, st = 0;
  double amx = 0.0, amy = 0.0, dtm = __longlong_as_double(0x7ff0000000000000LL);
  if (c < g.ncell) {
    // aux == null (global-stop mode): the temperature is the selected
    // iterate of the previous solve (mask midx - 1), i.e. that solve's
    // select pass is fused here
    const double T = aux ? aux[g.ncell + c] : fin.cand[(long long)halley_count(slots->mask[fin.midx - 1]) * g.ncell + c];
    chem_cell_step<DIM, WRITE_S, GEN, CELL>(m, g, U, T, out, fin, c, dt, shc + threadIdx.x, bits, st, amx, amy, dtm,
                                      slots);
  }
  if (WRITE_S)
    block_reduce_store(0.0, 0.0, 0.0, st << 16, slots, 0, false, false, -1);
  else
    finish_reduce(fin, amx, amy, dtm, bits | (st << 16), slots);
}

// ---------------------------------------------------------------------------
// U_to_prim (solver_{1D,2D}/aux_func.py:39-51): rho, u, [v,] Y, p, a
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void k_prim(MP m, Grid g, const double* __restrict__ U, const double* __restrict__ aux,
                       double* __restrict__ rho_o, double* __restrict__ u_o, double* __restrict__ v_o,
                       double* __restrict__ Y_o, double* __restrict__ p_o, double* __restrict__ a_o) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  constexpr int nv = nY + NR;
  const long long nc = g.ncell;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double q[nv];
#pragma unroll
  for (int f = 0; f < nv; ++f) q[f] = U[f * nc + c];
  Prim<DIM> pr = u_to_prim<DIM>(m, q, aux[c], aux[nc + c]);
  rho_o[c] = pr.rho;
  u_o[c] = pr.u;
  if (DIM == 2) v_o[c] = pr.v;
#pragma unroll
  for (int k = 0; k < NR; ++k) Y_o[k * nc + c] = q[nY + k] / pr.rho;
  p_o[c] = pr.p;
  a_o[c] = pr.a;
}

// ---------------------------------------------------------------------------
// thermo evaluation for state building (thermo_model.get_thermo)
// ---------------------------------------------------------------------------
__global__ void k_thermo(MP m, long long n, const double* __restrict__ T, const double* __restrict__ Y,
                         double* __restrict__ cp, double* __restrict__ gamma, double* __restrict__ h,
                         double* __restrict__ R, double* __restrict__ dcp) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double Y8[NR], Yf[NS];
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = Y[k * n + c];
  fill_Y(Y8, Yf);
  double r = get_R(m, Yf);
  Th t = thermo_mix(m, T[c], Yf);
  cp[c] = t.cp;
  gamma[c] = t.cp / (t.cp - r);
  h[c] = t.h;
  R[c] = r;
  dcp[c] = t.dcp;
}

// ---------------------------------------------------------------------------
// per-step slot bookkeeping (one thread)
// ---------------------------------------------------------------------------
__global__ void k_slots_reset(Slots* s) {
  for (int i = 0; i < 4; ++i) { s->ax[i] = 0ull; s->ay[i] = 0ull; s->mask[i] = 0u; }
  s->dtmin_next = 0x7ff0000000000000ull;
  s->dtnan = 0u;
  s->dt = 0.0;  // status is cleared only when the host reads it (jb_status)
}

// Start of a time step: alpha of stage 1 and the CFL minimum come from the
// previous select pass; dt = CFL * min (set_simulator.py:420-447) or given.
__global__ void k_step_begin(Slots* s, double cfl, double dt_fixed, double* dt_hist, int step) {
  s->ax[0] = s->ax[3];
  s->ay[0] = s->ay[3];
  double dt = cfl > 0.0 ? cfl * (s->dtnan ? __longlong_as_double(0x7ff8000000000000LL)
                                         : bitsd(s->dtmin_next))
                        : dt_fixed;
  s->dtnan = 0u;
  s->dt = dt;
  if (dt_hist) dt_hist[step] = dt;
  for (int i = 1; i < 4; ++i) { s->ax[i] = 0ull; s->ay[i] = 0ull; }
  for (int i = 0; i < 4; ++i) s->mask[i] = 0u;
  s->dtmin_next = 0x7ff0000000000000ull;
}

__global__ void k_dt_from_slots(const Slots* s, double cfl, double* dt_out) {
  *dt_out = cfl * (s->dtnan ? __longlong_as_double(0x7ff8000000000000LL) : bitsd(s->dtmin_next));
}

// ---------------------------------------------------------------------------
// x-slab decomposition (parallel/boundary_padding.py exchange_halo,
// parallel/boundary.py, the pmin of CFL_1D / CFL_2D in set_simulator.py)
// ---------------------------------------------------------------------------
// The 3 edge columns of each x side of (U, aux) as send[2][nv+2][3][ny]:
// side 0 holds columns 0..2 (the left neighbour's right halo), side 1 columns
// nx-3..nx-1 (the right neighbour's left halo), in halo_idx order.
__global__ void __launch_bounds__(256) k_halo_pack(Grid g, const double* __restrict__ U,
                                                   const double* __restrict__ aux, double* __restrict__ send) {
  const long long n = 6LL * (g.nv + 2) * g.ny;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int y = (int)(i % g.ny);
  long long r = i / g.ny;
  const int l = (int)(r % 3);
  r /= 3;
  const int q = (int)(r % (g.nv + 2));
  const int side = (int)(r / (g.nv + 2));
  const long long c = (long long)(side == 0 ? l : g.nx - 3 + l) * g.ny + y;
  send[i] = q < g.nv ? U[q * g.ncell + c] : aux[(q - g.nv) * g.ncell + c];
}

// The 3 edge rows of each y side of (U, aux) as send[2][nv+2][nx][3]:
// side 0 (bottom) rows 0..2, side 1 (top) rows ny-3..ny-1.
__global__ void __launch_bounds__(256) k_halo_pack_y(Grid g, const double* __restrict__ U,
                                                     const double* __restrict__ aux, double* __restrict__ send) {
  const long long n = 6LL * (g.nv + 2) * g.nx;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int l = (int)(i % 3);
  long long r = i / 3;
  const int x = (int)(r % g.nx);
  r /= g.nx;
  const int q = (int)(r % (g.nv + 2));
  const int side = (int)(r / (g.nv + 2));
  const long long c = (long long)x * g.ny + (side == 0 ? l : g.ny - 3 + l);
  send[i] = q < g.nv ? U[q * g.ncell + c] : aux[(q - g.nv) * g.ncell + c];
}

// Wave speeds of caller-computed ghost rows (JB_BC_HALO y sides) into the
// alpha maxima of slot aidx: every row of both ghost layers' columns.
__global__ void __launch_bounds__(128) k_halo_alpha_y(MP m, Grid g, Slots* slots, int aidx) {
  constexpr int nv = 12;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double amx = 0.0, amy = 0.0;
  if (t < 6 * g.nx) {
    const int side = 2 + t / (3 * g.nx), x = (t / 3) % g.nx, l = t % 3;
    if (g.bc[side] == JB_BC_HALO) {
      double q[nv + 2];
#pragma unroll
      for (int f = 0; f < nv + 2; ++f) q[f] = g.haloy[haloy_idx(g, side, l, f, x)];
      Prim<2> pr = u_to_prim<2>(m, q, q[nv], q[nv + 1]);
      amx = fabs(pr.u) + pr.a;
      amy = fabs(pr.v) + pr.a;
    }
  }
  block_reduce_store(amx, amy, 0.0, 0u, slots, aidx, true, false, -1);
}

// Wave speeds of the received ghost columns into the LF alpha maxima of slot
// aidx (flux_splitting/LF.py takes nanmax over the padded array).  A halo
// side contributes every row; a physical x side of a 2D slab only the rows
// its padded corners copy (y-periodic wrap: 1..3 and ny-4..ny-2), because the
// boundary condition overwrites the ghost columns' rows 3:-3 only.  Without
// the ring (caller-computed ghost columns) the corners are the single-domain
// periodic wrap of interior cells and add nothing.
template <int DIM>
__global__ void __launch_bounds__(128) k_halo_alpha(MP m, Grid g, Slots* slots, int aidx) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  constexpr int nv = nY + NR;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double amx = 0.0, amy = 0.0;
  if (t < 6 * g.ny) {
    const int side = t / (3 * g.ny), l = (t / g.ny) % 3, y = t % g.ny;
    const bool corner_row = (y >= 1 && y <= 3) || (y >= g.ny - 4 && y <= g.ny - 2);
    if (g.bc[side] == JB_BC_HALO || (DIM == 2 && g.halo_ring && corner_row)) {
      double q[nv + 2];
#pragma unroll
      for (int f = 0; f < nv + 2; ++f) q[f] = g.halo[halo_idx(g, side, l, f, y)];
      Prim<DIM> pr = u_to_prim<DIM>(m, q, q[nv], q[nv + 1]);
      amx = fabs(pr.u) + pr.a;
      amy = fabs(pr.v) + pr.a;
    }
  }
  block_reduce_store(amx, amy, 0.0, 0u, slots, aidx, true, false, -1);
}

// The CFL minimum and NaN flag as an int64 pair whose MIN over the ranks is
// the global pair: red[0] the bits of the (non-negative) minimum, red[1]
// minus the NaN flag.
__global__ void k_dt_pack(const Slots* s, long long* red) {
  red[0] = (long long)s->dtmin_next;
  red[1] = -(long long)s->dtnan;
}

__global__ void k_dt_unpack(Slots* s, const long long* red) {
  s->dtmin_next = (unsigned long long)red[0];
  s->dtnan = red[1] != 0 ? 1u : 0u;
}

#include "jb_godunov.cuh"
#include "jb_viscous.cuh"

}  // namespace
}  // namespace JB_NS
}  // namespace jb
