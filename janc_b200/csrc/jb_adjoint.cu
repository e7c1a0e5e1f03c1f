// Hand-written reverse-mode kernels of the reacting step (the adjoint), 2D
// and 1D (every kernel is a template on DIM; 1D has no y direction, the
// energy at field 2 and the species from field 3).
//
// The forward step being differentiated is the reference's advance_one_step
// (set_simulator.py:117-122) with its CFL time step (set_simulator.py:
// 420-447):
//   dt = CFL min 1/(sx/dx + sy/dy)  (2D),  CFL min dx/sx  (1D)   over (U, aux)
//   U1 = U  + dt L(U,  aux;  a1)           aux1 = update_aux(U1)
//   U2 = 3/4 U + 1/4 (U1 + dt L(U1, aux1; a2))   aux2 = update_aux(U2)
//   U3 = 1/3 U + 2/3 (U2 + dt L(U2, aux2; a3))   aux3 = update_aux(U3)
//   U4 = U3 + S(U3, T3, dt)                aux4 = update_aux(U4)
// with L = -(dF/dx + dG/dy) from LF splitting (a_k = max over the padded
// grid of |u|+a resp. |v|+a) and WENO5-JS, and S the point-implicit
// chemistry.  Derivative conventions are those of jax.grad of the
// reference: update_aux differentiates through get_T's custom VJP
// (thermo_model.py:155-190: implicit derivatives at the converged T, none
// through the initial guess), max / min split their gradient evenly among
// tied entries (entries within a relative 1e-13 count as tied), clip
// passes the gradient to whichever bound is active.
//
// Kernels (one thread per cell unless noted), in the order of one step:
//   k_vjp_begin     the probe term of the loss and update_aux of U4; the
//                   primitives and alpha / CFL tie counts of U, U1, U2
//   k_outlet_ghosts (pressure-outlet sides) the outlet ghost states of U,
//                   U1, U2 and their alpha tie counts
//   k_chem_vjp      chemistry: Ubar3 = Ubar4 + dS/dU3^T Ubar4, with the
//                   temperature, dt and ln A adjoints, then update_aux of U3
//   per RK stage (3, 2, 1):
//   k_flux_sweep    one thread per (direction, line, segment, field): the
//                   WENO5 / LF face adjoints along the line (registers only)
//   k_outlet_vjp    (pressure-outlet sides) the outlet ghosts' adjoints
//                   into their boundary cells
//   k_stage_merge   flux-function VJPs, ghost copies, RK combination, alpha
//                   (and CFL) ties, update_aux of the stage state
//   k_init_vjp      initial state from (P, T, Y): T adjoint
#define JB_NS adj
#define JB_FAST 1
#include "jb_kernels.cuh"

#include "jb_adjoint.h"

namespace jb {
namespace adj {

constexpr double TIE_REL = 1e-13;

// field layout of a DIM-D state: species from NYD, energy at EI, NVD fields
template <int DIM>
struct Lay {
  static constexpr int NY = DIM == 1 ? 3 : 4, EI = NY - 1, NV = NY + NR;
};

template <int N>
__device__ __forceinline__ void poly_d(const double* c, double T, double& p, double& dp) {
  p = c[0];
  dp = 0.0;
#pragma unroll
  for (int i = 1; i < N; ++i) {
    dp = dp * T + p;
    p = p * T + c[i];
  }
}

// ---------------------------------------------------------------------------
// get_T_bwd (thermo_model.py:155-190) at temperature T and mass fractions Yf
// ---------------------------------------------------------------------------
struct TBwd {
  double dT_de, dg_de;
  double dT_dY[NR], dg_dY[NR];
};

__device__ __forceinline__ void t_bwd(const MP& m, double T, const double* Yf, TBwd& o) {
  double cp = 0.0, dcp = 0.0, R = 0.0, cpi[NS], ei[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const bool lo = T < m.Tcr[k];
    const double cpk = lo ? poly5(m.cp_lo[k], T) : poly5(m.cp_hi[k], T);
    const double dck = lo ? poly4(m.dcp_lo[k], T) : poly4(m.dcp_hi[k], T);
    const double hk = lo ? poly6(m.h_lo[k], T) : poly6(m.h_hi[k], T);
    cp += cpk * Yf[k];
    dcp += dck * Yf[k];
    R += m.invM[k] * Yf[k];
    cpi[k] = cpk;
    ei[k] = hk - m.invM[k] * T;
  }
  const double cv = cp - R;
  const double icv2 = 1.0 / (cv * cv);
  o.dT_de = 1.0 / cv;
  const double dg_dT = (dcp * cv - dcp * cp) * icv2;
  o.dg_de = dg_dT * o.dT_de;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double dT_dY = (-ei[k] + ei[NR]) / cv;
    const double dR_dY = m.invM[k] - m.invM[NR];
    const double dcp_dY = cpi[k] - cpi[NR];
    const double dcv_dY = dcp_dY - dR_dY;
    o.dT_dY[k] = dT_dY;
    o.dg_dY[k] = dg_dT * dT_dY + (dcp_dY * cv - dcv_dY * cp) * icv2;
  }
}

// Mass fractions of a cell.
template <int DIM>
__device__ __forceinline__ void cell_Y(const double* q, double ri, double* Y8, double* Yf) {
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = q[Lay<DIM>::NY + k] * ri;
  fill_Y(Y8, Yf);
}

// ub += d(gamma, T)/dq^T (gb, Tb) for aux = update_aux(q)
// (solver_2D/aux_func.py:21-29, solver_1D/aux_func.py:21-28)
template <int DIM>
__device__ __forceinline__ void upd_vjp(const MP& m, const double* q, double T, double gb, double Tb, double* ub) {
  constexpr int NY = Lay<DIM>::NY, EI = Lay<DIM>::EI;
  if (gb == 0.0 && Tb == 0.0) return;
  const double rho = q[0], ri = 1.0 / rho;
  const double u = q[1] * ri, v = DIM == 2 ? q[2] * ri : 0.0;
  double Y8[NR], Yf[NS];
  cell_Y<DIM>(q, ri, Y8, Yf);
  TBwd b;
  t_bwd(m, T, Yf, b);
  const double eb = gb * b.dg_de + Tb * b.dT_de;
  double rb = eb * (-q[EI] * ri * ri + (u * u + v * v) * ri);
  ub[1] += eb * (-u * ri);
  if (DIM == 2) ub[2] += eb * (-v * ri);
  ub[EI] += eb * ri;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double yb = gb * b.dg_dY[k] + Tb * b.dT_dY[k];
    ub[NY + k] += yb * ri;
    rb -= yb * Y8[k] * ri;
  }
  ub[0] += rb;
}

// Adjoint of s = |u_dir| + a, a = sqrt(gamma p / rho), p = rho R T, with
// weight w: ub, gb, Tb accumulate.
template <int DIM>
__device__ __forceinline__ void speed_vjp(const MP& m, const double* q, double gamma, double T, int dir, double w,
                                          double* ub, double& gb, double& Tb) {
  constexpr int NY = Lay<DIM>::NY;
  if (w == 0.0) return;
  const double rho = q[0], ri = 1.0 / rho;
  double Y8[NR], Yf[NS];
  cell_Y<DIM>(q, ri, Y8, Yf);
  const double R = get_R(m, Yf);
  const double p = rho * R * T;
  const double a = sqrt(gamma * p / rho);
  const double un = q[dir] * ri;
  const double sg = un > 0.0 ? 1.0 : (un < 0.0 ? -1.0 : 0.0);
  const double unb = w * sg;
  gb += w * a / (2.0 * gamma);
  const double pb = w * a / (2.0 * p);
  double rb = -w * a / (2.0 * rho) + pb * R * T;
  const double Rb = pb * rho * T;
  Tb += pb * rho * R;
  ub[dir] += unb * ri;
  rb -= unb * un * ri;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double yb = Rb * (m.invM[k] - m.invM[NR]);
    ub[NY + k] += yb * ri;
    rb -= yb * Y8[k] * ri;
  }
  ub[0] += rb;
}

// block-wide sum into a global double (all threads call)
__device__ __forceinline__ void block_add(double v, double* dst) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int nt = blockDim.x * blockDim.y;
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  if ((t & 31) == 0) red[t >> 5] = v;
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    for (int i = 0; i < (nt + 31) / 32; ++i) s += red[i];
    if (s != 0.0) atomicAdd(dst, s);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// update_aux VJP over a whole state: Ubar += ..., abar consumed (zeroed)
// ---------------------------------------------------------------------------
// chemistry VJP (reaction_model.py:91-193)
// ---------------------------------------------------------------------------
// PA = LU of an 8x8 A in place (multipliers below the diagonal), partial
// pivoting with selects; piv[c] is the row exchanged with row c at step c.
__device__ __forceinline__ void lu8(double (&A)[NR][NR], int (&piv)[NR]) {
#pragma unroll
  for (int c = 0; c < NR; ++c) {
    int p = c;
    double best = fabs(A[c][c]);
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r > c) {
        const double v = fabs(A[r][c]);
        if (v > best) { best = v; p = r; }
      }
    piv[c] = p;
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r > c) {
        const bool sw = p == r;
#pragma unroll
        for (int j = 0; j < NR; ++j) {
          const double x0 = A[c][j], x1 = A[r][j];
          A[c][j] = sw ? x1 : x0;
          A[r][j] = sw ? x0 : x1;
        }
      }
    const double ip = 1.0 / A[c][c];
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r > c) {
        const double l = A[r][c] * ip;
        A[r][c] = l;
#pragma unroll
        for (int j = 0; j < NR; ++j)
          if (j > c) A[r][j] = A[r][j] - l * A[c][j];
      }
  }
}

// x = A^-1 b from lu8's factors
__device__ __forceinline__ void lu8_solve(const double (&A)[NR][NR], const int (&piv)[NR], const double* b,
                                          double* x) {
  double y[NR];
#pragma unroll
  for (int i = 0; i < NR; ++i) y[i] = b[i];
#pragma unroll
  for (int c = 0; c < NR; ++c)
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r > c) {
        const bool sw = piv[c] == r;
        const double y0 = y[c], y1 = y[r];
        y[c] = sw ? y1 : y0;
        y[r] = sw ? y0 : y1;
      }
#pragma unroll
  for (int i = 0; i < NR; ++i)
#pragma unroll
    for (int j = 0; j < NR; ++j)
      if (j < i) y[i] = y[i] - A[i][j] * y[j];
#pragma unroll
  for (int ii = 0; ii < NR; ++ii) {
    const int i = NR - 1 - ii;
    double t = y[i];
#pragma unroll
    for (int j = 0; j < NR; ++j)
      if (j > i) t = t - A[i][j] * x[j];
    x[i] = t / A[i][i];
  }
}

// y = A^-T c from lu8's factors (A^T = U^T L^T P)
__device__ __forceinline__ void lu8_solve_t(const double (&A)[NR][NR], const int (&piv)[NR], const double* c,
                                            double* y) {
  double z[NR];
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    double t = c[i];
#pragma unroll
    for (int j = 0; j < NR; ++j)
      if (j < i) t = t - A[j][i] * z[j];
    z[i] = t / A[i][i];
  }
#pragma unroll
  for (int ii = 0; ii < NR; ++ii) {
    const int i = NR - 1 - ii;
#pragma unroll
    for (int j = 0; j < NR; ++j)
      if (j > i) z[i] = z[i] - A[j][i] * z[j];
  }
#pragma unroll
  for (int cc = 0; cc < NR; ++cc) {
    const int k = NR - 1 - cc;
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r > k) {
        const bool sw = piv[k] == r;
        const double z0 = z[k], z1 = z[r];
        z[k] = sw ? z1 : z0;
        z[r] = sw ? z0 : z1;
      }
  }
#pragma unroll
  for (int i = 0; i < NR; ++i) y[i] = z[i];
}

constexpr int CHEM_ADJ_NT = 128;
constexpr int CHEM_ADJ_SH = 3 * NREAC;  // kf, kb, M per reaction

// Per cell: Ub3 = Ub4 + (dS/dU3)^T Ub4, then update_aux(U3)'s VJP with the
// chemistry's temperature adjoint; dt and ln A adjoints are reduced into
// dtb and lnAb.  Rates in log space: kf = exp(ln A + B ln T - Ea/T +
// sum vf ln X), kb = exp(ln kf0 - sum dv g - vsum ln(pref/T) + sum vb ln X).
template <int DIM>
__global__ void __launch_bounds__(CHEM_ADJ_NT, 2)
    k_chem_vjp(MP m, Grid g, const double* __restrict__ U3, const double* __restrict__ A3, const double* Ub4,
               double* Ub3, const double* __restrict__ slot_dt, double* dtb, double* lnAb) {
  constexpr int NY = Lay<DIM>::NY, NVD = Lay<DIM>::NV;
  extern __shared__ double shk[];
  const long long nc = g.ncell;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int NT = blockDim.x;
  double* sh = shk + threadIdx.x;
  const double dt = *slot_dt;
  double dtb_loc = 0.0;
  double* sA = shk + CHEM_ADJ_SH * NT + threadIdx.x;  // ln A adjoint per reaction, this thread's column
#pragma unroll 1
  for (int i = 0; i < NREAC; ++i) sA[i * NT] = 0.0;
  if (c < nc) {
    double q[NVD];
#pragma unroll
    for (int f = 0; f < NVD; ++f) q[f] = U3[f * nc + c];
    const double T = A3[nc + c];
    const double rho = q[0], ri = 1.0 / rho;
    double Y8[NR], Yf[NS], X[NS], Xc[NR], lnXc[NR], iXc[NR], gg[NR], dg[NR];
    cell_Y<DIM>(q, ri, Y8, Yf);
#pragma unroll
    for (int j = 0; j < NS; ++j) X[j] = rho * Yf[j] * m.invM[j];
#pragma unroll
    for (int n = 0; n < NR; ++n) {
      Xc[n] = X[n] < 1e-50 ? 1e-50 : X[n];
      lnXc[n] = log(Xc[n]);
      iXc[n] = 1.0 / Xc[n];
    }
    const double lT = log(T), iT = 1.0 / T;
    const double lT0T = lT + m.lnT0;
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const bool lo = T < m.Tcr[k];
      double s, ds, h, dh;
      poly_d<5>(lo ? m.s_lo[k] : m.s_hi[k], T, s, ds);
      poly_d<6>(lo ? m.hc_lo[k] : m.hc_hi[k], T, h, dh);
      const double lg = lo ? m.lg_lo[k] : m.lg_hi[k];
      gg[k] = s + lg * lT0T - h * iT;
      dg[k] = ds + lg * iT - dh * iT + h * iT * iT;
    }
    double w[NR], J[NR][NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      w[k] = 0.0;
#pragma unroll
      for (int n = 0; n < NR; ++n) J[k][n] = 0.0;
    }
#pragma unroll 1
    for (int i = 0; i < NREAC; ++i) {
      const double lkf0 = m.lnA[i] + m.B[i] * lT - m.EaR[i] * iT;
      double Ms = 1.0;
      if (m.is_tb[i] != 0.0) {
        Ms = 0.0;
#pragma unroll
        for (int j = 0; j < NS; ++j) Ms += m.tb[i][j] * X[j];
      }
      double sf = 0.0, sb = 0.0, sg = 0.0;
#pragma unroll
      for (int n = 0; n < NR; ++n) {
        sf += m.vf[i][n] * lnXc[n];
        sb += m.vb[i][n] * lnXc[n];
        sg += m.dv[i][n] * gg[n];
      }
      const double kf = exp(lkf0 + sf);
      const double kb = exp(lkf0 - sg - m.vsum[i] * (m.lnpref - lT) + sb);
      sh[(3 * i + 0) * NT] = kf;
      sh[(3 * i + 1) * NT] = kb;
      sh[(3 * i + 2) * NT] = Ms;
      const double net = kf - kb;
      double tn[NR];
#pragma unroll
      for (int n = 0; n < NR; ++n)
        tn[n] = net * m.tbinvM[i][n] + Ms * (m.vf[i][n] * kf - m.vb[i][n] * kb) * m.invM[n] * iXc[n];
#pragma unroll
      for (int k = 0; k < NR; ++k) {
        const double dvk = m.dv[i][k];
        if (dvk == 0.0) continue;
        const double mk = m.M[k] * dvk;
        w[k] += mk * Ms * net;
#pragma unroll
        for (int n = 0; n < NR; ++n) J[k][n] += mk * tn[n];
      }
    }
    const double idt = 1.0 / dt;
#pragma unroll
    for (int k = 0; k < NR; ++k)
#pragma unroll
      for (int n = 0; n < NR; ++n) J[k][n] = (k == n ? idt : 0.0) - J[k][n];  // J now holds A
    int piv[NR];
    lu8(J, piv);
    double x[NR];
    lu8_solve(J, piv, w, x);
    // S = rho clip(x / rho, -Y, 1 - Y)
    double rb = 0.0, Y8b[NR], xb[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const double Sb = Ub4[(NY + k) * nc + c];
      const double dY = x[k] * ri;
      const double lo = -Y8[k], hi = 1.0 - Y8[k];
      const double m1 = dY < lo ? lo : dY;
      const double cl = m1 > hi ? hi : m1;
      rb += Sb * cl;
      const double clb = rho * Sb;
      double dYb = 0.0;
      Y8b[k] = 0.0;
      if (m1 > hi) Y8b[k] -= clb;
      else if (dY < lo) Y8b[k] -= clb;
      else dYb = clb;
      xb[k] = dYb * ri;
      rb -= dYb * dY * ri;
    }
    double bb[NR];
    lu8_solve_t(J, piv, xb, bb);  // bbar = A^-T xbar
#pragma unroll
    for (int k = 0; k < NR; ++k) dtb_loc += bb[k] * x[k] * idt * idt;
    double Xb[NS], Xcb[NR], gb[NR], Tb = 0.0;
#pragma unroll
    for (int j = 0; j < NS; ++j) Xb[j] = 0.0;
#pragma unroll
    for (int n = 0; n < NR; ++n) { Xcb[n] = 0.0; gb[n] = 0.0; }
    double xw[NR];
#pragma unroll
    for (int n = 0; n < NR; ++n) xw[n] = x[n] * m.invM[n];
#pragma unroll 1
    for (int i = 0; i < NREAC; ++i) {
      double beta = 0.0;
#pragma unroll
      for (int k = 0; k < NR; ++k) beta += bb[k] * m.M[k] * m.dv[i][k];
      if (beta == 0.0) continue;
      const double kf = sh[(3 * i + 0) * NT], kb = sh[(3 * i + 1) * NT], Ms = sh[(3 * i + 2) * NT];
      double sF = 0.0, sB = 0.0, sMb = kf - kb;
#pragma unroll
      for (int n = 0; n < NR; ++n) {
        const double vfn = m.vf[i][n], vbn = m.vb[i][n], tbn = m.tb[i][n];
        sF += xw[n] * (tbn + Ms * vfn * iXc[n]);
        sB += xw[n] * (tbn + Ms * vbn * iXc[n]);
        const double d = vfn * kf - vbn * kb;
        sMb += xw[n] * d * iXc[n];
        Xcb[n] -= beta * Ms * xw[n] * d * iXc[n] * iXc[n];
      }
      const double kfb = beta * (Ms + sF);
      const double kbb = -beta * (Ms + sB);
      const double Mb = beta * sMb;
      if (m.is_tb[i] != 0.0) {
#pragma unroll
        for (int j = 0; j < NS; ++j) Xb[j] += Mb * m.tb[i][j];
      }
      const double fkf = kfb * kf, fkb = kbb * kb;
#pragma unroll
      for (int n = 0; n < NR; ++n) {
        Xcb[n] += (fkf * m.vf[i][n] + fkb * m.vb[i][n]) * iXc[n];
        gb[n] -= fkb * m.dv[i][n];
      }
      const double a0 = fkf + fkb;  // adjoint of ln kf0 (and of ln A_i)
      Tb += fkb * m.vsum[i] * iT + a0 * (m.B[i] * iT + m.EaR[i] * iT * iT);
      sA[i * NT] += a0;
    }
#pragma unroll
    for (int n = 0; n < NR; ++n) {
      Tb += gb[n] * dg[n];
      if (X[n] > 1e-50) Xb[n] += Xcb[n];
    }
    double Yfb[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) {
      const double ryb = Xb[j] * m.invM[j];
      rb += ryb * Yf[j];
      Yfb[j] = rho * ryb;
    }
    double ub[NVD];
#pragma unroll
    for (int f = 0; f < NVD; ++f) ub[f] = Ub4[f * nc + c];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const double yb = Y8b[k] + Yfb[k] - Yfb[NR];
      ub[NY + k] += yb * ri;
      rb -= yb * Y8[k] * ri;
    }
    ub[0] += rb;
    upd_vjp<DIM>(m, q, T, 0.0, Tb, ub);
#pragma unroll
    for (int f = 0; f < NVD; ++f) Ub3[f * nc + c] = ub[f];
  }
  block_add(dtb_loc, dtb);
#pragma unroll 1
  for (int i = 0; i < NREAC; ++i) block_add(sA[i * NT], lnAb + i);
}

// ---------------------------------------------------------------------------
// WENO5-JS value and partial derivatives (reconstruction/WENO5_JS.py)
// ---------------------------------------------------------------------------
// f = sum_k w_k q_k over v0..v4 (the left-biased form; the right-biased
// reconstruction is the same function of the mirrored stencil).
__device__ __forceinline__ double weno_d(double v0, double v1, double v2, double v3, double v4, double* dv) {
  const double d1 = v0 - 4.0 * v1 + 3.0 * v2, e1 = v0 - 2.0 * v1 + v2;
  const double d2 = v1 - v3, e2 = v1 - 2.0 * v2 + v3;
  const double d3 = 3.0 * v2 - 4.0 * v3 + v4, e3 = v2 - 2.0 * v3 + v4;
  const double b1 = 0.25 * d1 * d1 + 13.0 / 12.0 * e1 * e1;
  const double b2 = 0.25 * d2 * d2 + 13.0 / 12.0 * e2 * e2;
  const double b3 = 0.25 * d3 * d3 + 13.0 / 12.0 * e3 * e3;
  const double s1 = 1e-6 + b1, s2 = 1e-6 + b2, s3 = 1e-6 + b3;
  // one division for the three reciprocals (s_k lies in [1e-6, ~1e20])
  const double s12 = s1 * s2, r = 1.0 / (s12 * s3);
  const double i1 = s2 * s3 * r, i2 = s1 * s3 * r, i3 = s12 * r;
  const double a1 = 0.1 * i1 * i1, a2 = 0.6 * i2 * i2, a3 = 0.3 * i3 * i3;
  const double iS = 1.0 / (a1 + a2 + a3);
  const double w1 = a1 * iS, w2 = a2 * iS, w3 = a3 * iS;
  const double q1 = 1.0 / 3.0 * v0 - 7.0 / 6.0 * v1 + 11.0 / 6.0 * v2;
  const double q2 = -1.0 / 6.0 * v1 + 5.0 / 6.0 * v2 + 1.0 / 3.0 * v3;
  const double q3 = 1.0 / 3.0 * v2 + 5.0 / 6.0 * v3 - 1.0 / 6.0 * v4;
  const double f = w1 * q1 + w2 * q2 + w3 * q3;
  const double g1 = -2.0 * w1 * (q1 - f) * i1;
  const double g2 = -2.0 * w2 * (q2 - f) * i2;
  const double g3 = -2.0 * w3 * (q3 - f) * i3;
  dv[0] = w1 * (1.0 / 3.0) + g1 * (0.5 * d1 + 13.0 / 6.0 * e1);
  dv[1] = w1 * (-7.0 / 6.0) + w2 * (-1.0 / 6.0) + g1 * (-2.0 * d1 - 13.0 / 3.0 * e1) + g2 * (0.5 * d2 + 13.0 / 6.0 * e2);
  dv[2] = w1 * (11.0 / 6.0) + w2 * (5.0 / 6.0) + w3 * (1.0 / 3.0) + g1 * (1.5 * d1 + 13.0 / 6.0 * e1) +
          g2 * (-13.0 / 3.0 * e2) + g3 * (1.5 * d3 + 13.0 / 6.0 * e3);
  dv[3] = w2 * (1.0 / 3.0) + w3 * (5.0 / 6.0) + g2 * (-0.5 * d2 + 13.0 / 6.0 * e2) + g3 * (-2.0 * d3 - 13.0 / 3.0 * e3);
  dv[4] = w3 * (-1.0 / 6.0) + g3 * (0.5 * d3 + 13.0 / 6.0 * e3);
  return f;
}

// ---------------------------------------------------------------------------
// alpha (max over the padded grid) and CFL (min over cells) ties
// ---------------------------------------------------------------------------
struct Speeds {
  double sx, sy, d;
};

// wave speeds and the CFL candidate: 1 / (sx/dx + sy/dy) in 2D, dx / sx in 1D
template <int DIM>
__device__ __forceinline__ Speeds speeds_of(const Grid& g, const Prim<DIM>& pr) {
  Speeds s;
  s.sx = fabs(pr.u) + pr.a;
  s.sy = fabs(pr.v) + pr.a;
  s.d = DIM == 1 ? g.dx / s.sx : 1.0 / (s.sx / g.dx + s.sy / g.dy);
  return s;
}

__device__ __forceinline__ bool tied(double v, double ref) { return fabs(v - ref) <= TIE_REL * fabs(ref); }

// ---------------------------------------------------------------------------
// pressure-outlet sides (boundary_conditions_2D/pressure_outlet.py:5-66)
// ---------------------------------------------------------------------------
// The 3 ghost layers of an outlet side all hold the outlet state of the
// side's boundary cell.  They are padded entries of their own: the sweeps
// read them (og), the alpha maxima see their wave speeds (3 entries per
// boundary position), and their adjoints (flux, LF term, wave speeds) flow
// back into the boundary cell through the VJP of the outlet state (ogb).
//   og [stage][side][OG_F][lstrip]: ghost U (nv), then u, v, p at OG_U..OG_P
//   ogb[side][OG_B][lstrip]: the boundary cell's U adjoint (nv), T adjoint at
//   OG_T, gamma adjoint at OG_G (the blocked injector copies the cell's gamma)
// The rotating-detonation injector of the bottom side (2D) is handled the same
// way: its 3 ghost layers hold the injector state of the boundary cell.
constexpr int OG_F = 15, OG_B = 14, OG_U = 12, OG_V = 13, OG_P = 14, OG_T = 12, OG_G = 13;

__device__ __forceinline__ size_t og_idx(const Grid& g, int stage, int side, int f, int pos) {
  return (((size_t)stage * 4 + side) * OG_F + f) * g.lstrip + pos;
}

__device__ __forceinline__ bool outlet_side(const Grid& g, int side) {
  return g.bc[side] == JB_BC_PRESSURE_OUTLET;
}

// a side whose ghosts are states of their own (pressure outlet, injector)
__device__ __forceinline__ bool strip_side(const Grid& g, int side) {
  return g.bc[side] == JB_BC_PRESSURE_OUTLET || (side == 2 && g.bc[side] == JB_BC_RDC_INJECTOR);
}


// Boundary position t in [0, 2 ny + 2 nx): sides 0 and 1 (x = 0, nx - 1) by
// y, then sides 2 and 3 (y = 0, ny - 1) by x; side -1 past the end.
// In 1D only sides 0 and 1 (t = 0, 1).
template <int DIM>
__device__ __forceinline__ void boundary_pos(const Grid& g, int t, int& side, int& pos, int& x, int& y) {
  side = -1;
  pos = 0;
  if (t < 2 * g.ny) {
    side = t / g.ny;
    pos = t % g.ny;
  } else if (DIM == 2 && t < 2 * g.ny + 2 * g.nx) {
    side = 2 + (t - 2 * g.ny) / g.nx;
    pos = (t - 2 * g.ny) % g.nx;
  }
  x = side == 0 ? 0 : side == 1 ? g.nx - 1 : pos;
  y = side == 2 ? 0 : side == 3 ? g.ny - 1 : pos;
}

// normal velocity of boundary cell q, positive out of the domain
__device__ __forceinline__ double outlet_un(const double* q, int side) {
  const double un = (side < 2 ? q[1] : q[2]) / q[0];
  return (side == 0 || side == 2) ? -un : un;
}

// The ghost state (U, gamma, T) of strip side `side` at boundary cell q.
template <int DIM>
__device__ __forceinline__ void strip_state(const MP& m, const Grid& g, int side, int pos, const double* q,
                                            double gamma, double T, double* gs) {
  if constexpr (DIM == 2) {
    if (g.bc[side] == JB_BC_RDC_INJECTOR) {
      double Yi[NR];
#pragma unroll
      for (int k = 0; k < NR; ++k) Yi[k] = g.Yinj[k * g.nx + pos];
      injector_state(m, q, gamma, T, Yi, g.inj_block_p, gs);
      return;
    }
  }
  pressure_outlet_state<DIM>(m, q, gamma, T, outlet_un(q, side), g.Pb, gs);
}

// ub, Tb += the VJP of the outlet state (pressure_outlet.py:5-22) of boundary
// cell q with aux (gamma, T), given the adjoints of the ghost state (ob), of
// its gamma (gcb) and of its T (Tcb).  The subsonic / supersonic switch has
// no derivative and Pb is a parameter; gamma of the cell only enters the
// switch.  Subsonic: rho_c = Pb / (p / rho), p_c = Pb, T_c = p_c / (rho_c R);
// supersonic: the cell's rho, p, T.  Both: the ghost energy rho_c h(T_c) -
// p_c + rho_c |u|^2 / 2 and gamma_c = cp(T_c) / (cp(T_c) - R).
template <int DIM>
__device__ void outlet_vjp(const MP& m, const double* q, double gamma, double T, double un, double Pb,
                           const double* ob, double gcb, double Tcb, double* ub, double& Tb) {
  constexpr int NY = Lay<DIM>::NY, EI = Lay<DIM>::EI;
  const double rho = q[0], ri = 1.0 / rho;
  const double u = q[1] * ri, v = DIM == 2 ? q[2] * ri : 0.0;
  double Y8[NR], Yf[NS];
  cell_Y<DIM>(q, ri, Y8, Yf);
  const double R = get_R(m, Yf);
  const double p = rho * (R * T);
  const double a = sqrt(gamma * p / rho);
  const bool sub = un / a < 1.0;
  const double w = p / rho;
  const double rho_c = sub ? Pb / w : rho;
  const double T_c = sub ? Pb * 1.0 / (rho_c * R) : T;
  double cp = 0.0, dcp = 0.0, h = 0.0, cpi[NS], hi[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const bool lo = T_c < m.Tcr[k];
    cpi[k] = lo ? poly5(m.cp_lo[k], T_c) : poly5(m.cp_hi[k], T_c);
    hi[k] = lo ? poly6(m.h_lo[k], T_c) : poly6(m.h_hi[k], T_c);
    const double dck = lo ? poly4(m.dcp_lo[k], T_c) : poly4(m.dcp_hi[k], T_c);
    cp += cpi[k] * Yf[k];
    dcp += dck * Yf[k];
    h += hi[k] * Yf[k];
  }
  const double cv = cp - R, icv2 = 1.0 / (cv * cv);
  // ghost = [rho_c, rho_c u, (rho_c v,) rho_c h - p_c + rho_c ke, rho_c Y8]
  const double ke = 0.5 * (u * u + v * v);
  const double ob2 = DIM == 2 ? ob[2] : 0.0;
  double rcb = ob[0] + ob[1] * u + ob2 * v + ob[EI] * (h + ke);
  double Y8b[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    rcb += ob[NY + k] * Y8[k];
    Y8b[k] = ob[NY + k] * rho_c;
  }
  const double ubl = (ob[1] + ob[EI] * u) * rho_c, vbl = (ob2 + ob[EI] * v) * rho_c;
  const double hb = ob[EI] * rho_c, pcb = -ob[EI];
  // gamma_c = cp / (cp - R), h = sum h_k Y_k, cp = sum cp_k Y_k at T_c
  const double cpb = -gcb * R * icv2;
  double Rb = gcb * cp * icv2;
  const double Tct = Tcb + hb * cp + cpb * dcp;
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8b[k] += hb * (hi[k] - hi[NR]) + cpb * (cpi[k] - cpi[NR]);
  double rb, pb, Tl;
  if (sub) {
    // T_c = Pb / (rho_c R), rho_c = Pb / w, w = p / rho
    const double rcb2 = rcb - Tct * T_c / rho_c;
    Rb -= Tct * T_c / R;
    const double wb = -rcb2 * rho_c / w;
    pb = wb * ri;
    rb = -wb * w * ri;
    Tl = 0.0;
  } else {
    rb = rcb;
    pb = pcb;
    Tl = Tct;
  }
  // p = rho R T, R = sum Y_k / M_k
  rb += pb * R * T;
  Rb += pb * rho * T;
  Tl += pb * rho * R;
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8b[k] += Rb * (m.invM[k] - m.invM[NR]);
  ub[1] += ubl * ri;
  if (DIM == 2) ub[2] += vbl * ri;
  rb -= (ubl * u + vbl * v) * ri;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    ub[NY + k] += Y8b[k] * ri;
    rb -= Y8b[k] * Y8[k] * ri;
  }
  ub[0] += rb;
  Tb += Tl;
}

// ub, Tb, gb += the VJP of the rotating-detonation injector state of boundary
// cell q with aux (gamma, T) (examples/janc_basic_example2.ipynb
// bottom_boundary + inj_model, after Fievisohn et al. 2017), given the
// adjoints of the ghost U (ob), its gamma (gcb) and its T (Tcb).  The
// bisection's Mach number, the blocked / open switch (p >= block_p) and Yinj
// carry no derivative (comparisons and jnp.where selections of constants in
// the reference).  Open: rho_c = p / (R_i T_i), u_c = 0, v_c = V3,
// T_c = T_i = p / (R_i rho_i), rho_i = MFC / V3 / A3, V3 = -B + sqrt(B^2 - 2C),
// B = g/(g-1) p A3 / MFC, and the ghost energy rho_c h_i - p + rho_c V3^2 / 2
// with gamma_c = cp(T_i) / (cp(T_i) - R_i).  Blocked: the cell's rho, u, -v,
// T and gamma, the ghost energy rho h(T) - p + rho |u|^2 / 2.
__device__ void injector_vjp(const MP& m, const double* q, double gamma, double T, const double* Yinj8,
                             double block_p, const double* ob, double gcb, double Tcb, double* ub, double& Tb,
                             double& gb) {
  (void)gamma;
  const double rho = q[0], ri = 1.0 / rho;
  const double u = q[1] * ri, v = q[2] * ri;
  double Y8[NR], Yf[NS], Y8b[NR];
  cell_Y<2>(q, ri, Y8, Yf);
  const double R = get_R(m, Yf);
  const double p = rho * R * T;
  double rb = 0.0, pb = 0.0;
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8b[k] = 0.0;
  if (p >= block_p) {
    double h = 0.0, cp = 0.0, hk[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const bool lo = T < m.Tcr[k];
      hk[k] = lo ? poly6(m.h_lo[k], T) : poly6(m.h_hi[k], T);
      const double cpk = lo ? poly5(m.cp_lo[k], T) : poly5(m.cp_hi[k], T);
      h += hk[k] * Yf[k];
      cp += cpk * Yf[k];
    }
    // ghost = [rho, rho u, rho (-v), rho h - p + rho (u^2 + v^2) / 2, rho Y8]
    const double ubl = ob[1] * rho + ob[3] * rho * u;
    const double vbl = -ob[2] * rho + ob[3] * rho * v;
    rb += ob[0] + ob[1] * u - ob[2] * v + ob[3] * (h + 0.5 * (u * u + v * v));
    const double hb = ob[3] * rho;
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      rb += ob[4 + k] * Y8[k];
      Y8b[k] += ob[4 + k] * rho + hb * (hk[k] - hk[NR]);
    }
    Tb += hb * cp + Tcb;
    pb -= ob[3];
    gb += gcb;
    ub[1] += ubl * ri;
    ub[2] += vbl * ri;
    rb -= (ubl * u + vbl * v) * ri;
  } else {
    double Yi[NS];
    fill_Y(Yinj8, Yi);
    const double Ri = get_R(m, Yi);
    const double gam = 1.29, A1 = 1.0, A3 = 5.0;
    const double C0 = sqrt(gam * Ri * 1.0);
    const double gh = (gam - 1.0) / 2.0;
    const double e1 = -gam / (gam - 1.0), e2 = -(gam + 1.0) / 2.0 / (gam - 1.0), gg = gam / (gam - 1.0);
    const double C = -gam / (gam - 1.0) * Ri * 1.0;
    // the bisection of the forward (injector_state), for the last M's MFC
    double M1 = 0.0, M2 = 1.0, MFC = 0.0, V3 = 0.0;
    for (int it = 0; it < 20; ++it) {
      const double M = 0.5 * (M1 + M2);
      const double base = 1.0 + gh * (M * M);
      const double P1 = 1.0 * pow(base, e1);
      const double V1 = M * pow(base, -0.5) * C0;
      MFC = 1.0 * sqrt(gam / Ri) * M * pow(base, e2);
      const double B = gg * p * A3 / MFC;
      V3 = (-B + sqrt(B * B - 2.0 * C)) / 1.0;
      const double P2 = (MFC * (V3 - V1) - P1 * A1 + p * A3) / (A3 - A1);
      M2 = (P2 >= P1) ? M : M2;
      M1 = (P2 < P1) ? M : M1;
    }
    const double B = gg * p * A3 / MFC;
    const double sq = sqrt(B * B - 2.0 * C);
    const double dV3 = (-1.0 + B / sq) * (gg * A3 / MFC);  // dV3/dp
    const double rho_i = MFC / V3 / A3;
    const double drho_i = -rho_i / V3 * dV3;
    const double T_i = p / (Ri * rho_i);
    const double dT_i = 1.0 / (Ri * rho_i) - T_i / rho_i * drho_i;
    double h_i = 0.0, cp_i = 0.0, dcp_i = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const bool lo = T_i < m.Tcr[k];
      h_i += (lo ? poly6(m.h_lo[k], T_i) : poly6(m.h_hi[k], T_i)) * Yi[k];
      cp_i += (lo ? poly5(m.cp_lo[k], T_i) : poly5(m.cp_hi[k], T_i)) * Yi[k];
      dcp_i += (lo ? poly4(m.dcp_lo[k], T_i) : poly4(m.dcp_hi[k], T_i)) * Yi[k];
    }
    const double cvi = cp_i - Ri;
    const double dg_dT = -Ri * dcp_i / (cvi * cvi);
    const double rho_c = p / (Ri * T_i);
    const double drho_c = 1.0 / (Ri * T_i) - rho_c / T_i * dT_i;
    // ghost = [rho_c, 0, rho_c V3, rho_c h_i - p + rho_c V3^2 / 2, rho_c Yinj8]
    double rcb = ob[0] + ob[2] * V3 + ob[3] * (h_i + 0.5 * (V3 * V3));
#pragma unroll
    for (int k = 0; k < NR; ++k) rcb += ob[4 + k] * Yinj8[k];
    const double V3b = ob[2] * rho_c + ob[3] * rho_c * V3;
    const double hib = ob[3] * rho_c;
    pb += -ob[3] + rcb * drho_c + V3b * dV3 + (hib * cp_i + gcb * dg_dT + Tcb) * dT_i;
  }
  // p = rho R T, R = sum Y_k / M_k
  rb += pb * R * T;
  const double Rb = pb * rho * T;
  Tb += pb * rho * R;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    Y8b[k] += Rb * (m.invM[k] - m.invM[NR]);
    ub[4 + k] += Y8b[k] * ri;
    rb -= Y8b[k] * Y8[k] * ri;
  }
  ub[0] += rb;
}

// ---------------------------------------------------------------------------
// the probe term of the loss: L += dt_n * mean probe p(U_{n+1}), p = rho R T
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ void probe_vjp(const MP& m, const double* q, double T, double w, double* ub, double& Tb) {
  const double rho = q[0], ri = 1.0 / rho;
  double Y8[NR], Yf[NS];
  cell_Y<DIM>(q, ri, Y8, Yf);
  const double R = get_R(m, Yf);
  double rb = w * R * T;
  const double Rb = w * rho * T;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double yb = Rb * (m.invM[k] - m.invM[NR]);
    ub[Lay<DIM>::NY + k] += yb * ri;
    rb -= yb * Y8[k] * ri;
  }
  ub[0] += rb;
  Tb += w * rho * R;
}

// Start of one adjoint step, one thread per cell: the probe term and the
// update_aux VJP of U4 (the aux adjoint is consumed and cleared), the
// primitives (rho, u, v, p) of the three stage states U, U1, U2, and the
// alpha and CFL tie counts of the three stages.
template <int DIM>
__global__ void __launch_bounds__(128) k_vjp_begin(MP m, Grid g, const double* __restrict__ U4,
                                                   const double* __restrict__ A4, const double* __restrict__ pp_bar,
                                                   int px, int py, int wx, int wy, double* Ub, double* Ab,
                                                   const double* __restrict__ rec, double* prims,
                                                   const unsigned char* __restrict__ mult,
                                                   const double* __restrict__ slots_rec, double cfl, double* red) {
  constexpr int NVD = Lay<DIM>::NV;
  const long long nc = g.ncell, nU = NVD * nc;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double cnt[7];
#pragma unroll
  for (int i = 0; i < 7; ++i) cnt[i] = 0.0;
  if (c < nc) {
    const int x = (int)(c / g.ny), y = (int)(c % g.ny);
    double q[NVD], ub[NVD];
    double gb = Ab[c], Tb = Ab[nc + c];
#pragma unroll
    for (int f = 0; f < NVD; ++f) ub[f] = 0.0;
    const bool in_probe = pp_bar && x >= px && x < px + wx && y >= py && y < py + wy;
    if (in_probe || gb != 0.0 || Tb != 0.0) {
#pragma unroll
      for (int f = 0; f < NVD; ++f) q[f] = U4[f * nc + c];
      const double T = A4[nc + c];
      if (in_probe) probe_vjp<DIM>(m, q, T, *pp_bar / (double)(wx * wy), ub, Tb);
      upd_vjp<DIM>(m, q, T, gb, Tb, ub);
#pragma unroll
      for (int f = 0; f < NVD; ++f) Ub[f * nc + c] += ub[f];
      Ab[c] = 0.0;
      Ab[nc + c] = 0.0;
    }
    const jb_slots* rs = reinterpret_cast<const jb_slots*>(slots_rec);
#pragma unroll 1
    for (int s = 0; s < 3; ++s) {
      const double* S = rec + (long long)s * (nU + 2 * nc);
      const double* A = S + nU;
#pragma unroll
      for (int f = 0; f < NVD; ++f) q[f] = S[f * nc + c];
      const Prim<DIM> pr = u_to_prim<DIM>(m, q, A[c], A[nc + c]);
      double* P = prims + (long long)s * 4 * nc;
      P[c] = pr.rho;
      P[nc + c] = pr.u;
      P[2 * nc + c] = pr.v;
      P[3 * nc + c] = pr.p;
      const Speeds sp = speeds_of<DIM>(g, pr);
      if (tied(sp.sx, bitsd(rs->ax[s]))) cnt[2 * s] = mult[c];
      if (DIM == 2 && tied(sp.sy, bitsd(rs->ay[s]))) cnt[2 * s + 1] = mult[c];
      if (s == 0 && cfl > 0.0 && tied(sp.d, rs->dt / cfl)) cnt[6] = 1.0;
    }
  }
#pragma unroll 1
  for (int s = 0; s < 3; ++s) {
    block_add(cnt[2 * s], red + red_cnt(s, 0));
    block_add(cnt[2 * s + 1], red + red_cnt(s, 1));
  }
  block_add(cnt[6], red + red_cnt(0, 2));
}

// The outlet ghosts of the three stage states (blockIdx.y = stage), one
// thread per boundary position: og, and the ghosts' alpha tie counts (3
// padded entries per position).
template <int DIM>
__global__ void __launch_bounds__(128) k_outlet_ghosts(MP m, Grid g, const double* __restrict__ rec,
                                                       const double* __restrict__ slots_rec, double* og,
                                                       double* red) {
  constexpr int NVD = Lay<DIM>::NV;
  const long long nc = g.ncell, nU = NVD * nc;
  const int st = blockIdx.y;
  int side, pos, x, y;
  boundary_pos<DIM>(g, blockIdx.x * blockDim.x + threadIdx.x, side, pos, x, y);
  double cx = 0.0, cy = 0.0;
  if (side >= 0 && strip_side(g, side)) {
    const long long c = (long long)x * g.ny + y;
    const double* S = rec + (long long)st * (nU + 2 * nc);
    double q[NVD], gs[NVD + 2];
#pragma unroll
    for (int f = 0; f < NVD; ++f) q[f] = S[f * nc + c];
    strip_state<DIM>(m, g, side, pos, q, S[nU + c], S[nU + nc + c], gs);
    const Prim<DIM> pr = u_to_prim<DIM>(m, gs, gs[NVD], gs[NVD + 1]);
#pragma unroll
    for (int f = 0; f < NVD; ++f) og[og_idx(g, st, side, f, pos)] = gs[f];
    og[og_idx(g, st, side, OG_U, pos)] = pr.u;
    og[og_idx(g, st, side, OG_V, pos)] = pr.v;
    og[og_idx(g, st, side, OG_P, pos)] = pr.p;
    const jb_slots* rs = reinterpret_cast<const jb_slots*>(slots_rec);
    const Speeds sp = speeds_of<DIM>(g, pr);
    if (tied(sp.sx, bitsd(rs->ax[st]))) cx = 3.0;
    if (DIM == 2 && tied(sp.sy, bitsd(rs->ay[st]))) cy = 3.0;
  }
  block_add(cx, red + red_cnt(st, 0));
  block_add(cy, red + red_cnt(st, 1));
}

// ---------------------------------------------------------------------------
// flux VJP of one RK stage: line sweeps, then a per-cell merge
// ---------------------------------------------------------------------------
// The sweep thread of (direction D, line, segment, field f) owns SW_R
// consecutive padded cells of the line (ghosts included) and walks the
// faces that touch them, keeping a six-cell window of H+, H- and the field
// in registers: per face the two WENO5 reconstructions and their partials,
// scaled by the face-flux adjoint, accumulate into the window's cells, and a
// cell whose five + five contributions are complete is written out as the
// adjoint of its physical flux (Fb) and its LF term (Ua = alpha/2 (h+ - h-)).
// Only faces 0..n carry a flux into the interior, so faces outside are
// skipped.  No shared memory and no barriers: one thread's faces are
// independent of the other threads'.
constexpr int SW_R = 24;
constexpr int SW_NT = 128;

// H+ and H- of field f at padded cell a of a line, from the stage state and
// its primitives (those of the source cell; ghosts flip the momentum), or
// for a pressure-outlet ghost from the stage's outlet ghosts og.
template <int D, int DIM>
__device__ __forceinline__ void sweep_load(const Grid& g, const double* __restrict__ Uk,
                                           const double* __restrict__ Pk, const double* __restrict__ og, int f,
                                           int line, int a, double alpha, double& hp, double& hm, double& qv) {
  const Src s = map_cell<DIM>(g, D == 0 ? a : line, D == 0 ? line : a);
  const long long nc = g.ncell;
  double qf, rho, p, u, v;
  if (s.kind == 1) {
    const double* o = og + (size_t)s.side * OG_F * g.lstrip + s.pos;
    qf = o[(size_t)f * g.lstrip];
    rho = o[0];
    u = o[(size_t)OG_U * g.lstrip];
    v = o[(size_t)OG_V * g.lstrip];
    p = o[(size_t)OG_P * g.lstrip];
  } else {
    const long long src = (long long)s.xs * g.ny + s.ys;
    qf = Uk[f * nc + src];
    if ((s.flip >> f) & 1) qf = -qf;
    rho = Pk[src];
    p = Pk[3 * nc + src];
    u = Pk[nc + src];
    v = Pk[2 * nc + src];
    if (s.flip & 2) u = -u;
    if (s.flip & 4) v = -v;
  }
  const double un = D == 0 ? u : v;
  constexpr int mn = D == 0 ? 1 : 2;
  double F;
  if (f == 0) F = rho * un;
  else if (f == mn) F = rho * un * un + p;
  else if (DIM == 2 && f == 3 - mn) F = rho * u * v;
  else if (f == Lay<DIM>::EI) F = un * (qf + p);
  else F = un * qf;
  hp = 0.5 * (F + alpha * qf);
  hm = 0.5 * (F - alpha * qf);
  qv = qf;
}

template <int D, int DIM>
__device__ __forceinline__ void sweep_body(const Grid& g, const double* __restrict__ Uk,
                                           const double* __restrict__ Pk, const double* __restrict__ og,
                                           const double* __restrict__ Uo_b,
                                           double coef, double alpha, double dt, int f, int line, int seg,
                                           double* __restrict__ Fb, double* __restrict__ Ua, double& ab,
                                           double& dtb) {
  const int nA = D == 0 ? g.nx : g.ny;
  const long long nc = g.ncell;
  const double idA = 1.0 / (D == 0 ? g.dx : g.dy), dt_dA = dt * idA;
  const int a0 = -3 + seg * SW_R, a1 = min(a0 + SW_R, nA + 3);  // owned padded cells [a0, a1)
  const int flo = max(a0 - 2, 0), fhi = min(a1 + 2, nA);        // faces touching them
  const size_t npad = D == 0 ? (size_t)(g.nx + 6) * g.ny : (size_t)g.nx * (g.ny + 6);
  const double* ob = Uo_b + f * nc;
  double* fbo = Fb + f * npad;
  double* uao = Ua + f * npad;
  // adjoint of L at cell a of the line, without dt (zero outside the interior)
  auto lbar = [&](int a) -> double {
    if (a < 0 || a >= nA) return 0.0;
    return coef * ob[D == 0 ? (long long)a * g.ny + line : (long long)line * g.ny + a];
  };
  auto emit = [&](int a, double ap, double am, double qv) {
    ab += 0.5 * qv * (ap - am);
    const size_t k = D == 0 ? (size_t)(a + 3) * g.ny + line : (size_t)line * (g.ny + 6) + (a + 3);
    fbo[k] = 0.5 * (ap + am);
    uao[k] = 0.5 * alpha * (ap - am);
  };
  // window slot k holds padded cell fa - 3 + k while face fa is processed
  double Hp[6], Hm[6], Q[6], Ap[6], Am[6];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    sweep_load<D, DIM>(g, Uk, Pk, og, f, line, flo - 3 + k, alpha, Hp[k], Hm[k], Q[k]);
    Ap[k] = 0.0;
    Am[k] = 0.0;
  }
  Ap[5] = 0.0;
  Am[5] = 0.0;
  double lbm = lbar(flo - 1), Fprev = 0.0;
#pragma unroll 1
  for (int fa = flo; fa <= fhi; ++fa) {
    sweep_load<D, DIM>(g, Uk, Pk, og, f, line, fa + 2, alpha, Hp[5], Hm[5], Q[5]);
    const double lbp = lbar(fa);
    // L_i = -(F_{i+1} - F_i) / d  ->  Fbar_fa = dt (Lbar_fa - Lbar_{fa-1}) / d
    const double Fbf = dt_dA * (lbp - lbm);
    double dl[5], dr[5];
    const double vl = weno_d(Hp[0], Hp[1], Hp[2], Hp[3], Hp[4], dl);
    // right-biased: the left form of the mirrored stencil (cells fa+2 .. fa-2)
    const double vr = weno_d(Hm[5], Hm[4], Hm[3], Hm[2], Hm[1], dr);
    const double Fv = vl + vr;
    // dt adjoint: L of the owned interior cell fa-1, both of its faces known
    const int ci = fa - 1;
    if (fa > flo && ci >= a0 && ci < a1 && ci >= 0 && ci < nA) dtb -= (Fv - Fprev) * idA * lbm;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      Ap[j] += Fbf * dl[j];          // cell fa-3+j
      Am[j + 1] += Fbf * dr[4 - j];  // cell fa-2+j
    }
    // cell fa-3 has all of its contributions (faces fa-5 .. fa)
    if (fa - 3 >= a0 && fa - 3 < a1) emit(fa - 3, Ap[0], Am[0], Q[0]);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      Hp[k] = Hp[k + 1];
      Hm[k] = Hm[k + 1];
      Q[k] = Q[k + 1];
      Ap[k] = Ap[k + 1];
      Am[k] = Am[k + 1];
    }
    Ap[5] = 0.0;
    Am[5] = 0.0;
    lbm = lbp;
    Fprev = Fv;
  }
  // owned cells past the last face (it was clipped at the boundary): slot k
  // now holds cell fhi - 2 + k
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const int a = fhi - 2 + k;
    if (a >= a0 && a < a1) emit(a, Ap[k], Am[k], Q[k]);
  }
}

// Both directions of one RK stage: blocks [0, nbx) sweep x lines (SW_NT
// consecutive y per block), the rest y lines (SW_NT consecutive x); the
// field runs fastest over blocks, then the line block, then the segment.
template <int DIM>
__global__ void __launch_bounds__(SW_NT, 4) k_flux_sweep(Grid g, const double* __restrict__ Uk,
                                                      const double* __restrict__ Pk,
                                                      const double* __restrict__ og,
                                                      const double* __restrict__ Uo_b, double coef,
                                                      const double* __restrict__ slots_rec, int stage, double* FbX,
                                                      double* UaX, double* FbY, double* UaY, double* red, int nbx,
                                                      int nlx, int nly) {
  const jb_slots* rs = reinterpret_cast<const jb_slots*>(slots_rec);
  int b = blockIdx.x;
  const int D = b < nbx ? 0 : 1;
  if (D) b -= nbx;
  const int f = b % Lay<DIM>::NV;
  b /= Lay<DIM>::NV;
  const int nl = D == 0 ? nlx : nly;
  // 2D: a block sweeps SW_NT consecutive lines; 1D (one line): SW_NT
  // consecutive segments of it
  const int line = DIM == 1 ? 0 : (b % nl) * SW_NT + threadIdx.x;
  const int seg = DIM == 1 ? b * SW_NT + threadIdx.x : b / nl;
  double ab = 0.0, dtb = 0.0;
  if (D == 0) {
    if (line < g.ny && seg * SW_R < g.nx + 6)
      sweep_body<0, DIM>(g, Uk, Pk, og, Uo_b, coef, bitsd(rs->ax[stage]), rs->dt, f, line, seg, FbX, UaX, ab, dtb);
  } else if (DIM == 2) {
    if (line < g.nx)
      sweep_body<1, DIM>(g, Uk, Pk, og, Uo_b, coef, bitsd(rs->ay[stage]), rs->dt, f, line, seg, FbY, UaY, ab, dtb);
  }
  block_add(ab, red + red_ab(stage, D));
  block_add(dtb, red + RED_DTB);
}

// ub, Tb += the VJP of the direction-D physical flux F(q, T) (rho un, rho un
// u + p e_n, un (rho E + p), rho un Y) with adjoint Fb.
template <int D, int DIM>
__device__ __forceinline__ void flux_fn_vjp(const MP& m, const double* q, double T, const double* Fb, double* ub,
                                            double& Tb) {
  constexpr int NY = Lay<DIM>::NY, EI = Lay<DIM>::EI;
  const double rho = q[0], ri = 1.0 / rho;
  const double u = q[1] * ri, v = DIM == 2 ? q[2] * ri : 0.0;
  double Y8[NR], Yf[NS];
  cell_Y<DIM>(q, ri, Y8, Yf);
  const double R = get_R(m, Yf);
  const double p = rho * R * T;
  const double un = D == 0 ? u : v, ut = D == 0 ? v : u;
  constexpr int mn = D == 0 ? 1 : 2, mt = 3 - mn;
  const double fbt = DIM == 2 ? Fb[mt] : 0.0;  // the transverse momentum (2D)
  double rb = Fb[0] * un + Fb[mn] * un * un + fbt * u * v;
  double unb = Fb[0] * rho + Fb[mn] * 2.0 * rho * un + fbt * rho * ut + Fb[EI] * (q[EI] + p);
  const double utb = fbt * rho * un;
  const double pb = Fb[mn] + Fb[EI] * un;
  ub[EI] += Fb[EI] * un;
  double Yb[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    rb += Fb[NY + k] * un * Y8[k];
    unb += Fb[NY + k] * rho * Y8[k];
    Yb[k] = Fb[NY + k] * rho * un;
  }
  rb += pb * R * T;
  const double Rb = pb * rho * T;
  Tb += pb * rho * R;
#pragma unroll
  for (int k = 0; k < NR; ++k) Yb[k] += Rb * (m.invM[k] - m.invM[NR]);
  const double ubx = D == 0 ? unb : utb, uby = D == 0 ? utb : unb;
  ub[1] += ubx * ri;
  if (DIM == 2) ub[2] += uby * ri;
  rb -= ubx * u * ri + uby * v * ri;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    ub[NY + k] += Yb[k] * ri;
    rb -= Yb[k] * Y8[k] * ri;
  }
  ub[0] += rb;
}

// The ghost entries of the two direction-D sides that copy interior cell
// (x, y): their flux-function VJP at the ghost state (flipped momentum), with
// the flips undone on the way back.
template <int D, int DIM>
__device__ __forceinline__ void merge_ghosts(const MP& m, const Grid& g, const double* q, double T, int x, int y,
                                             const double* __restrict__ Fb, const double* __restrict__ Ua,
                                             double* ub, double& Tb) {
  constexpr int NVD = Lay<DIM>::NV;
  const int nA = D == 0 ? g.nx : g.ny;
  const size_t npad = D == 0 ? (size_t)(g.nx + 6) * g.ny : (size_t)g.nx * (g.ny + 6);
#pragma unroll 1
  for (int i = 0; i < 6; ++i) {
    const int a = i < 3 ? -1 - i : nA + i - 3;
    const Src s = map_cell<DIM>(g, D == 0 ? a : x, D == 0 ? y : a);
    if (s.kind != 0 || s.xs != x || s.ys != y) continue;
    const size_t k = D == 0 ? (size_t)(a + 3) * g.ny + y : (size_t)x * (g.ny + 6) + (a + 3);
    double qg[NVD], ug[NVD], fb[NVD];
#pragma unroll
    for (int f = 0; f < NVD; ++f) {
      qg[f] = ((s.flip >> f) & 1) ? -q[f] : q[f];
      ug[f] = Ua[f * npad + k];
      fb[f] = Fb[f * npad + k];
    }
    flux_fn_vjp<D, DIM>(m, qg, T, fb, ug, Tb);
#pragma unroll
    for (int f = 0; f < NVD; ++f) ub[f] += ((s.flip >> f) & 1) ? -ug[f] : ug[f];
  }
}

// The outlet sides of one RK stage, one thread per boundary position: the
// 3 ghost layers' flux and LF-term adjoints (sweeps) and their alpha ties,
// through the flux function and wave speeds at the ghost state, then the
// outlet state's VJP into the boundary cell: ogb.
template <int DIM>
__global__ void __launch_bounds__(128) k_outlet_vjp(MP m, Grid g, const double* __restrict__ Uk,
                                                    const double* __restrict__ Ak,
                                                    const double* __restrict__ slots_rec, int stage,
                                                    const double* __restrict__ red, const double* __restrict__ FbX,
                                                    const double* __restrict__ UaX, const double* __restrict__ FbY,
                                                    const double* __restrict__ UaY, double* ogb) {
  constexpr int NVD = Lay<DIM>::NV;
  const long long nc = g.ncell;
  int side, pos, x, y;
  boundary_pos<DIM>(g, blockIdx.x * blockDim.x + threadIdx.x, side, pos, x, y);
  if (side < 0 || !strip_side(g, side)) return;
  const long long c = (long long)x * g.ny + y;
  double q[NVD], gs[NVD + 2], ob[NVD], fb[NVD];
#pragma unroll
  for (int f = 0; f < NVD; ++f) q[f] = Uk[f * nc + c];
  const double gamma = Ak[c], T = Ak[nc + c];
  const double un = outlet_un(q, side);
  strip_state<DIM>(m, g, side, pos, q, gamma, T, gs);
  const int D = side < 2 ? 0 : 1;
  const int nA = D == 0 ? g.nx : g.ny;
  const size_t npad = D == 0 ? (size_t)(g.nx + 6) * g.ny : (size_t)g.nx * (g.ny + 6);
  const double* Fb = D == 0 ? FbX : FbY;
  const double* Ua = D == 0 ? UaX : UaY;
#pragma unroll
  for (int f = 0; f < NVD; ++f) {
    ob[f] = 0.0;
    fb[f] = 0.0;
  }
#pragma unroll 1
  for (int i = 0; i < 3; ++i) {
    const int a = (side == 0 || side == 2) ? -1 - i : nA + i;
    const size_t k = D == 0 ? (size_t)(a + 3) * g.ny + pos : (size_t)pos * (g.ny + 6) + (a + 3);
#pragma unroll
    for (int f = 0; f < NVD; ++f) {
      ob[f] += Ua[f * npad + k];
      fb[f] += Fb[f * npad + k];
    }
  }
  double gcb = 0.0, Tcb = 0.0;
  if (D == 0) flux_fn_vjp<0, DIM>(m, gs, gs[NVD + 1], fb, ob, Tcb);
  else if (DIM == 2) flux_fn_vjp<1, DIM>(m, gs, gs[NVD + 1], fb, ob, Tcb);
  const jb_slots* rs = reinterpret_cast<const jb_slots*>(slots_rec);
  const Speeds sp = speeds_of<DIM>(g, u_to_prim<DIM>(m, gs, gs[NVD], gs[NVD + 1]));
  const double cx = red[red_cnt(stage, 0)], cy = red[red_cnt(stage, 1)];
  const double wx = (cx > 0.0 && tied(sp.sx, bitsd(rs->ax[stage]))) ? red[red_ab(stage, 0)] * 3.0 / cx : 0.0;
  const double wy =
      (DIM == 2 && cy > 0.0 && tied(sp.sy, bitsd(rs->ay[stage]))) ? red[red_ab(stage, 1)] * 3.0 / cy : 0.0;
  speed_vjp<DIM>(m, gs, gs[NVD], gs[NVD + 1], 1, wx, ob, gcb, Tcb);
  if (DIM == 2) speed_vjp<DIM>(m, gs, gs[NVD], gs[NVD + 1], 2, wy, ob, gcb, Tcb);
  double ub[NVD], Tb = 0.0, gb = 0.0;
#pragma unroll
  for (int f = 0; f < NVD; ++f) ub[f] = 0.0;
  if constexpr (DIM == 2) {
    if (g.bc[side] == JB_BC_RDC_INJECTOR) {
      double Yi[NR];
#pragma unroll
      for (int k = 0; k < NR; ++k) Yi[k] = g.Yinj[k * g.nx + pos];
      injector_vjp(m, q, gamma, T, Yi, g.inj_block_p, ob, gcb, Tcb, ub, Tb, gb);
    } else {
      outlet_vjp<DIM>(m, q, gamma, T, un, g.Pb, ob, gcb, Tcb, ub, Tb);
    }
  } else {
    outlet_vjp<DIM>(m, q, gamma, T, un, g.Pb, ob, gcb, Tcb, ub, Tb);
  }
  double* o = ogb + (size_t)side * OG_B * g.lstrip + pos;
#pragma unroll
  for (int f = 0; f < NVD; ++f) o[(size_t)f * g.lstrip] = ub[f];
  o[(size_t)OG_T * g.lstrip] = Tb;
  o[(size_t)OG_G * g.lstrip] = gb;
}

// One RK stage U' = a Un + b (Uk + dt L(Uk, auxk)), per interior cell of Uk:
// the sweeps' LF terms of the cell and of the ghost entries that copy it,
// the flux-function VJPs of both directions, the RK combination (Ubar_k +=
// b Ubar', Ubar_n += a Ubar'), the alpha ties of the stage (and for stage 0
// the CFL ties of dt), then either the update_aux VJP of Uk with its
// completed aux adjoint (Ab null) or the aux adjoint itself added to Ab.
// ub_add / un_add: add to Ub / Un_b instead of storing.
template <int DIM>
__global__ void __launch_bounds__(128, 4) k_stage_merge(
    MP m, Grid g, const double* __restrict__ Uk, const double* __restrict__ Ak, const double* __restrict__ Uo_b,
    double coef, const double* __restrict__ slots_rec, int stage, double cfl, const unsigned char* __restrict__ mult,
    const double* __restrict__ red, const double* __restrict__ dt_bar_ext, const double* __restrict__ FbX,
    const double* __restrict__ UaX, const double* __restrict__ FbY, const double* __restrict__ UaY, double* Ub,
    int ub_add, double* Ab, double* Un_b, double un_coef, int un_add, const double* __restrict__ ogb) {
  constexpr int NVD = Lay<DIM>::NV;
  const long long nc = g.ncell;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int x = (int)(c / g.ny), y = (int)(c % g.ny);
  double q[NVD], ub[NVD], fb[NVD];
#pragma unroll
  for (int f = 0; f < NVD; ++f) q[f] = Uk[f * nc + c];
  const double gamma = Ak[c], T = Ak[nc + c];
  double Tb = 0.0, gb = 0.0;
  {
    const size_t npx = (size_t)(g.nx + 6) * g.ny, npy = (size_t)g.nx * (g.ny + 6);
    const size_t ix = (size_t)(x + 3) * g.ny + y, iy = (size_t)x * (g.ny + 6) + y + 3;
#pragma unroll
    for (int f = 0; f < NVD; ++f) {
      ub[f] = UaX[f * npx + ix] + (DIM == 2 ? UaY[f * npy + iy] : 0.0);
      fb[f] = FbX[f * npx + ix];
    }
    flux_fn_vjp<0, DIM>(m, q, T, fb, ub, Tb);
    if (DIM == 2) {
#pragma unroll
      for (int f = 0; f < NVD; ++f) fb[f] = FbY[f * npy + iy];
      flux_fn_vjp<1, DIM>(m, q, T, fb, ub, Tb);
    }
  }
  // only cells within four of a side are copied into ghosts
  if (x < 4 || x >= g.nx - 4) merge_ghosts<0, DIM>(m, g, q, T, x, y, FbX, UaX, ub, Tb);
  if (DIM == 2 && (y < 4 || y >= g.ny - 4)) merge_ghosts<1, DIM>(m, g, q, T, x, y, FbY, UaY, ub, Tb);
  // the outlet ghosts of the sides this cell borders (k_outlet_vjp)
  if (ogb && (x == 0 || x == g.nx - 1 || (DIM == 2 && (y == 0 || y == g.ny - 1)))) {
#pragma unroll 1
    for (int side = 0; side < 2 * DIM; ++side) {
      const bool on = side == 0 ? x == 0 : side == 1 ? x == g.nx - 1 : side == 2 ? y == 0 : y == g.ny - 1;
      if (!on || !strip_side(g, side)) continue;
      const double* o = ogb + (size_t)side * OG_B * g.lstrip + (side < 2 ? y : x);
#pragma unroll
      for (int f = 0; f < NVD; ++f) ub[f] += o[(size_t)f * g.lstrip];
      Tb += o[(size_t)OG_T * g.lstrip];
      gb += o[(size_t)OG_G * g.lstrip];
    }
  }
#pragma unroll
  for (int f = 0; f < NVD; ++f) {
    const double uo = Uo_b[f * nc + c];
    ub[f] += coef * uo;
    if (Un_b) Un_b[f * nc + c] = (un_add ? Un_b[f * nc + c] : 0.0) + un_coef * uo;
  }
  // alpha ties (evenly over the tied padded entries) and the CFL ties of dt
  const jb_slots* rs = reinterpret_cast<const jb_slots*>(slots_rec);
  const Prim<DIM> pr = u_to_prim<DIM>(m, q, gamma, T);
  const Speeds sp = speeds_of<DIM>(g, pr);
  double wx = 0.0, wy = 0.0;
  const double cx = red[red_cnt(stage, 0)], cy = red[red_cnt(stage, 1)];
  if (cx > 0.0 && tied(sp.sx, bitsd(rs->ax[stage]))) wx = red[red_ab(stage, 0)] * mult[c] / cx;
  if (DIM == 2 && cy > 0.0 && tied(sp.sy, bitsd(rs->ay[stage]))) wy = red[red_ab(stage, 1)] * mult[c] / cy;
  if (stage == 0 && cfl > 0.0) {
    const double cd = red[red_cnt(0, 2)];
    if (cd > 0.0 && tied(sp.d, rs->dt / cfl)) {
      // d = 1 / (sx/dx + sy/dy) (2D) or dx / sx (1D): dd/dsx = -d^2/dx either way
      const double db = cfl * (red[RED_DTB] + (dt_bar_ext ? *dt_bar_ext : 0.0)) / cd;
      wx += -db * sp.d * sp.d / g.dx;
      if (DIM == 2) wy += -db * sp.d * sp.d / g.dy;
    }
  }
  speed_vjp<DIM>(m, q, gamma, T, 1, wx, ub, gb, Tb);
  if (DIM == 2) speed_vjp<DIM>(m, q, gamma, T, 2, wy, ub, gb, Tb);
  if (Ab) {
    Ab[c] += gb;
    Ab[nc + c] += Tb;
  } else {
    upd_vjp<DIM>(m, q, T, gb, Tb, ub);
  }
#pragma unroll
  for (int f = 0; f < NVD; ++f) Ub[f * nc + c] = (ub_add ? Ub[f * nc + c] : 0.0) + ub[f];
}

// mean pressure over the probe rectangle (one block)
template <int DIM>
__global__ void k_probe_mean(MP m, Grid g, const double* __restrict__ U, const double* __restrict__ A, int px,
                             int py, int wx, int wy, double* out) {
  const long long nc = g.ncell;
  double s = 0.0;
  for (int t = threadIdx.x; t < wx * wy; t += blockDim.x) {
    const long long c = (long long)(px + t / wy) * g.ny + (py + t % wy);
    double q[Lay<DIM>::NV];
#pragma unroll
    for (int f = 0; f < Lay<DIM>::NV; ++f) q[f] = U[f * nc + c];
    const double rho = q[0], ri = 1.0 / rho;
    double Y8[NR], Yf[NS];
    cell_Y<DIM>(q, ri, Y8, Yf);
    s += rho * get_R(m, Yf) * A[nc + c];
  }
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x + 31) / 32; ++i) t += red[i];
    *out = t / (double)(wx * wy);
  }
}

// ---------------------------------------------------------------------------
// initial state (rho = P/(R T), rho E = rho h - P, aux = [gamma, T]) -> T adjoint
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void k_init_vjp(MP m, long long n, const double* __restrict__ P, const double* __restrict__ T,
                           const double* __restrict__ Y, const double* __restrict__ Ub, const double* __restrict__ Ab,
                           double* Tb) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double Y8[NR], Yf[NS];
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = Y[k * n + c];
  fill_Y(Y8, Yf);
  const double R = get_R(m, Yf);
  const double t = T[c], p = P[c];
  Th th = thermo_mix(m, t, Yf);
  const double rho = p / (R * t);
  const double drho = -rho / t;
  const double dE = drho * th.h + rho * th.cp;
  const double cv = th.cp - R;
  const double dgam = -th.dcp * R / (cv * cv);
  double tb = Ub[c] * drho + Ub[Lay<DIM>::EI * n + c] * dE + Ab[c] * dgam + Ab[n + c];
#pragma unroll
  for (int k = 0; k < NR; ++k) tb += Ub[(Lay<DIM>::NY + k) * n + c] * Y8[k] * drho;
  Tb[c] = tb;
}

}  // namespace adj
}  // namespace jb

// ---------------------------------------------------------------------------
// launchers (host)
// ---------------------------------------------------------------------------
namespace jb {
namespace adj {

static inline unsigned blocks_for(long long n, int nt) { return (unsigned)((n + nt - 1) / nt); }

// a pressure-outlet side, or the 2D injector side (ghosts that are states of their own)
static bool has_outlet(int dim, const jb_grid& g) {
  for (int s = 0; s < 2 * dim; ++s)
    if (g.bc[s] == JB_BC_PRESSURE_OUTLET || (dim == 2 && s == 2 && g.bc[s] == JB_BC_RDC_INJECTOR)) return true;
  return false;
}

// The scratch: FbX, UaX (nv x (nx+6) x ny each), in 2D FbY, UaY (nv x nx x
// (ny+6) each), og (3 x 4 x OG_F x lstrip), ogb (4 x OG_B x lstrip).
static size_t face_doubles(int dim, const jb_grid& g) {
  const size_t nx6 = (size_t)(g.nx + 6) * g.ny, ny6 = dim == 2 ? (size_t)g.nx * (g.ny + 6) : 0;
  return 2 * (size_t)g.nv * (nx6 + ny6);
}

static double* og_of(int dim, const jb_grid& g, double* scratch) { return scratch + face_doubles(dim, g); }

template <int DIM>
static cudaError_t vjp_begin_t(const jb_mech_params& m, const jb_grid& g, const double* U4, const double* A4,
                               const double* pp_bar, const int* probe, double* Ub, double* Ab, const double* rec,
                               double* prims, const unsigned char* mult, const double* slots_rec, double cfl,
                               double* red, double* scratch, cudaStream_t st) {
  k_vjp_begin<DIM><<<blocks_for(g.ncell, 128), 128, 0, st>>>(m, g, U4, A4, probe[2] * probe[3] > 0 ? pp_bar : nullptr,
                                                             probe[0], probe[1], probe[2], probe[3], Ub, Ab, rec,
                                                             prims, mult, slots_rec, cfl, red);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !has_outlet(DIM, g)) return e;
  const long long npos = DIM == 2 ? 2LL * (g.nx + g.ny) : 2;
  k_outlet_ghosts<DIM><<<dim3(blocks_for(npos, 128), 3), 128, 0, st>>>(m, g, rec, slots_rec, og_of(DIM, g, scratch),
                                                                     red);
  return cudaGetLastError();
}

cudaError_t vjp_begin(int dim, const jb_mech_params& m, const jb_grid& g, const double* U4, const double* A4,
                      const double* pp_bar, const int* probe, double* Ub, double* Ab, const double* rec,
                      double* prims, const unsigned char* mult, const double* slots_rec, double cfl, double* red,
                      double* scratch, cudaStream_t st) {
  return dim == 2 ? vjp_begin_t<2>(m, g, U4, A4, pp_bar, probe, Ub, Ab, rec, prims, mult, slots_rec, cfl, red,
                                   scratch, st)
                  : vjp_begin_t<1>(m, g, U4, A4, pp_bar, probe, Ub, Ab, rec, prims, mult, slots_rec, cfl, red,
                                   scratch, st);
}

cudaError_t chem_vjp(int dim, const jb_mech_params& m, const jb_grid& g, const double* U3, const double* A3,
                     const double* Ub4, double* Ub3, const double* slot_dt, double* dtb, double* lnAb,
                     cudaStream_t st) {
  const size_t sm = sizeof(double) * (CHEM_ADJ_SH + NREAC) * CHEM_ADJ_NT;
  if (dim == 2) {
    cudaError_t e = cudaFuncSetAttribute(k_chem_vjp<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_chem_vjp<2><<<blocks_for(g.ncell, CHEM_ADJ_NT), CHEM_ADJ_NT, sm, st>>>(m, g, U3, A3, Ub4, Ub3, slot_dt, dtb,
                                                                           lnAb);
  } else {
    cudaError_t e = cudaFuncSetAttribute(k_chem_vjp<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_chem_vjp<1><<<blocks_for(g.ncell, CHEM_ADJ_NT), CHEM_ADJ_NT, sm, st>>>(m, g, U3, A3, Ub4, Ub3, slot_dt, dtb,
                                                                           lnAb);
  }
  return cudaGetLastError();
}

size_t flux_scratch_doubles(int dim, const jb_grid& g) {
  return face_doubles(dim, g) + (size_t)(3 * 4 * OG_F + 4 * OG_B) * g.lstrip;
}

template <int DIM>
static cudaError_t flux_stage_t(const jb_mech_params& m, const jb_grid& g, const double* Uk, const double* Ak,
                                const double* Pk, const double* Uo_b, double coef, const double* slots_rec, int stage,
                                double cfl, const unsigned char* mult, double* red, const double* dt_bar_ext,
                                double* scratch, double* Ub, bool ub_add, double* Ab, double* Un_b, double un_coef,
                                bool un_add, cudaStream_t st) {
  constexpr int NVD = Lay<DIM>::NV;
  const size_t npx = NVD * (size_t)(g.nx + 6) * g.ny, npy = DIM == 2 ? NVD * (size_t)g.nx * (g.ny + 6) : 0;
  double *FbX = scratch, *UaX = FbX + npx, *FbY = UaX + npx, *UaY = FbY + npy;
  const int nlx = (g.ny + SW_NT - 1) / SW_NT, nsx = (g.nx + 6 + SW_R - 1) / SW_R;
  const int nly = (g.nx + SW_NT - 1) / SW_NT, nsy = (g.ny + 6 + SW_R - 1) / SW_R;
  const int nbx = (DIM == 2 ? nlx * nsx : (nsx + SW_NT - 1) / SW_NT) * NVD, nby = DIM == 2 ? nly * nsy * NVD : 0;
  const bool outlet = has_outlet(DIM, g);
  double* og = og_of(DIM, g, scratch);
  double* ogb = og + (size_t)3 * 4 * OG_F * g.lstrip;
  k_flux_sweep<DIM><<<nbx + nby, SW_NT, 0, st>>>(g, Uk, Pk,
                                                 outlet ? og + (size_t)stage * 4 * OG_F * g.lstrip : nullptr, Uo_b,
                                                 coef, slots_rec, stage, FbX, UaX, FbY, UaY, red, nbx, nlx, nly);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (outlet) {
    const long long npos = DIM == 2 ? 2LL * (g.nx + g.ny) : 2;
    k_outlet_vjp<DIM><<<blocks_for(npos, 128), 128, 0, st>>>(m, g, Uk, Ak, slots_rec, stage, red, FbX, UaX, FbY, UaY,
                                                             ogb);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  k_stage_merge<DIM><<<blocks_for(g.ncell, 128), 128, 0, st>>>(m, g, Uk, Ak, Uo_b, coef, slots_rec, stage, cfl, mult,
                                                               red, dt_bar_ext, FbX, UaX, FbY, UaY, Ub,
                                                               ub_add ? 1 : 0, Ab, Un_b, un_coef, un_add ? 1 : 0,
                                                               outlet ? ogb : nullptr);
  return cudaGetLastError();
}

cudaError_t flux_stage(int dim, const jb_mech_params& m, const jb_grid& g, const double* Uk, const double* Ak,
                       const double* Pk, const double* Uo_b, double coef, const double* slots_rec, int stage,
                       double cfl, const unsigned char* mult, double* red, const double* dt_bar_ext, double* scratch,
                       double* Ub, bool ub_add, double* Ab, double* Un_b, double un_coef, bool un_add,
                       cudaStream_t st) {
  return dim == 2 ? flux_stage_t<2>(m, g, Uk, Ak, Pk, Uo_b, coef, slots_rec, stage, cfl, mult, red, dt_bar_ext,
                                    scratch, Ub, ub_add, Ab, Un_b, un_coef, un_add, st)
                  : flux_stage_t<1>(m, g, Uk, Ak, Pk, Uo_b, coef, slots_rec, stage, cfl, mult, red, dt_bar_ext,
                                    scratch, Ub, ub_add, Ab, Un_b, un_coef, un_add, st);
}

cudaError_t probe_mean(int dim, const jb_mech_params& m, const jb_grid& g, const double* U, const double* A, int px,
                       int py, int wx, int wy, double* out, cudaStream_t st) {
  if (dim == 2) k_probe_mean<2><<<1, 128, 0, st>>>(m, g, U, A, px, py, wx, wy, out);
  else k_probe_mean<1><<<1, 128, 0, st>>>(m, g, U, A, px, py, wx, wy, out);
  return cudaGetLastError();
}

cudaError_t init_vjp(int dim, const jb_mech_params& m, long long n, const double* P, const double* T, const double* Y,
                     const double* Ub, const double* Ab, double* Tb, cudaStream_t st) {
  if (dim == 2) k_init_vjp<2><<<blocks_for(n, 128), 128, 0, st>>>(m, n, P, T, Y, Ub, Ab, Tb);
  else k_init_vjp<1><<<blocks_for(n, 128), 128, 0, st>>>(m, n, P, T, Y, Ub, Ab, Tb);
  return cudaGetLastError();
}

}  // namespace adj
}  // namespace jb
