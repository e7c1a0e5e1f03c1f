// Hand-written reverse-mode kernels of the 2D reacting step (the adjoint).
//
// The forward step being differentiated is the reference's advance_one_step
// (set_simulator.py:117-122) with its CFL time step (set_simulator.py:
// 420-447):
//   dt = CFL min 1/(sx/dx + sy/dy)         over (U, aux)
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
// Kernels (one thread per cell unless noted):
//   k_upd_vjp       Ubar += d(gamma,T)/dU^T abar           (update_aux)
//   k_chem_vjp      chemistry: Ubar3 = Ubar4 + dS/dU3^T Ubar4, with the
//                   temperature, dt and ln A adjoints, then update_aux of U3
//   k_flux_vjp      both directions of one RK stage's L (tile per block)
//   k_flux_merge    y-face adjoints and ghost-cell adjoints into the cells
//   k_speed_count / k_speed_scatter   alpha and CFL ties and their adjoint
//   k_probe_seed    the probe-pressure term of the loss
//   k_init_vjp      initial state from (P, T, Y): T adjoint
#define JB_NS adj
#define JB_FAST 1
#include "jb_kernels.cuh"

#include "jb_adjoint.h"

namespace jb {
namespace adj {

constexpr double TIE_REL = 1e-13;

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

// Mass fractions of a 2D cell.
__device__ __forceinline__ void cell_Y(const double* q, double ri, double* Y8, double* Yf) {
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = q[4 + k] * ri;
  fill_Y(Y8, Yf);
}

// ub += d(gamma, T)/dq^T (gb, Tb) for aux = update_aux(q) (solver_2D/aux_func.py:21-29)
__device__ __forceinline__ void upd_vjp(const MP& m, const double* q, double T, double gb, double Tb, double* ub) {
  if (gb == 0.0 && Tb == 0.0) return;
  const double rho = q[0], ri = 1.0 / rho;
  const double u = q[1] * ri, v = q[2] * ri;
  double Y8[NR], Yf[NS];
  cell_Y(q, ri, Y8, Yf);
  TBwd b;
  t_bwd(m, T, Yf, b);
  const double eb = gb * b.dg_de + Tb * b.dT_de;
  double rb = eb * (-q[3] * ri * ri + (u * u + v * v) * ri);
  ub[1] += eb * (-u * ri);
  ub[2] += eb * (-v * ri);
  ub[3] += eb * ri;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double yb = gb * b.dg_dY[k] + Tb * b.dT_dY[k];
    ub[4 + k] += yb * ri;
    rb -= yb * Y8[k] * ri;
  }
  ub[0] += rb;
}

// Adjoint of s = |u_dir| + a, a = sqrt(gamma p / rho), p = rho R T, with
// weight w: ub, gb, Tb accumulate.
__device__ __forceinline__ void speed_vjp(const MP& m, const double* q, double gamma, double T, int dir, double w,
                                          double* ub, double& gb, double& Tb) {
  if (w == 0.0) return;
  const double rho = q[0], ri = 1.0 / rho;
  double Y8[NR], Yf[NS];
  cell_Y(q, ri, Y8, Yf);
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
    ub[4 + k] += yb * ri;
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
__global__ void k_upd_vjp(MP m, Grid g, const double* __restrict__ U, const double* __restrict__ aux,
                          double* __restrict__ Ub, double* __restrict__ Ab) {
  const long long nc = g.ncell;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double gb = Ab[c], Tb = Ab[nc + c];
  if (gb == 0.0 && Tb == 0.0) return;
  double q[12], ub[12];
#pragma unroll
  for (int f = 0; f < 12; ++f) { q[f] = U[f * nc + c]; ub[f] = 0.0; }
  upd_vjp(m, q, aux[nc + c], gb, Tb, ub);
#pragma unroll
  for (int f = 0; f < 12; ++f) Ub[f * nc + c] += ub[f];
  Ab[c] = 0.0;
  Ab[nc + c] = 0.0;
}

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
__global__ void __launch_bounds__(CHEM_ADJ_NT, 2)
    k_chem_vjp(MP m, Grid g, const double* __restrict__ U3, const double* __restrict__ A3, const double* Ub4,
               double* Ub3, const double* __restrict__ slot_dt, double* dtb, double* lnAb) {
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
    double q[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) q[f] = U3[f * nc + c];
    const double T = A3[nc + c];
    const double rho = q[0], ri = 1.0 / rho;
    double Y8[NR], Yf[NS], X[NS], Xc[NR], lnXc[NR], iXc[NR], gg[NR], dg[NR];
    cell_Y(q, ri, Y8, Yf);
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
      const double Sb = Ub4[(4 + k) * nc + c];
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
    double ub[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) ub[f] = Ub4[f * nc + c];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const double yb = Y8b[k] + Yfb[k] - Yfb[NR];
      ub[4 + k] += yb * ri;
      rb -= yb * Y8[k] * ri;
    }
    ub[0] += rb;
    upd_vjp(m, q, T, 0.0, Tb, ub);
#pragma unroll
    for (int f = 0; f < 12; ++f) Ub3[f * nc + c] = ub[f];
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
// flux VJP of one direction of one RK stage
// ---------------------------------------------------------------------------
// Block: TO cells along the direction (padded coordinates, ghosts included)
// x TA cells across it (interior only).  threadIdx.x runs along y, so the
// y direction is the coalesced one for both kernels.
constexpr int TO = 16, TA = 16, NE = TO + 10, NF = TO + 5;
constexpr int NEP = NE + 1, NFP = NF;  // odd strides (in doubles) of the across-major layout
constexpr int EA = TA * NEP, FA = TA * NFP;  // doubles per extended-cell / face array

template <int D>
__device__ __forceinline__ int ie(int e, int c) { return D == 0 ? e * TA + c : c * NEP + e; }
template <int D>
__device__ __forceinline__ int iff(int f, int c) { return D == 0 ? f * TA + c : c * NFP + f; }

// One tile (bx, by) of one direction.  D = 0 (x faces) adds into Ub, Abk
// (T adjoint at Abk[nc + c]) and applies the RK combination; D = 1 (y faces)
// stores into its own Ub, Abk (T adjoint at Abk[c]), merged afterwards.
template <int D>  // 0: x faces (F), 1: y faces (G)
__device__ __forceinline__ void flux_vjp_body(const MP& m, const Grid& g, const double* __restrict__ Uk,
                                              const double* __restrict__ Ak, const double* __restrict__ Uo_b,
                                              double coef, const double* __restrict__ slots_rec, int stage,
                                              double* Ub, double* Abk, double* Un_b, double un_coef,
                                              double* ghost, double* red, int bx, int by) {
  // Shared arrays: per extended cell rho, u, v, p, the field, H+, H- and its
  // source (cell index, flip bits); per face the 5 + 5 WENO partials times
  // the face-flux adjoint and the face value.  The layout runs along the
  // across index for x faces and along the direction for y faces, so a
  // warp's accesses are unit-stride in both kernels.
  extern __shared__ __align__(16) double sm_flux[];
  double* sP = sm_flux;          // [4][EA]
  double* sQ = sP + 4 * EA;
  double* sHp = sQ + EA;
  double* sHm = sHp + EA;
  double* sPL = sHm + EA;        // [5][FA]
  double* sPR = sPL + 5 * FA;    // [5][FA]
  double* sFv = sPR + 5 * FA;    // [FA]
  long long* sSrc = reinterpret_cast<long long*>(sFv + FA);  // [EA], -1: outside the padded grid
  int* sFlip = reinterpret_cast<int*>(sSrc + EA);            // [EA]
  const int nA = D == 0 ? g.nx : g.ny;
  const int nC = D == 0 ? g.ny : g.nx;
  const long long nc = g.ncell;
  const int tA = D == 0 ? threadIdx.y : threadIdx.x;  // along index of the owned cell
  const int tC = D == 0 ? threadIdx.x : threadIdx.y;  // across index
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int a0 = -3 + bx * TO;
  const int c0 = by * TA;
  const double dA = D == 0 ? g.dx : g.dy;
  const jb_slots* rs = reinterpret_cast<const jb_slots*>(slots_rec);
  const double alpha = bitsd(D == 0 ? rs->ax[stage] : rs->ay[stage]);
  const double dt = rs->dt;
  const int dirf = D == 0 ? 1 : 2;  // normal momentum field
  // sources and primitives of the extended cells
  for (int i = tid; i < NE * TA; i += 256) {
    const int e = D == 0 ? i / TA : i % NE, cc = D == 0 ? i % TA : i / NE;
    const int a = a0 - 5 + e, cidx = c0 + cc;
    double q[12], T = 1.0;
    long long src = -1;
    int flip = 0;
    if (cidx < nC) {
      const int x = D == 0 ? a : cidx, y = D == 0 ? cidx : a;
      Src s = map_cell<2>(g, x, y);
      if (s.kind == 0) {
        src = (long long)s.xs * g.ny + s.ys;
        flip = s.flip;
      }
    }
    if (src >= 0) {
#pragma unroll
      for (int f = 0; f < 12; ++f) {
        const double v = Uk[f * nc + src];
        q[f] = ((flip >> f) & 1) ? -v : v;
      }
      T = Ak[nc + src];
    } else {
#pragma unroll
      for (int f = 0; f < 12; ++f) q[f] = 1.0;
    }
    const double rho = q[0], ri = 1.0 / rho;
    double Y8[NR], Yf[NS];
    cell_Y(q, ri, Y8, Yf);
    const int k = ie<D>(e, cc);
    sSrc[k] = src;
    sFlip[k] = flip;
    sP[k] = rho;
    sP[EA + k] = q[1] * ri;
    sP[2 * EA + k] = q[2] * ri;
    sP[3 * EA + k] = rho * get_R(m, Yf) * T;
  }
  __syncthreads();
  const int ao = a0 + tA;  // padded along coordinate of the owned cell
  const int co = c0 + tC;
  const bool owned = co < nC && ao < nA + 3;
  const bool interior = owned && ao >= 0 && ao < nA;
  const long long cell = D == 0 ? (long long)ao * g.ny + co : (long long)co * g.ny + ao;
  double Fb[12], Ua[12];
  double ab = 0.0, dtb = 0.0;
#pragma unroll 1
  for (int f = 0; f < 12; ++f) {
    // H+- of the field on the extended cells
    for (int i = tid; i < NE * TA; i += 256) {
      const int e = D == 0 ? i / TA : i % NE, cc = D == 0 ? i % TA : i / NE;
      const int k = ie<D>(e, cc);
      const long long src = sSrc[k];
      double qf = 1.0;
      if (src >= 0) {
        const double v = Uk[f * nc + src];
        qf = ((sFlip[k] >> f) & 1) ? -v : v;
      }
      const double rho = sP[k], u = sP[EA + k], v = sP[2 * EA + k], p = sP[3 * EA + k];
      const double un = D == 0 ? u : v;
      double F;
      if (f == 0) F = rho * un;
      else if (f == dirf) F = rho * un * un + p;
      else if (f == 3 - dirf) F = rho * u * v;
      else if (f == 3) F = un * (qf + p);
      else F = rho * un * (qf / rho);
      sQ[k] = qf;
      sHp[k] = 0.5 * (F + alpha * qf);
      sHm[k] = 0.5 * (F - alpha * qf);
    }
    __syncthreads();
    // faces: adjoint of the face flux and the WENO partials
    for (int i = tid; i < NF * TA; i += 256) {
      const int fl = D == 0 ? i / TA : i % NF, cc = D == 0 ? i % TA : i / NF;
      const int fa = a0 - 2 + fl;  // face between cells fa-1 and fa
      const int cidx = c0 + cc;
      double Lm = 0.0, Lp = 0.0;
      if (cidx < nC) {
        if (fa - 1 >= 0 && fa - 1 < nA) {
          const long long cl = D == 0 ? (long long)(fa - 1) * g.ny + cidx : (long long)cidx * g.ny + (fa - 1);
          Lm = coef * dt * Uo_b[f * nc + cl];
        }
        if (fa >= 0 && fa < nA) {
          const long long cr = D == 0 ? (long long)fa * g.ny + cidx : (long long)cidx * g.ny + fa;
          Lp = coef * dt * Uo_b[f * nc + cr];
        }
      }
      // L_i = -(F_{i+1} - F_i) / d  ->  Fbar_f = (Lbar_f - Lbar_{f-1}) / d
      const double Fb_face = (Lp - Lm) / dA;
      double dl[5], dr[5];
      const double vl = weno_d(sHp[ie<D>(fl, cc)], sHp[ie<D>(fl + 1, cc)], sHp[ie<D>(fl + 2, cc)],
                               sHp[ie<D>(fl + 3, cc)], sHp[ie<D>(fl + 4, cc)], dl);
      // right-biased: the left form of the mirrored stencil (cells fa+2 .. fa-2)
      const double vr = weno_d(sHm[ie<D>(fl + 5, cc)], sHm[ie<D>(fl + 4, cc)], sHm[ie<D>(fl + 3, cc)],
                               sHm[ie<D>(fl + 2, cc)], sHm[ie<D>(fl + 1, cc)], dr);
      const int kf = iff<D>(fl, cc);
      sFv[kf] = vl + vr;
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        sPL[j * FA + kf] = Fb_face * dl[j];      // cell fa-3+j
        sPR[j * FA + kf] = Fb_face * dr[4 - j];  // cell fa-2+j
      }
    }
    __syncthreads();
    if (owned) {
      const int o = tA;
      double hp = 0.0, hm = 0.0;
#pragma unroll
      for (int d = -1; d <= 3; ++d) hp += sPL[(3 - d) * FA + iff<D>(o + d + 2, tC)];
#pragma unroll
      for (int d = -2; d <= 2; ++d) hm += sPR[(2 - d) * FA + iff<D>(o + d + 2, tC)];
      const double qf = sQ[ie<D>(o + 5, tC)];
      Fb[f] = 0.5 * (hp + hm);
      Ua[f] = 0.5 * alpha * (hp - hm);
      ab += 0.5 * qf * (hp - hm);
      if (interior) {
        const double Lphys = -(sFv[iff<D>(o + 3, tC)] - sFv[iff<D>(o + 2, tC)]) / dA;
        dtb += Lphys * coef * Uo_b[f * nc + cell];
      }
    }
    __syncthreads();
  }
  if (owned) {
    // flux function VJP of this padded cell
    const int k = ie<D>(tA + 5, tC);
    const double rho = sP[k], u = sP[EA + k], v = sP[2 * EA + k], p = sP[3 * EA + k];
    const double un = D == 0 ? u : v, ut = D == 0 ? v : u;
    // the padded cell's own state (flipped for ghosts) for rho E and Y
    const long long src = sSrc[k] >= 0 ? sSrc[k] : 0;
    const int flip = sFlip[k];
    double q[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) {
      const double vv = Uk[f * nc + src];
      q[f] = ((flip >> f) & 1) ? -vv : vv;
    }
    const double T = Ak[nc + src];
    const double ri = 1.0 / rho;
    double Y8[NR], Yf[NS];
    cell_Y(q, ri, Y8, Yf);
    const double R = get_R(m, Yf);
    const int mn = dirf, mt = 3 - dirf;
    double rb = Fb[0] * un + Fb[mn] * un * un + Fb[mt] * u * v;
    double unb = Fb[0] * rho + Fb[mn] * 2.0 * rho * un + Fb[mt] * rho * ut + Fb[3] * (q[3] + p);
    double utb = Fb[mt] * rho * un;
    const double pb = Fb[mn] + Fb[3] * un;
    double ub[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) ub[f] = Ua[f];
    ub[3] += Fb[3] * un;
    double Yb[NR];
#pragma unroll
    for (int kk = 0; kk < NR; ++kk) {
      rb += Fb[4 + kk] * un * Y8[kk];
      unb += Fb[4 + kk] * rho * Y8[kk];
      Yb[kk] = Fb[4 + kk] * rho * un;
    }
    rb += pb * R * T;
    const double Rb = pb * rho * T;
    const double Tb = pb * rho * R;
#pragma unroll
    for (int kk = 0; kk < NR; ++kk) Yb[kk] += Rb * (m.invM[kk] - m.invM[NR]);
    const double ubx = D == 0 ? unb : utb, uby = D == 0 ? utb : unb;
    ub[1] += ubx * ri;
    ub[2] += uby * ri;
    rb -= ubx * u * ri + uby * v * ri;
#pragma unroll
    for (int kk = 0; kk < NR; ++kk) {
      ub[4 + kk] += Yb[kk] * ri;
      rb -= Yb[kk] * Y8[kk] * ri;
    }
    ub[0] += rb;
    if (interior) {
#pragma unroll
      for (int f = 0; f < 12; ++f) {
        double val = ub[f];
        if (D == 0) {
          const double uo = Uo_b[f * nc + cell];
          // the RK combination, once per cell and stage
          if (Un_b) Un_b[f * nc + cell] += un_coef * uo;
          val += coef * uo;
        }
        if (D == 0) Ub[f * nc + cell] += val;
        else Ub[f * nc + cell] = val;
      }
      if (D == 0) Abk[nc + cell] += Tb;
      else Abk[cell] = Tb;
    } else {
      // ghost entry: side, layer, position
      const int side = D == 0 ? (ao < 0 ? 0 : 1) : (ao < 0 ? 2 : 3);
      const int layer = ao < 0 ? -1 - ao : ao - nA;
      const int L = g.nx > g.ny ? g.nx : g.ny;
      double* gp = ghost + ((size_t)(side * 3 + layer) * 13) * L + co;
#pragma unroll
      for (int f = 0; f < 12; ++f) gp[(size_t)f * L] = ub[f];
      gp[(size_t)12 * L] = Tb;
    }
  }
  block_add(ab, red + (D == 0 ? 0 : 1));
  block_add(dtb, red + 2);
}

// Both directions of one RK stage in one launch: blocks [0, nbx) are x-face
// tiles (a grid of gxx tiles along x), the rest y-face tiles (gyy along y).
__global__ void __launch_bounds__(256, 3) k_flux_vjp(MP m, Grid g, const double* __restrict__ Uk,
                                                 const double* __restrict__ Ak, const double* __restrict__ Uo_b,
                                                 double coef, const double* __restrict__ slots_rec, int stage,
                                                 double* Ub, double* Abk, double* Ub2, double* Ab2, double* Un_b,
                                                 double un_coef, double* ghost, double* red, int nbx, int gxx,
                                                 int gyy) {
  const int b = blockIdx.x;
  if (b < nbx)
    flux_vjp_body<0>(m, g, Uk, Ak, Uo_b, coef, slots_rec, stage, Ub, Abk, Un_b, un_coef, ghost, red, b % gxx,
                     b / gxx);
  else
    flux_vjp_body<1>(m, g, Uk, Ak, Uo_b, coef, slots_rec, stage, Ub2, Ab2, nullptr, 0.0, ghost, red,
                     (b - nbx) % gyy, (b - nbx) / gyy);
}

// Per interior cell: add the y-face adjoints (Ub2, Ab2) and gather the
// adjoints of the ghost entries that copy this cell (the boundary map of
// every side, with the normal-momentum flips undone).
__global__ void k_flux_merge(Grid g, const double* __restrict__ ghost, const double* __restrict__ Ub2,
                             const double* __restrict__ Ab2, double* Ub, double* Ab) {
  const long long nc = g.ncell;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int x = (int)(c / g.ny), y = (int)(c % g.ny);
  const int L = g.nx > g.ny ? g.nx : g.ny;
  double ub[12];
#pragma unroll
  for (int f = 0; f < 12; ++f) ub[f] = Ub2[f * nc + c];
  double tb = Ab2[c];
  for (int side = 0; side < 4; ++side) {
    const int pos = side < 2 ? y : x;
    for (int layer = 0; layer < 3; ++layer) {
      const int gx = side == 0 ? -1 - layer : side == 1 ? g.nx + layer : x;
      const int gy = side == 2 ? -1 - layer : side == 3 ? g.ny + layer : y;
      Src s = map_cell<2>(g, gx, gy);
      if (s.kind != 0 || s.xs != x || s.ys != y) continue;
      const double* gp = ghost + ((size_t)(side * 3 + layer) * 13) * L + pos;
#pragma unroll
      for (int f = 0; f < 12; ++f) {
        const double v = gp[(size_t)f * L];
        ub[f] += ((s.flip >> f) & 1) ? -v : v;
      }
      tb += gp[(size_t)12 * L];
    }
  }
#pragma unroll
  for (int f = 0; f < 12; ++f) Ub[f * nc + c] += ub[f];
  Ab[nc + c] += tb;
}

// ---------------------------------------------------------------------------
// alpha (max over the padded grid) and CFL (min over cells) ties
// ---------------------------------------------------------------------------
struct Speeds {
  double sx, sy, d;
};

__device__ __forceinline__ Speeds speeds(const MP& m, const Grid& g, const double* q, double gamma, double T) {
  Prim<2> pr = u_to_prim<2>(m, q, gamma, T);
  Speeds s;
  s.sx = fabs(pr.u) + pr.a;
  s.sy = fabs(pr.v) + pr.a;
  s.d = 1.0 / (s.sx / g.dx + s.sy / g.dy);
  return s;
}

__device__ __forceinline__ bool tied(double v, double ref) { return fabs(v - ref) <= TIE_REL * fabs(ref); }

// red layout (doubles): [0] abar_x, [1] abar_y, [2] dtbar, [3] nx ties, [4] ny ties, [5] n CFL ties
__global__ void k_speed_count(MP m, Grid g, const double* __restrict__ U, const double* __restrict__ A,
                              const unsigned char* __restrict__ mult, const double* __restrict__ slots_rec,
                              int stage, double cfl, double* red) {
  const long long nc = g.ncell;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double cx = 0.0, cy = 0.0, cd = 0.0;
  if (c < nc) {
    const jb_slots* rs = reinterpret_cast<const jb_slots*>(slots_rec);
    double q[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) q[f] = U[f * nc + c];
    Speeds s = speeds(m, g, q, A[c], A[nc + c]);
    if (tied(s.sx, bitsd(rs->ax[stage]))) cx = mult[c];
    if (tied(s.sy, bitsd(rs->ay[stage]))) cy = mult[c];
    if (cfl > 0.0 && tied(s.d, rs->dt / cfl)) cd = 1.0;
  }
  block_add(cx, red + 3);
  block_add(cy, red + 4);
  block_add(cd, red + 5);
}

// UPD: then the update_aux VJP of the same state with the completed aux
// adjoint (consumed and zeroed), as k_upd_vjp.
template <bool UPD>
__global__ void k_speed_scatter(MP m, Grid g, const double* __restrict__ U, const double* __restrict__ A,
                                const unsigned char* __restrict__ mult, const double* __restrict__ slots_rec,
                                int stage, double cfl, const double* __restrict__ red, double* Ub, double* Ab) {
  const long long nc = g.ncell;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const jb_slots* rs = reinterpret_cast<const jb_slots*>(slots_rec);
  double q[12];
#pragma unroll
  for (int f = 0; f < 12; ++f) q[f] = U[f * nc + c];
  const double gamma = A[c], T = A[nc + c];
  Speeds s = speeds(m, g, q, gamma, T);
  double wx = 0.0, wy = 0.0;
  if (red[3] > 0.0 && tied(s.sx, bitsd(rs->ax[stage]))) wx = red[0] * mult[c] / red[3];
  if (red[4] > 0.0 && tied(s.sy, bitsd(rs->ay[stage]))) wy = red[1] * mult[c] / red[4];
  if (cfl > 0.0 && red[5] > 0.0 && tied(s.d, rs->dt / cfl)) {
    const double db = cfl * red[2] / red[5];
    wx += -db * s.d * s.d / g.dx;
    wy += -db * s.d * s.d / g.dy;
  }
  double gb = UPD ? Ab[c] : 0.0, Tb = UPD ? Ab[nc + c] : 0.0;
  if (wx == 0.0 && wy == 0.0 && gb == 0.0 && Tb == 0.0) return;
  double ub[12];
#pragma unroll
  for (int f = 0; f < 12; ++f) ub[f] = 0.0;
  speed_vjp(m, q, gamma, T, 1, wx, ub, gb, Tb);
  speed_vjp(m, q, gamma, T, 2, wy, ub, gb, Tb);
  if (UPD) {
    upd_vjp(m, q, T, gb, Tb, ub);
    Ab[c] = 0.0;
    Ab[nc + c] = 0.0;
  } else {
    Ab[c] += gb;
    Ab[nc + c] += Tb;
  }
#pragma unroll
  for (int f = 0; f < 12; ++f) Ub[f * nc + c] += ub[f];
}

// ---------------------------------------------------------------------------
// loss seed: L += dt_n * mean probe p(U_{n+1}); red[2] (dtbar) += dt_bar_ext
// ---------------------------------------------------------------------------
__global__ void k_probe_seed(MP m, Grid g, const double* __restrict__ U, const double* __restrict__ A,
                             const double* __restrict__ pp_bar, int px, int py, int wx, int wy, double* Ub,
                             double* Ab) {
  const int t = threadIdx.x;
  if (t >= wx * wy || !pp_bar) return;
  const long long nc = g.ncell;
  const long long c = (long long)(px + t / wy) * g.ny + (py + t % wy);
  const double w = *pp_bar / (double)(wx * wy);
  if (w == 0.0) return;
  double q[12];
#pragma unroll
  for (int f = 0; f < 12; ++f) q[f] = U[f * nc + c];
  const double T = A[nc + c];
  const double rho = q[0], ri = 1.0 / rho;
  double Y8[NR], Yf[NS];
  cell_Y(q, ri, Y8, Yf);
  const double R = get_R(m, Yf);
  // p = rho R T, R = sum Yf / M
  double rb = w * R * T;
  const double Rb = w * rho * T;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double yb = Rb * (m.invM[k] - m.invM[NR]);
    Ub[(4 + k) * nc + c] += yb * ri;
    rb -= yb * Y8[k] * ri;
  }
  Ub[c] += rb;
  Ab[nc + c] += w * rho * R;
}

// mean pressure over the probe rectangle (one block)
__global__ void k_probe_mean(MP m, Grid g, const double* __restrict__ U, const double* __restrict__ A, int px,
                             int py, int wx, int wy, double* out) {
  const long long nc = g.ncell;
  double s = 0.0;
  for (int t = threadIdx.x; t < wx * wy; t += blockDim.x) {
    const long long c = (long long)(px + t / wy) * g.ny + (py + t % wy);
    double q[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) q[f] = U[f * nc + c];
    const double rho = q[0], ri = 1.0 / rho;
    double Y8[NR], Yf[NS];
    cell_Y(q, ri, Y8, Yf);
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

__global__ void k_adj_begin(double* red, const double* __restrict__ dt_bar_ext) {
  for (int i = 0; i < 8; ++i) red[i] = 0.0;
  if (dt_bar_ext) red[2] = *dt_bar_ext;
}

__global__ void k_adj_clear_alpha(double* red) {
  red[0] = 0.0;
  red[1] = 0.0;
  red[3] = 0.0;
  red[4] = 0.0;
}

// ---------------------------------------------------------------------------
// initial state (rho = P/(R T), rho E = rho h - P, aux = [gamma, T]) -> T adjoint
// ---------------------------------------------------------------------------
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
  double tb = Ub[c] * drho + Ub[3 * n + c] * dE + Ab[c] * dgam + Ab[n + c];
#pragma unroll
  for (int k = 0; k < NR; ++k) tb += Ub[(4 + k) * n + c] * Y8[k] * drho;
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

cudaError_t upd_vjp(const jb_mech_params& m, const jb_grid& g, const double* U, const double* A, double* Ub,
                    double* Ab, cudaStream_t st) {
  k_upd_vjp<<<blocks_for(g.ncell, 128), 128, 0, st>>>(m, g, U, A, Ub, Ab);
  return cudaGetLastError();
}

cudaError_t chem_vjp(const jb_mech_params& m, const jb_grid& g, const double* U3, const double* A3,
                     const double* Ub4, double* Ub3, const double* slot_dt, double* dtb, double* lnAb,
                     cudaStream_t st) {
  const size_t sm = sizeof(double) * (CHEM_ADJ_SH + NREAC) * CHEM_ADJ_NT;
  cudaError_t e = cudaFuncSetAttribute(k_chem_vjp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k_chem_vjp<<<blocks_for(g.ncell, CHEM_ADJ_NT), CHEM_ADJ_NT, sm, st>>>(m, g, U3, A3, Ub4, Ub3, slot_dt, dtb, lnAb);
  return cudaGetLastError();
}

constexpr size_t FLUX_VJP_SMEM = sizeof(double) * (7 * EA + 11 * FA) + (sizeof(long long) + sizeof(int)) * EA;

cudaError_t flux_vjp(const jb_mech_params& m, const jb_grid& g, const double* Uk, const double* Ak,
                     const double* Uo_b, double coef, const double* slots_rec, int stage, double* Ub, double* Abk,
                     double* Un_b, double un_coef, double* ghost, double* Ub2, double* Ab2, double* red,
                     cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(k_flux_vjp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FLUX_VJP_SMEM);
  if (e != cudaSuccess) return e;
  const int gxx = (g.nx + 6 + TO - 1) / TO, gxy = (g.ny + TA - 1) / TA;
  const int gyy = (g.ny + 6 + TO - 1) / TO, gyx = (g.nx + TA - 1) / TA;
  const int nbx = gxx * gxy, nby = gyy * gyx;
  k_flux_vjp<<<nbx + nby, dim3(16, 16), FLUX_VJP_SMEM, st>>>(m, g, Uk, Ak, Uo_b, coef, slots_rec, stage, Ub, Abk, Ub2,
                                                             Ab2, Un_b, un_coef, ghost, red, nbx, gxx, gyy);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_flux_merge<<<blocks_for(g.ncell, 128), 128, 0, st>>>(g, ghost, Ub2, Ab2, Ub, Abk);
  return cudaGetLastError();
}

cudaError_t speed_vjp(const jb_mech_params& m, const jb_grid& g, const double* U, const double* A,
                      const unsigned char* mult, const double* slots_rec, int stage, double cfl, double* red,
                      double* Ub, double* Ab, bool upd, cudaStream_t st) {
  k_speed_count<<<blocks_for(g.ncell, 128), 128, 0, st>>>(m, g, U, A, mult, slots_rec, stage, cfl, red);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (upd)
    k_speed_scatter<true><<<blocks_for(g.ncell, 128), 128, 0, st>>>(m, g, U, A, mult, slots_rec, stage, cfl, red, Ub, Ab);
  else
    k_speed_scatter<false><<<blocks_for(g.ncell, 128), 128, 0, st>>>(m, g, U, A, mult, slots_rec, stage, cfl, red, Ub, Ab);
  return cudaGetLastError();
}

cudaError_t probe_seed(const jb_mech_params& m, const jb_grid& g, const double* U, const double* A,
                       const double* pp_bar, int px, int py, int wx, int wy, double* Ub, double* Ab, cudaStream_t st) {
  if (!pp_bar || wx * wy <= 0) return cudaSuccess;
  k_probe_seed<<<1, 32 * ((wx * wy + 31) / 32), 0, st>>>(m, g, U, A, pp_bar, px, py, wx, wy, Ub, Ab);
  return cudaGetLastError();
}

cudaError_t probe_mean(const jb_mech_params& m, const jb_grid& g, const double* U, const double* A, int px, int py,
                       int wx, int wy, double* out, cudaStream_t st) {
  k_probe_mean<<<1, 128, 0, st>>>(m, g, U, A, px, py, wx, wy, out);
  return cudaGetLastError();
}

cudaError_t adj_begin(double* red, const double* dt_bar_ext, cudaStream_t st) {
  k_adj_begin<<<1, 1, 0, st>>>(red, dt_bar_ext);
  return cudaGetLastError();
}

cudaError_t clear_alpha(double* red, cudaStream_t st) {
  k_adj_clear_alpha<<<1, 1, 0, st>>>(red);
  return cudaGetLastError();
}

cudaError_t init_vjp(const jb_mech_params& m, long long n, const double* P, const double* T, const double* Y,
                     const double* Ub, const double* Ab, double* Tb, cudaStream_t st) {
  k_init_vjp<<<blocks_for(n, 128), 128, 0, st>>>(m, n, P, T, Y, Ub, Ab, Tb);
  return cudaGetLastError();
}

}  // namespace adj
}  // namespace jb
