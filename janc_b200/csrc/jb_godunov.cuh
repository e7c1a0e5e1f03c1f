// Godunov path of the advective flux (solver_{1D,2D}/flux.py godunov_flux):
// WENO5-JS face states of the primitives w = [rho, u, (v), p, Y], then an
// HLLC (riemann_solver/HLLC.py) or AUSMPW+ (riemann_solver/AUSMPW_plus.py)
// flux per face.  Included by jb_kernels.cuh inside namespace jb::JB_NS.
// The reconstruction runs in RW (float32 in the mixed variant), the Riemann
// solver, RK combination and Halley iterates in float64; operation order as
// the reference's expressions evaluate.
#pragma once

constexpr int RS_HLLC = 0, RS_AUSMPW = 1;


// gamma and h of a reconstructed face state from T = p / (R rho)
// (HLLC.py:8-12 / AUSMPW_plus.py:86-92 in 2D).
__device__ __forceinline__ void face_thermo(const MP& m, double rho, double p, const double* Y8, double& gamma,
                                            double& h) {
  double Yf[NS];
  fill_Y(Y8, Yf);
  const double R = get_R(m, Yf);
  const double T = p / (R * rho);
  const Th t = thermo_mix(m, T, Yf);
  h = t.h;
  gamma = t.cp / (t.cp - R);
}

// HLLC flux through a face with normal velocity component N (1: x, 2: y) of
// face states w = [rho, vel[DIM], p, Y8] (2D HLLC.py:15-43 x, :45-73 y;
// 1D HLLC.py:13-42).  F is in the conserved layout [rho, rho vel, rho E, rho Y].
template <int DIM, int N>
__device__ __forceinline__ void hllc_flux(const MP& m, const double* wL, const double* wR, double* F) {
  constexpr int IP = DIM + 1, IY = DIM + 2;
  const double rL = wL[0], rR = wR[0], pL = wL[IP], pR = wR[IP];
  double gL, hL, gR, hR;
  face_thermo(m, rL, pL, wL + IY, gL, hL);
  face_thermo(m, rR, pR, wR + IY, gR, hR);
  const double aL = sqrt(gL * pL / rL);
  const double aR = sqrt(gR * pR / rR);
  const double unL = wL[N], unR = wR[N];
  const double kL = DIM == 2 ? wL[1] * wL[1] + wL[2] * wL[2] : wL[1] * wL[1];
  const double kR = DIM == 2 ? wR[1] * wR[1] + wR[2] * wR[2] : wR[1] * wR[1];
  const double EL = rL * hL - pL + 0.5 * rL * kL;
  const double ER = rR * hR - pR + 0.5 * rR * kR;
  const double sL = nan_min(unL - aL, unR - aR);
  const double sR = nan_max(unL + aL, unR + aR);
  const double sM = (pR - pL + rL * unL * (sL - unL) - rR * unR * (sR - unR)) / (rL * (sL - unL) - rR * (sR - unR));
  const bool c1 = sL >= 0.0, c2 = sL <= 0.0 && sM >= 0.0, c3 = sM <= 0.0 && sR >= 0.0;
  // the star-state factor and energy of each side
  const double fL = rL * (sL - unL) / (sL - sM), fR = rR * (sR - unR) / (sR - sM);
  const double eL = EL / rL + (sM - unL) * (sM + pL / (rL * (sL - unL)));
  const double eR = ER / rR + (sM - unR) * (sM + pR / (rR * (sR - unR)));
  // component c: conserved U, star U_M, physical flux of each side
  auto pick = [&](double UL, double UML, double FL_, double UR, double UMR, double FR_) {
    const double FLM = FL_ + sL * (UML - UL);
    const double FRM = FR_ + sR * (UMR - UR);
    double f = c1 ? FL_ : FR_;
    f = c2 ? FLM : f;
    return c3 ? FRM : f;
  };
  F[0] = pick(rL, fL * 1.0, rL * unL, rR, fR * 1.0, rR * unR);
#pragma unroll
  for (int k = 1; k <= DIM; ++k) {
    const double vL = wL[k], vR = wR[k];
    const double mL = k == N ? rL * (unL * unL) + pL : (N == 1 ? rL * unL * vL : rL * vL * unL);
    const double mR = k == N ? rR * (unR * unR) + pR : (N == 1 ? rR * unR * vR : rR * vR * unR);
    F[k] = pick(rL * vL, fL * (k == N ? sM : vL), mL, rR * vR, fR * (k == N ? sM : vR), mR);
  }
  F[DIM + 1] = pick(EL, fL * eL, unL * (EL + pL), ER, fR * eR, unR * (ER + pR));
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double yL = wL[IY + k], yR = wR[IY + k];
    F[IY + k] = pick(rL * yL, fL * yL, rL * unL * yL, rR * yR, fR * yR, rR * unR * yR);
  }
}

__device__ __forceinline__ double ausm_sign(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : (x == 0.0 ? 0.0 : x)); }

// AUSMPW+ flux (2D AUSMPW_plus.py:77-131, 1D AUSMPW_plus.py:53-82; split
// polynomials :5-11, pressure weights :13-24).  The y faces use their own
// gamma_R (the reference's 2D code takes the x-face gamma_R there, whose
// shape does not broadcast with the y-face arrays).
template <int DIM, int N>
__device__ __forceinline__ void ausmpw_flux(const MP& m, const double* wL, const double* wR, double* F) {
  constexpr int IP = DIM + 1, IY = DIM + 2;
  const double rL = wL[0], rR = wR[0], pL = wL[IP], pR = wR[IP];
  double gL, hL, gR, hR;
  face_thermo(m, rL, pL, wL + IY, gL, hL);
  face_thermo(m, rR, pR, wR + IY, gR, hR);
  const double cL = sqrt(gL * pL / rL), cR = sqrt(gR * pR / rR);
  const double c = 0.5 * (cL + cR);
  const double ML = wL[N] / c, MR = wR[N] / c;
  // split Mach numbers and pressures
  double MLp, PLp, MRm, PRm;
  if (fabs(ML) <= 1.0) {
    const double t = (ML + 1.0) * (ML + 1.0);
    MLp = 1.0 / 4.0 * t;
    PLp = 1.0 / 4.0 * t * (2.0 - ML);
  } else {
    MLp = 1.0 / 2.0 * (ML + fabs(ML));
    PLp = 1.0 / 2.0 * (1.0 + ausm_sign(ML));
  }
  if (fabs(MR) <= 1.0) {
    const double t = (MR - 1.0) * (MR - 1.0);
    MRm = -1.0 / 4.0 * t;
    PRm = 1.0 / 4.0 * t * (2.0 + MR);
  } else {
    MRm = 1.0 / 2.0 * (MR - fabs(MR));
    PRm = 1.0 / 2.0 * (1.0 - ausm_sign(MR));
  }
  const double ps = PLp * pL + PRm * pR;
  const double mk = nan_min(pL / pR, pR / pL);
  const double w = 1.0 - mk * (mk * mk);
  const double fl = fabs(ML) < 1.0 ? pL / ps - 1.0 : 0.0;
  const double fr = fabs(MR) < 1.0 ? pR / ps - 1.0 : 0.0;
  double MLa, MRa;
  if (MLp + MRm >= 0.0) {
    MLa = MLp + MRm * ((1.0 - w) * (1.0 + fr) - fl);
    MRa = MRm * w * (1.0 + fr);
  } else {
    MLa = MLp * w * (1.0 + fl);
    MRa = MRm + MLp * ((1.0 - w) * (1.0 + fl) - fr);
  }
  const double aL = MLa * c, aR = MRa * c;
  const double kL = DIM == 2 ? wL[1] * wL[1] + wL[2] * wL[2] : wL[1] * wL[1];
  const double kR = DIM == 2 ? wR[1] * wR[1] + wR[2] * wR[2] : wR[1] * wR[1];
  // phi = [rho, rho vel, rho h + rho |vel|^2 / 2, rho Y]; pressure in the normal momentum
  F[0] = aL * rL + aR * rR + (PLp * 0.0 + PRm * 0.0);
#pragma unroll
  for (int k = 1; k <= DIM; ++k)
    F[k] = aL * (rL * wL[k]) + aR * (rR * wR[k]) + (k == N ? PLp * pL + PRm * pR : PLp * 0.0 + PRm * 0.0);
  F[DIM + 1] = aL * (rL * hL + 0.5 * rL * kL) + aR * (rR * hR + 0.5 * rR * kR) + (PLp * 0.0 + PRm * 0.0);
#pragma unroll
  for (int k = 0; k < NR; ++k)
    F[IY + k] = aL * (rL * wL[IY + k]) + aR * (rR * wR[IY + k]) + (PLp * 0.0 + PRm * 0.0);
}

template <int DIM, int N, int RS>
__device__ __forceinline__ void riemann_flux(const MP& m, const double* wL, const double* wR, double* F) {
  if (RS == RS_HLLC) hllc_flux<DIM, N>(m, wL, wR, F);
  else ausmpw_flux<DIM, N>(m, wL, wR, F);
}

// Primitives w = [rho, u, (v), p, Y8] of one padded cell from its conserved
// state q and temperature (U_to_prim, solver_{1D,2D}/aux_func.py:39-51).
template <int DIM>
__device__ __forceinline__ void cons_to_w(const MP& m, const double* q, double T, double* w) {
  constexpr int nY = DIM == 1 ? 3 : 4;
  const double rho = q[0];
  w[0] = rho;
  w[1] = q[1] / rho;
  if (DIM == 2) w[2] = q[2] / rho;
  double Y8[NR], Yf[NS];
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = q[nY + k] / rho;
  fill_Y(Y8, Yf);
  w[DIM + 1] = rho * get_R(m, Yf) * T;
#pragma unroll
  for (int k = 0; k < NR; ++k) w[DIM + 2 + k] = Y8[k];
}

// ---------------------------------------------------------------------------
// stage kernels (STAGE as k_flux2d / k_flux1d: 0 flux_func, 1..3 RK stage
// followed by the Halley iterates of update_aux)
// ---------------------------------------------------------------------------
// Shared memory: the padded tile's primitives in RW (float32 in the mixed
// variant: the reconstruction runs in RW; the Riemann solver, RK and Halley
// stay float64), then the face fluxes in float64 at a 16-byte aligned offset.
// float64: the region first receives the TMA boxes of the padded tile
// (TQ_N fields at the staged layout, tile_ci), which the primitives then
// replace
template <class RW>
__host__ __device__ constexpr size_t god2_wbytes() {
  return sizeof(RW) == sizeof(double) ? sizeof(double) * TQ_N * SM2_QF : (sizeof(RW) * 12 * SM2_Q + 15) / 16 * 16;
}
template <class RW>
__host__ __device__ constexpr size_t god2_smem() {
  return god2_wbytes<RW>() + sizeof(double) * 12 * (SM2_FX + SM2_FY);
}

// 2D: the tile of k_flux2d (15 x 16 cells, 3-cell halo); primitives of the
// padded tile in shared memory, then one thread per x face and per y face
// reconstructs all 12 components on both sides and solves the Riemann
// problem.
template <int STAGE, int RS, class RW>
__global__ void __launch_bounds__(NT2, 2) k_god2d(MP m, Grid g, const double* __restrict__ Uk,
                                                 const double* __restrict__ auxk, const double* __restrict__ Un,
                                                 double* __restrict__ out,
                                                 const double* __restrict__ strips, Slots* slots, jb_fin fin,
                                                 double dt_arg, const __grid_constant__ CUtensorMap tmU,
                                                 const __grid_constant__ CUtensorMap tmA, int use_tma) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ __align__(8) unsigned long long tma_bar;
  RW* sW = reinterpret_cast<RW*>(smraw);                                // [12][PX2][PY2]
  double* sFx = reinterpret_cast<double*>(smraw + god2_wbytes<RW>());  // [12][TX2+1][TY2]
  double* sFy = sFx + 12 * SM2_FX;                 // [12][TX2][TY2+1]
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * TX2, y0 = blockIdx.y * TY2;
  const long long nc = g.ncell;
  const double dt = STAGE == 0 ? dt_arg : slots->dt;
  // float64 tiles: the conserved fields and (gamma, T) of the padded tile by
  // two TMA boxes into the start of the region (staged layout, tile_ci); the
  // cells inside the domain are read from there, the others (ghost cells)
  // by their boundary mapping.  The primitives overwrite the region, so each
  // thread converts its cells (at most two) into registers first.
  constexpr bool EXACT = sizeof(RW) == sizeof(double);
  const bool tma = EXACT && use_tma;
  const double* sS = reinterpret_cast<const double*>(smraw);
  if (tma) {
    if (tid == 0) mbar_init(&tma_bar, 1);
    __syncthreads();
    if (tid == 0) {
      mbar_expect_tx(&tma_bar, (unsigned)(sizeof(double) * (TQ_N * SM2_QF)));
      tma_load_3d(smraw, &tmU, y0 - 4, x0 - 3, 0, &tma_bar);
      tma_load_3d(smraw + sizeof(double) * TQ_G * SM2_QF, &tmA, y0 - 4, x0 - 3, 0, &tma_bar);
    }
    if (!mbar_wait_bounded(&tma_bar)) {
      if (tid == 0) atomicOr(&slots->status, (unsigned)JB_ERR_TIMEOUT);
      mbar_wait_bounded(&tma_bar);  // the copy must not land after the block has left
      return;
    }
  }
  constexpr int NCELL_T = (SM2_Q + NT2 - 1) / NT2;  // padded cells per thread (2)
  double wk[NCELL_T][12];
#pragma unroll
  for (int r = 0; r < NCELL_T; ++r) {
    const int i = tid + r * NT2;
    if (i >= SM2_Q) break;
    const int px = i / PY2, py = i % PY2;
    const int x = x0 + px - 3, y = y0 + py - 3;
    double q[12], T = 1.0;
    if (tma && x >= 0 && x < g.nx && y >= 0 && y < g.ny) {
      const int k = tile_ci(px, py);
#pragma unroll
      for (int f = 0; f < 12; ++f) q[f] = sS[f * SM2_QF + k];
      T = sS[TQ_T * SM2_QF + k];
    } else {
      const Src s = map_cell<2>(g, x, y);
      if (s.kind == 0) {
        const size_t c = (size_t)s.xs * g.ny + s.ys;
#pragma unroll
        for (int f = 0; f < 12; ++f) {
          const double v = Uk[f * nc + c];
          q[f] = ((s.flip >> f) & 1) ? -v : v;
        }
        T = auxk[nc + c];
      } else if (s.kind == 1) {
#pragma unroll
        for (int f = 0; f < 12; ++f) q[f] = ghost(g, strips, s, f);
        T = ghost(g, strips, s, 13);
      } else {
#pragma unroll
        for (int f = 0; f < 12; ++f) q[f] = 1.0;
      }
    }
    cons_to_w<2>(m, q, T, wk[r]);
  }
  if (tma) __syncthreads();  // every cell has been read from the staged boxes
#pragma unroll
  for (int r = 0; r < NCELL_T; ++r) {
    const int i = tid + r * NT2;
    if (i >= SM2_Q) break;
#pragma unroll
    for (int f = 0; f < 12; ++f) sW[f * SM2_Q + i] = (RW)wk[r][f];
  }
  __syncthreads();
  {
    // x face t: cells (x0 + mxf - 1 | x0 + mxf) of row y0 + jy
    const int mxf = tid / TY2, jy = tid % TY2;
    double wL[12], wR[12], F[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) {
      const RW* b = sW + f * SM2_Q + mxf * PY2 + jy + 3;
      wL[f] = recon_L(g, b[0], b[PY2], b[2 * PY2], b[3 * PY2], b[4 * PY2]);
      wR[f] = recon_R(g, b[PY2], b[2 * PY2], b[3 * PY2], b[4 * PY2], b[5 * PY2]);
    }
    riemann_flux<2, 1, RS>(m, wL, wR, F);
#pragma unroll
    for (int f = 0; f < 12; ++f) sFx[f * SM2_FX + mxf * TY2 + jy] = F[f];
  }
  if (tid < SM2_FY) {
    const int jx = tid / (TY2 + 1), myf = tid % (TY2 + 1);
    double wL[12], wR[12], F[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) {
      const RW* b = sW + f * SM2_Q + (jx + 3) * PY2 + myf;
      wL[f] = recon_L(g, b[0], b[1], b[2], b[3], b[4]);
      wR[f] = recon_R(g, b[1], b[2], b[3], b[4], b[5]);
    }
    riemann_flux<2, 2, RS>(m, wL, wR, F);
#pragma unroll
    for (int f = 0; f < 12; ++f) sFy[f * SM2_FY + jx * (TY2 + 1) + myf] = F[f];
  }
  __syncthreads();
  const bool owner = tid < TX2 * TY2;
  const int ix = owner ? tid / TY2 : 0, iy = owner ? tid % TY2 : 0;
  const int gx = x0 + ix, gy = y0 + iy;
  const bool live = owner && gx < g.nx && gy < g.ny;
  const size_t cell = (size_t)gx * g.ny + gy;
  unsigned bits = 0;
  double amx = 0.0, amy = 0.0, dtm = __longlong_as_double(0x7ff0000000000000LL);
  if (live) {
    double q[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) {
      const double dF = sFx[f * SM2_FX + (ix + 1) * TY2 + iy] - sFx[f * SM2_FX + ix * TY2 + iy];
      const double dG = sFy[f * SM2_FY + ix * (TY2 + 1) + iy + 1] - sFy[f * SM2_FY + ix * (TY2 + 1) + iy];
#if JB_FAST
      const double rhs = dt * visc_add(g, f, cell, -(dF * g.idx + dG * g.idy));
#else
      const double rhs = dt * visc_add(g, f, cell, -(dF / g.dx + dG / g.dy));
#endif
      const double uk = Uk[f * nc + cell];
      double r;
      if (STAGE == 0) r = rhs;
      else if (STAGE == 1) r = uk + rhs;
      else if (STAGE == 2) r = 3.0 / 4.0 * Un[f * nc + cell] + 1.0 / 4.0 * (uk + rhs);
      else r = 1.0 / 3.0 * Un[f * nc + cell] + 2.0 / 3.0 * (uk + rhs);
      out[f * nc + cell] = r;
      q[f] = r;
    }
    // float32 reconstruction = the mixed variant: per-cell temperature solve
    if (STAGE != 0)
      bits = finish_state<2, sizeof(RW) == 4>(m, g, fin, q, auxk[nc + cell], cell, amx, amy, dtm, slots);
  }
  if (STAGE != 0) finish_reduce(fin, amx, amy, dtm, bits, slots);
}

// 1D: a block of NT1 threads covers NT1 - 1 cells and their NT1 faces.
template <class RW>
__host__ __device__ constexpr size_t god1_wbytes() {
  return (sizeof(RW) * 11 * (NT1 + 5) + 15) / 16 * 16;
}
template <class RW>
__host__ __device__ constexpr size_t god1_smem() {
  return god1_wbytes<RW>() + sizeof(double) * 11 * NT1;
}

template <int STAGE, int RS, class RW>
__global__ void __launch_bounds__(NT1) k_god1d(MP m, Grid g, const double* __restrict__ Uk,
                                              const double* __restrict__ auxk, const double* __restrict__ Un,
                                              double* __restrict__ out, double* __restrict__ cand,
                                              const double* __restrict__ strips, Slots* slots, int midx,
                                              double dt_arg) {
  constexpr int PW = NT1 + 5;
  extern __shared__ __align__(128) unsigned char smraw[];
  RW* sW = reinterpret_cast<RW*>(smraw);                               // [11][PW]: padded cell x0 - 3 + j
  double* sF = reinterpret_cast<double*>(smraw + god1_wbytes<RW>());  // [11][NT1]: face x0 + t
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * (NT1 - 1);
  const long long nc = g.ncell;
  const double dt = STAGE == 0 ? dt_arg : slots->dt;
  for (int j = tid; j < PW; j += NT1) {
    const Src s = map_cell<1>(g, x0 - 3 + j, 0);
    double q[11], T = 1.0;
    if (s.kind == 0) {
      const size_t c = (size_t)s.xs;
#pragma unroll
      for (int f = 0; f < 11; ++f) {
        const double v = Uk[f * nc + c];
        q[f] = ((s.flip >> f) & 1) ? -v : v;
      }
      T = auxk[nc + c];
    } else if (s.kind == 1) {
#pragma unroll
      for (int f = 0; f < 11; ++f) q[f] = ghost(g, strips, s, f);
      T = ghost(g, strips, s, 12);
    } else {
#pragma unroll
      for (int f = 0; f < 11; ++f) q[f] = 1.0;
    }
    double w[11];
    cons_to_w<1>(m, q, T, w);
#pragma unroll
    for (int f = 0; f < 11; ++f) sW[f * PW + j] = (RW)w[f];
  }
  __syncthreads();
  {
    // face x0 + t: left-biased from padded j = t .. t+4, right from t+1 .. t+5
    double wL[11], wR[11], F[11];
#pragma unroll
    for (int f = 0; f < 11; ++f) {
      const RW* b = sW + f * PW + tid;
      wL[f] = recon_L(g, b[0], b[1], b[2], b[3], b[4]);
      wR[f] = recon_R(g, b[1], b[2], b[3], b[4], b[5]);
    }
    riemann_flux<1, 1, RS>(m, wL, wR, F);
#pragma unroll
    for (int f = 0; f < 11; ++f) sF[f * NT1 + tid] = F[f];
  }
  __syncthreads();
  const int gx = x0 + tid;
  const bool live = tid < NT1 - 1 && gx < g.nx;
  unsigned bits = 0;
  if (live) {
    const size_t cell = (size_t)gx;
    double q[11];
#pragma unroll
    for (int f = 0; f < 11; ++f) {
      const double dF = sF[f * NT1 + tid + 1] - sF[f * NT1 + tid];
#if JB_FAST
      const double rhs = dt * visc_add(g, f, cell, -(dF * g.idx));
#else
      const double rhs = dt * visc_add(g, f, cell, -(dF / g.dx));
#endif
      const double uk = Uk[f * nc + cell];
      double r;
      if (STAGE == 0) r = rhs;
      else if (STAGE == 1) r = uk + rhs;
      else if (STAGE == 2) r = 3.0 / 4.0 * Un[f * nc + cell] + 1.0 / 4.0 * (uk + rhs);
      else r = 1.0 / 3.0 * Un[f * nc + cell] + 2.0 / 3.0 * (uk + rhs);
      out[f * nc + cell] = r;
      q[f] = r;
    }
    if (STAGE != 0) {
      const double rho = q[0];
      const double u = q[1] / rho;
      const double e = q[2] / rho - 0.5 * (u * u);
      double Y8[NR], Yf[NS];
#pragma unroll
      for (int k = 0; k < NR; ++k) Y8[k] = q[3 + k] / rho;
      fill_Y(Y8, Yf);
      double cnd[JB_NCAND];
      bits = halley_any(m, e, Yf, get_R(m, Yf), auxk[nc + cell], cnd);
#pragma unroll
      for (int i = 0; i < JB_NCAND; ++i) cand[i * nc + cell] = cnd[i];
    }
  }
  if (STAGE != 0) block_reduce_store(0.0, 0.0, 0.0, bits, slots, 0, false, false, midx);
}
