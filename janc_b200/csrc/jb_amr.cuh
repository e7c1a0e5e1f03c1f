// Block-structured AMR stepping on blocks with their ghost layers
// (src/janc_v2/simulation/time_step/TVD_RK3.py:15-36 advance_one_step_amr,
// with the block functions of simulation/set_simulator.py:37-42 and
// :97-113): the block layer (the external jaxamr package) fills each
// block's 3-cell ghost layers; the reference then applies, per block,
//   flux_func(U, aux) = pad(dt * total_flux(U, aux), 3)   (vmapped)
//   update_func       = update_aux                          (vmapped)
// on the ghost-padded block, and after the three stages the chemistry and
// update_aux on the unpadded blocks.  vmap makes every reduction per block:
// the LF wave-speed maxima are nanmax over the block's padded array, and the
// temperature solve stops when the block's own max |res| <= tol (JAX's
// batched while_loop keeps each block's carry once its predicate is false).
//
// Layout: blocks [nb][nv + 2][PX][PY] float64, C-contiguous (the reference's
// blk_data: U fields then gamma, T), PX = bx + 6, PY = by + 6 for padded
// blocks; the chemistry takes unpadded blocks [nb][nv + 2][bx][by].
//
// One CTA per block, so each block's reductions stay inside its CTA:
//   k_amr_stage  alpha of the padded block; the interior in tiles of
//                ATX x ATY cells (LF + WENO5-JS / MUSCL faces in shared
//                memory, the RK combination); every ghost entry takes the
//                combination with a zero right-hand side (the reference pads
//                the rhs with zeros); update_aux over the whole padded block
//                with the block's global stop: a first pass ORs the Halley
//                residual masks, a second recomputes the iterates and takes
//                the block's iteration count (no iterate buffer)
//   k_amr_chem   point-implicit chemistry per cell, U + S, and update_aux
//                over the block with its global stop (two passes as above)

namespace {  // internal linkage

constexpr int AMR_NT = 256;
constexpr int ATX = 15, ATY = 16;  // interior tile: 16 x 16 x faces for 256 threads
constexpr int APX = ATX + 6, APY = ATY + 6, AQ = APX * APY;
constexpr int A_HX = APX * ATY, A_HY = ATX * APY, A_FX = (ATX + 1) * ATY, A_FY = ATX * (ATY + 1);
constexpr size_t AMR_STAGE_SMEM = sizeof(double) * (14 * AQ + 4 * AQ + 2 * A_HX + 2 * A_HY + A_FX + A_FY);

struct AmrBlocks {
  int nb, bx, by, padded;  // padded: the arrays carry the 3-cell ghost layers
  double dx, dy, idx, idy;
};

// Block-wide reductions (all threads of the CTA call them).
__device__ __forceinline__ void amr_block_max2(double& a, double& b) {
  __shared__ double ra[32], rb[32];
  a = warp_max(a);
  b = warp_max(b);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { ra[w] = a; rb[w] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) { a = fmax(a, ra[i]); b = fmax(b, rb[i]); }
    ra[0] = a;
    rb[0] = b;
  }
  __syncthreads();
  a = ra[0];
  b = rb[0];
  __syncthreads();
}

__device__ __forceinline__ unsigned amr_block_or(unsigned v) {
  __shared__ unsigned ro[32];
  v = warp_or(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) ro[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) v |= ro[i];
    ro[0] = v;
  }
  __syncthreads();
  v = ro[0];
  __syncthreads();
  return v;
}

// e, Y and R of a 2D state cell c (field stride nc): update_aux
// (solver_2D/aux_func.py:21-29) as the select pass forms them.
__device__ __forceinline__ void amr_eYR(const MP& m, const double* Ub, long long nc, long long c, double& e,
                                        double* Yf, double& R) {
  constexpr int nY = 4;
  const double rho = Ub[c];
  const double u = Ub[nc + c] / rho, v = Ub[2 * nc + c] / rho;
  e = Ub[3 * nc + c] / rho - 0.5 * (u * u + v * v);
  double Y8[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = Ub[(nY + k) * nc + c] / rho;
  fill_Y(Y8, Yf);
  R = get_R(m, Yf);
}

// update_aux of the nc cells of one block (state Ub, initial temperatures
// T0b, result into Ab = [gamma][T]) with the block's global stop.
__device__ void amr_update_block(const MP& m, const double* Ub, const double* T0b, double* Ab, long long nc,
                                 unsigned& st) {
  unsigned bits = 0;
  for (long long c = threadIdx.x; c < nc; c += blockDim.x) {
    double e, Yf[NS], R, cnd[JB_NCAND];
    amr_eYR(m, Ub, nc, c, e, Yf, R);
    bits |= halley_any(m, e, Yf, R, T0b[c], cnd);
  }
  const int n = halley_count(amr_block_or(bits));
  for (long long c = threadIdx.x; c < nc; c += blockDim.x) {
    double e, Yf[NS], R, cnd[JB_NCAND];
    amr_eYR(m, Ub, nc, c, e, Yf, R);
    halley_any(m, e, Yf, R, T0b[c], cnd);
    const double T = cnd[n];
    const double cp = cp_mix(m, T, Yf);
    Ab[c] = cp / (cp - R);
    Ab[nc + c] = T;
    if (!(T == T)) st |= JB_ERR_NONFINITE;
  }
}

typedef jb_amr_io AmrIO;  // the stage call's block arrays (jb_ops.h)

// STAGE 1..3: one SSP-RK3 stage of every padded block (TVD_RK3.py:17-35):
// out = a U0 + b (G + pad(dt L(G))) and its update_aux started from G's T.
// STAGE 0: the block flux function alone, out = pad(dt L(G))
// (set_simulator.py:37-40).  G: the stage input with its ghost layers
// filled; U0: the step's first stage input.
template <int STAGE>
__global__ void __launch_bounds__(AMR_NT) k_amr_stage(MP m, Grid g, AmrBlocks B, AmrIO io, Slots* slots,
                                                    double dt) {
  extern __shared__ __align__(128) unsigned char smraw[];
  constexpr int nv = 12;
  double* sQ = reinterpret_cast<double*>(smraw);  // [14][APX][APY]: U, gamma, T
  double* sP = sQ + 14 * AQ;                       // [4][APX][APY]: rho, u, v, p
  double* sHxp = sP + 4 * AQ;                      // [APX][ATY]
  double* sHxm = sHxp + A_HX;
  double* sHyp = sHxm + A_HX;                      // [ATX][APY]
  double* sHym = sHyp + A_HY;
  double* sFx = sHym + A_HY;                       // [ATX+1][ATY]
  double* sFy = sFx + A_FX;                        // [ATX][ATY+1]
  const int tid = threadIdx.x;
  const int PX = B.bx + 6, PY = B.by + 6;
  const long long nc = (long long)PX * PY;
  const long long b = blockIdx.x;
  const double* gU = io.gU + b * io.gsU;
  const double* gA = io.gA + b * io.gsA;
  const double* u0 = STAGE >= 2 ? io.u0 + b * io.u0s : nullptr;
  double* oU = io.oU + b * io.osU;
  unsigned st = 0;
  // field q of padded cell c of the stage input (q < nv: U, nv: gamma, nv + 1: T)
  auto gq = [&](int q, long long c) { return q < nv ? gU[q * nc + c] : gA[(q - nv) * nc + c]; };

  // ---- LF wave speeds: nanmax(|u| + a), nanmax(|v| + a) over the padded
  // block (flux_splitting/LF.py:11-12 on the vmapped block)
  double ax = 0.0, ay = 0.0;
  for (long long c = tid; c < nc; c += AMR_NT) {
    double q[nv];
#pragma unroll
    for (int f = 0; f < nv; ++f) q[f] = gU[f * nc + c];
    const Prim<2> pr = u_to_prim<2>(m, q, gA[c], gA[nc + c]);
    ax = fmax(ax, fabs(pr.u) + pr.a);
    ay = fmax(ay, fabs(pr.v) + pr.a);
  }
  amr_block_max2(ax, ay);

  // ---- the interior, tile by tile
  const bool owner = tid < ATX * ATY;
  const int ix = owner ? tid / ATY : 0, iy = owner ? tid % ATY : 0;
  const int ntx = (B.bx + ATX - 1) / ATX, nty = (B.by + ATY - 1) / ATY;
  for (int t = 0; t < ntx * nty; ++t) {
    const int x0 = (t / nty) * ATX, y0 = (t % nty) * ATY;  // interior coordinates of the tile
    // padded tile: block padded rows x0 .. x0 + APX - 1, columns y0 .. y0 + APY - 1
    for (int i = tid; i < AQ; i += AMR_NT) {
      const int px = x0 + i / APY, py = y0 + i % APY;
      if (px < PX && py < PY) {
        const long long c = (long long)px * PY + py;
#pragma unroll
        for (int q = 0; q < 14; ++q) sQ[q * AQ + i] = gq(q, c);
      } else {
        // beyond the padded block: read only by faces of cells outside the block
#pragma unroll
        for (int q = 0; q < 14; ++q) sQ[q * AQ + i] = 1.0;
      }
    }
    __syncthreads();
    for (int i = tid; i < AQ; i += AMR_NT) {
      double q[nv];
#pragma unroll
      for (int f = 0; f < nv; ++f) q[f] = sQ[f * AQ + i];
      double rho, u, v, p;
      flux_prims<2>(m, q, sQ[13 * AQ + i], rho, u, v, p);
      sP[i] = rho;
      sP[AQ + i] = u;
      sP[2 * AQ + i] = v;
      sP[3 * AQ + i] = p;
    }
    __syncthreads();
    const int gx = x0 + ix, gy = y0 + iy;
    const bool live = owner && gx < B.bx && gy < B.by;
    const long long cell = (long long)(gx + 3) * PY + (gy + 3);
    for (int f = 0; f < nv; ++f) {
      // split fluxes H+- = 0.5 (F +- alpha U) (flux_splitting/LF.py:4-16)
      for (int i = tid; i < A_HX + A_HY; i += AMR_NT) {
        int px, py, dir;
        if (i < A_HX) { px = i / ATY; py = i % ATY + 3; dir = 0; }
        else { const int j = i - A_HX; px = j / APY + 3; py = j % APY; dir = 1; }
        const int c = px * APY + py;
        const double qf = sQ[f * AQ + c];
        const double F = lf_flux<2>(f, dir, qf, sP[c], sP[AQ + c], sP[2 * AQ + c], sP[3 * AQ + c], sQ[3 * AQ + c]);
        const double al = dir == 0 ? ax : ay;
        const double hp = 0.5 * (F + al * qf), hm = 0.5 * (F - al * qf);
        if (dir == 0) { sHxp[px * ATY + (py - 3)] = hp; sHxm[px * ATY + (py - 3)] = hm; }
        else { sHyp[(px - 3) * APY + py] = hp; sHym[(px - 3) * APY + py] = hm; }
      }
      __syncthreads();
      // face values F = L(H+) + R(H-) (flux.py:56-68, WENO5_JS.py / MUSCL.py)
      {
        const int mxf = tid / ATY, jy = tid % ATY;  // x faces: (ATX + 1) x ATY = 256
        const double* hp = sHxp + jy;
        const double* hm = sHxm + jy;
        const double L = recon_L(g, hp[mxf * ATY], hp[(mxf + 1) * ATY], hp[(mxf + 2) * ATY], hp[(mxf + 3) * ATY],
                                 hp[(mxf + 4) * ATY]);
        const double Rr = recon_R(g, hm[(mxf + 1) * ATY], hm[(mxf + 2) * ATY], hm[(mxf + 3) * ATY],
                                  hm[(mxf + 4) * ATY], hm[(mxf + 5) * ATY]);
        sFx[mxf * ATY + jy] = L + Rr;
        if (tid < A_FY) {
          const int jx = tid / (ATY + 1), myf = tid % (ATY + 1);
          const double* gp = sHyp + jx * APY + myf;
          const double* gm = sHym + jx * APY + myf;
          const double Lg = recon_L(g, gp[0], gp[1], gp[2], gp[3], gp[4]);
          const double Rg = recon_R(g, gm[1], gm[2], gm[3], gm[4], gm[5]);
          sFy[jx * (ATY + 1) + myf] = Lg + Rg;
        }
      }
      __syncthreads();
      // divergence and the RK combination (TVD_RK3.py:17, 24, 31)
      if (live) {
        const double dF = sFx[(ix + 1) * ATY + iy] - sFx[ix * ATY + iy];
        const double dG = sFy[ix * (ATY + 1) + iy + 1] - sFy[ix * (ATY + 1) + iy];
#if JB_FAST
        const double rhs = dt * (-(dF * B.idx + dG * B.idy));
#else
        const double rhs = dt * (-(dF / B.dx + dG / B.dy));
#endif
        const double uk = sQ[f * AQ + (ix + 3) * APY + (iy + 3)];
        double r;
        if (STAGE == 0) r = rhs;
        else if (STAGE == 1) r = uk + rhs;
        else if (STAGE == 2) r = 3.0 / 4.0 * u0[f * nc + cell] + 1.0 / 4.0 * (uk + rhs);
        else r = 1.0 / 3.0 * u0[f * nc + cell] + 2.0 / 3.0 * (uk + rhs);
        oU[f * nc + cell] = r;
      }
      __syncthreads();
    }
  }
  // ---- ghost entries: the combination with the zero-padded rhs
  for (long long c = tid; c < nc; c += AMR_NT) {
    const int px = (int)(c / PY), py = (int)(c % PY);
    if (px >= 3 && px < PX - 3 && py >= 3 && py < PY - 3) continue;
    for (int f = 0; f < nv; ++f) {
      const double rhs = 0.0;
      double r;
      if (STAGE == 0) r = rhs;
      else if (STAGE == 1) r = gU[f * nc + c] + rhs;
      else if (STAGE == 2) r = 3.0 / 4.0 * u0[f * nc + c] + 1.0 / 4.0 * (gU[f * nc + c] + rhs);
      else r = 1.0 / 3.0 * u0[f * nc + c] + 2.0 / 3.0 * (gU[f * nc + c] + rhs);
      oU[f * nc + c] = r;
    }
  }
  if (!(ax == ax) || !(ay == ay)) st |= JB_ERR_NONFINITE;
  if (STAGE > 0) {
    __syncthreads();
    // ---- update_aux of the padded block from G's temperatures
    amr_update_block(m, oU, gA + nc, io.oA + b * io.osA, nc, st);
  }
  st = amr_block_or(st);
  if (tid == 0 && st) atomicOr(&slots->status, st);
}

// update_aux of every block (vmap(update_aux), set_simulator.py:41) with
// each block's own stop: U [nb][nv][X][Y], aux_in / aux_out [nb][2][X][Y].
template <int UNUSED>
__global__ void __launch_bounds__(AMR_NT) k_amr_update(MP m, long long nc, const double* __restrict__ U,
                                                     const double* __restrict__ aux_in, double* __restrict__ aux_out,
                                                     Slots* slots) {
  const long long b = blockIdx.x;
  unsigned st = 0;
  amr_update_block(m, U + b * 12 * nc, aux_in + b * 2 * nc + nc, aux_out + b * 2 * nc, nc, st);
  st = amr_block_or(st);
  if (threadIdx.x == 0 && st) atomicOr(&slots->status, st);
}

// Chemistry of every unpadded block (set_simulator.py:106-113):
// out = U + S(U, T, dt) and update_aux of the block started from its T.
// GEN: the specialised chemistry (CHEM_SH shared doubles per thread).
template <bool GEN>
__global__ void __launch_bounds__(128) k_amr_chem(MP m, AmrBlocks B, const double* __restrict__ blk,
                                                  double* __restrict__ out, Slots* slots, double dt) {
  extern __shared__ double shc[];
  constexpr int nY = 4, nv = 12;
  const long long nc = (long long)B.bx * B.by;
  const double* Ib = blk + (long long)blockIdx.x * (nv + 2) * nc;
  double* Ob = out + (long long)blockIdx.x * (nv + 2) * nc;
  unsigned st = 0;
  for (long long c = threadIdx.x; c < nc; c += blockDim.x) {
    const double T = Ib[(nv + 1) * nc + c];
    const double rho = Ib[c];
    double Y8[NR], S[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) Y8[k] = Ib[(nY + k) * nc + c] / rho;
#if JB_FAST
    if (GEN) chem_cell_gen(m, rho, Y8, T, dt, S, st, shc + threadIdx.x, blockDim.x);
    else chem_cell(m, rho, Y8, T, dt, S, st);
#else
    chem_cell(m, rho, Y8, T, dt, S, st);
#endif
#pragma unroll
    for (int f = 0; f < nY; ++f) Ob[f * nc + c] = Ib[f * nc + c];
#pragma unroll
    for (int k = 0; k < NR; ++k) Ob[(nY + k) * nc + c] = Ib[(nY + k) * nc + c] + S[k];
  }
  __syncthreads();
  amr_update_block(m, Ob, Ib + (nv + 1) * nc, Ob + nv * nc, nc, st);
  st = amr_block_or(st);
  if (threadIdx.x == 0 && st) atomicOr(&slots->status, st);
}

}  // namespace
