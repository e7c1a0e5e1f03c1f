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
//   k_amr_stage   alpha of the padded block; the interior in tiles of
//                 tx x ty cells, a shape the host picks per block size so
//                 that few, well-filled tiles cover the block (LF + WENO5-JS
//                 / MUSCL faces in shared memory, the RK combination); every
//                 ghost entry takes the combination with a zero right-hand
//                 side (the reference pads the rhs with zeros); update_aux
//                 over the whole padded block
//   k_amr_update  update_aux of blocks alone
// update_aux runs the reference's loop in lockstep over the block: one
// Halley iteration of every cell per round, the block's OR of "residual
// above tol" / "residual NaN" deciding whether another round follows (the
// iterates live in the output's gamma / T slots), so a cell is evaluated
// once per iteration the block takes.
//   k_amr_chem    point-implicit chemistry, one thread per cell of all
//                 blocks, U + S; k_amr_update then solves the temperatures

namespace {  // internal linkage

constexpr int AMR_NT = 256;
constexpr int AMR_AQ_MAX = 640;  // padded cells of a tile, (tx + 6)(ty + 6)
constexpr int AMR_H_MAX = 420;   // (tx + 6) ty and tx (ty + 6) when (tx + 1) ty, tx (ty + 1) <= 256
constexpr size_t AMR_STAGE_SMEM = sizeof(double) * (4 * AMR_AQ_MAX + 4 * AMR_H_MAX + 2 * AMR_NT);

struct AmrBlocks {
  int nb, bx, by, tx, ty;  // blocks, block cells, interior tile of k_amr_stage
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
// T0b, result into Ab = [gamma][T]) with the block's global stop
// (thermo_model.py:135-153 on the vmapped block): round i evaluates the
// residual at every cell's i-th iterate; the loop ends when no residual
// exceeds tol, when one is NaN (jnp.max is then NaN and the test false) or
// after 5 iterations.  T0b may equal Ab + nc.
__device__ void amr_update_block(const MP& m, const double* Ub, const double* T0b, double* Ab, long long nc,
                                 unsigned& st) {
  double* Tn = Ab;       // each cell's next iterate (the gamma slot until the end)
  double* Tc = Ab + nc;  // its current iterate
  for (long long c = threadIdx.x; c < nc; c += blockDim.x) Tc[c] = T0b[c];
  for (int i = 0;; ++i) {
    unsigned bits = 0;
    for (long long c = threadIdx.x; c < nc; c += blockDim.x) {
      double e, Yf[NS], R;
      amr_eYR(m, Ub, nc, c, e, Yf, R);
      const double T = Tc[c];
      const Th t = thermo_mix(m, T, Yf);
      const double res = (t.h - R * T) - e;
      const double d1 = t.cp - R, d2 = t.dcp;
      if (fabs(res) > HALLEY_TOL) bits |= 1u;
      if (res != res) bits |= 2u;
      Tn[c] = T + ((-2.0 * res) * d1) / ((2.0 * (d1 * d1)) - res * d2);
    }
    bits = amr_block_or(bits);
    if (!(bits & 1u) || (bits & 2u) || i == HALLEY_MAX) break;
    for (long long c = threadIdx.x; c < nc; c += blockDim.x) Tc[c] = Tn[c];
  }
  for (long long c = threadIdx.x; c < nc; c += blockDim.x) {
    double e, Yf[NS], R;
    amr_eYR(m, Ub, nc, c, e, Yf, R);
    const double T = Tc[c];
    const double cp = cp_mix(m, T, Yf);
    Ab[c] = cp / (cp - R);
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
#ifndef JB_AMR_MINB
#define JB_AMR_MINB 4  // 64 registers (8 B of spills)
#endif
__global__ void __launch_bounds__(AMR_NT, JB_AMR_MINB) k_amr_stage(MP m, Grid g, AmrBlocks B, AmrIO io, Slots* slots,
                                                    double dt) {
  extern __shared__ __align__(128) unsigned char smraw[];
  constexpr int nv = 12;
  const int TX = B.tx, TY = B.ty, APX = TX + 6, APY = TY + 6, AQ = APX * APY;
  const int HX = APX * TY, HY = TX * APY;
  double* sP = reinterpret_cast<double*>(smraw);  // [4][APX][APY]: rho, u, v, p
  double* sHxp = sP + 4 * AQ;                      // [APX][TY]
  double* sHxm = sHxp + HX;
  double* sHyp = sHxm + HX;                        // [TX][APY]
  double* sHym = sHyp + HY;
  double* sFx = sHym + HY;                         // [TX+1][TY]
  double* sFy = sFx + (TX + 1) * TY;               // [TX][TY+1]
  const int tid = threadIdx.x;
  const int PX = B.bx + 6, PY = B.by + 6;
  const long long nc = (long long)PX * PY;
  const long long b = blockIdx.x;
  const double* gU = io.gU + b * io.gsU;
  const double* gA = io.gA + b * io.gsA;
  const double* u0 = STAGE >= 2 ? io.u0 + b * io.u0s : nullptr;
  double* oU = io.oU + b * io.osU;
  unsigned st = 0;

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
  const bool owner = tid < TX * TY;
  const int ix = owner ? tid / TY : 0, iy = owner ? tid % TY : 0;
  const int ntx = (B.bx + TX - 1) / TX, nty = (B.by + TY - 1) / TY;
  for (int t = 0; t < ntx * nty; ++t) {
    const int x0 = (t / nty) * TX, y0 = (t % nty) * TY;  // interior coordinates of the tile
    // primitives of the padded tile (block padded rows x0 .. x0 + APX - 1,
    // columns y0 .. y0 + APY - 1); cells beyond the padded block are read
    // only by faces of cells outside the block
    for (int i = tid; i < AQ; i += AMR_NT) {
      const int px = x0 + i / APY, py = y0 + i % APY;
      double rho = 1.0, u = 1.0, v = 1.0, p = 1.0;
      if (px < PX && py < PY) {
        const long long c = (long long)px * PY + py;
        double q[nv];
#pragma unroll
        for (int f = 0; f < nv; ++f) q[f] = gU[f * nc + c];
        flux_prims<2>(m, q, gA[nc + c], rho, u, v, p);
      }
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
      for (int i = tid; i < HX + HY; i += AMR_NT) {
        int px, py, dir;
        if (i < HX) { px = i / TY; py = i % TY + 3; dir = 0; }
        else { const int j = i - HX; px = j / APY + 3; py = j % APY; dir = 1; }
        const int c = px * APY + py;
        const int bxp = x0 + px, byp = y0 + py;
        const long long gc = (long long)bxp * PY + byp;
        const bool in = bxp < PX && byp < PY;
        const double qf = in ? gU[f * nc + gc] : 1.0;
        const double E = in ? gU[3 * nc + gc] : 1.0;
        const double F = lf_flux<2>(f, dir, qf, sP[c], sP[AQ + c], sP[2 * AQ + c], sP[3 * AQ + c], E);
        const double al = dir == 0 ? ax : ay;
        const double hp = 0.5 * (F + al * qf), hm = 0.5 * (F - al * qf);
        if (dir == 0) { sHxp[px * TY + (py - 3)] = hp; sHxm[px * TY + (py - 3)] = hm; }
        else { sHyp[(px - 3) * APY + py] = hp; sHym[(px - 3) * APY + py] = hm; }
      }
      __syncthreads();
      // face values F = L(H+) + R(H-) (flux.py:56-68, WENO5_JS.py / MUSCL.py)
      if (tid < (TX + 1) * TY) {
        const int mxf = tid / TY, jy = tid % TY;
        const double* hp = sHxp + jy;
        const double* hm = sHxm + jy;
        const double L = recon_L(g, hp[mxf * TY], hp[(mxf + 1) * TY], hp[(mxf + 2) * TY], hp[(mxf + 3) * TY],
                                 hp[(mxf + 4) * TY]);
        const double Rr = recon_R(g, hm[(mxf + 1) * TY], hm[(mxf + 2) * TY], hm[(mxf + 3) * TY],
                                  hm[(mxf + 4) * TY], hm[(mxf + 5) * TY]);
        sFx[mxf * TY + jy] = L + Rr;
      }
      if (tid < TX * (TY + 1)) {
        const int jx = tid / (TY + 1), myf = tid % (TY + 1);
        const double* gp = sHyp + jx * APY + myf;
        const double* gm = sHym + jx * APY + myf;
        const double Lg = recon_L(g, gp[0], gp[1], gp[2], gp[3], gp[4]);
        const double Rg = recon_R(g, gm[1], gm[2], gm[3], gm[4], gm[5]);
        sFy[jx * (TY + 1) + myf] = Lg + Rg;
      }
      __syncthreads();
      // divergence and the RK combination (TVD_RK3.py:17, 24, 31)
      if (live) {
        const double dF = sFx[(ix + 1) * TY + iy] - sFx[ix * TY + iy];
        const double dG = sFy[ix * (TY + 1) + iy + 1] - sFy[ix * (TY + 1) + iy];
#if JB_FAST
        const double rhs = dt * (-(dF * B.idx + dG * B.idy));
#else
        const double rhs = dt * (-(dF / B.dx + dG / B.dy));
#endif
        const double uk = gU[f * nc + cell];
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
// each block's own stop: U [nb][nv][X][Y] (field stride nc, block stride
// su), aux_in / aux_out [nb][2][X][Y] (block stride sa).
template <int UNUSED>
__global__ void __launch_bounds__(AMR_NT) k_amr_update(MP m, long long nc, const double* U, long long su,
                                                     const double* aux_in, double* aux_out, long long sa,
                                                     Slots* slots) {
  const long long b = blockIdx.x;
  unsigned st = 0;
  amr_update_block(m, U + b * su, aux_in + b * sa + nc, aux_out + b * sa, nc, st);
  st = amr_block_or(st);
  if (threadIdx.x == 0 && st) atomicOr(&slots->status, st);
}

// Chemistry of every cell of nb unpadded blocks (the vmapped
// reaction_source_terms of set_simulator.py:109-111): out = U + S(U, T, dt),
// the flow fields copied; one thread per cell.  out may equal blk.
// GEN: the specialised chemistry (CHEM_SH shared doubles per thread).
template <bool GEN>
__global__ void __launch_bounds__(128, 3) k_amr_chem(MP m, AmrBlocks B, const double* blk, double* out,
                                                     Slots* slots, double dt) {
  extern __shared__ double shc[];
  constexpr int nY = 4, nv = 12;
  const long long nc = (long long)B.bx * B.by;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned st = 0;
  if (i < nc * B.nb) {
    const long long b = i / nc, c = i % nc;
    const double* Ib = blk + b * (nv + 2) * nc;
    double* Ob = out + b * (nv + 2) * nc;
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
  block_reduce_store(0.0, 0.0, 0.0, st << 16, slots, 0, false, false, -1);
}

}  // namespace
