// Batched ensemble of 1D reacting-flow instances (detonation tubes of uneven
// length and composition) advanced by ONE persistent kernel per run.
//
// Each instance is served by its own group of CTAs.  A time step of one
// instance is the reference's advance_one_step (set_simulator.py:117-122:
// TVD_RK3 over flux_func, then reaction_source_terms and update_aux) with
// its own CFL time step (set_simulator.py:420-447) and its own LF alpha per
// RK stage; the reductions that need every cell of the instance (alpha,
// the CFL minimum, the global Halley stopping mask of thermo_model.py:
// 157-172) are atomics into the instance's slots followed by a barrier of
// its CTA group.  The kernel is launched cooperatively, so all CTAs are
// resident together and the group barriers cannot wait on a CTA that never
// runs; every wait is still bounded in time and gives up with
// JB_ERR_TIMEOUT instead of hanging.
//
// The phases of one step and the buffers they touch (per instance):
//   stage 1  U, aux           -> W0, cand      (Halley mask 0)
//   select 1 W0, cand         -> A0            (alpha 1)
//   stage 2  W0, A0, U        -> W1, cand      (mask 1)
//   select 2 W1, cand         -> A1            (alpha 2)
//   stage 3  W1, A1, U        -> W0, cand      (mask 2)
//   chem     W0, cand[mask 2] -> U, cand       (mask 3; the stage-3
//            temperature is taken straight from the Halley iterates)
//   select 4 U, cand          -> aux           (alpha of the next stage 1,
//                                               CFL minimum of the next dt)
// with a group barrier after each, seven per step (the float64 ensemble,
// whose instances keep the reference's global stop of the temperature
// solve).  The mixed variant solves each cell's temperature where its new
// state is written (as its single-case step does), so no select pass
// follows and a step has four phases:
//   stage 1  U, aux      -> W0, A0      (alpha 1)
//   stage 2  W0, A0, U   -> W1, A1      (alpha 2)
//   stage 3  W1, A1, U   -> W0, A0
//   chem     W0, A0      -> U, aux      (alpha of the next stage 1, CFL
//                                        minimum of the next dt)
// each also writing the outlet ghost strips of its new state.  Slot sets
// alternate between even and odd steps, so clearing one never races with
// reading the other.
#define JB_NS ens
#define JB_FAST 1
#include "jb_kernels.cuh"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/janc_b200.h"
#include "jb_ensemble.h"
#include "jb_ops.h"

namespace jb {
namespace ens {

static_assert(sizeof(jb_ens_inst) % 8 == 0, "instance table entries are copied as 8-byte words");

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr long long SPIN_MAX = 1LL << 26;  // polls of one wait (>= 64 ns apart)

// Barrier of the CTAs serving one instance; every thread of the block calls
// it.  Returns false when the run was aborted (a wait here or elsewhere gave
// up), in which case the caller returns.
__device__ __forceinline__ bool group_sync(const jb_ens_inst& I, unsigned& target, jb_ens_ctl* ctl,
                                           unsigned long long limit_ns, int inst, int phase) {
  __shared__ int s_go;
  __syncthreads();
  if (threadIdx.x == 0) {
    int go = 1;
    if (I.ncta > 1) {
      target += (unsigned)I.ncta;
      __threadfence();
      atomicAdd(I.bar, 1u);
      const unsigned long long t0 = global_ns();
      for (long long it = 0;; ++it) {
        if (ld_acquire_u32(I.bar) >= target) break;
        if (*(volatile unsigned*)&ctl->abort) { go = 0; break; }
        if (it >= SPIN_MAX || global_ns() - t0 > limit_ns) {
          if (atomicExch(&ctl->timeout, 1u) == 0u) {
            ctl->where_inst = (unsigned)inst;
            ctl->where_phase = (unsigned)phase;
          }
          atomicExch(&ctl->abort, 1u);
          go = 0;
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
    } else if (*(volatile unsigned*)&ctl->abort) {
      go = 0;
    }
    s_go = go;
  }
  __syncthreads();
  return s_go != 0;
}

// Clear one slot set for reuse; the status word accumulates over the run.
__device__ __forceinline__ void slots_clear(Slots* s) {
  for (int i = 0; i < 4; ++i) { s->ax[i] = 0ull; s->ay[i] = 0ull; s->mask[i] = 0u; }
  s->dtmin_next = 0x7ff0000000000000ull;
  s->dtnan = 0u;
  s->dt = 0.0;
}

template <int NT>
struct Shape {
  // 170 registers a thread at most for 64 and 128 threads (the chemistry's
  // footprint), one CTA an SM at 256
  static constexpr int MINB = NT == 64 ? 6 : NT == 128 ? 3 : 1;
};

template <class R, int NT>
__host__ __device__ constexpr size_t ens_smem_bytes() {
  return smem1d_bytes<R, NT>(12) > sizeof(double) * CHEM_SH * NT ? smem1d_bytes<R, NT>(12)
                                                                  : sizeof(double) * CHEM_SH * NT;
}

// The mechanism of the running ensemble.  Each launch copies it here from
// the ensemble's device copy (a node of the same graph), so ensembles with
// different mechanisms may alternate on one stream.
__constant__ MP c_mech;

// The phases below are separate (non-inlined) functions so that each is
// register-allocated on its own: the chemistry needs most of the register
// file, the loop state of the step only a few registers.

// Select pass over this CTA's cells of one instance, reduced into `s`
// (alpha into ax[aidx]; with CFL also the CFL minimum of the next step).
template <bool SELECT, bool CFL, int NT>
__device__ __noinline__ void select_pass(const jb_ens_inst& I, int rank, const double* U, const double* aux_in,
                                         double* aux_out, unsigned mask, Slots* s, int aidx) {
  const Grid& g = I.g;
  double amx = 0.0, amy = 0.0, dtm = __longlong_as_double(0x7ff0000000000000LL);
  unsigned st = 0;
  for (int j = rank; j < I.nchunks; j += I.ncta) {
    long long c = (long long)j * NT + threadIdx.x;
    if (c < g.ncell)
      select_cell<1, SELECT, true, CFL>(c_mech, g, U, aux_in, I.cand, aux_out, I.strips, s, mask, c, amx, amy,
                                        dtm, st);
  }
  block_reduce_store(amx, amy, dtm, st << 16, s, aidx, true, CFL, -1);
}

// The outlet ghost strips of this instance from the boundary cells' new
// (U, gamma, T), computed by the CTA that wrote those cells (its writes are
// visible to its own threads after a block barrier), their wave speeds
// folded into amx.  chunk: cells per work item of the pass that wrote them.
__device__ __forceinline__ void ens_strips(const jb_ens_inst& I, int rank, int chunk, int nitems,
                                           const double* U, const double* aux, double& amx) {
  __syncthreads();
  if (threadIdx.x < 2) {
    const int side = threadIdx.x;
    const int x = side == 0 ? 0 : I.g.nx - 1;
    const int kind = I.g.bc[side];
    if ((kind == JB_BC_PRESSURE_OUTLET || kind == JB_BC_RDC_INJECTOR) && (x / chunk) % I.ncta == rank &&
        x / chunk < nitems) {
      double amy = 0.0;
      strip_one<1>(c_mech, I.g, U, aux, I.strips, side, 0, amx, amy);
    }
  }
}

// One RK stage over this CTA's tiles.  Global-stop mode (float64 tiles):
// Halley mask into s->mask[STAGE - 1]; per-cell mode (float tiles of the
// mixed variant): each cell's temperature solve into fin.aux, and the new
// state's alpha (with the outlet strips) into s->ax[fin.aidx].
template <int STAGE, class R, int NT>
__device__ __noinline__ void flux_pass(const jb_ens_inst& I, int rank, const double* Uk, const double* auxk,
                                       double* out, double alpha, double dt, Slots* s, unsigned char* smraw,
                                       const jb_fin& fin) {
  unsigned bits = 0;
  double amx = 0.0, dtm = __longlong_as_double(0x7ff0000000000000LL);
  for (int t = rank; t < I.ntiles; t += I.ncta)
    bits |= flux1d_tile<STAGE, R, NT>(c_mech, I.g, Uk, auxk, I.U, out, fin, I.strips, alpha, dt, t * (NT - 1),
                                      smraw, amx, dtm, s);
  if (fin.aux && fin.aidx >= 0) ens_strips(I, rank, NT - 1, I.ntiles, out, fin.aux, amx);
  finish_reduce(fin, amx, 0.0, dtm, bits, s);
}

// Per-cell mode: chemistry of this CTA's cells at the stage-3 temperature
// in A0, then each cell's temperature solve into aux, the new state's alpha
// (with the outlet strips) into s->ax[3] and its CFL minimum.
template <int NT>
__device__ __noinline__ void chem_pass_cell(const jb_ens_inst& I, int rank, double dt, Slots* s,
                                            unsigned char* smraw) {
  const Grid& g = I.g;
  const long long nc = g.ncell;
  double* sh = reinterpret_cast<double*>(smraw) + threadIdx.x;
  const jb_fin fin = jb_fin_cell(I.aux, nullptr, 3, 1);
  unsigned bits = 0, st = 0;
  double amx = 0.0, amy = 0.0, dtm = __longlong_as_double(0x7ff0000000000000LL);
  for (int j = rank; j < I.nchunks; j += I.ncta) {
    long long c = (long long)j * NT + threadIdx.x;
    if (c < nc)
      chem_cell_step<1, false, true, true>(c_mech, g, I.W0, I.A0[nc + c], I.U, fin, c, dt, sh, bits, st, amx, amy,
                                           dtm, s);
  }
  ens_strips(I, rank, NT, I.nchunks, I.U, I.aux, amx);
  finish_reduce(fin, amx, 0.0, dtm, bits | (st << 16), s);
}

// Chemistry of this CTA's cells at the stage-3 temperature (iterate n3 of
// the last solve), then the final Halley iterates; mask into s->mask[3].
template <int NT>
__device__ __noinline__ void chem_pass(const jb_ens_inst& I, int rank, int n3, double dt, Slots* s,
                                       unsigned char* smraw) {
  const Grid& g = I.g;
  const long long nc = g.ncell;
  double* sh = reinterpret_cast<double*>(smraw) + threadIdx.x;
  unsigned bits = 0, st = 0;
  for (int j = rank; j < I.nchunks; j += I.ncta) {
    long long c = (long long)j * NT + threadIdx.x;
    double amx = 0.0, amy = 0.0, dtm = 0.0;
    if (c < nc)
      chem_cell_step<1, false, true>(c_mech, g, I.W0, I.cand[n3 * nc + c], I.U, jb_fin_cand(I.cand, 0), c, dt, sh,
                                     bits, st, amx, amy, dtm, nullptr);
  }
  block_reduce_store(0.0, 0.0, 0.0, bits | (st << 16), s, 0, false, false, 3);
}

template <class R, int NT>
__global__ void __launch_bounds__(NT, Shape<NT>::MINB)
    k_ensemble(const jb_ens_inst* __restrict__ insts, const int* __restrict__ cta_inst, int nsteps,
               double* dt_hist, jb_ens_ctl* ctl, unsigned long long limit_ns) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ jb_ens_inst sI;
  const int tid = threadIdx.x;
  const int ii = cta_inst[blockIdx.x];
  {
    const long long* src = reinterpret_cast<const long long*>(insts + ii);
    long long* dst = reinterpret_cast<long long*>(&sI);
    for (int w = tid; w < (int)(sizeof(jb_ens_inst) / 8); w += NT) dst[w] = src[w];
  }
  __syncthreads();
  const jb_ens_inst& I = sI;
  const int rank = blockIdx.x - I.cta0;
  Slots* sl = I.slots;
  unsigned target = 0;
  int phase = 0;
#define JB_ENS_SYNC() \
  if (!group_sync(I, target, ctl, limit_ns, ii, phase++)) return

  if (rank == 0 && tid == 0) {
    slots_clear(&sl[0]);
    slots_clear(&sl[1]);
  }
  JB_ENS_SYNC();
  // alpha and CFL minimum of the initial state (slot set 1 plays the previous step)
  select_pass<false, true, NT>(I, rank, I.U, I.aux, nullptr, 0u, &sl[1], 3);
  JB_ENS_SYNC();

  for (int step = 0; step < nsteps; ++step) {
    Slots* cur = sl + (step & 1);
    Slots* prv = sl + ((step & 1) ^ 1);
    const double dt = I.cfl > 0.0 ? I.cfl * (__ldcg(&prv->dtnan) ? __longlong_as_double(0x7ff8000000000000LL)
                                                                  : bitsd(__ldcg(&prv->dtmin_next)))
                                  : I.dt;
    if (dt_hist && rank == 0 && tid == 0) dt_hist[(long long)ii * nsteps + step] = dt;
    if constexpr (sizeof(R) == sizeof(float)) {
      // mixed variant, per-cell temperature solves: four phases a step
      // stage 1: U1 = U + L(U), (gamma, T)_1 and alpha 1
      flux_pass<1, R, NT>(I, rank, I.U, I.aux, I.W0, bitsd(__ldcg(&prv->ax[3])), dt, cur, smraw,
                          jb_fin_cell(I.A0, nullptr, 1, 0));
      JB_ENS_SYNC();
      if (rank == 0 && tid == 0) slots_clear(prv);  // every CTA has read it
      // stage 2: U2 = 3/4 U + 1/4 (U1 + L(U1))
      flux_pass<2, R, NT>(I, rank, I.W0, I.A0, I.W1, bitsd(__ldcg(&cur->ax[1])), dt, cur, smraw,
                          jb_fin_cell(I.A1, nullptr, 2, 0));
      JB_ENS_SYNC();
      // stage 3: U3 = 1/3 U + 2/3 (U2 + L(U2)), T3 into A0
      flux_pass<3, R, NT>(I, rank, I.W1, I.A1, I.W0, bitsd(__ldcg(&cur->ax[2])), dt, cur, smraw,
                          jb_fin_cell(I.A0, nullptr, -1, 0));
      JB_ENS_SYNC();
      // chemistry, the final solve, alpha and CFL minimum of the next step
      chem_pass_cell<NT>(I, rank, dt, cur, smraw);
      JB_ENS_SYNC();
    } else {
    // stage 1: U1 = U + L(U)
    flux_pass<1, R, NT>(I, rank, I.U, I.aux, I.W0, bitsd(__ldcg(&prv->ax[3])), dt, cur, smraw,
                        jb_fin_cand(I.cand, 0));
    JB_ENS_SYNC();
    if (rank == 0 && tid == 0) slots_clear(prv);  // every CTA has read it
    select_pass<true, false, NT>(I, rank, I.W0, nullptr, I.A0, __ldcg(&cur->mask[0]), cur, 1);
    JB_ENS_SYNC();
    // stage 2: U2 = 3/4 U + 1/4 (U1 + L(U1))
    flux_pass<2, R, NT>(I, rank, I.W0, I.A0, I.W1, bitsd(__ldcg(&cur->ax[1])), dt, cur, smraw,
                        jb_fin_cand(I.cand, 1));
    JB_ENS_SYNC();
    select_pass<true, false, NT>(I, rank, I.W1, nullptr, I.A1, __ldcg(&cur->mask[1]), cur, 2);
    JB_ENS_SYNC();
    // stage 3: U3 = 1/3 U + 2/3 (U2 + L(U2))
    flux_pass<3, R, NT>(I, rank, I.W1, I.A1, I.W0, bitsd(__ldcg(&cur->ax[2])), dt, cur, smraw,
                        jb_fin_cand(I.cand, 2));
    JB_ENS_SYNC();
    chem_pass<NT>(I, rank, halley_count(__ldcg(&cur->mask[2])), dt, cur, smraw);
    JB_ENS_SYNC();
    select_pass<true, true, NT>(I, rank, I.U, nullptr, I.aux, __ldcg(&cur->mask[3]), cur, 3);
    JB_ENS_SYNC();
    }
  }
#undef JB_ENS_SYNC
}

template <class R, int NT>
cudaError_t launch_t(const jb_ens_inst* insts, const int* cta_inst, int nblocks, int nsteps,
                     double* dt_hist, jb_ens_ctl* ctl, unsigned long long limit_ns, cudaStream_t st) {
  // the shared-memory attribute was set by occupancy_t when the shape was chosen
  constexpr size_t smem = ens_smem_bytes<R, NT>();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblocks);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_ensemble<R, NT>, insts, cta_inst, nsteps, dt_hist, ctl, limit_ns);
}

template <class R, int NT>
cudaError_t occupancy_t(int* per_sm) {
  constexpr size_t smem = ens_smem_bytes<R, NT>();
  cudaError_t e = cudaFuncSetAttribute(k_ensemble<R, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_ensemble<R, NT>, NT, smem);
}

}  // namespace ens
}  // namespace jb

// ---------------------------------------------------------------------------
// host side: the jb_ensemble handle (C ABI in include/janc_b200.h)
// ---------------------------------------------------------------------------
namespace {

constexpr int kBlocks[3] = {64, 128, 256};
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // one barrier wait: 2 s
constexpr int kMaxSteps = 100000;                          // per call (barrier counters stay < 2^32)

bool block_ok(int b) { return b == 64 || b == 128 || b == 256; }

cudaError_t ens_launch(bool mixed, int block, const jb_ens_inst* insts,
                       const int* cta_inst, int nblocks, int nsteps, double* dt_hist, jb_ens_ctl* ctl,
                       cudaStream_t st, unsigned long long lim = kWaitLimitNs) {
  using namespace jb::ens;
  if (mixed) {
    if (block == 64) return launch_t<float, 64>(insts, cta_inst, nblocks, nsteps, dt_hist, ctl, lim, st);
    if (block == 128) return launch_t<float, 128>(insts, cta_inst, nblocks, nsteps, dt_hist, ctl, lim, st);
    return launch_t<float, 256>(insts, cta_inst, nblocks, nsteps, dt_hist, ctl, lim, st);
  }
  if (block == 64) return launch_t<double, 64>(insts, cta_inst, nblocks, nsteps, dt_hist, ctl, lim, st);
  if (block == 128) return launch_t<double, 128>(insts, cta_inst, nblocks, nsteps, dt_hist, ctl, lim, st);
  return launch_t<double, 256>(insts, cta_inst, nblocks, nsteps, dt_hist, ctl, lim, st);
}

cudaError_t ens_occupancy(bool mixed, int block, int* per_sm) {
  using namespace jb::ens;
  if (mixed) {
    if (block == 64) return occupancy_t<float, 64>(per_sm);
    if (block == 128) return occupancy_t<float, 128>(per_sm);
    return occupancy_t<float, 256>(per_sm);
  }
  if (block == 64) return occupancy_t<double, 64>(per_sm);
  if (block == 128) return occupancy_t<double, 128>(per_sm);
  return occupancy_t<double, 256>(per_sm);
}

}  // namespace

struct jb_ensemble {
  jb_mech_params mech;
  int n;
  int precision;
  int device;
  int nsm;
  std::vector<int> nx;
  std::vector<long long> off;   // first cell of each instance in the packed buffers
  long long cells;              // sum of nx
  long long cells_alloc;        // packed length (instances start on 32-cell boundaries)
  std::vector<jb_ens_inst> host_insts;
  double* state;                // per instance: U [11][nx] then aux [2][nx]
  double* work;                 // per instance: W0, W1 [11][nx], A0, A1 [2][nx], cand [6][nx]
  double* strips;               // [n][4][13]
  jb_slots* slots;              // [n][2]
  unsigned* sync;               // [n] barrier counters, then a jb_ens_ctl
  jb_ens_ctl* ctl;
  jb_ens_inst* d_insts;
  jb_mech_params* d_mech;       // device copy, loaded into constant memory by each launch
  int* d_cta_inst;
  int block, bpsm, nblocks, max_tiles;
  // captured graph of one persistent launch
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  int graph_steps;
  double* graph_dt_hist;
  cudaStream_t graph_stream;
  int graph_mode;  // 1: stream capture, 2: graph built node by node
  char err[512];
};

namespace {

int set_err(jb_ensemble* e, int code, const char* fmt, ...) {
  if (e) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(e->err, sizeof(e->err), fmt, ap);
    va_end(ap);
  }
  return code;
}

#define JB_ETRY(expr, what)                                                          \
  do {                                                                               \
    cudaError_t _e = (expr);                                                         \
    if (_e != cudaSuccess) return set_err(e, JB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(_e)); \
  } while (0)

// barrier counters (cleared before every launch), then the run control
// (sticky: cleared when jb_ens_status reports it)
size_t counter_bytes(int n) { return sizeof(unsigned) * (size_t)((n + 3) / 4 * 4); }
size_t sync_bytes(int n) { return counter_bytes(n) + sizeof(jb_ens_ctl); }

void drop_graph(jb_ensemble* e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->exec = nullptr;
  e->graph = nullptr;
  e->graph_steps = 0;
  e->graph_dt_hist = nullptr;
  e->graph_stream = nullptr;
}

// Static assignment of CTAs to instances for `total` CTAs of `block`
// threads: the smallest bound B on flux tiles per CTA such that giving each
// instance ceil(tiles / B) CTAs fits; work per CTA and step is then at most
// B tiles of each phase for every instance.
bool assign(const std::vector<int>& nx, int block, int total, std::vector<int>& ncta, int& used, int& bound) {
  const int n = (int)nx.size();
  std::vector<int> tiles(n);
  int tmax = 0;
  for (int i = 0; i < n; ++i) {
    tiles[i] = (nx[i] + block - 2) / (block - 1);
    tmax = std::max(tmax, tiles[i]);
  }
  if (total < n) return false;
  int lo = 1, hi = tmax;
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    long long s = 0;
    for (int i = 0; i < n; ++i) s += (tiles[i] + mid - 1) / mid;
    if (s <= total) hi = mid;
    else lo = mid + 1;
  }
  bound = lo;
  ncta.assign(n, 0);
  used = 0;
  for (int i = 0; i < n; ++i) {
    ncta[i] = (tiles[i] + lo - 1) / lo;
    used += ncta[i];
  }
  return used <= total;
}

int configure(jb_ensemble* e, int block, int bpsm) {
  if (!block_ok(block)) return set_err(e, JB_ERR_ARG, "block must be 64, 128 or 256");
  int occ = 0;
  JB_ETRY(ens_occupancy(e->precision == JB_PREC_MIXED, block, &occ), "occupancy");
  if (occ < 1) return set_err(e, JB_ERR_UNSUPPORTED, "ensemble kernel does not fit an SM with %d threads", block);
  if (bpsm < 1 || bpsm > occ) return set_err(e, JB_ERR_ARG, "blocks per SM must be in 1..%d for %d threads", occ, block);
  std::vector<int> ncta;
  int used = 0, bound = 0;
  if (!assign(e->nx, block, e->nsm * bpsm, ncta, used, bound))
    return set_err(e, JB_ERR_ARG, "%d instances need more than %d CTAs", e->n, e->nsm * bpsm);
  // largest instances first in block order
  std::vector<int> order(e->n);
  for (int i = 0; i < e->n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e->nx[a] > e->nx[b]; });
  std::vector<int> cta_inst(used);
  int c = 0;
  for (int i : order) {
    jb_ens_inst& I = e->host_insts[i];
    I.cta0 = c;
    I.ncta = ncta[i];
    I.ntiles = (e->nx[i] + block - 2) / (block - 1);
    I.nchunks = (e->nx[i] + block - 1) / block;
    for (int j = 0; j < ncta[i]; ++j) cta_inst[c++] = i;
  }
  drop_graph(e);
  if (e->d_cta_inst) cudaFree(e->d_cta_inst);
  e->d_cta_inst = nullptr;
  JB_ETRY(cudaMalloc(&e->d_cta_inst, sizeof(int) * used), "cta table");
  JB_ETRY(cudaMemcpy(e->d_cta_inst, cta_inst.data(), sizeof(int) * used, cudaMemcpyHostToDevice), "cta table copy");
  JB_ETRY(cudaMemcpy(e->d_insts, e->host_insts.data(), sizeof(jb_ens_inst) * e->n, cudaMemcpyHostToDevice),
          "instance table copy");
  e->block = block;
  e->bpsm = bpsm;
  e->nblocks = used;
  e->max_tiles = bound;
  return JB_OK;
}

// One persistent launch, preceded by loading the mechanism into constant
// memory and clearing the barrier counters.
int launch_once(jb_ensemble* e, int nsteps, double* dt_hist, cudaStream_t st) {
  JB_ETRY(cudaMemcpyToSymbolAsync(jb::ens::c_mech, e->d_mech, sizeof(jb_mech_params), 0, cudaMemcpyDeviceToDevice, st),
          "mechanism to constant memory");
  JB_ETRY(cudaMemsetAsync(e->sync, 0, counter_bytes(e->n), st), "clear barriers");
  JB_ETRY(ens_launch(e->precision == JB_PREC_MIXED, e->block, e->d_insts, e->d_cta_inst, e->nblocks, nsteps,
                     dt_hist, e->ctl, st),
          "ensemble launch");
  return JB_OK;
}

}  // namespace

extern "C" {

int jb_ens_create(const jb_mech_params* mech, int n, const int* nx, const double* dx, const int* bc,
                  const double* cfl, const double* dt, int precision, jb_ensemble** out) {
  if (!out || !mech || !nx || !dx || !bc || !cfl) return JB_ERR_ARG;
  *out = nullptr;
  if (n < 1) return JB_ERR_ARG;
  if (mech->ns != 9 || mech->nr != 8 || mech->nreac != 19) return JB_ERR_UNSUPPORTED;
  if (precision != JB_PREC_FP64 && precision != JB_PREC_MIXED) return JB_ERR_UNSUPPORTED;
  for (int i = 0; i < n; ++i) {
    if (nx[i] < 4 || !(dx[i] > 0.0)) return JB_ERR_ARG;
    if (!(cfl[i] > 0.0) && !(dt && dt[i] > 0.0)) return JB_ERR_ARG;
    for (int s = 0; s < 2; ++s) {
      int b = bc[2 * i + s];
      if (b < JB_BC_PERIODIC || b > JB_BC_PRESSURE_OUTLET) return b == JB_BC_RDC_INJECTOR ? JB_ERR_UNSUPPORTED : JB_ERR_ARG;
    }
  }
  jb_ensemble* e = new (std::nothrow) jb_ensemble();
  if (!e) return JB_ERR_ARG;
  e->mech = *mech;
  jb::derive_mech(e->mech);
  if (!e->mech.gen_ok) {
    delete e;
    return JB_ERR_UNSUPPORTED;  // the ensemble kernel has the specialised chemistry only
  }
  e->n = n;
  e->precision = precision;
  cudaGetDevice(&e->device);
  cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, e->device);
  e->nx.assign(nx, nx + n);
  e->off.resize(n);
  long long o = 0;
  e->cells = 0;
  for (int i = 0; i < n; ++i) {
    e->off[i] = o;
    o += (nx[i] + 31) / 32 * 32;
    e->cells += nx[i];
  }
  e->cells_alloc = o;
  cudaError_t ce = cudaMalloc(&e->state, sizeof(double) * 13 * (size_t)o);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->work, sizeof(double) * 32 * (size_t)o);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->strips, sizeof(double) * 52 * (size_t)n);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->slots, sizeof(jb_slots) * 2 * (size_t)n);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->sync, sync_bytes(n));
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_insts, sizeof(jb_ens_inst) * (size_t)n);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_mech, sizeof(jb_mech_params));
  if (ce == cudaSuccess) ce = cudaMemcpy(e->d_mech, &e->mech, sizeof(jb_mech_params), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemset(e->state, 0, sizeof(double) * 13 * (size_t)o);
  if (ce == cudaSuccess) ce = cudaMemset(e->strips, 0, sizeof(double) * 52 * (size_t)n);
  if (ce == cudaSuccess) ce = cudaMemset(e->slots, 0, sizeof(jb_slots) * 2 * (size_t)n);
  if (ce == cudaSuccess) ce = cudaMemset(e->sync, 0, sync_bytes(n));
  if (ce != cudaSuccess) {
    jb_ens_destroy(e);
    return JB_ERR_CUDA;
  }
  e->ctl = reinterpret_cast<jb_ens_ctl*>(reinterpret_cast<unsigned char*>(e->sync) + counter_bytes(n));
  e->host_insts.resize(n);
  for (int i = 0; i < n; ++i) {
    jb_ens_inst& I = e->host_insts[i];
    std::memset(&I, 0, sizeof(I));
    jb_grid& g = I.g;
    g.nx = nx[i];
    g.ny = 1;
    g.nv = 11;
    g.nY = 3;
    g.ncell = nx[i];
    g.dx = dx[i];
    g.dy = 1.0;
    g.idx = 1.0 / dx[i];
    g.idy = 1.0;
    g.bc[0] = bc[2 * i];
    g.bc[1] = bc[2 * i + 1];
    g.bc[2] = g.bc[3] = JB_BC_PERIODIC;
    g.Pb = 0.0;
    g.Yinj = nullptr;
    g.inj_block_p = 1.0;
    g.lstrip = 1;
    const size_t c = (size_t)nx[i];
    I.U = e->state + 13 * (size_t)e->off[i];
    I.aux = I.U + 11 * c;
    double* w = e->work + 32 * (size_t)e->off[i];
    I.W0 = w;
    I.W1 = w + 11 * c;
    I.A0 = w + 22 * c;
    I.A1 = w + 24 * c;
    I.cand = w + 26 * c;
    I.strips = e->strips + 52 * (size_t)i;
    I.slots = e->slots + 2 * (size_t)i;
    I.bar = e->sync + i;
    I.dt_hist = nullptr;
    I.cfl = cfl[i];
    I.dt = dt ? dt[i] : 0.0;
  }
  int rc = configure(e, 128, 3);
  if (rc) {
    // fall back to the largest shape this device fits
    rc = configure(e, 128, 1);
  }
  if (rc) {
    jb_ens_destroy(e);
    return rc;
  }
  *out = e;
  return JB_OK;
}

int jb_ens_destroy(jb_ensemble* e) {
  if (!e) return JB_OK;
  drop_graph(e);
  if (e->state) cudaFree(e->state);
  if (e->work) cudaFree(e->work);
  if (e->strips) cudaFree(e->strips);
  if (e->slots) cudaFree(e->slots);
  if (e->sync) cudaFree(e->sync);
  if (e->d_insts) cudaFree(e->d_insts);
  if (e->d_mech) cudaFree(e->d_mech);
  if (e->d_cta_inst) cudaFree(e->d_cta_inst);
  delete e;
  return JB_OK;
}

int jb_ens_instance(jb_ensemble* e, int i, double** U, double** aux, int* nx) {
  if (!e || i < 0 || i >= e->n) return set_err(e, JB_ERR_ARG, "instance index out of range");
  if (U) *U = e->host_insts[i].U;
  if (aux) *aux = e->host_insts[i].aux;
  if (nx) *nx = e->nx[i];
  return JB_OK;
}

long long jb_ens_total_cells(const jb_ensemble* e) { return e ? e->cells : 0; }

int jb_ens_configure(jb_ensemble* e, int block, int blocks_per_sm) {
  if (!e) return JB_ERR_ARG;
  return configure(e, block, blocks_per_sm);
}

int jb_ens_set_back_pressure(jb_ensemble* e, const double* pb) {
  if (!e || !pb) return set_err(e, JB_ERR_ARG, "null pointer");
  for (int i = 0; i < e->n; ++i)
    if (!(pb[i] >= 0.0)) return set_err(e, JB_ERR_ARG, "back pressure of instance %d is not >= 0", i);
  for (int i = 0; i < e->n; ++i) e->host_insts[i].g.Pb = pb[i];
  drop_graph(e);
  JB_ETRY(cudaMemcpy(e->d_insts, e->host_insts.data(), sizeof(jb_ens_inst) * e->n, cudaMemcpyHostToDevice),
          "instance table copy");
  return JB_OK;
}

int jb_ens_launch_shape(const jb_ensemble* e, int* block, int* blocks_per_sm, int* nblocks, int* max_tiles,
                        int* graph_mode) {
  if (!e) return JB_ERR_ARG;
  if (block) *block = e->block;
  if (blocks_per_sm) *blocks_per_sm = e->bpsm;
  if (nblocks) *nblocks = e->nblocks;
  if (max_tiles) *max_tiles = e->max_tiles;
  if (graph_mode) *graph_mode = e->graph_mode;
  return JB_OK;
}

int jb_ens_advance(jb_ensemble* e, int nsteps, double* dt_hist, void* stream) {
  if (!e) return JB_ERR_ARG;
  if (nsteps < 1 || nsteps > kMaxSteps) return set_err(e, JB_ERR_ARG, "nsteps must be in 1..%d", kMaxSteps);
  cudaStream_t st = (cudaStream_t)stream;
  if (!e->exec || e->graph_steps != nsteps || e->graph_dt_hist != dt_hist) {
    drop_graph(e);
    // capture the clearing memset and the cooperative launch
    cudaStream_t cs = nullptr;
    JB_ETRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
    cudaError_t ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    int rc = JB_OK;
    if (ce == cudaSuccess) {
      rc = launch_once(e, nsteps, dt_hist, cs);
      cudaGraph_t g = nullptr;
      cudaError_t ee = cudaStreamEndCapture(cs, &g);
      if (rc == JB_OK && ee == cudaSuccess) {
        e->graph = g;
        e->graph_mode = 1;
      } else if (g) {
        cudaGraphDestroy(g);
      }
    }
    cudaStreamDestroy(cs);
    cudaGetLastError();
    if (!e->graph) {
      // build the same three nodes explicitly, the kernel node marked cooperative
      JB_ETRY(cudaGraphCreate(&e->graph, 0), "graph create");
      cudaGraphNode_t mcpy = nullptr, mset = nullptr, kn = nullptr;
      JB_ETRY(cudaGraphAddMemcpyNodeToSymbol(&mcpy, e->graph, nullptr, 0, jb::ens::c_mech, e->d_mech,
                                             sizeof(jb_mech_params), 0, cudaMemcpyDeviceToDevice),
              "mechanism node");
      cudaMemsetParams mp = {};
      mp.dst = e->sync;
      mp.value = 0;
      mp.elementSize = 1;
      mp.width = counter_bytes(e->n);
      mp.height = 1;
      mp.pitch = 0;
      JB_ETRY(cudaGraphAddMemsetNode(&mset, e->graph, &mcpy, 1, &mp), "memset node");
      (void)rc;
      const bool mixed = e->precision == JB_PREC_MIXED;
      void* fn = nullptr;
      size_t smem = 0;
      using namespace jb::ens;
#define JB_ENS_PICK(RT, NTV)                                              \
  if ((mixed == (sizeof(RT) == 4)) && e->block == NTV) {                  \
    fn = reinterpret_cast<void*>(&k_ensemble<RT, NTV>);                   \
    smem = ens_smem_bytes<RT, NTV>();                                     \
  }
      JB_ENS_PICK(float, 64)
      JB_ENS_PICK(float, 128)
      JB_ENS_PICK(float, 256)
      JB_ENS_PICK(double, 64)
      JB_ENS_PICK(double, 128)
      JB_ENS_PICK(double, 256)
#undef JB_ENS_PICK
      unsigned long long lim = kWaitLimitNs;
      int ns = nsteps;
      void* args[] = {&e->d_insts, &e->d_cta_inst, &ns, &dt_hist, &e->ctl, &lim};
      cudaKernelNodeParams kp = {};
      kp.func = fn;
      kp.gridDim = dim3(e->nblocks);
      kp.blockDim = dim3(e->block);
      kp.sharedMemBytes = (unsigned)smem;
      kp.kernelParams = args;
      JB_ETRY(cudaGraphAddKernelNode(&kn, e->graph, &mset, 1, &kp), "kernel node");
      cudaLaunchAttributeValue v = {};
      v.cooperative = 1;
      JB_ETRY(cudaGraphKernelNodeSetAttribute(kn, cudaLaunchAttributeCooperative, &v), "cooperative node");
      e->graph_mode = 2;
    }
    cudaError_t ie = cudaGraphInstantiate(&e->exec, e->graph, 0);
    if (ie != cudaSuccess) {
      drop_graph(e);
      return set_err(e, JB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
    }
    e->graph_steps = nsteps;
    e->graph_dt_hist = dt_hist;
  }
  JB_ETRY(cudaGraphLaunch(e->exec, st), "graph launch");
  return JB_OK;
}

int jb_ens_advance_direct(jb_ensemble* e, int nsteps, double* dt_hist, void* stream) {
  if (!e) return JB_ERR_ARG;
  if (nsteps < 1 || nsteps > kMaxSteps) return set_err(e, JB_ERR_ARG, "nsteps must be in 1..%d", kMaxSteps);
  return launch_once(e, nsteps, dt_hist, (cudaStream_t)stream);
}

int jb_ens_autotune(jb_ensemble* e, int trial_steps, void* stream, int* best_block, int* best_bpsm,
                    double* best_ms) {
  if (!e) return JB_ERR_ARG;
  if (trial_steps < 1 || trial_steps > 1000) return set_err(e, JB_ERR_ARG, "trial_steps must be in 1..1000");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t bytes = sizeof(double) * 13 * (size_t)e->cells_alloc;
  double* backup = nullptr;
  JB_ETRY(cudaMalloc(&backup, bytes), "autotune backup");
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  int bb = e->block, bp = e->bpsm;
  double bms = 1e300;
  int rc = JB_OK;
  cudaError_t ce = cudaMemcpyAsync(backup, e->state, bytes, cudaMemcpyDeviceToDevice, st);
  for (int bi = 0; bi < 3 && rc == JB_OK && ce == cudaSuccess; ++bi) {
    int occ = 0;
    if (ens_occupancy(e->precision == JB_PREC_MIXED, kBlocks[bi], &occ) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    for (int p = 1; p <= occ && rc == JB_OK; ++p) {
      if (e->nsm * p < e->n) continue;
      if (configure(e, kBlocks[bi], p) != JB_OK) continue;
      float ms = 0.f;
      for (int rep = 0; rep < 2 && rc == JB_OK; ++rep) {
        ce = cudaMemcpyAsync(e->state, backup, bytes, cudaMemcpyDeviceToDevice, st);
        if (ce != cudaSuccess) break;
        cudaEventRecord(a, st);
        rc = launch_once(e, trial_steps, nullptr, st);
        cudaEventRecord(b, st);
      }
      if (rc != JB_OK || ce != cudaSuccess) break;
      ce = cudaEventSynchronize(b);
      if (ce != cudaSuccess) break;
      cudaEventElapsedTime(&ms, a, b);
      jb_ens_ctl c = {};
      ce = cudaMemcpy(&c, e->ctl, sizeof(c), cudaMemcpyDeviceToHost);
      if (ce != cudaSuccess) break;
      if (c.timeout) {
        rc = set_err(e, JB_ERR_TIMEOUT, "barrier wait gave up (instance %u, phase %u)", c.where_inst, c.where_phase);
        break;
      }
      if (ms < bms) {
        bms = ms;
        bb = kBlocks[bi];
        bp = p;
      }
    }
  }
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(e->state, backup, bytes, cudaMemcpyDeviceToDevice, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  cudaFree(backup);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (ce != cudaSuccess) return set_err(e, JB_ERR_CUDA, "autotune: %s", cudaGetErrorString(ce));
  if (rc != JB_OK) return rc;
  rc = configure(e, bb, bp);
  if (rc) return rc;
  if (best_block) *best_block = bb;
  if (best_bpsm) *best_bpsm = bp;
  if (best_ms) *best_ms = bms;
  return JB_OK;
}

int jb_ens_status(jb_ensemble* e, unsigned* per_instance, unsigned* combined, void* stream) {
  if (!e) return JB_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<jb_slots> s(2 * (size_t)e->n);
  jb_ens_ctl c = {};
  JB_ETRY(cudaMemcpyAsync(s.data(), e->slots, sizeof(jb_slots) * s.size(), cudaMemcpyDeviceToHost, st), "status copy");
  JB_ETRY(cudaMemcpyAsync(&c, e->ctl, sizeof(c), cudaMemcpyDeviceToHost, st), "ctl copy");
  JB_ETRY(cudaStreamSynchronize(st), "status sync");
  unsigned all = c.timeout ? (unsigned)JB_ERR_TIMEOUT : 0u;
  for (int i = 0; i < e->n; ++i) {
    unsigned v = s[2 * i].status | s[2 * i + 1].status;
    if (per_instance) per_instance[i] = v;
    all |= v;
  }
  for (int i = 0; i < 2 * e->n; ++i)
    JB_ETRY(cudaMemsetAsync(&e->slots[i].status, 0, sizeof(unsigned), st), "status clear");
  if (c.timeout) {
    set_err(e, JB_ERR_TIMEOUT, "barrier wait gave up (instance %u, phase %u)", c.where_inst, c.where_phase);
    JB_ETRY(cudaMemsetAsync(e->ctl, 0, sizeof(jb_ens_ctl), st), "ctl clear");
  }
  if (combined) *combined = all;
  return JB_OK;
}

const char* jb_ens_last_error(const jb_ensemble* e) { return e ? e->err : "null ensemble"; }

int jb_ens_selftest_timeout(jb_ensemble* e, double wait_limit_ms, unsigned* combined, void* stream) {
  if (!e || !combined) return JB_ERR_ARG;
  if (!(wait_limit_ms > 0.0) || wait_limit_ms > 1000.0) return set_err(e, JB_ERR_ARG, "wait limit must be in (0, 1000] ms");
  cudaStream_t st = (cudaStream_t)stream;
  // instance 0's group waits for one CTA more than is launched
  std::vector<jb_ens_inst> t = e->host_insts;
  t[0].ncta += 1;
  JB_ETRY(cudaMemcpyAsync(e->d_insts, t.data(), sizeof(jb_ens_inst) * e->n, cudaMemcpyHostToDevice, st),
          "selftest table");
  JB_ETRY(cudaMemcpyToSymbolAsync(jb::ens::c_mech, e->d_mech, sizeof(jb_mech_params), 0, cudaMemcpyDeviceToDevice, st),
          "mechanism to constant memory");
  JB_ETRY(cudaMemsetAsync(e->sync, 0, counter_bytes(e->n), st), "clear barriers");
  JB_ETRY(ens_launch(e->precision == JB_PREC_MIXED, e->block, e->d_insts, e->d_cta_inst, e->nblocks, 1, nullptr,
                     e->ctl, st, (unsigned long long)(wait_limit_ms * 1e6)),
          "selftest launch");
  JB_ETRY(cudaMemcpyAsync(e->d_insts, e->host_insts.data(), sizeof(jb_ens_inst) * e->n, cudaMemcpyHostToDevice, st),
          "restore table");
  return jb_ens_status(e, nullptr, combined, stream);
}

}  // extern "C"
