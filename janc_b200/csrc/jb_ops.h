// Host-side launch table: one instance per compiled arithmetic variant
// (jb::strict_ops from jb_strict.cu, jb::fast_ops from jb_fast.cu).
#pragma once
#include <cuda_runtime.h>

#include "jb_fin.h"
#include "jb_types.h"

namespace jb {

// Block arrays of one AMR stage call: U fields and (gamma, T) of each block
// at its own block stride (one [nb][nv+2][X][Y] array gives U = base,
// A = base + nv X Y and both strides (nv+2) X Y; separate [nb][nv][X][Y] and
// [nb][2][X][Y] arrays give strides nv X Y and 2 X Y).
struct jb_amr_io {
  const double* gU;  // stage input
  const double* gA;
  long long gsU, gsA;
  const double* u0;  // U fields of the step's first stage input (stage 2, 3)
  long long u0s;
  double* oU;        // result
  double* oA;        // (gamma, T) of the result (stage 1..3)
  long long osU, osA;
};

struct Ops {
  const char* name;
  // stepping (jb_advance) solves each new state's temperature per cell
  // (jb_fin per-cell mode) instead of the global-stop iterates + select: the
  // mixed variant only (2D, and 1D with flux splitting); strict and fp64
  // keep the reference's global stop
  bool per_cell;
  // STAGE 0 writes dt * flux; STAGE 1..3 writes the RK stage and finishes
  // its temperature solve as fin says (jb_fin.h).  aidx: the alpha slot the
  // stage reads.  prims: float32 u, v, p of the stage state (mixed 2D) and
  // work: float32 scratch of the x flux differences [12][ncell], or null.
  cudaError_t (*flux)(int dim, int stage, const jb_mech_params& m, const jb_grid& g,
                      const double* Uk, const double* auxk, const double* Un, double* out,
                      const double* strips, jb_slots* slots, int aidx, const jb_fin& fin,
                      const float* prims, void* work, double dt, cudaStream_t st);
  // work: where the pass writes the float32 u, v, p of its state when it
  // computes alpha (mixed 2D), or null
  cudaError_t (*select)(int dim, bool select, bool alpha, bool cfl, const jb_mech_params& m,
                        const jb_grid& g, const double* U, const double* aux_in,
                        const double* cand, double* aux_out, double* strips, jb_slots* slots,
                        int midx, int aidx, void* work, cudaStream_t st);
  cudaError_t (*halley)(int dim, const jb_mech_params& m, const jb_grid& g, const double* U,
                        const double* aux, double* cand, jb_slots* slots, int midx,
                        cudaStream_t st);
  // write_s: reaction_source_terms into out; else out = U + S and its
  // temperature solve as fin says (aux == null: the stage-3 temperature is
  // the global-stop iterate of mask fin.midx - 1)
  cudaError_t (*chem)(int dim, bool write_s, const jb_mech_params& m, const jb_grid& g,
                      const double* U, const double* aux, double* out, const jb_fin& fin,
                      jb_slots* slots, double dt, cudaStream_t st);
  cudaError_t (*thermo)(const jb_mech_params& m, long long n, const double* T, const double* Y,
                        double* cp, double* gamma, double* h, double* R, double* dcp,
                        cudaStream_t st);
  cudaError_t (*prim)(int dim, const jb_mech_params& m, const jb_grid& g, const double* U,
                      const double* aux, double* rho, double* u, double* v, double* Y, double* p,
                      double* a, cudaStream_t st);
  // viscous rhs of (Uk, auxk) into V; vbuf: visc_scratch_doubles(dim, g)
  cudaError_t (*visc)(int dim, const jb_mech_params& m, const jb_grid& g, const jb_transport& tr,
                      const double* Uk, const double* auxk, const double* strips, double* vbuf, double* V,
                      cudaStream_t st);
  cudaError_t (*slots_reset)(jb_slots* s, cudaStream_t st);
  cudaError_t (*step_begin)(jb_slots* s, double cfl, double dt_fixed, double* dt_hist, int step,
                            cudaStream_t st);
  cudaError_t (*dt_from_slots)(const jb_slots* s, double cfl, double* dt_out, cudaStream_t st);
  // exchange (jb_exchange_flags): pack the CFL pair into red and the edge
  // columns (rows) of (U, aux) into send (sendy); after the exchange,
  // unpack the pair and fold the ghost layers' wave speeds into alpha slot aidx
  cudaError_t (*xch_pre)(int dim, const jb_grid& g, const double* U, const double* aux, double* send,
                         double* sendy, const jb_slots* slots, long long* red, int flags, cudaStream_t st);
  cudaError_t (*xch_post)(int dim, const jb_mech_params& m, const jb_grid& g, jb_slots* slots,
                          const long long* red, int aidx, int flags, cudaStream_t st);
  // ghost-padded copies of (U, aux) (the ghost strips and ghost layers must be current)
  cudaError_t (*pad)(int dim, const jb_grid& g, const double* U, const double* aux, const double* strips,
                     double* Up, double* auxp, cudaStream_t st);
  // ghost strips of the pressure-outlet / injector sides of (U, aux) and their
  // wave speeds into alpha slot aidx (no launch without such sides)
  cudaError_t (*strips)(int dim, const jb_mech_params& m, const jb_grid& g, const double* U, const double* aux,
                        double* strips, jb_slots* slots, int aidx, cudaStream_t st);
  // block-structured AMR (2D, flux splitting): one SSP-RK3 stage (1..3) of nb
  // ghost-padded blocks [nb][nv+2][bx+6][by+6] (G the stage input, U0 the
  // step's first stage input), and the chemistry with its temperature solve
  // of nb unpadded blocks [nb][nv+2][bx][by]; g supplies the reconstruction
  // (stage 0: out = pad(dt L(G)) alone) and update_aux of nb blocks of nc
  // cells with each block's own stop (U [nb][nv][..], aux [nb][2][..])
  cudaError_t (*amr_stage)(const jb_mech_params& m, const jb_grid& g, int nb, int bx, int by, double dx,
                           double dy, int stage, const jb_amr_io& io, jb_slots* slots, double dt, cudaStream_t st);
  cudaError_t (*amr_update)(const jb_mech_params& m, int nb, long long nc, const double* U, const double* aux_in,
                            double* aux_out, jb_slots* slots, cudaStream_t st);
  cudaError_t (*amr_chem)(const jb_mech_params& m, int nb, int bx, int by, const double* blk, double* out,
                          jb_slots* slots, double dt, cudaStream_t st);
};

// Doubles of the viscous scratch (node planes and node fluxes) of a grid.
inline long long visc_scratch_doubles(int dim, const jb_grid& g) {
  const long long PY = dim == 2 ? g.ny + 6 : 1, np = (long long)(g.nx + 6) * PY;
  const long long sF = dim == 2 ? (long long)(g.nx + 6) * g.ny : g.nx + 6;
  const long long sG = dim == 2 ? (long long)g.nx * PY : 0;
  return (dim == 2 ? 13 : 12) * np + (dim == 2 ? 12 : 11) * (sF + sG);
}

extern const Ops strict_ops;
extern const Ops fast_ops;
extern const Ops mixed_ops;

// Fill the derived fields of a mechanism block (ln A, tb/M, ln pref, ln T0)
// and flag whether its structure matches the generated chemistry.
void derive_mech(jb_mech_params& m);

}  // namespace jb
