// Launchers of the adjoint kernels (jb_adjoint.cu), used by the C ABI.
#pragma once
#include <cuda_runtime.h>

#include "jb_types.h"

namespace jb {
namespace adj {

// Reduction slots of one adjoint step (device doubles, cleared before it):
// [0] the dt adjoint; per RK stage s = 0, 1, 2 from 1 + 5 s: the alpha_x and
// alpha_y adjoints, the alpha_x and alpha_y tie counts (padded-grid
// multiplicity) and, for stage 0, the CFL tie count.
constexpr int RED_DTB = 0, RED_N = 16;
__host__ __device__ constexpr int red_ab(int s, int d) { return 1 + 5 * s + d; }
__host__ __device__ constexpr int red_cnt(int s, int d) { return 3 + 5 * s + d; }

// dim: 1 or 2 (1D: py = 0, wy = 1).  probe = {px, py, wx, wy}; pp_bar may
// be null.  prims: 3 x 4 x ncell (rho, u, v, p; v = 0 in 1D).
// scratch: flux_scratch_doubles(g) doubles (the outlet ghosts of the three
// stage states go there when a side is a pressure outlet).
cudaError_t vjp_begin(int dim, const jb_mech_params& m, const jb_grid& g, const double* U4, const double* A4,
                      const double* pp_bar, const int* probe, double* Ub, double* Ab, const double* rec,
                      double* prims, const unsigned char* mult, const double* slots_rec, double cfl, double* red,
                      double* scratch, cudaStream_t st);
cudaError_t chem_vjp(int dim, const jb_mech_params& m, const jb_grid& g, const double* U3, const double* A3,
                     const double* Ub4, double* Ub3, const double* slot_dt, double* dtb, double* lnAb,
                     cudaStream_t st);
// Doubles of the scratch that flux_stage needs (the per-face-direction
// flux and LF-term adjoints of the padded cells; the pressure-outlet ghost
// states of the three stage states and their adjoints).
size_t flux_scratch_doubles(int dim, const jb_grid& g);
// One RK stage U' = a Un + b (Uk + dt L(Uk)) with b = coef, a = un_coef:
// Ub (store, or add with ub_add) = Ubar_k; Un_b (store / add) += a Ubar'.
// Ab null: the update_aux VJP of Uk is applied; else its aux adjoint is
// added to Ab.  cfl > 0 only for stage 0 (the CFL time step).
cudaError_t flux_stage(int dim, const jb_mech_params& m, const jb_grid& g, const double* Uk, const double* Ak,
                       const double* Pk, const double* Uo_b, double coef, const double* slots_rec, int stage,
                       double cfl, const unsigned char* mult, double* red, const double* dt_bar_ext, double* scratch,
                       double* Ub, bool ub_add, double* Ab, double* Un_b, double un_coef, bool un_add,
                       cudaStream_t st);
cudaError_t probe_mean(int dim, const jb_mech_params& m, const jb_grid& g, const double* U, const double* A, int px, int py,
                       int wx, int wy, double* out, cudaStream_t st);
cudaError_t init_vjp(int dim, const jb_mech_params& m, long long n, const double* P, const double* T, const double* Y,
                     const double* Ub, const double* Ab, double* Tb, cudaStream_t st);

}  // namespace adj
}  // namespace jb
