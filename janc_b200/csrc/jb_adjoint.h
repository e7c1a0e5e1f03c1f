// Launchers of the adjoint kernels (jb_adjoint.cu), used by the C ABI.
#pragma once
#include <cuda_runtime.h>

#include "jb_types.h"

namespace jb {
namespace adj {

// red: 8 device doubles [abar_x, abar_y, dtbar, ties_x, ties_y, ties_cfl, -, -]
cudaError_t upd_vjp(const jb_mech_params& m, const jb_grid& g, const double* U, const double* A, double* Ub,
                    double* Ab, cudaStream_t st);
cudaError_t chem_vjp(const jb_mech_params& m, const jb_grid& g, const double* U3, const double* A3,
                     const double* Ub4, double* Ub3, const double* slot_dt, double* dtb, double* lnAb,
                     cudaStream_t st);
// Ub2 (nv x ncell), Ab2 (ncell): scratch for the y-face adjoints
cudaError_t flux_vjp(const jb_mech_params& m, const jb_grid& g, const double* Uk, const double* Ak,
                     const double* Uo_b, double coef, const double* slots_rec, int stage, double* Ub, double* Abk,
                     double* Un_b, double un_coef, double* ghost, double* Ub2, double* Ab2, double* red,
                     cudaStream_t st);
// upd: also the update_aux VJP of (U, A) with the completed aux adjoint
cudaError_t speed_vjp(const jb_mech_params& m, const jb_grid& g, const double* U, const double* A,
                      const unsigned char* mult, const double* slots_rec, int stage, double cfl, double* red,
                      double* Ub, double* Ab, bool upd, cudaStream_t st);
cudaError_t probe_seed(const jb_mech_params& m, const jb_grid& g, const double* U, const double* A,
                       const double* pp_bar, int px, int py, int wx, int wy, double* Ub, double* Ab, cudaStream_t st);
cudaError_t probe_mean(const jb_mech_params& m, const jb_grid& g, const double* U, const double* A, int px, int py,
                       int wx, int wy, double* out, cudaStream_t st);
cudaError_t adj_begin(double* red, const double* dt_bar_ext, cudaStream_t st);
cudaError_t clear_alpha(double* red, cudaStream_t st);
cudaError_t init_vjp(const jb_mech_params& m, long long n, const double* P, const double* T, const double* Y,
                     const double* Ub, const double* Ab, double* Tb, cudaStream_t st);

}  // namespace adj
}  // namespace jb
