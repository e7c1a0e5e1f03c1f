// Plain-old-data types shared by the host launcher and the device kernels.
// No torch or CUDA-runtime types appear here so the C ABI header can mirror
// the layouts one-for-one.
#ifndef JB_TYPES_H
#define JB_TYPES_H
#include <stdint.h>

#define JB_NS_MAX 9      // species including the implicit last (inert) one
#define JB_NR_MAX 8      // reactive species (the linear system size)
#define JB_NREAC_MAX 19  // reactions
#define JB_NCAND 6       // Halley iterates kept per cell: T_0 .. T_5

// Mechanism tables in the reference's packing (preprocess/load.py:91-135 and
// :8-88), already non-dimensionalised.  Polynomials are highest power first
// (numpy/jax polyval order).
typedef struct jb_mech_params {
  int ns, nr, nreac, pad_;
  double M[JB_NS_MAX];      // species_M
  double invM[JB_NS_MAX];   // 1/species_M (thermo_model.py:91 "1/Mex")
  double Tcr[JB_NS_MAX];
  double cp_lo[JB_NS_MAX][5], cp_hi[JB_NS_MAX][5];
  double dcp_lo[JB_NS_MAX][4], dcp_hi[JB_NS_MAX][4];
  double h_lo[JB_NS_MAX][6], h_hi[JB_NS_MAX][6];
  double hc_lo[JB_NS_MAX][6], hc_hi[JB_NS_MAX][6];  // h/R (chemistry)
  double s_lo[JB_NS_MAX][5], s_hi[JB_NS_MAX][5];
  double lg_lo[JB_NS_MAX], lg_hi[JB_NS_MAX];
  double A[JB_NREAC_MAX], B[JB_NREAC_MAX], EaR[JB_NREAC_MAX];
  double vsum[JB_NREAC_MAX], is_tb[JB_NREAC_MAX];
  double vf[JB_NREAC_MAX][JB_NR_MAX], vb[JB_NREAC_MAX][JB_NR_MAX];
  double dv[JB_NREAC_MAX][JB_NR_MAX];  // vb - vf
  double tb[JB_NREAC_MAX][JB_NS_MAX];  // third-body efficiencies (scaled)
  double T0;        // nondim reference temperature (gibbs uses log(T0*T))
  double pref;      // 101325 / P0 (reaction_model.py:113)
  // derived by jb_create (callers leave these zero)
  double lnA[JB_NREAC_MAX];
  double tbinvM[JB_NREAC_MAX][JB_NR_MAX];  // tb[i][n] / M[n]
  double lnpref, lnT0;
  int gen_ok;       // structure matches the generated specialised chemistry
  int tcr_uniform;  // every species switches NASA7 ranges at the same temperature
} jb_mech_params;

enum jb_bc_kind {
  JB_BC_PERIODIC = 0,
  JB_BC_SLIP_WALL = 1,
  JB_BC_ZERO_GRADIENT = 2,
  JB_BC_NO_SLIP_WALL = 3,
  JB_BC_PRESSURE_OUTLET = 4,
  JB_BC_RDC_INJECTOR = 5,
  // side whose 3 ghost layers come from a buffer filled before each flux
  // evaluation: an x slab's neighbour columns (parallel/boundary.py), or the
  // caller's boundary function of the 3 edge layers (a Python callable
  // boundary, boundary/boundary.py:16-21)
  JB_BC_HALO = 6
};

// What jb_exchange_fn is asked to do (bit flags).
enum jb_exchange_flags {
  JB_XCH_DT = 1,   // all-reduce MIN over the ranks of the int64 pair red[0..1]
  JB_XCH_HALO = 2  // send send[side] to the neighbour across side, receive halo[side]
};

// kernel categories reported by jb_kernel_times
enum jb_kernel_cat {
  JB_KCAT_FLUX = 0,    // LF + WENO5 + RK stage + Halley iterates
  JB_KCAT_SELECT = 1,  // Halley selection, wave-speed / CFL reductions, ghost strips
  JB_KCAT_CHEM = 2,    // point-implicit chemistry + final Halley iterates
  JB_KCAT_OTHER = 3,   // per-step bookkeeping
  JB_KCAT_COUNT = 4
};
#define JB_TIMED_MAX 64  // timed launches buffered between jb_kernel_times calls

enum jb_precision { JB_PREC_STRICT = 0, JB_PREC_FP64 = 1, JB_PREC_MIXED = 2 };

// Advective flux (solver_{1D,2D}/flux.py set_flux_solver): flux splitting
// (LF or Steger-Warming, the face reconstruction on the split fluxes) or
// Godunov (the reconstruction on the primitives and a Riemann solver).
enum jb_flux_scheme { JB_FLUX_LF = 0, JB_FLUX_HLLC = 1, JB_FLUX_AUSMPW = 2, JB_FLUX_SW = 3 };

// Face reconstruction (solver_{1D,2D}/reconstruction): WENO5-JS or MUSCL
// (minmod limiter, kappa = 1/3, beta = 1).
enum jb_reconstruction { JB_RECON_WENO5 = 0, JB_RECON_MUSCL = 1 };

// Laminar transport (model/transport_model.py set_transport): viscosity
// 0 Sutherland mu_ref (T/T_ref)^1.5 (T_ref+S)/(T+S), 1 constant rho nu0;
// conductivity 0 Prandtl number mu cp/Pr, 1 constant k0; diffusivity 0 Lewis
// number rho D_k = k_k/(Le cp_k) (a Schmidt number gives Le = Sc/Pr), 1
// constant D0.  turbulence_model 0 laminar, 1 LES with the 2D Vreman
// sub-grid viscosity mu_t = 0.07 rho sqrt(B / (a_ij a_ij))
// (model/LES/Verman.py); mu_t adds to mu and enters k and D through Pr_t and
// Le_t (transport_model.py:117-157).
typedef struct jb_transport {
  int viscosity_model, conductivity_model, diffusivity_model, turbulence_model;
  double mu_ref, T_ref, S, nu0, Pr, Le, k0, D0, Pr_t, Le_t;
} jb_transport;

// status bits (device status word and C-ABI return codes)
enum jb_status {
  JB_OK = 0,
  JB_ERR_ARG = 1,
  JB_ERR_CUDA = 2,
  JB_ERR_NONFINITE = 4,
  JB_ERR_SINGULAR = 8,
  JB_ERR_TIMEOUT = 16,
  JB_ERR_UNSUPPORTED = 32
};

// Grid, boundary and theta parameters of one configured solver.
typedef struct jb_grid {
  int nx, ny;            // ny == 1 in 1D
  int nv, nY;            // number of conserved fields, index of first species
  long long ncell;
  double dx, dy;
  double idx, idy;       // 1/dx, 1/dy
  int bc[4];             // left, right, bottom, top (jb_bc_kind)
  double Pb;             // pressure_outlet back pressure (theta['Pb'])
  const double* Yinj;    // injector mass fractions [nr][nx] (theta['Yinj'])
  double inj_block_p;    // injector blocked when p_in >= this (1.0 nondim)
  int lstrip;            // ghost strip length max(nx, ny)
  int scheme;            // advective flux (jb_flux_scheme): LF splitting or Godunov + Riemann solver
  int recon;             // face reconstruction (jb_reconstruction): WENO5-JS or MUSCL
  const double* visc;    // viscous rhs of the stage state (ncell x nv) or null: Euler fluxes
  const double* halo;    // ghost columns [2][nv+2][3][ny] of the JB_BC_HALO x sides, else null
  int halo_ring;         // 1: x slabs (neighbours' columns, ring corners); 0: caller-computed ghost columns
  const double* haloy;   // ghost rows [2][nv+2][nx][3] of JB_BC_HALO y sides (caller-computed), else null
} jb_grid;

// Per-step reduction results.  Doubles reduced with atomics are stored as
// their bit patterns: for non-negative values integer order is float order.
typedef struct jb_slots {
  unsigned long long ax[4], ay[4];  // [0..2]: LF alpha of RK stage 1..3; [3]: next step
  unsigned long long dtmin_next;    // CFL minimum for the next step
  unsigned int mask[4];             // Halley masks of the 4 temperature solves
  unsigned int status;              // jb_status bits seen on the device
  unsigned int dtnan;               // a CFL candidate was NaN (jnp.min propagates it)
  double dt;                        // time step of the current step
} jb_slots;

#endif  // JB_TYPES_H
