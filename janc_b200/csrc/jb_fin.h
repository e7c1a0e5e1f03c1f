// Where a kernel that writes a new state (an RK stage, the chemistry) puts
// the temperature solve of that state: update_aux after every stage and
// after the chemistry (src/janc_v2/simulation/set_simulator.py:117-122,
// simulation/time_step/TVD_RK3.py:5-12).
#pragma once

#ifdef __CUDACC__
#define JB_HD __host__ __device__
#else
#define JB_HD
#endif

struct jb_fin {
  // Global-stop mode (aux == nullptr): every cell keeps the Halley iterates
  // T_0..T_5 in cand[6][ncell] and ORs its residual bits into mask slot midx;
  // a select pass then takes the iterate of the reference's global iteration
  // count (model/thermo_model.py:135-153).  The parity build uses this mode.
  double* cand;
  int midx;
  // Per-cell mode (aux != nullptr; the mixed variant in 2D): each cell
  // iterates until its own residual is within tol, takes one more step, and
  // writes (gamma, T) into aux; the
  // wave speeds |u| + a, |v| + a of the new state go to alpha slot aidx
  // (< 0: none), with cfl != 0 also the CFL minimum, and the float32 u, v, p
  // of the new state into prims (the next mixed-precision stage's input; may
  // be null).
  double* aux;
  float* prims;
  int aidx;
  int cfl;
};

// jb_fin of the global-stop mode
JB_HD inline jb_fin jb_fin_cand(double* cand, int midx) {
  jb_fin f;
  f.cand = cand;
  f.midx = midx;
  f.aux = nullptr;
  f.prims = nullptr;
  f.aidx = -1;
  f.cfl = 0;
  return f;
}

// jb_fin of the per-cell mode
JB_HD inline jb_fin jb_fin_cell(double* aux, float* prims, int aidx, int cfl) {
  jb_fin f;
  f.cand = nullptr;
  f.midx = -1;
  f.aux = aux;
  f.prims = prims;
  f.aidx = aidx;
  f.cfl = cfl;
  return f;
}
