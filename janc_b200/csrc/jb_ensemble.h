// Device-resident description of a batched ensemble of 1D instances.
#ifndef JB_ENSEMBLE_H
#define JB_ENSEMBLE_H

#include "jb_types.h"

// One instance (a detonation tube).  Every pointer is device memory owned by
// the ensemble; the state U / aux is advanced in place.
typedef struct jb_ens_inst {
  jb_grid g;            // nx = cells, ny = 1, ncell = nx, lstrip = 1
  double* U;            // [11][nx] conserved state
  double* aux;          // [2][nx]  gamma, T
  double* W0;           // [11][nx] RK stage buffers
  double* W1;
  double* A0;           // [2][nx]  aux of the RK stages
  double* A1;
  double* cand;         // [6][nx]  Halley iterates
  double* strips;       // [4][13][1] ghost states of outlet sides
  jb_slots* slots;      // [2]: even / odd steps
  unsigned* bar;        // arrival counter of this instance's CTA group
  double* dt_hist;      // [max steps] time steps of the last run, or null
  double cfl;           // > 0: CFL time step
  double dt;            // fixed time step when cfl <= 0
  int cta0, ncta;       // the CTAs [cta0, cta0 + ncta) serve this instance
  int ntiles;           // flux tiles of (block - 1) cells
  int nchunks;          // cell chunks of block cells (select / chemistry)
} jb_ens_inst;

// Run control shared by all CTAs of one launch (cleared before each launch).
typedef struct jb_ens_ctl {
  unsigned abort;       // set when any wait gave up; every CTA then returns
  unsigned timeout;     // a group barrier exceeded its time limit
  unsigned where_inst;  // instance and phase of the first wait that gave up
  unsigned where_phase;
} jb_ens_ctl;

#endif  // JB_ENSEMBLE_H
