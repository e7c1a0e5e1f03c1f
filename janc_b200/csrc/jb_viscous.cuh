// Laminar viscous flux (solver_{1D,2D}/flux.py viscous_flux_node /
// viscous_flux; model/transport_model.py; finite_difference/CENTRAL6.py;
// reconstruction/CENTRAL6.py).  Three passes over the ghost-padded grid:
//   k_visc_nodes  rho, u, (v), T, Y (9, filled) of every padded node,
//                 corners included (they hold the periodic wrap of the pad)
//   k_visc_flux   the node fluxes F_hat (x) and G_hat (y) from sixth-order
//                 derivatives (one-sided at the padded array's ends) and the
//                 transport model
//   k_visc_div    sixth-order interface values and their divergence per cell
// The result V = dF_hat/dx (+ dG_hat/dy) is added to the advective rhs by the
// stage kernels (NS_flux = advective + viscous, solver_2D/flux.py:117-118).
// Included by jb_kernels.cuh inside namespace jb::JB_NS.
#pragma once

// The padded grid's entry (x, y): interior, side ghost (boundary conditions)
// or corner (periodic wrap of both axes, boundary_padding.py pad_2D).  In
// x-slab mode the x pad is the exchanged neighbour columns on both sides,
// physical sides included (parallel/boundary_padding.py exchange_halo; the
// boundary conditions overwrite only the rows 3:-3), so a corner is the
// y-periodic wrap of a halo column.
template <int DIM>
__device__ __forceinline__ Src map_padded(const Grid& g, int x, int y) {
  if (DIM == 2 && (x < 0 || x >= g.nx) && (y < 0 || y >= g.ny)) {
    Src s;
    s.kind = 0;
    s.xs = x < 0 ? g.nx - 1 + x : x - g.nx + 1;
    s.ys = y < 0 ? g.ny - 1 + y : y - g.ny + 1;
    s.side = 0;
    s.pos = 0;
    s.flip = 0;
    s.layer = -1;
    if (g.halo && g.halo_ring) {
      s.kind = 1;
      s.side = x < 0 ? 0 : 1;
      s.layer = x < 0 ? x + 3 : x - g.nx;
      s.pos = s.ys;
    }
    return s;
  }
  return map_cell<DIM>(g, x, y);
}

// node planes: 2D rho, u, v, T, Y0..Y8 (13); 1D rho, u, T, Y0..Y8 (12)
template <int DIM>
__global__ void __launch_bounds__(256) k_visc_nodes(MP m, Grid g, const double* __restrict__ Uk,
                                                    const double* __restrict__ auxk,
                                                    const double* __restrict__ strips, double* __restrict__ nodes) {
  constexpr int nY = DIM == 1 ? 3 : 4, nv = nY + NR;
  const int PY = DIM == 2 ? g.ny + 6 : 1;
  const long long np = (long long)(g.nx + 6) * PY;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int px = (int)(i / PY), py = (int)(i % PY);
  const Src s = map_padded<DIM>(g, px - 3, DIM == 2 ? py - 3 : 0);
  const long long nc = g.ncell;
  double q[nv], T = 1.0;
  if (s.kind == 0) {
    const long long c = DIM == 2 ? (long long)s.xs * g.ny + s.ys : s.xs;
#pragma unroll
    for (int f = 0; f < nv; ++f) {
      const double v = Uk[f * nc + c];
      q[f] = ((s.flip >> f) & 1) ? -v : v;
    }
    T = auxk[nc + c];
  } else {
#pragma unroll
    for (int f = 0; f < nv; ++f) q[f] = ghost(g, strips, s, f);
    T = ghost(g, strips, s, nv + 1);
  }
  const double rho = q[0];
  double Y8[NR], Yf[NS];
#pragma unroll
  for (int k = 0; k < NR; ++k) Y8[k] = q[nY + k] / rho;
  fill_Y(Y8, Yf);
  nodes[i] = rho;
  nodes[np + i] = q[1] / rho;
  if (DIM == 2) nodes[2 * np + i] = q[2] / rho;
  nodes[(DIM + 1) * np + i] = T;
#pragma unroll
  for (int k = 0; k < NS; ++k) nodes[(DIM + 2 + k) * np + i] = Yf[k];
}

// d/dx of a node plane along one line (finite_difference/CENTRAL6.py d_dx):
// f points at position 0 of the line, stride st, n positions, at position p.
// The fast variants multiply by the stencils' reciprocal denominators.
__device__ __forceinline__ double d_line(const double* f, long long st, int n, int p, double d) {
  auto F = [&](int j) { return f[(long long)j * st]; };
#if JB_FAST
  const double id = 1.0 / d;
  if (p >= 3 && p < n - 3)
    return (-F(p - 3) + 9.0 * F(p - 2) - 45.0 * F(p - 1) + 45.0 * F(p + 1) - 9.0 * F(p + 2) + F(p + 3)) *
           (id * (1.0 / 60.0));
  if (p == 0) return (F(1) - F(0)) * id;
  if (p == 1) return (F(2) - F(0)) * (0.5 * id);
  if (p == 2) return (F(0) - 8.0 * F(1) + 8.0 * F(3) - F(4)) * (id * (1.0 / 12.0));
  if (p == n - 3) return (F(n - 5) - 8.0 * F(n - 4) + 8.0 * F(n - 2) - F(n - 1)) * (id * (1.0 / 12.0));
  if (p == n - 2) return (F(n - 1) - F(n - 3)) * (0.5 * id);
  return (F(n - 1) - F(n - 2)) * id;
#else
  if (p >= 3 && p < n - 3)
    return (-F(p - 3) + 9.0 * F(p - 2) - 45.0 * F(p - 1) + 45.0 * F(p + 1) - 9.0 * F(p + 2) + F(p + 3)) /
           (60.0 * d);
  if (p == 0) return (F(1) - F(0)) / d;
  if (p == 1) return (F(2) - F(0)) / (2.0 * d);
  if (p == 2) return (F(0) - 8.0 * F(1) + 8.0 * F(3) - F(4)) / (12.0 * d);
  if (p == n - 3) return (F(n - 5) - 8.0 * F(n - 4) + 8.0 * F(n - 2) - F(n - 1)) / (12.0 * d);
  if (p == n - 2) return (F(n - 1) - F(n - 3)) / (2.0 * d);
  return (F(n - 1) - F(n - 2)) / d;
#endif
}

// transport at one node (transport_model.py:106-157); mu_t is the LES
// sub-grid viscosity (0 for the laminar model), mu the total
struct NodeTransport {
  double mu, k, D[NS], h[NS];
};

// Vreman's sub-grid viscosity in 2D (model/LES/Verman.py:5-27) from the
// node's velocity gradient, in the reference's order of operations.
__device__ __forceinline__ double vreman_mu_t(double rho, double dx, double dy, double du_dx, double du_dy,
                                              double dv_dx, double dv_dy) {
  const double d1s = dx * dx, d2s = dy * dy;
  const double a11 = du_dx, a12 = dv_dx, a21 = du_dy, a22 = dv_dy;
  const double b11 = d1s * a11 * a11 + d2s * a21 * a21;
  const double b12 = d1s * a11 * a12 + d2s * a21 * a22;
  const double b22 = d1s * a12 * a12 + d2s * a22 * a22;
  double B = fabs(b11 * b22 - b12 * b12);
  if (!(B >= 0.0)) B = 0.0;  // jnp.where(B >= 0, B, 0): NaN -> 0
  const double a_sum = a11 * a11 + a12 * a12 + a21 * a21 + a22 * a22;
  const double ratio = a_sum > 0.0 ? B / a_sum : 0.0;
  return rho * 0.07 * sqrt(ratio);
}

__device__ __forceinline__ void node_transport(const MP& m, const jb_transport& tr, double rho, double T,
                                               const double* Yf, double mu_t, NodeTransport& o) {
  double cpk[NS], cp = 0.0;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const bool lo = T < m.Tcr[k];
    cpk[k] = lo ? poly5(m.cp_lo[k], T) : poly5(m.cp_hi[k], T);
    o.h[k] = lo ? poly6(m.h_lo[k], T) : poly6(m.h_hi[k], T);
    cp = k == 0 ? cpk[0] * Yf[0] : cp + cpk[k] * Yf[k];
  }
#if JB_FAST
  if (tr.viscosity_model == 0) {
    const double x = T / tr.T_ref;
    o.mu = tr.mu_ref * (x * sqrt(x)) * (tr.T_ref + tr.S) / (T + tr.S);
  } else {
    o.mu = rho * tr.nu0;
  }
  if (tr.turbulence_model) o.mu = o.mu + mu_t;
  if (tr.conductivity_model == 0 && tr.diffusivity_model == 0 && !tr.turbulence_model) {
    // Prandtl and Lewis numbers: rho D_k = mu / (Pr Le) for every species
    // (cp_k cancels), k = mu cp / Pr
    o.k = o.mu * cp / tr.Pr;
    const double D = o.mu / (tr.Pr * tr.Le * rho);
#pragma unroll
    for (int k = 0; k < NS; ++k) o.D[k] = D;
    return;
  }
#else
  if (tr.viscosity_model == 0) o.mu = tr.mu_ref * pow(T / tr.T_ref, 1.5) * (tr.T_ref + tr.S) / (T + tr.S);
  else o.mu = rho * tr.nu0;
  if (tr.turbulence_model) o.mu = o.mu + mu_t;  // mu_LES returns mu + mu_t
#endif
  if (tr.conductivity_model == 0) o.k = o.mu * cp / tr.Pr + mu_t * cp / tr.Pr_t;
  else o.k = tr.k0 + mu_t * cp / tr.Pr_t;
  const double pr_on = tr.conductivity_model == 0 ? 1.0 : 0.0, k_on = tr.conductivity_model == 0 ? 0.0 : 1.0;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    if (tr.diffusivity_model == 0) {
      const double k_i = pr_on * o.mu * cpk[k] / tr.Pr + k_on * tr.k0;
      const double rhoD_i = k_i / (tr.Le * cpk[k]);
      const double k_t = mu_t / tr.Pr_t;
      const double rhoD_t = k_t / (tr.Le_t * cpk[k]);
      o.D[k] = (rhoD_i + rhoD_t) / rho;
    } else {
      const double k_t = mu_t / tr.Pr_t;
      const double rhoD_t = k_t / tr.Le_t * cpk[k];
      o.D[k] = tr.D0 + rhoD_t / rho;
    }
  }
}

// Node fluxes, one thread per node.  2D threads [0, nF) take the nodes of
// the F_hat region (padded px in [0, nx+6), py in [3, ny+3) ->
// fh[c][px][py-3]); those with px in [3, nx+3) also lie in the G_hat region
// and write G_hat (gh[c][px-3][py]) from the same transport and velocity
// derivatives.  The rest are the G_hat-only nodes of the 3 + 3 ghost rows.
// 1D: F_hat at every padded px.
template <int DIM>
__global__ void __launch_bounds__(128) k_visc_flux(MP m, Grid g, jb_transport tr, const double* __restrict__ nodes,
                                                   double* __restrict__ fh, double* __restrict__ gh) {
  const int PX = g.nx + 6, PY = DIM == 2 ? g.ny + 6 : 1;
  const long long np = (long long)PX * PY;
  const long long nF = DIM == 2 ? (long long)PX * g.ny : PX;
  const long long nGo = DIM == 2 ? (long long)g.nx * 6 : 0;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nF + nGo) return;
  int px, py;
  bool do_f, do_g;
  if (DIM == 1) {
    px = (int)t;
    py = 0;
    do_f = true;
    do_g = false;
  } else if (t < nF) {
    px = (int)(t / g.ny);
    py = (int)(t % g.ny) + 3;
    do_f = true;
    do_g = px >= 3 && px < g.nx + 3;
  } else {
    const int j = (int)((t - nF) % 6);
    px = (int)((t - nF) / 6) + 3;
    py = j < 3 ? j : g.ny + j;
    do_f = false;
    do_g = true;
  }
  const long long i = (long long)px * PY + py;
  const double* N = nodes;
  const double rho = N[i], u = N[np + i];
  const double v = DIM == 2 ? N[2 * np + i] : 0.0;
  const double T = N[(DIM + 1) * np + i];
  double Yf[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) Yf[k] = N[(DIM + 2 + k) * np + i];
  NodeTransport tp;
  // derivatives along x (stride PY, PX positions) and y (stride 1, PY positions)
  const double* lx = N + (long long)py;           // line at this y, position px
  const double* ly = N + (long long)px * PY;      // line at this x, position py
  auto ddx = [&](int plane) { return d_line(lx + plane * np, PY, PX, px, g.dx); };
  auto ddy = [&](int plane) { return d_line(ly + plane * np, 1, PY, py, g.dy); };
  if (DIM == 1) {
    node_transport(m, tr, rho, T, Yf, 0.0, tp);
    double* out;
    long long ostride, oidx;
    const double du_dx = ddx(1), dT_dx = ddx(2);
    const double div_u = du_dx;
    const double tau = 2.0 * tp.mu * du_dx - 2.0 / 3.0 * tp.mu * div_u;
    const double qx = -tp.k * dT_dx;
    double jx[NS], e = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      jx[k] = -rho * tp.D[k] * ddx(3 + k);
      e = k == 0 ? jx[0] * tp.h[0] : e + jx[k] * tp.h[k];
    }
    out = fh;
    ostride = PX;
    oidx = px;
    out[oidx] = 0.0;
    out[ostride + oidx] = tau;
    out[2 * ostride + oidx] = u * tau - qx - e;
#pragma unroll
    for (int k = 0; k < NR; ++k) out[(3 + k) * ostride + oidx] = -jx[k];
    return;
  }
  const double du_dx = ddx(1), du_dy = ddy(1), dv_dx = ddx(2), dv_dy = ddy(2);
  const double mu_t = tr.turbulence_model ? vreman_mu_t(rho, g.dx, g.dy, du_dx, du_dy, dv_dx, dv_dy) : 0.0;
  node_transport(m, tr, rho, T, Yf, mu_t, tp);
  const double lam = -2.0 / 3.0 * tp.mu;
  const double S12 = 0.5 * (du_dy + dv_dx);
  const double div_u = du_dx + dv_dy;
  const double tau_xy = 2.0 * tp.mu * S12;
  // one direction's heat and species fluxes and its node flux vector
  auto emit = [&](bool xdir) {
    double jn[NS], e = 0.0;
    const double dTn = xdir ? ddx(3) : ddy(3);
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      jn[k] = -rho * tp.D[k] * (xdir ? ddx(4 + k) : ddy(4 + k));
      e = k == 0 ? jn[0] * tp.h[0] : e + jn[k] * tp.h[k];
    }
    const double qn = -tp.k * dTn;
    double f1, f2, f3;
    double* o;
    long long os, oi;
    if (xdir) {
      const double tau_xx = 2.0 * tp.mu * du_dx + lam * div_u;
      f1 = tau_xx;
      f2 = tau_xy;
      f3 = u * tau_xx + v * tau_xy - qn - e;
      o = fh;
      os = (long long)PX * g.ny;
      oi = (long long)px * g.ny + (py - 3);
    } else {
      const double tau_yy = 2.0 * tp.mu * dv_dy + lam * div_u;
      f1 = tau_xy;
      f2 = tau_yy;
      f3 = u * tau_xy + v * tau_yy - qn - e;
      o = gh;
      os = (long long)g.nx * PY;
      oi = (long long)(px - 3) * PY + py;
    }
    o[oi] = 0.0;
    o[os + oi] = f1;
    o[2 * os + oi] = f2;
    o[3 * os + oi] = f3;
#pragma unroll
    for (int k = 0; k < NR; ++k) o[(4 + k) * os + oi] = -jn[k];
  };
  if (do_f) emit(true);
  if (do_g) emit(false);
}

// interface value from six node fluxes (reconstruction/CENTRAL6.py)
__device__ __forceinline__ double central6(const double* f, long long st) {
  return (3.0 * f[0] - 25.0 * f[st] + 150.0 * f[2 * st] + 150.0 * f[3 * st] - 25.0 * f[4 * st] + 3.0 * f[5 * st]) /
         256.0;
}

template <int DIM>
__global__ void __launch_bounds__(128) k_visc_div(Grid g, const double* __restrict__ fh,
                                                  const double* __restrict__ gh, double* __restrict__ V) {
  constexpr int nv = DIM == 1 ? 11 : 12;
  const long long nc = g.ncell;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int x = DIM == 2 ? (int)(c / g.ny) : (int)c, y = DIM == 2 ? (int)(c % g.ny) : 0;
  const int PX = g.nx + 6, PY = g.ny + 6;
  const long long sF = DIM == 2 ? (long long)PX * g.ny : PX, sG = (long long)g.nx * PY;
#pragma unroll
  for (int f = 0; f < nv; ++f) {
    // faces x and x+1 of this cell: node fluxes at padded x .. x+6
    const double* a = fh + f * sF + (DIM == 2 ? (long long)x * g.ny + y : x);
    const long long st = DIM == 2 ? g.ny : 1;
#if JB_FAST
    double r = (central6(a + st, st) - central6(a, st)) * g.idx;
    if (DIM == 2) {
      const double* b = gh + f * sG + (long long)x * PY + y;
      r = r + (central6(b + 1, 1) - central6(b, 1)) * g.idy;
    }
#else
    double r = (central6(a + st, st) - central6(a, st)) / g.dx;
    if (DIM == 2) {
      const double* b = gh + f * sG + (long long)x * PY + y;
      r = r + (central6(b + 1, 1) - central6(b, 1)) / g.dy;
    }
#endif
    V[f * nc + c] = r;
  }
}

// The ghost-padded arrays themselves (boundary/boundary.py:120-132,
// boundary_conditions_{1D,2D}): every padded entry from the same mapping
// the stencils read, corners included (their periodic wrap, or the ring's
// on an x slab).  Up [nv][nx+6][ny+6], auxp [2][nx+6][ny+6] (1D: [.][nx+6]).
template <int DIM>
__global__ void __launch_bounds__(256) k_pad(Grid g, const double* __restrict__ U, const double* __restrict__ aux,
                                             const double* __restrict__ strips, double* __restrict__ Up,
                                             double* __restrict__ auxp) {
  constexpr int nv = DIM == 1 ? 11 : 12;
  const int PY = DIM == 2 ? g.ny + 6 : 1;
  const long long np = (long long)(g.nx + 6) * PY;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int px = (int)(i / PY), py = (int)(i % PY);
  const Src s = map_padded<DIM>(g, px - 3, DIM == 2 ? py - 3 : 0);
  const long long nc = g.ncell;
  if (s.kind == 0) {
    const long long c = DIM == 2 ? (long long)s.xs * g.ny + s.ys : s.xs;
#pragma unroll
    for (int f = 0; f < nv; ++f) {
      const double v = U[f * nc + c];
      Up[f * np + i] = ((s.flip >> f) & 1) ? -v : v;
    }
    auxp[i] = aux[c];
    auxp[np + i] = aux[nc + c];
  } else if (s.kind == 1) {
#pragma unroll
    for (int f = 0; f < nv; ++f) Up[f * np + i] = ghost(g, strips, s, f);
    auxp[i] = ghost(g, strips, s, nv);
    auxp[np + i] = ghost(g, strips, s, nv + 1);
  } else {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int f = 0; f < nv; ++f) Up[f * np + i] = nan;
    auxp[i] = auxp[np + i] = nan;
  }
}
