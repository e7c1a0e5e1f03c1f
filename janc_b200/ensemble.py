"""Batched ensemble of 1D reacting-flow instances on one GPU.

Many independent detonation tubes (different lengths, spacings, boundary
pairs, compositions, ignition states) advance together in ONE persistent
cooperative kernel per call, replayed from a CUDA graph.  Each instance
takes exactly the steps a single-case ``Solver`` takes (the reference's
``Simulator.advance_func`` loop, src/janc_v2/simulation/set_simulator.py:
412-447, with the RK3 step of set_simulator.py:117-122), with its own CFL
time step and Lax-Friedrichs alpha, so instance i of an ensemble equals a
``Solver`` run of that instance alone in the same precision.

    ens = Ensemble(nx_list, dx_list, cfl=0.1, precision="mixed")
    for i, (U, aux) in enumerate(states):
        ens.set_state(i, U, aux)
    ens.autotune()                  # picks block size and CTAs per SM
    dts = ens.advance(2000, record_dt=True)
    U, aux = ens.get_state(0)
"""
import ctypes

import numpy as np
import torch

from . import _native
from . import mechanism as _mech

ATM = 101325.0


class _DeviceArray:
    """A float64 device buffer exposed through __cuda_array_interface__."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(int(s) for s in shape), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 2, "strides": None}


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _per_instance(v, n, name):
    if np.ndim(v) == 0:
        return [v] * n
    v = list(v)
    if len(v) != n:
        raise ValueError(f"{name}: expected {n} values, got {len(v)}")
    return v


class Ensemble:
    """``nx[i]`` cells of spacing ``dx[i]`` per instance; ``boundary`` is a
    (left, right) pair of boundary names for all instances or a list of
    pairs; ``cfl`` (scalar or list) > 0 selects CFL time steps, otherwise
    ``dt`` (scalar or list) is the fixed step.  ``Pb`` (scalar or list) is
    the back pressure of pressure-outlet sides (the reference's
    theta['Pb']); required when an instance has one, as the reference's
    boundary function requires it."""

    def __init__(self, nx, dx, boundary=("slip_wall", "zero_gradient"), cfl=0.1, dt=None,
                 mechanism=_mech.DEFAULT_MECHANISM, nondim_config=None, precision="mixed", device=None, Pb=None):
        if precision not in ("fp64", "mixed"):
            raise KeyError("ensemble precision must be 'fp64' or 'mixed'")
        n = len(nx)
        if n < 1:
            raise ValueError("an ensemble needs at least one instance")
        self.n = n
        self.nx = [int(v) for v in nx]
        self.dx = [float(v) for v in _per_instance(dx, n, "dx")]
        if isinstance(boundary, (tuple, list)) and len(boundary) == 2 and isinstance(boundary[0], str):
            boundary = [tuple(boundary)] * n
        boundary = _per_instance(boundary, n, "boundary")
        kinds = []
        for pair in boundary:
            for name in pair:
                if callable(name):
                    raise NotImplementedError("Python callables cannot run inside the kernels")
                if name not in _native.BC_KIND:
                    raise KeyError(f"unknown boundary condition {name!r}")
                kinds.append(_native.BC_KIND[name])
        if Pb is None and _native.BC_KIND["pressure_outlet"] in kinds:
            raise KeyError("Pb")
        self.Pb = [float(v) for v in _per_instance(0.0 if Pb is None else Pb, n, "Pb")]
        self.cfl = [float(v) for v in _per_instance(0.0 if cfl is None else cfl, n, "cfl")]
        self.dt = [float(v) for v in _per_instance(0.0 if dt is None else dt, n, "dt")]
        self.precision = precision
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.mech = mechanism if isinstance(mechanism, _mech.Mechanism) else _mech.load(mechanism, nondim_config)
        self._params = _mech.pack(self.mech)
        self._lib = _native.lib()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            rc = self._lib.jb_ens_create(
                ctypes.byref(self._params), n, (ctypes.c_int * n)(*self.nx), (ctypes.c_double * n)(*self.dx),
                (ctypes.c_int * (2 * n))(*kinds), (ctypes.c_double * n)(*self.cfl),
                (ctypes.c_double * n)(*self.dt), _native.PRECISION[precision], ctypes.byref(h))
        _native.check(rc, None, "jb_ens_create")
        self._h = h
        if any(v != 0.0 for v in self.Pb):
            _native.check(self._lib.jb_ens_set_back_pressure(h, (ctypes.c_double * n)(*self.Pb)), h,
                          "jb_ens_set_back_pressure", ensemble=True)
        self._U, self._aux = [], []
        for i in range(n):
            pu, pa, m = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int()
            _native.check(self._lib.jb_ens_instance(h, i, ctypes.byref(pu), ctypes.byref(pa), ctypes.byref(m)),
                          h, "jb_ens_instance", ensemble=True)
            self._U.append(torch.as_tensor(_DeviceArray(pu.value, (11, m.value)), device=self.device))
            self._aux.append(torch.as_tensor(_DeviceArray(pa.value, (2, m.value)), device=self.device))
        self._thermo = None

    # ------------------------------------------------------------- lifetime
    def close(self):
        if getattr(self, "_h", None):
            self._U, self._aux = [], []
            self._lib.jb_ens_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ----------------------------------------------------------------- state
    @property
    def total_cells(self):
        return int(self._lib.jb_ens_total_cells(self._h))

    def state(self, i):
        """Views (U (11, nx_i), aux (2, nx_i)) of instance i's live state."""
        return self._U[i], self._aux[i]

    def set_state(self, i, U, aux):
        for dst, src, nv in ((self._U[i], U, 11), (self._aux[i], aux, 2)):
            t = torch.as_tensor(src, dtype=torch.float64)
            if tuple(t.shape) != (nv, self.nx[i]):
                raise ValueError(f"instance {i}: expected shape {(nv, self.nx[i])}, got {tuple(t.shape)}")
            dst.copy_(t.to(self.device))

    def get_state(self, i):
        return self._U[i].clone(), self._aux[i].clone()

    def state_from_PTY(self, P, T, Y):
        """(U, aux) of one 1D instance at rest from pressure (1, n),
        temperature (1, n) and mass fractions (8, n), as the reference's
        examples build it (rho = P/(R T), rho E = rho h - P)."""
        if self._thermo is None:
            from .solver import Solver
            self._thermo = Solver(1, 4, dx=1.0, mechanism=self.mech, precision="fp64", device=self.device)
        f = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=self.device)
        return self._thermo.state_from_PTY(f(P), f(T), f(Y))

    # ----------------------------------------------------------- launching
    def configure(self, block=128, blocks_per_sm=3):
        _native.check(self._lib.jb_ens_configure(self._h, int(block), int(blocks_per_sm)), self._h,
                      "jb_ens_configure", ensemble=True)

    def autotune(self, trial_steps=20):
        """Time every launch shape on ``trial_steps`` steps (state restored)
        and keep the fastest; returns {block, blocks_per_sm, ms}."""
        b, p, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _native.check(self._lib.jb_ens_autotune(self._h, int(trial_steps), _stream(), ctypes.byref(b),
                                                ctypes.byref(p), ctypes.byref(ms)),
                      self._h, "jb_ens_autotune", ensemble=True)
        return {"block": b.value, "blocks_per_sm": p.value, "ms": ms.value}

    def launch_shape(self):
        v = [ctypes.c_int() for _ in range(5)]
        _native.check(self._lib.jb_ens_launch_shape(self._h, *[ctypes.byref(x) for x in v]), self._h,
                      "jb_ens_launch_shape", ensemble=True)
        mode = {0: "none yet", 1: "stream capture", 2: "explicit nodes"}[v[4].value]
        return {"block": v[0].value, "blocks_per_sm": v[1].value, "ctas": v[2].value,
                "max_tiles_per_cta": v[3].value, "graph": mode}

    def advance(self, nsteps, record_dt=False, graph=True):
        """Advance every instance ``nsteps`` steps in place.  Returns the
        (n, nsteps) device tensor of time steps when ``record_dt``."""
        hist = None
        if record_dt:
            # reuse the buffer so that the captured graph (which holds its
            # address) is replayed rather than rebuilt
            if getattr(self, "_hist", None) is None or tuple(self._hist.shape) != (self.n, int(nsteps)):
                self._hist = torch.empty((self.n, int(nsteps)), dtype=torch.float64, device=self.device)
            hist = self._hist
        p = ctypes.c_void_p(hist.data_ptr()) if hist is not None else None
        fn = self._lib.jb_ens_advance if graph else self._lib.jb_ens_advance_direct
        _native.check(fn(self._h, int(nsteps), p, _stream()), self._h, "jb_ens_advance", ensemble=True)
        return hist.clone() if hist is not None else None

    def status(self):
        """(combined, per-instance) jb_status bits since the last call;
        combined includes JB_ERR_TIMEOUT if a barrier wait gave up."""
        per = (ctypes.c_uint * self.n)()
        comb = ctypes.c_uint()
        _native.check(self._lib.jb_ens_status(self._h, per, ctypes.byref(comb), _stream()), self._h,
                      "jb_ens_status", ensemble=True)
        return comb.value, list(per)


def detonation_tubes(n=64, seed=4, cells=(1000, 16000), phi=(0.6, 1.4), T_ign=(2500.0, 3500.0), dx=5e-5,
                     slab=0.02, p_ign=30 * ATM, p0=ATM, T0=300.0, mech=None):
    """The batched-ensemble workload: ``n`` 1D H2-air tubes at rest with
    lengths drawn log-uniform in ``cells``, equivalence ratio uniform in
    ``phi`` and ignition temperature uniform in ``T_ign`` (numpy
    default_rng(seed)), spacing ``dx``, and an ignition slab over the first
    ``slab`` fraction of cells at ``p_ign``.  Returns a list of dicts with
    nx, phi, T_ign, and the P, T, Y arrays of the initial state."""
    if mech is None:
        mech = _mech.load(_mech.DEFAULT_MECHANISM)
    rng = np.random.default_rng(seed)
    lengths = np.round(np.exp(rng.uniform(np.log(cells[0]), np.log(cells[1]), n))).astype(int)
    phis = rng.uniform(phi[0], phi[1], n)
    Tign = rng.uniform(T_ign[0], T_ign[1], n)
    out = []
    for nx, ph, Ti in zip(lengths, phis, Tign):
        nx = int(nx)
        ns = max(1, int(round(slab * nx)))
        P = np.full((1, nx), p0)
        T = np.full((1, nx), T0)
        P[:, :ns] = p_ign
        T[:, :ns] = Ti
        Y = np.tile(_mech.stoichiometric_Y(mech, float(ph))[:, None], (1, nx))
        out.append({"nx": nx, "phi": float(ph), "T_ign": float(Ti), "dx": dx, "P": P, "T": T, "Y": Y})
    return out
