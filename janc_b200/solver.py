"""One configured solver = one native handle (grid, boundaries, mechanism,
arithmetic variant) with the reference's call signatures.

Tensors are torch CUDA float64, C-contiguous, in the reference layout
(``U`` (nv, nx[, ny]), ``aux`` (2, nx[, ny])).  PyTorch only provides the
device buffers and the current stream; every computation is a kernel of
``libjanc_b200.so``.
"""
import ctypes

import numpy as np
import torch

from . import _native
from . import mechanism as _mech

BOUNDARY_KEYS = ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def flux_scheme(flux_config):
    """Validate a reference ``flux_solver_config`` (set_flux_solver,
    solver_2D/flux.py:19-40) and name the native flux: ``LF``, ``SW``
    (flux splitting) or ``HLLC``, ``AUSMPW_plus`` (Godunov).  Raises as the
    reference does: KeyError for an unknown solver type or dictionary
    entry."""
    if flux_config is None:
        return "LF"
    solver_type = flux_config["solver_type"]
    if solver_type not in ("godunov", "flux_splitting"):
        raise KeyError("JANC only support 'godunov' and 'flux_splitting'")
    recon = flux_config["interface_reconstruction"]
    if recon not in _native.RECONSTRUCTION:
        raise KeyError(recon)
    if solver_type == "godunov":
        rs = flux_config["riemann_solver"]
        if rs not in ("HLLC", "AUSMPW_plus"):
            raise KeyError(rs)
        return rs
    split = flux_config["split_method"]
    if split not in ("LF", "SW"):
        raise KeyError(split)
    return split


def transport_params(transport_config, dim=2):
    """jb_transport from a reference ``transport_config`` (set_transport,
    model/transport_model.py:26-104), with its defaults and errors: laminar,
    or LES with the Vreman sub-grid model, the only one the reference has
    (``LES_model`` 'Verman', 2D; another model name raises the KeyError the
    reference raises at its first flux evaluation)."""
    c = transport_config
    t = _native.Transport()
    t.mu_ref, t.T_ref, t.S, t.nu0 = 1.716e-5, 273.15, 110.4, 1e-4
    t.Pr, t.Pr_t, t.Le, t.Le_t, t.k0, t.D0 = 0.72, 0.72, 1.0, 1.0, 0.0, 0.0
    if c["viscosity_model"] == "constant":
        t.viscosity_model, t.nu0 = 1, c["dynamic_viscosity"]
    elif c["viscosity_model"] == "Sutherland":
        t.mu_ref = c.get("reference_viscosity", t.mu_ref)
        t.T_ref = c.get("reference_temperature", t.T_ref)
        t.S = c.get("effective_temperature", t.S)
    else:
        raise KeyError("Only 'Sutherland' and 'constant' viscosity model are supported.")
    if c["thermal_conductivity_model"] == "constant":
        t.conductivity_model, t.k0 = 1, c["thermal_conductivity"]
    elif c["thermal_conductivity_model"] == "Prandtl number":
        assert "Pr" in c, "Key 'Pr' must be provided"
        t.Pr = c["Pr"]
    else:
        raise KeyError("Only 'Prandtl number' and 'constant' thermal conductivity model are supported.")
    if c["species_diffusivity_model"] == "constant":
        t.diffusivity_model, t.D0 = 1, c["species_diffusivity"]
    elif c["species_diffusivity_model"] == "Schmidt number":
        assert "Sc" in c, "Key 'Sc' must be provided"
        t.Le = c["Sc"] / t.Pr
    elif c["species_diffusivity_model"] == "Lewis number":
        assert "Le" in c, "Key 'Le' must be provided"
        t.Le = c["Le"]
    else:
        raise KeyError("Only 'Schmidt number', 'Lewis number', and 'constant' species diffusivity model "
                       "are supported.")
    model = c.get("turbulence_model", "laminar")
    if model == "LES":
        assert "LES_model" in c, "Please specify the SGS model of LES."
        assert "Pr_t" in c, "Key 'Pr_t'(turbulent Prandtl number) must be provided"
        assert ("Le_t" in c) or ("Sc_t" in c), \
            "Key 'Sc_t'(turbulent Schmidt number) or 'Le_t'(turbulent Lewis number) must be provided"
        name = f"{c['LES_model']}_{'2D' if dim == 2 else '1D'}"
        if name != "Verman_2D":
            raise KeyError(name)
        t.turbulence_model = 1
        t.Pr_t = c["Pr_t"]
        t.Le_t = c["Le_t"] if "Le_t" in c else c["Sc_t"] / t.Pr_t
    elif model != "laminar":
        raise KeyError("Only 'laminar' and 'LES' model are supported.")
    return t


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class _GhostCells:
    """Boundary functions (boundary/boundary.py:16-21, 37-42, 58-63, 79-84):
    before each flux evaluation the library packs the 3 boundary-adjacent
    layers of (U, aux) and calls back here; each function gets them as the
    reference passes them (left ``padded_U[:, 3:6(, 3:-3)]``, right
    ``[:, -6:-3]``, bottom ``[:, 3:-3, 3:6]``, top ``[:, 3:-3, -6:-3]``, as
    CUDA tensors) with theta, and returns the 3 ghost layers in padded
    order, which go to the kernels' ghost buffers (``jb_set_ghost_cells``)."""

    def __init__(self, solver, fns):
        nv, nx, ny, dev = solver.nv, solver.nx, solver.ny, solver.device
        self.sendx = torch.zeros((2, nv + 2, 3, ny), dtype=torch.float64, device=dev)
        self.halox = torch.zeros_like(self.sendx)
        self.sendy = torch.zeros((2, nv + 2, nx, 3), dtype=torch.float64, device=dev)
        self.haloy = torch.zeros_like(self.sendy)
        self.fns = [fns.get(k) for k in BOUNDARY_KEYS]
        self.solver = solver
        self.error = None
        self.calls = 0
        self._fn = _native.EXCHANGE_FN(self._callback)

    def attach(self, lib, h):
        _native.check(lib.jb_set_ghost_cells(h, _ptr(self.sendx), _ptr(self.halox), _ptr(self.sendy),
                                             _ptr(self.haloy), self._fn, None), h, "jb_set_ghost_cells")

    def _callback(self, user, flags, stream):
        try:
            dev = self.sendx.device
            if stream and torch.cuda.current_stream(dev).cuda_stream != stream:
                with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=dev)):
                    self._fill()
            else:
                self._fill()
            self.calls += 1
            return 0
        except BaseException as e:  # reported by the library as a failed call
            self.error = e
            return 1

    def _fill(self):
        s = self.solver
        nv = s.nv
        for side, fn in enumerate(self.fns):
            if fn is None:
                continue
            send, halo = (self.sendx, self.halox) if side < 2 else (self.sendy, self.haloy)
            b = side % 2
            Ub, ab = send[b, :nv], send[b, nv:]
            if s.dim == 1:
                Ub, ab = Ub[..., 0], ab[..., 0]
            Ug, ag = fn(Ub, ab, s._theta)
            halo[b, :nv].copy_(torch.as_tensor(Ug, device=halo.device).reshape(halo[b, :nv].shape))
            halo[b, nv:].copy_(torch.as_tensor(ag, device=halo.device).reshape(halo[b, nv:].shape))


class Solver:
    """Native solver for a fixed grid.

    ``boundary_config`` maps ``left_boundary``/``right_boundary``
    (``bottom_boundary``/``top_boundary`` in 2D) to one of ``periodic``,
    ``slip_wall``, ``zero_gradient``, ``no_slip_wall``, ``pressure_outlet`` or
    ``rdc_injector`` (the rotating-detonation injector of the reference's
    example 2, bottom side only).

    ``flux_config`` is the reference's ``flux_solver_config``
    (solver_{1D,2D}/flux.py set_flux_solver): ``solver_type``
    ``flux_splitting`` (``split_method`` ``LF`` or ``SW``) or ``godunov``
    (``riemann_solver`` ``HLLC`` or ``AUSMPW_plus``), with
    ``interface_reconstruction`` ``WENO5_JS`` or ``MUSCL``.  Default: LF flux
    splitting with WENO5_JS.
    ``viscosity`` ``on`` adds the laminar viscous fluxes of
    ``transport_config`` (the reference's transport_config: Sutherland or
    constant viscosity, Prandtl-number or constant conductivity, Lewis /
    Schmidt-number or constant diffusivity).

    ``slab`` (a ``janc_b200.slab.Slab``) makes this solver one x slab of a
    grid decomposed over the ranks of a process group (the reference's
    ``is_parallel`` mode): ``nx`` is the slab's column count, the
    ``boundary_config`` is the global domain's, and every flux evaluation
    exchanges 3 ghost columns with the neighbouring slabs.
    """

    def __init__(self, dim, nx, ny=None, dx=1.0, dy=None, boundary_config=None,
                 mechanism=_mech.DEFAULT_MECHANISM, nondim_config=None, precision="fp64",
                 device=None, flux_config=None, transport_config=None, slab=None):
        if dim in ("1D", 1):
            dim = 1
        elif dim in ("2D", 2):
            dim = 2
        else:
            raise KeyError(f"unsupported dimension {dim!r}")
        if precision not in _native.PRECISION:
            raise KeyError(f"precision must be one of {sorted(_native.PRECISION)}")
        self.dim, self.nx = dim, int(nx)
        self.ny = int(ny) if dim == 2 else 1
        self.dx = float(dx)
        self.dy = float(dy) if dim == 2 else 1.0
        self.nv = 12 if dim == 2 else 11
        self.precision = precision
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.mech = mechanism if isinstance(mechanism, _mech.Mechanism) else _mech.load(mechanism, nondim_config)
        self._params = _mech.pack(self.mech)
        bc = boundary_config or {}
        kinds = []
        ghost_fns = {}
        for key in BOUNDARY_KEYS[: 2 * dim]:
            name = bc.get(key, "periodic")
            if callable(name):
                ghost_fns[key] = name
                kinds.append(_native.BC_HALO)
                continue
            if name not in _native.BC_KIND:
                raise KeyError(f"{key}: unknown boundary condition {name!r}")
            kinds.append(_native.BC_KIND[name])
        kinds += [0] * (4 - len(kinds))
        if ghost_fns and slab is not None:
            raise NotImplementedError("boundary functions on x slabs")
        self._theta = None
        self.slab = slab
        if slab is not None:
            kinds = slab.boundary_kinds(kinds)
        self.boundary_kinds = kinds
        self._theta_key = None
        self._theta_keep = None
        L = _native.lib()
        h = ctypes.c_void_p()
        arr = (ctypes.c_int * 4)(*kinds)
        with torch.cuda.device(self.device):
            rc = L.jb_create(ctypes.byref(self._params), dim, self.nx, self.ny, self.dx, self.dy, arr,
                             _native.PRECISION[precision], ctypes.byref(h))
        _native.check(rc, None, "jb_create")
        self._h = h
        self._lib = L
        self._exchange = None
        if slab is not None:
            from .slab import SlabExchange
            self._exchange = SlabExchange(slab, self.nv, self.ny, self.device)
            self._exchange.attach(L, h)
        elif ghost_fns:
            self._exchange = _GhostCells(self, ghost_fns)
            self._exchange.attach(L, h)
        self.flux_scheme = flux_scheme(flux_config)
        _native.check(L.jb_set_flux_scheme(h, _native.FLUX_SCHEME[self.flux_scheme]), h, "jb_set_flux_scheme")
        self.reconstruction = (flux_config or {}).get("interface_reconstruction", "WENO5_JS")
        _native.check(L.jb_set_reconstruction(h, _native.RECONSTRUCTION[self.reconstruction]), h,
                      "jb_set_reconstruction")
        self.viscous = bool(flux_config) and flux_config.get("viscosity", "off") == "on"
        if self.viscous:
            if transport_config is None:
                raise KeyError("transport_config")  # set_flux_solver passes it to set_transport
            self._transport = transport_params(transport_config, dim)
            with torch.cuda.device(self.device):
                _native.check(L.jb_set_transport(h, ctypes.byref(self._transport)), h, "jb_set_transport")

    # ------------------------------------------------------------------ utils
    def close(self):
        if getattr(self, "_h", None):
            self._lib.jb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return (self.nx, self.ny) if self.dim == 2 else (self.nx,)

    def _check_state(self, U, aux=None):
        for name, t, nv in (("U", U, self.nv), ("aux", aux, 2)):
            if t is None:
                continue
            if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
                raise TypeError(f"{name} must be a CUDA tensor")
            if t.dtype != torch.float64:
                raise TypeError(f"{name} must be float64")
            if tuple(t.shape) != (nv,) + self.shape:
                raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {(nv,) + self.shape}")
            if not t.is_contiguous():
                raise ValueError(f"{name} must be contiguous")

    def _check(self, rc, what):
        """Raise for a failed call; a failed slab exchange raises its own error."""
        if rc != 0 and self._exchange is not None and self._exchange.error is not None:
            err, self._exchange.error = self._exchange.error, None
            raise _native.JancError(f"{what}: slab exchange failed: {err!r}") from err
        _native.check(rc, self._h, what)

    def _spacing(self, dx, dy):
        dx = self.dx if dx is None else float(dx)
        dy = self.dy if (dy is None or self.dim == 1) else float(dy)
        if dx != self.dx or dy != self.dy:
            _native.check(self._lib.jb_set_spacing(self._h, dx, dy), self._h, "jb_set_spacing")
            self.dx, self.dy = dx, dy

    def set_theta(self, theta):
        """theta['Pb'] for pressure outlets; theta['Yinj'] (8, nx[, 1]) or (8,)
        for the injector."""
        self._theta = theta
        if theta is None:
            theta = {}
        Pb = float(theta.get("Pb", 0.0))
        Yinj = theta.get("Yinj", None)
        key = (Pb, None if Yinj is None else id(Yinj))
        if key == self._theta_key:
            return
        yptr = None
        if Yinj is not None:
            y = torch.as_tensor(np.asarray(Yinj.cpu() if isinstance(Yinj, torch.Tensor) else Yinj),
                                dtype=torch.float64)
            if y.ndim == 1:
                y = y[:, None].expand(y.shape[0], self.nx)
            y = y.reshape(y.shape[0], -1)
            if self.slab is not None and y.shape[1] == self.nx * self.slab.size:
                y = y[:, self.slab.rank * self.nx:(self.slab.rank + 1) * self.nx]  # PartitionDict along x
            y = y.reshape(y.shape[0], self.nx).contiguous().to(self.device)
            self._theta_keep = y
            yptr = _ptr(y)
        if any(k == _native.BC_KIND["pressure_outlet"] for k in self.boundary_kinds[: 2 * self.dim]) \
                and "Pb" not in theta:
            raise KeyError("Pb")
        if any(k == _native.BC_KIND["rdc_injector"] for k in self.boundary_kinds[: 2 * self.dim]) \
                and Yinj is None:
            raise KeyError("Yinj")
        _native.check(self._lib.jb_set_theta(self._h, Pb, yptr, 1.0), self._h, "jb_set_theta")
        self._theta_key = key

    def status(self):
        st = ctypes.c_uint()
        _native.check(self._lib.jb_status(self._h, ctypes.byref(st), _stream()), self._h, "jb_status")
        return st.value

    def set_kernel_timing(self, enable=True):
        _native.check(self._lib.jb_set_kernel_timing(self._h, int(enable)), self._h, "jb_set_kernel_timing")

    def kernel_times(self):
        """{category: (milliseconds, launches)} accumulated since
        set_kernel_timing (categories: flux, select, chem, other)."""
        ms = (ctypes.c_double * 4)()
        n = (ctypes.c_longlong * 4)()
        _native.check(self._lib.jb_kernel_times(self._h, ms, n), self._h, "jb_kernel_times")
        return {k: (ms[i], n[i]) for i, k in enumerate(("flux", "select", "chem", "other"))}

    def workspace_bytes(self):
        return int(self._lib.jb_workspace_bytes(self._h))

    # ------------------------------------------------ reference entry points
    def flux_func(self, U, aux, dx=None, dy=None, dt=1.0, theta=None):
        """dt * total_flux(BC(U, aux)) (set_simulator.py:26-29 / 44-47)."""
        self._check_state(U, aux)
        self._spacing(dx, dy)
        self.set_theta(theta)
        out = torch.empty_like(U)
        self._check(self._lib.jb_flux_func(self._h, _ptr(U), _ptr(aux), float(dt), _ptr(out), _stream()),
                    "jb_flux_func")
        return out

    def boundary_conditions(self, U, aux, theta=None):
        """boundary_conditions_1D / _2D (boundary/boundary.py:120-132; on a
        slab parallel/boundary.py): the ghost-padded (U, aux), (nv, nx+6[,
        ny+6]) and (2, nx+6[, ny+6]), corners included."""
        self._check_state(U, aux)
        self.set_theta(theta)
        pad = (self.nx + 6,) + ((self.ny + 6,) if self.dim == 2 else ())
        Up = torch.empty((self.nv,) + pad, dtype=torch.float64, device=U.device)
        Ap = torch.empty((2,) + pad, dtype=torch.float64, device=U.device)
        self._check(self._lib.jb_boundary_conditions(self._h, _ptr(U), _ptr(aux), _ptr(Up), _ptr(Ap), _stream()),
                    "jb_boundary_conditions")
        return Up, Ap

    def update_aux(self, U, aux):
        """aux_func.update_aux: (gamma, T) from the Halley solve."""
        self._check_state(U, aux)
        out = torch.empty_like(aux)
        _native.check(self._lib.jb_update_aux(self._h, _ptr(U), _ptr(aux), _ptr(out), _stream()),
                      self._h, "jb_update_aux")
        return out

    def reaction_source_terms(self, U, aux, dt, theta=None):
        """reaction_model.reaction_source_terms: point-implicit chemistry dU."""
        self._check_state(U, aux)
        out = torch.empty_like(U)
        _native.check(self._lib.jb_reaction_source_terms(self._h, _ptr(U), _ptr(aux), float(dt), _ptr(out),
                                                         _stream()), self._h, "jb_reaction_source_terms")
        return out

    def _check_blocks(self, blk, padded, name):
        if self.dim != 2:
            raise ValueError("block AMR needs a 2D solver")
        if not isinstance(blk, torch.Tensor) or blk.device.type != "cuda" or blk.dtype != torch.float64:
            raise TypeError(f"{name} must be a float64 CUDA tensor")
        if blk.ndim != 4 or blk.shape[1] != self.nv + 2 or (padded and min(blk.shape[2:]) < 7):
            raise ValueError(f"{name} has shape {tuple(blk.shape)}, expected (nb, {self.nv + 2}, X, Y)"
                             + (" with 3 ghost layers on each side" if padded else ""))
        if not blk.is_contiguous():
            raise ValueError(f"{name} must be contiguous")

    def amr_stage(self, G, U0, stage, dx, dy, dt):
        """One SSP-RK3 stage of ghost-padded AMR blocks (TVD_RK3.py:15-36 with
        the vmapped block flux and update_aux of set_simulator.py:37-42):
        G, U0 [nb][nv+2][bx+6][by+6] (U fields, gamma, T; U0 the step's
        first stage input, unused for stage 1).  Returns the new padded
        blocks (ghost entries combined with a zero rhs) with their (gamma,
        T) from the block's own temperature solve."""
        self._check_blocks(G, True, "G")
        if stage > 1:
            self._check_blocks(U0, True, "U0")
            if U0.shape != G.shape:
                raise ValueError("U0 and G differ in shape")
        out = torch.empty_like(G)
        nb, _, X, Y = G.shape
        _native.check(self._lib.jb_amr_stage(self._h, nb, X - 6, Y - 6, float(dx), float(dy), int(stage), _ptr(G),
                                             _ptr(U0) if stage > 1 else None, float(dt), _ptr(out), _stream()),
                      self._h, "jb_amr_stage")
        return out

    def amr_flux(self, U, aux, dx, dy, dt):
        """The vmapped block flux function (set_simulator.py:37-40): padded
        blocks U [nb][nv][bx+6][by+6], aux [nb][2][..] -> pad(dt * total_flux,
        3) with zeros in the ghost entries."""
        for name, t, nf in (("U", U, self.nv), ("aux", aux, 2)):
            if not isinstance(t, torch.Tensor) or t.device.type != "cuda" or t.dtype != torch.float64:
                raise TypeError(f"{name} must be a float64 CUDA tensor")
            if t.ndim != 4 or t.shape[1] != nf or min(t.shape[2:]) < 7 or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous (nb, {nf}, X, Y) array of padded blocks")
        if U.shape[0] != aux.shape[0] or U.shape[2:] != aux.shape[2:]:
            raise ValueError("U and aux differ in their blocks")
        out = torch.empty_like(U)
        nb, _, X, Y = U.shape
        _native.check(self._lib.jb_amr_flux(self._h, nb, X - 6, Y - 6, float(dx), float(dy), _ptr(U), _ptr(aux),
                                            float(dt), _ptr(out), _stream()), self._h, "jb_amr_flux")
        return out

    def amr_update_aux(self, U, aux):
        """vmap(update_aux) (set_simulator.py:41): U [nb][nv][X][Y], aux
        [nb][2][X][Y]; each block's temperature solve stops on its own
        residuals."""
        for name, t, nf in (("U", U, self.nv), ("aux", aux, 2)):
            if not isinstance(t, torch.Tensor) or t.device.type != "cuda" or t.dtype != torch.float64:
                raise TypeError(f"{name} must be a float64 CUDA tensor")
            if t.ndim != 4 or t.shape[1] != nf or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous (nb, {nf}, X, Y) array of blocks")
        if U.shape[0] != aux.shape[0] or U.shape[2:] != aux.shape[2:]:
            raise ValueError("U and aux differ in their blocks")
        out = torch.empty_like(aux)
        nb, _, X, Y = U.shape
        _native.check(self._lib.jb_amr_update_aux(self._h, nb, X, Y, _ptr(U), _ptr(aux), _ptr(out), _stream()),
                      self._h, "jb_amr_update_aux")
        return out

    def amr_chem(self, blk, dt, out=None):
        """Chemistry and update_aux of unpadded AMR blocks [nb][nv+2][bx][by]
        (set_simulator.py:106-113), each block's temperature solve stopping
        on its own residuals."""
        self._check_blocks(blk, False, "blk")
        out = torch.empty_like(blk) if out is None else out
        nb, _, X, Y = blk.shape
        _native.check(self._lib.jb_amr_chem(self._h, nb, X, Y, _ptr(blk), float(dt), _ptr(out), _stream()),
                      self._h, "jb_amr_chem")
        return out

    def advance(self, U, aux, nsteps=1, dt=None, cfl=None, theta=None, dt_hist=None):
        """``nsteps`` fused steps; CFL time steps when ``cfl`` is given,
        otherwise the fixed ``dt``.  Returns (U, aux, dt_hist) with dt_hist a
        device tensor of the step sizes."""
        self._check_state(U, aux)
        self.set_theta(theta)
        if cfl is None and dt is None:
            raise ValueError("need dt or cfl")
        U_out = torch.empty_like(U)
        aux_out = torch.empty_like(aux)
        if dt_hist is None:
            dt_hist = torch.empty(nsteps, dtype=torch.float64, device=U.device)
        rc = self._lib.jb_advance(self._h, _ptr(U), _ptr(aux), _ptr(U_out), _ptr(aux_out),
                                  float(dt or 0.0), float(cfl or 0.0), int(nsteps), _ptr(dt_hist), _stream())
        self._check(rc, "jb_advance")
        return U_out, aux_out, dt_hist

    def advance_host(self, inputs, outputs, nsteps=1, dt=None, cfl=None, theta=None):
        """Advance host states through the device with the copies hidden
        behind the steps: ``inputs`` and ``outputs`` are equal-length lists of
        (U, aux) pinned CPU float64 tensors; item i is copied in on one
        stream, advanced ``nsteps`` on the current stream and copied out on a
        third, so the copy-in of item i+1 and the copy-out of item i-1 overlap
        the steps of item i (two device buffer sets).  Items are independent
        states (a parameter sweep, a queue of cases); a single time-stepping
        chain keeps its state on the device instead.  Returns when every
        result is in ``outputs``."""
        if cfl is None and dt is None:
            raise ValueError("need dt or cfl")
        if len(inputs) != len(outputs):
            raise ValueError("inputs and outputs differ in length")
        for hU, haux in list(inputs) + list(outputs):
            if hU.device.type != "cpu" or haux.device.type != "cpu" or not (hU.is_pinned() and haux.is_pinned()):
                raise ValueError("advance_host takes pinned CPU tensors")
            if tuple(hU.shape) != (self.nv,) + self.shape or tuple(haux.shape) != (2,) + self.shape:
                raise ValueError("state shape does not match the solver")
        self.set_theta(theta)
        dev = self.device
        buf = [[torch.empty((self.nv,) + self.shape, dtype=torch.float64, device=dev),
                torch.empty((2,) + self.shape, dtype=torch.float64, device=dev)] for _ in range(4)]
        din, dout = buf[:2], buf[2:]
        hist = torch.empty(max(nsteps, 1), dtype=torch.float64, device=dev)
        comp = torch.cuda.current_stream(dev)
        s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        ev = lambda: torch.cuda.Event()  # noqa: E731
        loaded, computed, drained = [ev(), ev()], [ev(), ev()], [ev(), ev()]
        started = ev()
        started.record(comp)
        s_in.wait_event(started)
        s_out.wait_event(started)
        for i, ((hU, haux), (oU, oaux)) in enumerate(zip(inputs, outputs)):
            b = i % 2
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(computed[b])  # the step that read din[b] is done
                din[b][0].copy_(hU, non_blocking=True)
                din[b][1].copy_(haux, non_blocking=True)
                loaded[b].record(s_in)
            comp.wait_event(loaded[b])
            if i >= 2:
                comp.wait_event(drained[b])  # dout[b] has been copied out
            rc = self._lib.jb_advance(self._h, _ptr(din[b][0]), _ptr(din[b][1]), _ptr(dout[b][0]),
                                      _ptr(dout[b][1]), float(dt or 0.0), float(cfl or 0.0), int(nsteps),
                                      _ptr(hist), ctypes.c_void_p(comp.cuda_stream))
            self._check(rc, "jb_advance")
            computed[b].record(comp)
            with torch.cuda.stream(s_out):
                s_out.wait_event(computed[b])
                oU.copy_(dout[b][0], non_blocking=True)
                oaux.copy_(dout[b][1], non_blocking=True)
                drained[b].record(s_out)
        comp.wait_stream(s_in)
        comp.wait_stream(s_out)
        for t in din + dout:
            for x in t:
                x.record_stream(s_in)
                x.record_stream(s_out)
        # the copies into ``outputs`` are asynchronous: wait for the last one
        # so the host can read every result when this returns
        s_out.synchronize()
        return outputs

    def advance_one_step(self, U, aux, dx=None, dy=None, dt=None, theta=None):
        """set_advance_func's advance_one_step(U, aux, dx, dy, dt, theta)."""
        self._spacing(dx, dy)
        U, aux, _ = self.advance(U, aux, 1, dt=dt, theta=theta)
        return U, aux

    def rk3(self, U, aux, dx=None, dy=None, dt=None, theta=None):
        """time_step_dict['TVD_RK3'] with this solver's flux_func/update_aux:
        the SSP-RK3 flux step without chemistry (TVD_RK3.py:5-12)."""
        self._check_state(U, aux)
        self._spacing(dx, dy)
        self.set_theta(theta)
        U_out = torch.empty_like(U)
        aux_out = torch.empty_like(aux)
        self._check(self._lib.jb_rk3(self._h, _ptr(U), _ptr(aux), _ptr(U_out), _ptr(aux_out), float(dt),
                                     _stream()), "jb_rk3")
        return U_out, aux_out

    def u_to_prim(self, U, aux):
        """aux_func.U_to_prim: (rho, u, [v,] Y, p, a) with the reference's shapes."""
        self._check_state(U, aux)
        sh = (1,) + self.shape
        rho, u, v, p, a = (torch.empty(sh, dtype=torch.float64, device=U.device) for _ in range(5))
        Y = torch.empty((8,) + self.shape, dtype=torch.float64, device=U.device)
        _native.check(self._lib.jb_u_to_prim(self._h, _ptr(U), _ptr(aux), _ptr(rho), _ptr(u), _ptr(v), _ptr(Y),
                                             _ptr(p), _ptr(a), _stream()), self._h, "jb_u_to_prim")
        if self.dim == 1:
            return rho, u, Y, p, a
        return rho, u, v, Y, p, a

    def cfl_dt(self, U, aux, cfl):
        self._check_state(U, aux)
        out = torch.empty((), dtype=torch.float64, device=U.device)
        self._check(self._lib.jb_cfl_dt(self._h, _ptr(U), _ptr(aux), float(cfl), _ptr(out), _stream()),
                    "jb_cfl_dt")
        return out

    def get_thermo(self, T, Y):
        """thermo_model.get_thermo(T, Y) -> (cp, gamma, h, R, dcp), each with
        T's shape; T is (1, ...) and Y (8, ...)."""
        T = T.contiguous()
        Y = Y.contiguous()
        n = T.numel()
        outs = [torch.empty_like(T) for _ in range(5)]
        _native.check(self._lib.jb_get_thermo(self._h, n, _ptr(T), _ptr(Y), *[_ptr(o) for o in outs], _stream()),
                      self._h, "jb_get_thermo")
        return tuple(outs)

    def state_from_PTY(self, P, T, Y, vel=None):
        """Conserved state from pressure, temperature and mass fractions as the
        reference's examples build it: rho = P/(R T), rho E = rho h - P
        (+ kinetic), aux = [gamma, T]."""
        _, gamma, h, R, _ = self.get_thermo(T, Y)
        rho = P / (R * T)
        E = rho * h - P
        nd = T.ndim - 1
        if vel is None:
            vel = [torch.zeros_like(T) for _ in range(nd)]
        for v in vel:
            E = E + 0.5 * rho * v ** 2
        U = torch.cat([rho] + [rho * v for v in vel] + [E, rho * Y], dim=0).contiguous()
        aux = torch.cat([gamma, T], dim=0).contiguous()
        return U, aux
