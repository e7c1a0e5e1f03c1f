"""Solver wiring and the time loop (src/janc_v2/simulation/set_simulator.py):
``set_rhs``, ``set_advance_func`` and ``Simulator`` with the reference's
configuration dictionary.  One ``advance_func`` call is one fused native
step (``jb_advance``): CFL dt, SSP-RK3 flux stages with update_aux,
point-implicit chemistry and the final update_aux."""
from .. import _state
from ..boundary import boundary
from ..model import reaction_model, thermo_model
from ..solver_1D import aux_func as aux_func_1D
from ..solver_1D import flux as flux_1D
from ..solver_2D import aux_func
from ..solver_2D import flux
from .time_step import time_step_dict


def set_rhs(dim, reaction_config, source_config=None, is_parallel=False, is_amr=False):
    """(flux_func, update_func, source_func) as set_simulator.py:20-71.
    ``is_parallel``: the arrays are this rank's x slab (one process per GPU
    in an initialised torch.distributed group); ghost columns come from the
    neighbouring slabs (parallel/boundary.py)."""
    if is_amr:
        return _set_rhs_amr(dim, reaction_config, source_config)
    if is_parallel and _state.config["slab"] is None:
        from ...slab import Slab
        _state.config["slab"] = Slab()
    elif not is_parallel:
        _state.config["slab"] = None
    if not reaction_config["is_detailed_chemistry"]:
        raise NotImplementedError("non-detailed chemistry (an N2-only state) is outside the 9-species path")

    def flux_func(U, aux, dx, dy, dt, theta):
        Ud, kind = _state.to_device(U)
        auxd, _ = _state.to_device(aux)
        s = _state.solver_for(tuple(Ud.shape[1:]), dx, dy if dim == "2D" else None)
        return _state.back(s.flux_func(Ud, auxd, dx, dy if dim == "2D" else None, float(dt), theta), kind)

    flux_func._janc_b200_flux = True
    update_func = aux_func_1D.update_aux if dim == "1D" else aux_func.update_aux
    update_func._janc_b200_update = True
    # detailed chemistry: a user source is added to the flux (set_simulator.py:50-54)
    source_func = source_config["self_defined_source_terms"] if source_config is not None else None
    return flux_func, update_func, source_func


def set_advance_func(dim, flux_config, reaction_config, time_control, is_amr, flux_func, update_func,
                     source_func):
    """advance_one_step(U, aux, dx, dy, dt, theta) as set_simulator.py:73-125
    (Lie splitting: time-stepped flux, chemistry, update_aux).  TVD_RK3
    without a user source is one fused native call; RK2 or a user source is
    composed as the reference composes it, from the native flux_func,
    update_aux and reaction_source_terms and the user's callable."""
    if is_amr:
        return _set_advance_func_amr(flux_config, reaction_config, time_control, flux_func, update_func,
                                     source_func)
    scheme = time_control["temporal_evolution_scheme"]
    if scheme not in time_step_dict:
        raise KeyError(scheme)
    step = time_step_dict[scheme]
    if source_func is not None or scheme != "TVD_RK3" or not reaction_config["is_detailed_chemistry"]:
        if source_func is None:
            def advance_flux(U, aux, dx, dy, dt, theta=None):
                return step(U, aux, dx, dy, dt, theta, flux_func, update_func)
        elif flux_config["solver_type"] == "flux_splitting":
            def rhs_func(U, aux, dx, dy, dt, theta=None):
                return flux_func(U, aux, dx, dy, dt, theta) + source_func(U, aux, dt, theta)

            def advance_flux(U, aux, dx, dy, dt, theta=None):
                return step(U, aux, dx, dy, dt, theta, rhs_func, update_func)
        else:  # godunov: the source as a second time-stepped pass
            def wrapped_source_func(U, aux, dx, dy, dt, theta=None):
                return source_func(U, aux, dt, theta)

            def advance_flux(U, aux, dx, dy, dt, theta=None):
                U_adv, aux_adv = step(U, aux, dx, dy, dt, theta, flux_func, update_func)
                return step(U_adv, aux_adv, dx, dy, dt, theta, wrapped_source_func, update_func)
        if not reaction_config["is_detailed_chemistry"]:
            return advance_flux

        def advance_composed(U, aux, dx, dy, dt, theta=None):
            U, aux = advance_flux(U, aux, dx, dy, dt, theta)
            dU = reaction_model.reaction_source_terms(U, aux, dt, theta)
            U = U + dU
            aux = update_func(U, aux)
            return U, aux
        advance_composed._janc_b200_composed = True
        return advance_composed

    def advance_one_step(U, aux, dx, dy, dt, theta=None):
        Ud, kind = _state.to_device(U)
        auxd, _ = _state.to_device(aux)
        s = _state.solver_for(tuple(Ud.shape[1:]), dx, dy if dim == "2D" else None)
        U1, aux1 = s.advance_one_step(Ud, auxd, dx, dy if dim == "2D" else None, float(dt), theta)
        return _state.back(U1, kind), _state.back(aux1, kind)
    return advance_one_step


def _set_rhs_amr(dim, reaction_config, source_config):
    """set_rhs(is_amr=True) (set_simulator.py:37-42, 64-70): the block flux
    function pad(dt * total_flux(U, aux), 3) and update_aux of ghost-padded
    blocks [nb][nv][bx+6][by+6], every reduction per block (vmapped in the
    reference), as native calls.  Flux splitting with LF only (the kernels'
    scheme), detailed chemistry, no user source: the reference adds the
    interior-shaped AMR source to the padded flux, which cannot broadcast."""
    if dim != "2D":
        raise NotImplementedError("block AMR is 2D (AMR_Simulator fixes dim = '2D')")
    fc = _state.config["flux"]
    if (fc.get("solver_type") != "flux_splitting" or fc.get("split_method", "LF") != "LF"
            or fc.get("viscosity", "off") == "on"):
        raise NotImplementedError("block AMR runs flux splitting with LF (WENO5-JS or MUSCL) without viscosity")
    if not reaction_config["is_detailed_chemistry"]:
        raise NotImplementedError("non-detailed chemistry (an N2-only state) is outside the 9-species path")
    if source_config is not None:
        raise NotImplementedError("a user source with AMR: the reference adds an interior-shaped source to the "
                                  "padded block flux (set_simulator.py:66-70), which cannot broadcast")

    def flux_func(U, aux, dx, dy, dt, theta):
        Ud, kind = _state.to_device(U)
        auxd, _ = _state.to_device(aux)
        return _state.back(_state.solver_for_amr().amr_flux(Ud, auxd, dx, dy, float(dt)), kind)

    def update_func(U, aux):
        Ud, kind = _state.to_device(U)
        auxd, _ = _state.to_device(aux)
        return _state.back(_state.solver_for_amr().amr_update_aux(Ud, auxd), kind)

    flux_func._janc_b200_amr_flux = True
    update_func._janc_b200_amr_update = True
    return flux_func, update_func, None


def _set_advance_func_amr(flux_config, reaction_config, time_control, flux_func, update_func, source_func):
    """set_advance_func(is_amr=True) (set_simulator.py:73-110): the time
    scheme's AMR form on the blocks, then the blocks' chemistry and
    update_aux (one native call, ``jb_amr_chem``)."""
    scheme = time_control["temporal_evolution_scheme"] + "_amr"
    if scheme not in time_step_dict:
        raise KeyError(scheme)
    step = time_step_dict[scheme]
    if source_func is not None:
        raise NotImplementedError("a user source with AMR (see set_rhs)")

    def advance_flux(level, blk_data, dx, dy, dt, ref_blk_data, ref_blk_info, theta=None):
        return step(level, blk_data, dx, dy, dt, ref_blk_data, ref_blk_info, theta, flux_func, update_func)
    if not reaction_config["is_detailed_chemistry"]:
        return advance_flux

    def advance_one_step(level, blk_data, dx, dy, dt, ref_blk_data, ref_blk_info, theta=None):
        blk = advance_flux(level, blk_data, dx, dy, dt, ref_blk_data, ref_blk_info, theta=None)
        blkd, kind = _state.to_device(blk)
        return _state.back(_state.solver_for_amr().amr_chem(blkd, float(dt)), kind)
    return advance_one_step


def AMR_Simulator(simulation_config):  # noqa: N802 (the reference's name)
    """(advance_func_amr, advance_func_base) as set_simulator.py:496-532:
    ``advance_func_amr(level, blk_data, dx, dy, dt, ref_blk_data,
    ref_blk_info, theta=None)`` advances one refinement level's blocks
    (``blk_data``: the coarser level's blocks, ``ref_blk_data``: this
    level's; the ghost layers come from the block layer, see
    ``time_step.set_amr_module``); ``advance_func_base(blk_data, dx, dy, dt,
    theta=None)`` advances the level-0 array [1][nv+2][nx][ny] with the
    boundary conditions of ``boundary_config``."""
    import torch
    dim = "2D"
    thermo_config = simulation_config["thermo_config"]
    reaction_config = simulation_config["reaction_config"]
    transport_config = simulation_config.get("transport_config", None)
    flux_config = simulation_config["flux_config"]
    boundary_config = simulation_config["boundary_config"]
    source_config = simulation_config.get("source_config", None)
    nondim_config = simulation_config.get("nondim_config", None)
    time_control = simulation_config["time_config"]
    _state.reset_solvers()
    _state.config["slab"] = None
    _state.config["precision"] = simulation_config.get("precision", "fp64")
    thermo_model.set_thermo(thermo_config, nondim_config, dim)
    reaction_model.set_reaction(reaction_config, nondim_config, dim)
    flux.set_flux_solver(flux_config, transport_config, nondim_config)
    boundary.set_boundary(boundary_config, dim)
    ff, uf, sf = set_rhs(dim, reaction_config, source_config, False, True)
    advance_func_amr = set_advance_func(dim, flux_config, reaction_config, time_control, True, ff, uf, sf)
    ff, uf, sf = set_rhs(dim, reaction_config, source_config, False, False)
    advance_func_body = set_advance_func(dim, flux_config, reaction_config, time_control, False, ff, uf, sf)

    def advance_func_base(blk_data, dx, dy, dt, theta=None):
        b, kind = _state.to_device(blk_data)
        U, aux = b[0, :-2].contiguous(), b[0, -2:].contiguous()
        U, aux = advance_func_body(U, aux, dx, dy, dt, theta)
        return _state.back(torch.cat([U, aux], dim=0)[None], kind)
    return advance_func_amr, advance_func_base


def _h5_module():
    """h5py when importable, else the built-in HDF5 subset (janc_b200.h5lite)."""
    try:
        import h5py
        return h5py
    except ImportError:
        from ... import h5lite
        return h5lite


class H5Saver:
    """Snapshot file in the reference's layout (set_simulator.py:126-318):
    one group ``save_step{k}`` per snapshot with attributes ``time`` and
    ``step`` and a dataset per saved array (``u``: the conserved state,
    gzip-compressed).  ``parallel_save`` writes ``save_step{k}_device{d}``
    groups, one per x slab, and ``collect`` concatenates them into
    ``save_step{k}``.  Fixed from the reference: ``collect`` has its
    defaultdict, ``get_prim`` uses the 2D aux functions, ``parallel_save``
    gathers the slabs to rank 0, the only process that opens the file (no
    I/O inside a mapped function), and a saved ``aux`` (the temperature and
    gamma of the state) is used by ``load`` instead of the reference's
    gamma = 1.4, T = 500 K initial guesses."""

    def __init__(self, filepath, data_dim, slab=None, mode="a"):
        from pathlib import Path
        self.filepath = Path(filepath)
        self.dim = data_dim
        self.slab = slab
        self._h5 = _h5_module()
        self.file = self._h5.File(self.filepath, mode) if (self._writer or mode == "r") else None

    @property
    def _writer(self):
        return self.slab is None or self.slab.rank == 0

    def get_prim(self, U, aux):
        """(density, x-velocity[, y-velocity], pressure, tempreature,
        species) of a state, as the reference names them."""
        if self.dim == "1D":
            aux = aux_func_1D.update_aux(U, aux)
            rho, u, Y, p, a = aux_func_1D.U_to_prim(U, aux)
            return {"density": rho[0], "x-velocity": u[0], "pressure": p[0], "tempreature": aux[1], "species": Y}
        aux = aux_func.update_aux(U, aux)
        rho, u, v, Y, p, a = aux_func.U_to_prim(U, aux)
        return {"density": rho[0], "x-velocity": u[0], "y-velocity": v[0], "pressure": p[0],
                "tempreature": aux[1], "species": Y}

    @staticmethod
    def _host(a):
        import numpy as np
        if hasattr(a, "detach"):
            a = a.detach().cpu().numpy()
        return np.asarray(a)

    def _write(self, key, t, step, arrays):
        import numpy as np
        if key in self.file:
            del self.file[key]
        grp = self.file.create_group(key)
        grp.attrs["time"] = np.float64(float(t))
        grp.attrs["step"] = np.int64(int(step))
        for name, arr in arrays.items():
            grp.create_dataset(name, data=self._host(arr), compression="gzip")
        self.file.flush()

    def save(self, save_step, t, step, **arrays):
        """One snapshot group ``save_step{save_step}`` (replaced if present)."""
        if self._writer:
            self._write(f"save_step{save_step}", t, step, arrays)

    def parallel_save(self, save_step, t, step, **arrays):
        """Each rank's slab as ``save_step{k}_device{rank}``, written by rank 0
        (every rank must call it)."""
        if self.slab is None:
            self._write(f"save_step{save_step}_device0", t, step, arrays)
            return
        from ...slab import gather_grid
        import torch
        full = {n: gather_grid(torch.as_tensor(a).to(dtype=torch.float64).contiguous(), self.slab)
                for n, a in arrays.items()}
        if not self._writer:
            return
        for d in range(self.slab.size):
            part = {n: torch.chunk(a, self.slab.size, dim=1)[d] for n, a in full.items()}
            self._write(f"save_step{save_step}_device{d}", t, step, part)

    def list_snapshots(self):
        return list(self.file.keys())

    def collect(self, concat_axis=1):
        """Concatenate the ``_device{d}`` groups of every snapshot into
        ``save_step{k}`` (attributes from the last device)."""
        import numpy as np
        from collections import defaultdict
        groups = defaultdict(list)
        for g in list(self.file.keys()):
            if g.startswith("save_step") and "_device" in g:
                groups[g.split("_device")[0]].append(g)
        for step, names in groups.items():
            names.sort(key=lambda x: int(x.split("_device")[-1]))
            data, attrs = {}, {}
            for g in names:
                grp = self.file[g]
                attrs = dict(grp.attrs)
                for k in grp.keys():
                    data.setdefault(k, []).append(np.asarray(grp[k]))
            if step in self.file:
                del self.file[step]
            new = self.file.create_group(step)
            for k, v in attrs.items():
                new.attrs[k] = v
            for k, parts in data.items():
                new.create_dataset(k, data=np.concatenate(parts, axis=concat_axis), compression="gzip")
        self.file.flush()

    def _state_of(self, grp):
        import numpy as np
        U = np.asarray(grp["u"])
        if "aux" in grp:
            aux = np.asarray(grp["aux"])
        else:  # the reference's initial guesses for the temperature solve
            aux = np.concatenate([np.full_like(U[0:1], 1.4), np.full_like(U[0:1], 500.0)], axis=0)
        return U, aux

    def load(self, key):
        """(time, primitive dict) of snapshot ``key``."""
        grp = self.file[key]
        U, aux = self._state_of(grp)
        return grp.attrs["time"], self.get_prim(U, aux)

    def load_state(self, key=None):
        """(U, aux, time, step) of snapshot ``key`` (default: the latest
        ``save_step{k}``) for a restart.  A snapshot without ``aux`` (written
        by the reference, which saves ``u`` only) gets its (gamma, T) from
        the temperature solve started at the reference's gamma = 1.4,
        T = 500 K guesses, as its ``load`` does."""
        if key is None:
            keys = [k for k in self.file.keys() if k.startswith("save_step") and "_device" not in k]
            key = max(keys, key=lambda k: int(k[len("save_step"):]))
        grp = self.file[key]
        U, aux = self._state_of(grp)
        if "aux" not in grp:
            aux = (aux_func_1D if self.dim == "1D" else aux_func).update_aux(U, aux)
        return U, aux, float(grp.attrs["time"]), int(grp.attrs["step"])

    def load_all(self):
        """(times, primitive dict with a leading snapshot axis) over all
        snapshots in step order."""
        import numpy as np
        keys = sorted(self.file.keys(), key=lambda s: int("".join(ch for ch in s if ch.isdigit())))
        times, prims = [], []
        for k in keys:
            t, q = self.load(k)
            times.append(t)
            prims.append({n: self._host(v) for n, v in q.items()})
        return np.stack(times), {n: np.stack([q[n] for q in prims]) for n in prims[0]}

    def close(self):
        if self.file is not None:
            self.file.close()
            self.file = None


class Simulator:
    """Simulator(simulation_config) with advance_func(U, aux, t, theta) ->
    (U, aux, t + dt, dt) and run(U_init, aux_init) (set_simulator.py:320-494).
    ``computation_config['output_settings']`` (``save_dt``, ``results_path``)
    sets the snapshots run() writes with H5Saver (default: the initial and
    final states in results.h5); the file is opened when run() starts.
    ``computation_config['is_parallel']`` decomposes x into one slab per rank
    of the initialised torch.distributed group (one process per GPU);
    advance_func then takes and returns this rank's slab."""

    def __init__(self, simulation_config):
        dim = simulation_config["dimension"]
        grid_config = simulation_config["grid_config"]
        thermo_config = simulation_config["thermo_config"]
        reaction_config = simulation_config["reaction_config"]
        flux_config = simulation_config["flux_config"]
        boundary_config = simulation_config["boundary_config"]
        nondim_config = simulation_config.get("nondim_config", None)
        time_control = simulation_config["time_config"]
        self.t_end = time_control["t_end"]
        self.theta = simulation_config.get("solver_parameters", None)
        comp = simulation_config.get("computation_config", {})
        self.is_parallel = bool(comp.get("is_parallel", False))
        out = comp.get("output_settings", {})
        self.save_dt = out.get("save_dt", self.t_end)
        self.results_path = out.get("results_path", "results.h5")
        _state.reset_solvers()
        _state.config["slab"] = None
        _state.config["precision"] = simulation_config.get("precision", "fp64")
        thermo_model.set_thermo(thermo_config, nondim_config, dim)
        reaction_model.set_reaction(reaction_config, nondim_config, dim)
        (flux_1D if dim == "1D" else flux).set_flux_solver(
            flux_config, simulation_config.get("transport_config", None), nondim_config)
        boundary.set_boundary(boundary_config, dim)
        if time_control["temporal_evolution_scheme"] not in time_step_dict:
            raise KeyError(time_control["temporal_evolution_scheme"])
        self.dim = dim
        self.dx = grid_config["dx"]
        self.dy = grid_config.get("dy") if dim == "2D" else None
        source_config = simulation_config.get("source_config", None)
        self.flux_func, self.update_func, self.source_func = set_rhs(dim, reaction_config, source_config,
                                                                     self.is_parallel)
        self.slab = _state.config["slab"]
        self._advance_body = set_advance_func(dim, flux_config, reaction_config, time_control, False,
                                              self.flux_func, self.update_func, self.source_func)
        self._composed = getattr(self._advance_body, "_janc_b200_composed", False)
        self.dt = time_control.get("dt", None)
        self.CFL = time_control.get("CFL", None)
        if self.dt is None and self.CFL is None:
            raise KeyError("time_config needs 'dt' or 'CFL'")

    def advance_func(self, U, aux, t, theta=None):
        Ud, kind = _state.to_device(U)
        auxd, _ = _state.to_device(aux)
        s = _state.solver_for(tuple(Ud.shape[1:]), self.dx, self.dy)
        if self._composed:  # RK2 or a user source: CFL dt, then the composed step
            dt = s.cfl_dt(Ud, auxd, self.CFL) if self.CFL is not None else self.dt
            if kind == "numpy":
                dt = float(dt)
            U1, aux1 = self._advance_body(U, aux, self.dx, self.dy, dt, theta)
            return U1, aux1, t + dt, dt
        if self.CFL is not None:
            U1, aux1, dts = s.advance(Ud, auxd, 1, cfl=self.CFL, theta=theta)
            dt = dts[0]
        else:
            U1, aux1, _ = s.advance(Ud, auxd, 1, dt=self.dt, theta=theta)
            dt = self.dt
        if kind == "numpy":
            dt = float(dt)
        return _state.back(U1, kind), _state.back(aux1, kind), t + dt, dt

    def run(self, U_init, aux_init, t0=0.0, step0=0, save=True):
        """Advance to t_end, writing a snapshot (u and aux) at the start and
        whenever t passes the next multiple of save_dt (set_simulator.py:
        457-494).  ``t0``/``step0`` restart from a saved state (the reference
        always starts at t = 0; see ``restart``).  In the is_parallel mode the
        global initial arrays are split into this rank's x slab first, the
        snapshots hold one group per slab, and the slab is returned (the
        reference returns its device-sharded arrays)."""
        U, aux, t, step = U_init, aux_init, float(t0), int(step0)
        if self.is_parallel:
            from ...slab import split_and_distribute_grid
            U = split_and_distribute_grid(U, self.slab)
            aux = split_and_distribute_grid(aux, self.slab)
        saver = H5Saver(self.results_path, self.dim, self.slab) if save else None
        put = (lambda *a, **k: None) if saver is None else (saver.parallel_save if self.is_parallel else saver.save)
        save_step = 0
        if step == 0:
            put(0, t, step, u=U, aux=aux)
            save_step = 1
        else:
            save_step = 1 + int(t // self.save_dt)
        next_save = save_step * self.save_dt if step else self.save_dt
        try:
            while t < self.t_end:
                U, aux, t, dt = self.advance_func(U, aux, t, self.theta)
                t = float(t)
                step += 1
                if t >= next_save or t >= self.t_end:
                    put(save_step, t, step, u=U, aux=aux)
                    next_save += self.save_dt
                    save_step += 1
        finally:
            if saver is not None:
                saver.close()
        return U, aux, t

    def restart(self, key=None):
        """(U, aux, t, step) of a snapshot in results_path (default: the
        latest) for ``run(U, aux, t0=t, step0=step)``; a parallel file is
        collected first."""
        if self.slab is None or self.slab.rank == 0:
            saver = H5Saver(self.results_path, self.dim)
            try:
                if any("_device" in k for k in saver.list_snapshots()):
                    saver.collect()
            finally:
                saver.close()
        if self.slab is not None:
            import torch.distributed as dist
            dist.barrier(group=self.slab.group)
        saver = H5Saver(self.results_path, self.dim, mode="r")
        try:
            return saver.load_state(key)
        finally:
            saver.close()
