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
        raise NotImplementedError("AMR is not part of this build")
    if is_parallel and _state.config["slab"] is None:
        from ...slab import Slab
        _state.config["slab"] = Slab()
    elif not is_parallel:
        _state.config["slab"] = None
    if source_config is not None:
        raise NotImplementedError("user source terms are outside the detailed-chemistry path")

    def flux_func(U, aux, dx, dy, dt, theta):
        Ud, kind = _state.to_device(U)
        auxd, _ = _state.to_device(aux)
        s = _state.solver_for(tuple(Ud.shape[1:]), dx, dy if dim == "2D" else None)
        return _state.back(s.flux_func(Ud, auxd, dx, dy if dim == "2D" else None, float(dt), theta), kind)

    flux_func._janc_b200_flux = True
    update_func = aux_func_1D.update_aux if dim == "1D" else aux_func.update_aux
    update_func._janc_b200_update = True
    source_func = None
    return flux_func, update_func, source_func


def set_advance_func(dim, flux_config, reaction_config, time_control, is_amr, flux_func, update_func,
                     source_func):
    """advance_one_step(U, aux, dx, dy, dt, theta) as set_simulator.py:73-125
    (Lie splitting: RK3 flux, chemistry, update_aux) -- one fused call."""
    if is_amr:
        raise NotImplementedError("AMR is not part of this build")
    if not reaction_config["is_detailed_chemistry"]:
        def advance_flux(U, aux, dx, dy, dt, theta=None):
            return time_step_dict[time_control["temporal_evolution_scheme"]](
                U, aux, dx, dy, dt, theta, flux_func, update_func)
        return advance_flux

    def advance_one_step(U, aux, dx, dy, dt, theta=None):
        Ud, kind = _state.to_device(U)
        auxd, _ = _state.to_device(aux)
        s = _state.solver_for(tuple(Ud.shape[1:]), dx, dy if dim == "2D" else None)
        U1, aux1 = s.advance_one_step(Ud, auxd, dx, dy if dim == "2D" else None, float(dt), theta)
        return _state.back(U1, kind), _state.back(aux1, kind)
    return advance_one_step


class Simulator:
    """Simulator(simulation_config) with advance_func(U, aux, t, theta) ->
    (U, aux, t + dt, dt) and run(U_init, aux_init) (set_simulator.py:320-494).
    Snapshot output (H5Saver) is not part of this build; run() returns the
    final state.  ``computation_config['is_parallel']`` decomposes x into one
    slab per rank of the initialised torch.distributed group (one process per
    GPU); advance_func then takes and returns this rank's slab."""

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
        _state.reset_solvers()
        _state.config["slab"] = None
        _state.config["precision"] = simulation_config.get("precision", "fp64")
        thermo_model.set_thermo(thermo_config, nondim_config, dim)
        reaction_model.set_reaction(reaction_config, nondim_config, dim)
        (flux_1D if dim == "1D" else flux).set_flux_solver(
            flux_config, simulation_config.get("transport_config", None), nondim_config)
        boundary.set_boundary(boundary_config, dim)
        if time_control["temporal_evolution_scheme"] != "TVD_RK3":
            raise KeyError("only 'TVD_RK3' time stepping is built")
        self.dim = dim
        self.dx = grid_config["dx"]
        self.dy = grid_config.get("dy") if dim == "2D" else None
        self.flux_func, self.update_func, _ = set_rhs(dim, reaction_config, None, self.is_parallel)
        self.slab = _state.config["slab"]
        self._advance_body = set_advance_func(dim, flux_config, reaction_config, time_control, False,
                                              self.flux_func, self.update_func, None)
        self.dt = time_control.get("dt", None)
        self.CFL = time_control.get("CFL", None)
        if self.dt is None and self.CFL is None:
            raise KeyError("time_config needs 'dt' or 'CFL'")

    def advance_func(self, U, aux, t, theta=None):
        Ud, kind = _state.to_device(U)
        auxd, _ = _state.to_device(aux)
        s = _state.solver_for(tuple(Ud.shape[1:]), self.dx, self.dy)
        if self.CFL is not None:
            U1, aux1, dts = s.advance(Ud, auxd, 1, cfl=self.CFL, theta=theta)
            dt = dts[0]
        else:
            U1, aux1, _ = s.advance(Ud, auxd, 1, dt=self.dt, theta=theta)
            dt = self.dt
        if kind == "numpy":
            dt = float(dt)
        return _state.back(U1, kind), _state.back(aux1, kind), t + dt, dt

    def run(self, U_init, aux_init):
        """Advance to t_end.  In the is_parallel mode the global initial
        arrays are split into this rank's x slab first and the slab is
        returned (the reference returns its device-sharded arrays)."""
        U, aux, t = U_init, aux_init, 0.0
        if self.is_parallel:
            from ...slab import split_and_distribute_grid
            U = split_and_distribute_grid(U, self.slab)
            aux = split_and_distribute_grid(aux, self.slab)
        while t < self.t_end:
            U, aux, t, dt = self.advance_func(U, aux, t, self.theta)
            t = float(t)
        return U, aux, t
