"""Advective flux selection (src/janc_v2/solver_2D/flux.py set_flux_solver)."""
from .. import _state


def set_flux_solver(flux_solver_config, transport_config=None, nondim_config=None):
    """Validate as set_flux_solver does and keep the configuration for the
    native solvers: LF flux splitting or Godunov (HLLC / AUSMPW+), WENO5_JS,
    optionally with the laminar viscous fluxes of transport_config."""
    from ...solver import flux_scheme, transport_params
    flux_scheme(flux_solver_config)
    if flux_solver_config.get("viscosity", "off") == "on":
        transport_params(transport_config)
    _state.config["flux"] = dict(flux_solver_config)
    _state.config["transport"] = dict(transport_config) if transport_config else None
