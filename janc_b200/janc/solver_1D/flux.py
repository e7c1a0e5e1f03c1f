"""Advective flux selection (src/janc_v2/solver_1D/flux.py set_flux_solver)."""
from .. import _state


def set_flux_solver(flux_solver_config, transport_config=None, nondim_config=None):
    """Validate as set_flux_solver does and keep the configuration for the
    native solvers: LF or Steger-Warming flux splitting, or Godunov (HLLC /
    AUSMPW+), with WENO5_JS or MUSCL, optionally with the viscous fluxes of
    transport_config (laminar or LES)."""
    from ...solver import flux_scheme, transport_params
    flux_scheme(flux_solver_config)
    if flux_solver_config.get("viscosity", "off") == "on":
        transport_params(transport_config)
    _state.config["flux"] = dict(flux_solver_config)
    _state.config["transport"] = dict(transport_config) if transport_config else None


def total_flux(U, aux, dx):
    """total_flux (solver_1D/flux.py:107-108) of ghost-padded arrays
    (nv, nx+6), (2, nx+6): -dF/dx (+ the viscous part when 'viscosity' is
    on), with the configured flux and the arrays' ghost cells."""
    Ud, kind = _state.to_device(U)
    ad, _ = _state.to_device(aux)
    s, Ui, ai = _state.solver_for_padded(Ud, ad, dx)
    return _state.back(s.flux_func(Ui, ai, dx, None, 1.0), kind)
