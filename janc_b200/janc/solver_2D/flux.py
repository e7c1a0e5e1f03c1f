"""Advective flux selection (src/janc_v2/solver_2D/flux.py set_flux_solver)."""
from .. import _state


def set_flux_solver(flux_solver_config, transport_config=None, nondim_config=None):
    solver_type = flux_solver_config["solver_type"]
    if solver_type == "godunov":
        raise NotImplementedError("the Godunov (HLLC/AUSMPW+) path is not built; use 'flux_splitting'")
    elif solver_type != "flux_splitting":
        raise KeyError("JANC only support 'godunov' and 'flux_splitting'")
    if flux_solver_config["interface_reconstruction"] != "WENO5_JS":
        raise KeyError("only 'WENO5_JS' reconstruction is built")
    if flux_solver_config["split_method"] != "LF":
        raise KeyError("only the 'LF' flux splitting is built")
    if flux_solver_config.get("viscosity", "off") == "on":
        raise NotImplementedError("viscous fluxes are not built")
    _state.config["flux"] = dict(flux_solver_config)
