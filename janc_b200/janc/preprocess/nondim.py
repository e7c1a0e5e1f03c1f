"""Reference scales (src/janc_v2/preprocess/nondim.py): P0, T0, R0, x0 and
the derived rho0, M0, e0, u0, t0; all 1 (SI) until set_nondim is called."""
import math

from .. import _state

Rg = 8.314463
P0 = T0 = R0 = x0 = 1.0
rho0 = P0 / (R0 * T0)
M0 = Rg / R0
e0 = P0 / rho0
u0 = math.sqrt(P0 / rho0)
t0 = x0 / u0


def set_nondim(nondim_config):
    global P0, T0, R0, x0, rho0, M0, e0, u0, t0
    if nondim_config is not None:
        P0, T0, R0, x0 = (nondim_config[k] for k in ("P0", "T0", "R0", "x0"))
        rho0 = P0 / (R0 * T0)
        M0 = Rg / R0
        e0 = P0 / rho0
        u0 = math.sqrt(P0 / rho0)
        t0 = x0 / u0
        _state.config["nondim"] = dict(nondim_config)
