"""NASA7 mixture thermo (src/janc_v2/model/thermo_model.py) on the GPU."""
import os

import torch

from .. import _state
from ..preprocess import nondim as _nondim

max_iter = 5
tol = 5e-9


def set_thermo(thermo_config, nondim_config=None, dim="2D"):
    """thermo_model.py:42-77: validates like the reference; only 'nasa7'."""
    if thermo_config["thermo_model"] == "nasa7":
        assert "mechanism_directory" in thermo_config, \
            "Please specify 'mechanism_directory' in your dict of settings"
        _, ext = os.path.splitext(thermo_config["mechanism_directory"])
        assert ext.lower() == ".yaml", "janc only read mech file with .yaml format"
        if not os.path.isfile(thermo_config["mechanism_directory"]):
            raise FileNotFoundError("No mechanism file detected in the specified directory.")
    elif thermo_config["thermo_model"] == "constant_gamma":
        raise NotImplementedError("the constant_gamma model is not part of the detailed-chemistry path")
    else:
        raise KeyError("The thermo model you specified is not supported, only 'nasa7' or "
                       "'constant_gamma' can be specified.")
    _state.config["mechanism"] = thermo_config["mechanism_directory"]
    _state.config["dim"] = dim
    if nondim_config is not None:
        _nondim.set_nondim(nondim_config)
    _state.config["nondim"] = nondim_config


def fill_Y(Y):
    """thermo_model.py:80-82"""
    Y, kind = _state.to_device(Y)
    return _state.back(torch.cat([Y, 1.0 - Y.sum(0, keepdim=True)], 0), kind)


def get_R(Y):
    """thermo_model.py:87-92: R = sum_k Y_k / M_k"""
    Yd, kind = _state.to_device(Y)
    m = _state.mechanism()
    invM = torch.tensor(1 / m.tables["species_M"], device="cuda").reshape((-1,) + (1,) * (Yd.ndim - 1))
    Yf = torch.cat([Yd, 1.0 - Yd.sum(0, keepdim=True)], 0)
    return _state.back((invM * Yf).sum(0, keepdim=True), kind)


def get_thermo(T, Y):
    """thermo_model.py:115-126 -> (cp, gamma, h, R, dcp), kernel jb_get_thermo."""
    Td, kind = _state.to_device(T)
    Yd, _ = _state.to_device(Y)
    s = _state.solver_for((4,))  # get_thermo does not depend on the grid
    outs = s.get_thermo(Td, Yd)
    return tuple(_state.back(o, kind) for o in outs)


def get_thermo_properties(T):
    """thermo_model.py:107-112: per-species (cp_k, dcp_k, h_k), each of shape
    (9,) + T.shape, from the NASA7 kernel (jb_get_thermo) evaluated with
    one-hot mass fractions, whose mixture sums hold a single nonzero term."""
    Td, kind = _state.to_device(T)
    s = _state.solver_for((4,))
    T1 = Td.reshape(1, -1).contiguous()
    cps, dcps, hs = [], [], []
    for k in range(9):
        Y = torch.zeros((8, T1.shape[1]), dtype=torch.float64, device=T1.device)
        if k < 8:
            Y[k] = 1.0  # the ninth (N2) is the filled remainder of all-zero Y
        cp, _, h, _, dcp = s.get_thermo(T1, Y)
        cps.append(cp.reshape(Td.shape))
        dcps.append(dcp.reshape(Td.shape))
        hs.append(h.reshape(Td.shape))
    return tuple(_state.back(torch.stack(x), kind) for x in (cps, dcps, hs))


def get_T(e, Y, initial_T):
    """thermo_model.py:135-153 (Halley with the global stopping rule):
    returns concat([gamma, T]).  Runs the update_aux kernel on a unit-density
    state carrying the given specific internal energy."""
    ed, kind = _state.to_device(e)
    Yd, _ = _state.to_device(Y)
    Td, _ = _state.to_device(initial_T)
    n = ed.numel()
    U = torch.cat([torch.ones_like(ed).reshape(1, n), torch.zeros_like(ed).reshape(1, n),
                   ed.reshape(1, n), Yd.reshape(Yd.shape[0], n)], 0).contiguous()
    aux = torch.cat([torch.ones_like(Td).reshape(1, n), Td.reshape(1, n)], 0).contiguous()
    if n < 4:
        raise ValueError("get_T needs at least 4 points")
    s = _state.solver_for((n,))
    out = s.update_aux(U, aux)
    return _state.back(out.reshape((2,) + tuple(ed.shape[1:])), kind)
