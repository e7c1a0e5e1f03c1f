"""Point-implicit detailed chemistry (src/janc_v2/model/reaction_model.py)."""
import os

from .. import _state


def set_reaction(reaction_config, nondim_config=None, dim="2D"):
    """reaction_model.py:37-75: validates like the reference."""
    if reaction_config["is_detailed_chemistry"]:
        assert "mechanism_directory" in reaction_config, \
            "You choosed detailed chemistry without specifying the directory of your mechanism files"
        _, ext = os.path.splitext(reaction_config["mechanism_directory"])
        assert ext.lower() == ".yaml", "janc only read mech file with .yaml format"
        if not os.path.isfile(reaction_config["mechanism_directory"]):
            raise FileNotFoundError("No mechanism file detected in the specified directory.")
        _state.config["mechanism"] = reaction_config["mechanism_directory"]
    else:
        raise NotImplementedError("user-defined reaction sources are outside the detailed-chemistry path")
    _state.config["detailed_chemistry"] = True
    _state.config["dim"] = dim
    if nondim_config is not None:
        _state.config["nondim"] = nondim_config


def reaction_source_terms(U, aux, dt, theta=None):
    """reaction_model.py:202-203 -> detailed_reaction (:183-193)."""
    Ud, kind = _state.to_device(U)
    auxd, _ = _state.to_device(aux)
    s = _state.solver_for(tuple(Ud.shape[1:]))
    return _state.back(s.reaction_source_terms(Ud, auxd, float(dt)), kind)
