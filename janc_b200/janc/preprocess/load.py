"""Mechanism tables (src/janc_v2/preprocess/load.py:8-135) without Cantera."""
from ... import mechanism as _mech


def _expand(a, dim):
    extra = {"1D": 1, "2D": 2, "3D": 3}[dim]
    return a.reshape(a.shape + (1,) * extra)


def read_reaction_mechanism(file_path, nondim_config=None, dim="2D"):
    """ReactionParams dict of the reference (load.py:8-88)."""
    m = _mech.load(file_path, nondim_config)
    t = m.tables
    return {
        "species": list(m.species),
        "vf": _expand(t["vf"], dim), "vb": _expand(t["vb"], dim),
        "A": t["A"], "B": t["B"], "Ea/Ru": t["EaR"],
        "third_body_coeffs": _expand(t["third_body"], dim),
        "is_third_body": t["is_third_body"],
        "num_of_reactions": t["vf"].shape[0], "num_of_species": m.ns,
        "num_of_inert_species": m.ns - t["vf"].shape[1],
        "vsum": t["vsum"],
    }


def get_cantera_coeffs(species_list, mech=_mech.DEFAULT_MECHANISM, nondim_config=None, dim="2D"):
    """(species_M, Mex, Tcr, cp/dcp/h/h_chem/s low/high, logcof low/high)
    of the reference (load.py:91-135), for species in ``species_list``."""
    m = _mech.load(mech, nondim_config)
    idx = [m.species.index(s) for s in species_list]
    t = m.tables
    pick = lambda k: t[k][idx]  # noqa: E731
    species_M = pick("species_M")
    return (species_M, _expand(species_M, dim), pick("Tcr"), pick("cp_cof_low"), pick("cp_cof_high"),
            pick("dcp_cof_low"), pick("dcp_cof_high"), pick("h_cof_low"), pick("h_cof_high"),
            pick("h_cof_low_chem"), pick("h_cof_high_chem"), pick("s_cof_low"), pick("s_cof_high"),
            pick("logcof_low"), pick("logcof_high"))
