"""PyYAML-backed stand-in for the slice of Cantera's Python API that JANC's
``janc_v2/preprocess/load.py`` reads (Cantera is not installed here).

Test infrastructure only.  It restates the Cantera 3.x conventions the loader
depends on:

* ``Solution.species_names`` follows the phase's ``species:`` list order.
* ``reactant_stoich_coeffs`` / ``product_stoich_coeffs``: dense
  (n_species, n_reactions) float arrays; the third-body ``M`` is not a species.
* ``reaction.rate.pre_exponential_factor`` is in SI with kmol:
  A_yaml * (1e-3)**(order-1) for a mechanism in cm/mol units, where
  ``order`` counts the third body for three-body reactions.
* ``reaction.rate.activation_energy`` is in J/kmol: Ea[cal/mol] * 4184.
* ``reaction.reaction_type`` is ``'three-body-Arrhenius'`` or ``'Arrhenius'``;
  ``reaction.third_body.efficiencies`` holds only the listed efficiencies.
* ``species(name).thermo.coeffs`` is ``[Tmid, high[7], low[7]]`` (NASA7).
* ``species(name).molecular_weight`` sums IUPAC conventional atomic weights
  (H 1.008, N 14.007, O 15.999, He 4.002602, Ar 39.95, C 12.011).
"""
import re

import numpy as np
import yaml

_ATOMIC_WEIGHT = {"H": 1.008, "He": 4.002602, "C": 12.011, "N": 14.007,
                  "O": 15.999, "Ar": 39.95}

_ENERGY_TO_J_PER_KMOL = {"cal/mol": 4184.0, "kcal/mol": 4184000.0,
                         "J/mol": 1000.0, "kJ/mol": 1.0e6, "J/kmol": 1.0,
                         "K": 8314.462618}


class _Thermo:
    def __init__(self, coeffs):
        self.coeffs = np.asarray(coeffs, dtype=np.float64)


class _Species:
    def __init__(self, d, element_order):
        self.name = d["name"]
        comp = d["composition"]
        w = 0.0
        for el in element_order:
            if el in comp:
                w += comp[el] * _ATOMIC_WEIGHT[el]
        self.molecular_weight = w
        th = d["thermo"]
        assert th["model"] == "NASA7"
        tmid = th["temperature-ranges"][1]
        low, high = th["data"][0], th["data"][1]
        self.thermo = _Thermo([tmid] + list(high) + list(low))


class _Rate:
    def __init__(self, A, b, Ea):
        self.pre_exponential_factor = A
        self.temperature_exponent = b
        self.activation_energy = Ea


class _ThirdBody:
    def __init__(self, eff):
        self.efficiencies = dict(eff)


def _parse_side(side):
    out = {}
    has_m = False
    for tok in side.split(" + "):
        tok = tok.strip()
        if tok == "M":
            has_m = True
            continue
        m = re.match(r"^(\d+(?:\.\d+)?)\s+(\S+)$", tok)
        if m:
            nu, sp = float(m.group(1)), m.group(2)
        else:
            nu, sp = 1.0, tok
        out[sp] = out.get(sp, 0.0) + nu
    return out, has_m


class _Reaction:
    def __init__(self, d, length_factor, quantity_factor, ea_factor):
        eq = d["equation"]
        for arrow in ("<=>", "=>", "="):
            if arrow in eq:
                lhs, rhs = eq.split(arrow)
                break
        self.reactants, m_l = _parse_side(lhs)
        self.products, _ = _parse_side(rhs)
        three_body = d.get("type", "elementary") == "three-body" or m_l
        self.reaction_type = "three-body-Arrhenius" if three_body else "Arrhenius"
        self.third_body = _ThirdBody(d.get("efficiencies", {})) if three_body else None
        rc = d["rate-constant"]
        order = sum(self.reactants.values()) + (1 if three_body else 0)
        if (length_factor, quantity_factor) == (0.01, 1.0e-3):
            A = float(rc["A"]) * (1.0e-3) ** (order - 1)
        elif (length_factor, quantity_factor) == (1.0, 1.0):
            A = float(rc["A"])
        else:
            raise NotImplementedError("unit system not covered by this stand-in")
        self.rate = _Rate(A, float(rc["b"]), float(rc["Ea"]) * ea_factor)


class Solution:
    def __init__(self, path):
        with open(path) as f:
            doc = yaml.safe_load(f)
        units = doc.get("units", {})
        length_factor = {"cm": 0.01, "m": 1.0}[units.get("length", "m")]
        quantity_factor = {"mol": 1.0e-3, "kmol": 1.0}[units.get("quantity", "kmol")]
        ea_factor = _ENERGY_TO_J_PER_KMOL[units.get("activation-energy", "J/kmol")]
        phase = doc["phases"][0]
        self.species_names = list(phase["species"])
        elements = list(phase["elements"])
        by_name = {s["name"]: s for s in doc["species"]}
        self._species = {n: _Species(by_name[n], elements) for n in self.species_names}
        self._reactions = [_Reaction(r, length_factor, quantity_factor, ea_factor)
                           for r in doc.get("reactions", [])]
        ns, nr = len(self.species_names), len(self._reactions)
        self.reactant_stoich_coeffs = np.zeros((ns, nr))
        self.product_stoich_coeffs = np.zeros((ns, nr))
        idx = {n: i for i, n in enumerate(self.species_names)}
        for j, r in enumerate(self._reactions):
            for sp, nu in r.reactants.items():
                self.reactant_stoich_coeffs[idx[sp], j] = nu
            for sp, nu in r.products.items():
                self.product_stoich_coeffs[idx[sp], j] = nu

    def reactions(self):
        return list(self._reactions)

    def species(self, name):
        return self._species[name]
