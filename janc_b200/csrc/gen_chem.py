"""Generate ``jb_chem_gen.cuh``: point-implicit chemistry specialised to one
mechanism's structure.

The stoichiometry (which species each reaction consumes and produces, with
what coefficients), the third-body pattern and the sparsity of the analytic
Jacobian become compile-time constants, so the kernel is straight-line code
with no table loops.  Rate parameters, efficiencies and thermo coefficients
stay runtime values read from the kernel's parameter block, so the same
binary serves any non-dimensionalisation.  ``jb_create`` compares the loaded
mechanism's structure with ``GEN_*`` below and falls back to the generic
kernel when they differ.

The arithmetic restates ``src/janc_v2/model/reaction_model.py:91-193``
with one exponential per reaction and one per species:
k0 = exp(ln A + B ln T - Ea/(R T)), kf = k0 prod Xc^vf,
kb = k0 prod E^(-dv) (T P0/101325)^vsum prod Xc^vb with E_k = exp(g_k) the
exponentiated Gibbs terms and Xc the molar concentrations clipped at 1e-50
(the reference's exp(sum vf log Xc), exp(sum dv g) and
(101325/(P0 T))^vsum, whose exponents are small integers); the Jacobian
entry is
J_kn = M_k sum_i dv_ik [q_i a_in / M_n + (vf_in M_i kf_i - vb_in M_i kb_i)/(M_n X_n)].

Usage: python gen_chem.py [mechanism.yaml] > jb_chem_gen.cuh
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def _num(v):
    v = float(v)
    return repr(v) if v != int(v) else f"{int(v)}.0"


def generate(path=None):
    from janc_b200 import mechanism as jm
    mech = jm.load(path or jm.DEFAULT_MECHANISM)
    t = mech.tables
    vf, vb, tb = t["vf"], t["vb"], t["third_body"]
    is_tb = t["is_third_body"]
    vsum = t["vsum"]
    nreac, nr = vf.shape
    ns = tb.shape[1]
    out = []
    w = out.append
    w("// Generated by janc_b200/csrc/gen_chem.py from "
      f"{os.path.basename(path or jm.DEFAULT_MECHANISM)}; do not edit.")
    w("// Species: " + ", ".join(mech.species))
    w("#pragma once")
    w("")
    w(f"#define JB_GEN_NREAC {nreac}")
    w(f"#define JB_GEN_NR {nr}")
    w(f"#define JB_GEN_NS {ns}")
    w("// structure signature (compared with the loaded mechanism by jb_create)")
    w("static const signed char JB_GEN_VF[%d][%d] = {%s};" % (
        nreac, nr, ", ".join("{" + ", ".join(str(int(x)) for x in row) + "}" for row in vf)))
    w("static const signed char JB_GEN_VB[%d][%d] = {%s};" % (
        nreac, nr, ", ".join("{" + ", ".join(str(int(x)) for x in row) + "}" for row in vb)))
    w("static const signed char JB_GEN_TBNZ[%d][%d] = {%s};" % (
        nreac, ns, ", ".join("{" + ", ".join(str(int(x != 0)) for x in row) + "}" for row in tb)))
    w("static const signed char JB_GEN_ISTB[%d] = {%s};" % (nreac, ", ".join(str(int(x)) for x in is_tb)))
    w("static const signed char JB_GEN_VSUM[%d] = {%s};" % (nreac, ", ".join(str(int(x)) for x in vsum)))
    w("")
    w("#ifdef JB_NS")
    w("namespace jb {")
    w("namespace JB_NS {")
    w("namespace {")
    w("")
    w("// Phase A: rates of every reaction for one cell.  Writes q_i = kf - kb,")
    w("// F_i = M_i kf and B_i = M_i kb to shared memory (layout [i][3][stride])")
    w("// and accumulates w_k = sum_i dv_ik M_i q_i.  Xc: clipped concentrations;")
    w("// E, iE: exp(g_k) and 1 / exp(g_k); Tp = T / pref, pT = pref / T.")
    w("__device__ __forceinline__ void chem_rates_gen(const MP& m, double lT, double invT, double Tp, double pT,")
    w("    const double* X, const double* Xc, const double* E, const double* iE, double* sh, int stride,")
    w("    double* wk) {")
    for k in range(nr):
        w(f"  wk[{k}] = 0.0;")
    for i in range(nreac):
        reac = [(k, int(vf[i, k])) for k in range(nr) if vf[i, k] != 0]
        prod = [(k, int(vb[i, k])) for k in range(nr) if vb[i, k] != 0]
        dv = [(k, int(vb[i, k] - vf[i, k])) for k in range(nr) if vb[i, k] != vf[i, k]]

        def powers(terms, arr):
            # prod arr[k]^c as repeated products (c a small positive integer)
            return [f"{arr}[{k}]" for k, c in terms for _ in range(c)]

        w(f"  {{  // reaction {i}")
        w(f"    const double k0 = exp(m.lnA[{i}] + m.B[{i}] * lT - m.EaR[{i}] * invT);")
        if is_tb[i]:
            terms = [f"m.tb[{i}][{j}] * X[{j}]" for j in range(ns) if tb[i, j] != 0]
            w(f"    const double Mi = {' + '.join(terms)};")
        else:
            w("    const double Mi = 1.0;")
        fac_f = powers(reac, "Xc")
        eg = [f"E[{k}]" for k, c in dv if c < 0 for _ in range(-c)] + \
             [f"iE[{k}]" for k, c in dv if c > 0 for _ in range(c)]
        vs = int(vsum[i])
        pw = ["Tp"] * vs if vs > 0 else ["pT"] * (-vs)
        fac_b = eg + pw + powers(prod, "Xc")
        w(f"    const double kf = {' * '.join(['k0'] + fac_f)};")
        w(f"    const double kb = {' * '.join(['k0'] + fac_b)};")
        w("    const double q = kf - kb;")
        w("    const double Mq = Mi * q;")
        for k, c in dv:
            if c == 1:
                w(f"    wk[{k}] += Mq;")
            elif c == -1:
                w(f"    wk[{k}] -= Mq;")
            else:
                w(f"    wk[{k}] += {_num(c)} * Mq;")
        w(f"    sh[({3 * i} + 0) * stride] = q;")
        w(f"    sh[({3 * i} + 1) * stride] = Mi * kf;")
        w(f"    sh[({3 * i} + 2) * stride] = Mi * kb;")
        w("  }")
    w("}")
    w("")
    w("// Phase B: the analytic Jacobian J[k][n] (without the M_k row factor).")
    w("__device__ __forceinline__ void chem_jac_gen(const MP& m, const double* rMX, const double* sh,")
    w("    int stride, double (&J)[8][8]) {")
    w("#pragma unroll")
    w("  for (int k = 0; k < 8; ++k)")
    w("#pragma unroll")
    w("    for (int n = 0; n < 8; ++n) J[k][n] = 0.0;")
    for i in range(nreac):
        dv = [(k, int(vb[i, k] - vf[i, k])) for k in range(nr) if vb[i, k] != vf[i, k]]
        if not dv:
            continue
        w(f"  {{  // reaction {i}")
        if is_tb[i]:
            w(f"    const double q = sh[({3 * i} + 0) * stride];")
        w(f"    const double F = sh[({3 * i} + 1) * stride];")
        w(f"    const double B = sh[({3 * i} + 2) * stride];")
        for n in range(nr):
            parts = []
            if tb[i, n] != 0:
                parts.append(f"q * m.tbinvM[{i}][{n}]")
            a, b = int(vf[i, n]), int(vb[i, n])
            if a or b:
                inner = []
                if a:
                    inner.append("F" if a == 1 else f"{_num(a)} * F")
                if b:
                    inner.append(("- B" if b == 1 else f"- {_num(b)} * B"))
                expr = " ".join(inner) if a else inner[0].replace("- ", "-", 1)
                parts.append(f"({expr}) * rMX[{n}]")
            if not parts:
                continue
            w(f"    {{ const double c = {' + '.join(parts)};")
            for k, c in dv:
                if c == 1:
                    w(f"      J[{k}][{n}] += c;")
                elif c == -1:
                    w(f"      J[{k}][{n}] -= c;")
                else:
                    w(f"      J[{k}][{n}] += {_num(c)} * c;")
            w("    }")
        w("  }")
    w("}")
    w("")
    w("}  // namespace")
    w("}  // namespace JB_NS")
    w("}  // namespace jb")
    w("#endif")
    return "\n".join(out) + "\n"


if __name__ == "__main__":
    sys.stdout.write(generate(sys.argv[1] if len(sys.argv) > 1 else None))
