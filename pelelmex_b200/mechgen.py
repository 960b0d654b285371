"""Mechanism-specific CUDA code for the right-hand side (like CEPTR does for
the reference's mechanisms).

For a flattened mechanism this writes a device function

    void gen_rhs_<name>(const double* y, const double* F, double* out)

with every rate constant, stoichiometric coefficient, efficiency and NASA-7
coefficient as an immediate, so that concentrations, g/RT and production
rates live in registers and no table is read.  The formulas are the ones of
the table-driven right-hand side (Chemkin formalism: Arrhenius, third body,
Lindemann / Troe falloff, reverse rates from Kc), evaluated in the same
order per reaction.

The function is selected at handle creation by a 64-bit FNV-1a digest of the
mechanism description (mechanism_digest), computed identically here and in
the library.
"""
from __future__ import annotations

import numpy as np

FNV_OFFSET = 0xcbf29ce484222325
FNV_PRIME = 0x100000001b3


def _fnv(h: int, data: bytes) -> int:
    for b in data:
        h ^= b
        h = (h * FNV_PRIME) & 0xFFFFFFFFFFFFFFFF
    return h


def mechanism_digest(flat) -> int:
    """FNV-1a over the description arrays in b200chem_mech_desc order."""
    a = flat.arrays
    h = FNV_OFFSET
    h = _fnv(h, np.array([flat.n_species, flat.n_reactions, flat.n_eff], np.int32).tobytes())
    for key, dt in (("mw", np.float64), ("nasa", np.float64), ("rtype", np.int32), ("rflags", np.int32),
                    ("arr", np.float64), ("arr_lo", np.float64), ("arr_rev", np.float64), ("troe", np.float64),
                    ("sp", np.int32), ("nu", np.int32), ("eff_ptr", np.int32)):
        h = _fnv(h, np.ascontiguousarray(a[key], dt).tobytes())
    ne = flat.n_eff
    h = _fnv(h, np.ascontiguousarray(a["eff_sp"][:ne], np.int32).tobytes())
    h = _fnv(h, np.ascontiguousarray(a["eff_val"][:ne], np.float64).tobytes())
    return h


def _d(x: float) -> str:
    return repr(float(x))


def generate(flat, name: str) -> str:
    a = flat.arrays
    N, R = flat.n_species, flat.n_reactions
    mw = a["mw"]
    nasa = a["nasa"]  # [N][15]
    out = []
    w = out.append
    w(f"// mechanism {name}: {N} species, {R} reactions")
    w(f"constexpr unsigned long long kGenDigest_{name} = {mechanism_digest(flat)}ull;")
    w(f"__device__ __forceinline__ void gen_rhs_{name}(const double* __restrict__ y, "
      f"const double* __restrict__ F, double* __restrict__ out) {{")
    w(f"  const double T = y[{N}];")
    w("  const double lnT = log(T), invT = 1.0 / T;")
    w("  const double lnPRT = log(kPatm / (kRu * T));")
    w("  const bool lo = T < " + _d(nasa[0, 0]) + ";")
    if not np.all(nasa[:, 0] == nasa[0, 0]):
        raise ValueError("generated right-hand side needs one common NASA-7 midpoint temperature")
    w(f"  double C[{N}], g[{N}], wd[{N}];")
    w("  double Ctot = 0.0, rcp = 0.0;")
    for k in range(N):
        lo = nasa[k, 1:8]
        hi = nasa[k, 8:15]
        cs = ", ".join(f"lo ? {_d(lo[i])} : {_d(hi[i])}" for i in range(7))
        w(f"  {{ const double c[7] = {{{cs}}};")
        w("    const double cpR = c[0] + T * (c[1] + T * (c[2] + T * (c[3] + T * c[4])));")
        w("    const double hRT = c[0] + T * (c[1] / 2 + T * (c[2] / 3 + T * (c[3] / 4 + T * c[4] / 5))) + c[5] * invT;")
        w("    const double sR = c[0] * lnT + T * (c[1] + T * (c[2] / 2 + T * (c[3] / 3 + T * c[4] / 4))) + c[6];")
        w(f"    g[{k}] = hRT - sR; C[{k}] = y[{k}] * {_d(1.0 / mw[k])}; wd[{k}] = 0.0;")
        w(f"    Ctot += C[{k}]; rcp += y[{k}] * cpR * {_d(8.31446261815324e7 / mw[k])}; }}")
    sp, nu = a["sp"], a["nu"]
    effp, effs, effv = a["eff_ptr"], a["eff_sp"], a["eff_val"]
    for j in range(R):
        typ, fl = int(a["rtype"][j]), int(a["rflags"][j])
        lnA, b, ea = a["arr"][j]
        w(f"  {{ // reaction {j}")
        arg = _d(lnA)
        if b != 0.0:
            arg += f" + {_d(b)} * lnT"
        if ea != 0.0:
            arg += f" - {_d(ea)} * invT"
        w(f"    double kf = gexp({arg});")
        if typ != 0:
            terms = "Ctot"
            for q in range(effp[j], effp[j + 1]):
                e = effv[q] - 1.0
                if e != 0.0:
                    terms += f" + {_d(e)} * C[{int(effs[q])}]"
            w(f"    const double M = {terms};")
        if typ >= 2:
            l0, b0, e0 = a["arr_lo"][j]
            arg0 = _d(l0)
            if b0 != 0.0:
                arg0 += f" + {_d(b0)} * lnT"
            if e0 != 0.0:
                arg0 += f" - {_d(e0)} * invT"
            w(f"    const double k0 = gexp({arg0});")
            w("    const double Pr = k0 * M / kf;")
            if typ == 3:
                ta, t3, t1, t2 = a["troe"][j]
                fc = f"(1.0 - {_d(ta)}) * gexp(-T / {_d(t3)}) + {_d(ta)} * gexp(-T / {_d(t1)})"
                if fl & 4:
                    fc += f" + gexp(-{_d(t2)} * invT)"
                w(f"    const double Fc = {fc};")
                w("    const double logFc = log10(fmax(Fc, 1e-300));")
                w("    const double cc = -0.4 - 0.67 * logFc, nn = 0.75 - 1.27 * logFc;")
                w("    const double u = log10(fmax(Pr, 1e-300)) + cc;")
                w("    const double f1 = u / (nn - 0.14 * u);")
                w(f"    const double Fb = gexp({_d(np.log(10.0))} * (logFc / (1.0 + f1 * f1)));")
                w("    kf = kf * Pr / (1.0 + Pr) * Fb;")
            else:
                w("    kf = kf * Pr / (1.0 + Pr);")
        pf, pr, sg = [], [], []
        sd = 0
        for s in range(8):
            k = int(sp[j, s])
            if k < 0:
                continue
            v = int(nu[j, s])
            sgn = -1 if s < 4 else 1
            sd += sgn * v
            (pf if s < 4 else pr).extend([f"C[{k}]"] * v)
            sg.append(f"{'-' if sgn < 0 else '+'} {v}.0 * g[{k}]" if v != 1 else f"{'-' if sgn < 0 else '+'} g[{k}]")
        pfs = " * ".join(pf) if pf else "1.0"
        prs = " * ".join(pr) if pr else "1.0"
        if fl & 2:
            lr, br, er = a["arr_rev"][j]
            argr = _d(lr)
            if br != 0.0:
                argr += f" + {_d(br)} * lnT"
            if er != 0.0:
                argr += f" - {_d(er)} * invT"
            w(f"    const double kr = gexp({argr});")
        elif fl & 1:
            sgs = " ".join(sg).lstrip("+ ")
            w(f"    const double kr = kf * gexp({sgs} - {_d(float(sd))} * lnPRT);")
        else:
            w("    const double kr = 0.0;")
        w(f"    double q = kf * ({pfs}) - kr * ({prs});")
        if typ == 1:
            w("    q *= M;")
        for s in range(8):
            k = int(sp[j, s])
            if k < 0:
                continue
            v = int(nu[j, s])
            op = "-=" if s < 4 else "+="
            w(f"    wd[{k}] {op} {'' if v == 1 else f'{v}.0 * '}q;")
        w("  }")
    w("  double hs = 0.0;")
    for k in range(N):
        lo = nasa[k, 1:8]
        hi = nasa[k, 8:15]
        cs = ", ".join(f"lo ? {_d(lo[i])} : {_d(hi[i])}" for i in range(6))
        w(f"  {{ const double c[6] = {{{cs}}};")
        w("    const double hRT = c[0] + T * (c[1] / 2 + T * (c[2] / 3 + T * (c[3] / 4 + T * c[4] / 5))) + c[5] * invT;")
        w(f"    const double yd = wd[{k}] * {_d(mw[k])} + F[{k}];")
        w(f"    out[{k}] = yd; hs += hRT * {_d(8.31446261815324e7 / mw[k])} * T * yd; }}")
    w(f"  out[{N}] = (F[{N}] - hs) / rcp;")
    w("}")
    return "\n".join(out) + "\n"


def generate_bundled() -> str:
    """Header with the generated right-hand sides of the bundled mechanisms."""
    from . import mechanism as mechmod
    parts = ["// gen_mechs.cuh -- generated by pelelmex_b200.mechgen; do not edit.",
             "#pragma once", "// included after mech_dev.cuh (kPatm, kRu)", "namespace b200 {", "namespace gen {",
             "// out-of-line FP64 exp: one copy of the code for every call site",
             "__device__ __noinline__ double gexp(double x) { return exp(x); }"]
    for name in ("synth_h2_9", "synth_ch4_21", "synth_c12_53"):
        flat = mechmod.flatten(mechmod.builtin(name))
        parts.append(generate(flat, name))
    parts += ["}  // namespace gen", "}  // namespace b200"]
    return "\n".join(parts) + "\n"


def _c_array(ctype: str, name: str, values, per_line: int = 6) -> str:
    vals = [repr(float(v)) if ctype == "double" else str(int(v)) for v in np.ravel(values)]
    if not vals:
        vals = ["0"]
    lines = [", ".join(vals[i:i + per_line]) for i in range(0, len(vals), per_line)]
    return f"static const {ctype} {name}[{len(vals)}] = {{\n  " + ",\n  ".join(lines) + "\n};\n"


def generate_mech_desc(flat, name: str) -> str:
    """C++ translation unit defining b200chem_make_mech_desc() for one
    mechanism: the flat description (the data a CEPTR-generated mechanism
    bakes into code) as static tables, so a PelePhysics build links the
    ReactorB200 shim without hand-written mechanism code.  The digest it
    carries in a comment is the one the library computes for it."""
    a = flat.arrays
    ne = flat.n_eff
    out = [f"// b200chem mechanism description of {name}: {flat.n_species} species, {flat.n_reactions} "
           f"reactions.", "// Generated by pelelmex_b200.mechgen; do not edit.",
           f"// digest 0x{mechanism_digest(flat):016x}", '#include "b200chem.h"', "", "namespace {"]
    for key, ct in (("mw", "double"), ("nasa", "double"), ("rtype", "int32_t"), ("rflags", "int32_t"),
                    ("arr", "double"), ("arr_lo", "double"), ("arr_rev", "double"), ("troe", "double"),
                    ("sp", "int32_t"), ("nu", "int32_t"), ("eff_ptr", "int32_t")):
        out.append(_c_array(ct, f"k_{key}", a[key]))
    out.append(_c_array("int32_t", "k_eff_sp", a["eff_sp"][:max(ne, 0)]))
    out.append(_c_array("double", "k_eff_val", a["eff_val"][:max(ne, 0)]))
    out += ["}  // namespace", "", "b200chem_mech_desc b200chem_make_mech_desc() {", "  b200chem_mech_desc d{};",
            f"  d.n_species = {flat.n_species};", f"  d.n_reactions = {flat.n_reactions};", f"  d.n_eff = {ne};"]
    for key in ("mw", "nasa", "rtype", "rflags", "arr", "arr_lo", "arr_rev", "troe", "sp", "nu", "eff_ptr",
                "eff_sp", "eff_val"):
        out.append(f"  d.{key} = k_{key};")
    out += ["  return d;", "}", ""]
    return "\n".join(out)


def main(argv=None):
    """python -m pelelmex_b200.mechgen --mech-desc MECHANISM --out FILE.cpp

    MECHANISM is a bundled mechanism name or a Cantera-style YAML file."""
    import argparse
    from pathlib import Path
    from . import mechanism as mechmod
    p = argparse.ArgumentParser()
    p.add_argument("--mech-desc", required=True)
    p.add_argument("--out", required=True)
    a = p.parse_args(argv)
    src = a.mech_desc
    mech = mechmod.load(src) if Path(src).exists() else mechmod.builtin(src)
    Path(a.out).write_text(generate_mech_desc(mechmod.flatten(mech), mech.name if hasattr(mech, "name") else src))


if __name__ == "__main__":
    main()
