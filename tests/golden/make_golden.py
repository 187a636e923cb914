"""Regenerate tests/golden/reference_tables.json from the reference source text.

Reads (as text, nothing is compiled or run) the Gauss-Legendre tables of
src/numeric/Numeric.cpp:9-46 and the RK coefficient tables of
src/numeric/Numeric.H:111-282 of slug-cfd/kfvm-kokkos, evaluates the literal
expressions (e.g. "1.0 / 3.0") in double precision, and writes them as JSON.
Usage: python tests/golden/make_golden.py <path of the reference checkout>
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py <path of the reference checkout>")
ref = sys.argv[1]
cpp = open(os.path.join(ref, "src/numeric/Numeric.cpp")).read()
hdr = open(os.path.join(ref, "src/numeric/Numeric.H")).read()


def ev(expr):
    expr = expr.strip()
    if not re.fullmatch(r"[-+0-9.eE/* ()]+", expr):
        raise ValueError(expr)
    return float(eval(expr))  # literal arithmetic only (checked above)


def arr(body):
    return [ev(x) for x in body.replace("\n", " ").split(",") if x.strip()]


out = {"quad": {}, "rk": {}}
for nq in (1, 2, 3):
    for name in ("ab", "wt"):
        m = re.search(r"QuadRuleLUT<%d>::%s\s*(?:=\s*)?\{([^}]*)\}" % (nq, name), cpp)
        out["quad"].setdefault(str(nq), {})[name] = arr(m.group(1))
for scheme in ("SSP4_3_2", "SSP10_4_3", "ThreeStarP", "FourStarP"):
    m = re.search(r"struct RKCoeff<RKType::%s> \{(.*?)\n\};" % scheme, hdr, re.S)
    body = m.group(1)
    tab = {}
    for key in ("gam1", "gam2", "gam3", "delta", "beta", "bhat", "c"):
        mm = re.search(r"std::array<Real, \d+> %s = \{(.*?)\};" % key, body, re.S)
        tab[key] = arr(mm.group(1))
    for key in ("bhatfsal", "ep1", "ep2"):
        mm = re.search(r"Real %s = ([^;]*);" % key, body)
        tab[key] = ev(mm.group(1))
    tab["nStages"] = int(re.search(r"nStages = (\d+);", body).group(1))
    out["rk"][scheme] = tab
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_tables.json")
with open(path, "w") as f:
    json.dump(out, f, indent=1)
print("wrote", path)
