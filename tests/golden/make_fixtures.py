"""Generate the golden fixtures under tests/golden/ from the reference tree.

Run as `python tests/golden/make_fixtures.py <path of the HigherHarmonics
source tree>` where the reference sources are available.  Nothing at test time
reads the reference; the tests only read the JSON files written here.

* gauss_tables.json -- every gauss::container<N> table of
  sources/HHG/thread_gauss.hpp (positive abscissae ascending, weights), parsed
  as text, plus the 30-point [0,1] table of sources/HHG/Laser/gauss.hpp.
* magnus_dirac.json -- the Magnus generator Omega of helper/magnus_dirac.py,
  evaluated with sympy at seeded sample points (k, k_z, kappa, alpha..delta).
* piflux_ic.json -- the thermal PiFlux initial state <sigma> of
  helper/piflux_initial_conditions.py (the state alpha|a> + beta|b> written
  through the helper's V and normalisation), evaluated with sympy at seeded
  (t, beta_T, E_F, k) with alpha^2, beta^2 the reference's band occupations
  (PiFlux.cpp:420-426, GlobalDefinitions.hpp:36-41), together with the
  helper's closed form of |<sigma(0)>|^2.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def gauss_tables(ref: str) -> dict:
    txt = open(os.path.join(ref, "sources/HHG/thread_gauss.hpp")).read()
    out = {}
    starts = [(m.start(), int(m.group(1))) for m in re.finditer(r"struct container<(\d+)>\s*\{", txt)]
    for idx, (pos, n) in enumerate(starts):
        end = starts[idx + 1][0] if idx + 1 < len(starts) else len(txt)
        body = txt[pos:end]
        arrs = [re.search(name + r"\s*=\s*\{(.*?)\};", body, re.S).group(1)
                for name in ("abscissa", "weights")]
        vals = [[float(v.strip().rstrip("L")) for v in a.split(",") if v.strip()] for a in arrs]
        out[str(n)] = {"abscissa": vals[0], "weights": vals[1]}
    g = open(os.path.join(ref, "sources/HHG/Laser/gauss.hpp")).read()
    ab = re.search(r"abscissa\s*=\s*\{(.*?)\};", g, re.S).group(1)
    wt = re.search(r"weights\s*=\s*\{(.*?)\};", g, re.S).group(1)
    xs = [float(x) for x in re.findall(r"0\.5 \* \(([-+0-9.e]+) \+ 1\.\)", ab)]
    ws = [float(x) for x in re.findall(r"0\.5 \* ([-+0-9.e]+)", wt)]
    out["laser30"] = {"nodes_pm1": xs, "weights_pm1": ws}
    return out


def magnus_dirac(ref: str, n_points: int = 6, seed: int = 20261203) -> dict:
    import sympy
    sys.path.insert(0, os.path.join(ref, "helper"))
    src = open(os.path.join(ref, "helper/magnus_dirac.py")).read()
    # execute the derivation up to the symbolic Omega (drop the print loop)
    src = src.split("for i in range(3):")[0]
    ns: dict = {}
    exec(compile(src, "magnus_dirac.py", "exec"), ns)
    omega = ns["expr_simplified"]
    syms = {s.name: s for s in omega.free_symbols}
    rng = np.random.default_rng(seed)
    pts = []
    for _ in range(n_points):
        vals = {"k": float(rng.uniform(0.01, 0.5)), "k_z": float(rng.uniform(-0.3, 0.3)),
                "kappa": float(rng.uniform(0.01, 0.4)), "alpha": float(rng.uniform(-2, 2)),
                "beta": float(rng.uniform(-1, 1)), "gamma": float(rng.uniform(-0.5, 0.5)),
                "delta": float(rng.uniform(-0.3, 0.3))}
        sub = {syms[n]: sympy.Float(v, 30) for n, v in vals.items() if n in syms}
        om = [[float(sympy.N(omega[i, j].subs(sub), 25)) for j in range(3)] for i in range(3)]
        pts.append({"inputs": vals, "omega": om})
    return {"points": pts}


def piflux_ic(ref: str, n_points: int = 12, seed: int = 20261203) -> dict:
    import contextlib
    import io
    import math

    import sympy
    src = open(os.path.join(ref, "helper/piflux_initial_conditions.py")).read()
    ns: dict = {}
    with contextlib.redirect_stdout(io.StringIO()):
        exec(compile(src, "piflux_initial_conditions.py", "exec"), ns)
    a, b, x, y, z = (ns[n] for n in ("alpha", "beta", "x", "y", "z"))
    phi, V, nrm = ns["phi"], ns["V"], ns["normalization"]
    exprs = [sympy.simplify(nrm * (phi.H * V.H * s * V * phi)[0])
             for s in (ns["sigma_x"], ns["sigma_y"], ns["sigma_z"])]
    norm2 = ns["norm"]

    def fermi(e, beta_t):
        return 1.0 / (1.0 + math.exp(beta_t * e))

    rng = np.random.default_rng(seed)
    pts = []
    for _ in range(n_points):
        t = float(rng.uniform(0.5, 1.5))
        beta_t = float(rng.uniform(0.05, 3.0))
        ef = float(rng.uniform(-1.0, 1.0))
        k = [float(v) for v in rng.uniform(-math.pi, math.pi, 3)]
        c = [math.cos(v) for v in k]
        disp = math.sqrt(sum(v * v for v in c))
        a2 = fermi(-ef + 2 * t * disp, beta_t)
        b2 = fermi(-ef - 2 * t * disp, beta_t)
        sub = {a: sympy.sqrt(sympy.Float(a2, 30)), b: sympy.sqrt(sympy.Float(b2, 30)),
               x: sympy.Float(c[0], 30), y: sympy.Float(c[1], 30), z: sympy.Float(c[2], 30)}
        sigma = [float(sympy.re(sympy.N(e.subs(sub), 25))) for e in exprs]
        n2 = float(sympy.N(norm2.subs({a: sub[a], b: sub[b]}), 25))
        pts.append({"hopping": t, "beta": beta_t, "fermi_energy": ef, "k": k,
                    "alpha2": a2, "beta2": b2, "sigma": sigma, "norm2": n2})
    return {"points": pts}


def main() -> None:
    if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], "sources")):
        sys.exit("usage: make_fixtures.py <HigherHarmonics source tree (holds sources/ and helper/)>")
    ref = sys.argv[1]
    with open(os.path.join(HERE, "gauss_tables.json"), "w") as f:
        json.dump(gauss_tables(ref), f)
    with open(os.path.join(HERE, "magnus_dirac.json"), "w") as f:
        json.dump(magnus_dirac(ref), f, indent=1)
    with open(os.path.join(HERE, "piflux_ic.json"), "w") as f:
        json.dump(piflux_ic(ref), f, indent=1)


if __name__ == "__main__":
    main()
