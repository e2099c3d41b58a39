"""Loader for the golden fixtures (tests/golden/*.npz) shared by the tests."""

from __future__ import annotations

import json
import pathlib

import numpy as np

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"

CASES = sorted(p.stem for p in GOLDEN.glob("c[23]d_*.npz"))


def load_case(name: str) -> dict:
    d = np.load(GOLDEN / f"{name}.npz")
    c = {k: d[k] for k in d.files}
    c["kwargs"] = json.loads(str(d["kwargs"]))
    for k in ("dims", "nx", "ny", "nz", "steps"):
        c[k] = int(c[k])
    for k in ("omega", "u0", "D"):
        c[k] = float(c[k])
    c["hist"] = {k[5:]: c[k] for k in d.files if k.startswith("hist_")}
    if c["phi"].dtype == object or c["phi"].shape == ():
        c["phi"] = None
    return c


def make_oracle(c: dict, **extra):
    from oracle.oracle import OracleSolver
    kw = dict(c["kwargs"])
    kw.update(extra)
    o = OracleSolver(solid=c["solid"], omega=c["omega"], u0=c["u0"], D=c["D"], phi=c["phi"], **kw)
    o.f = c["f0"].copy()
    if "g0" in c:
        o.g = c["g0"].copy()
    return o
