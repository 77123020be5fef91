"""Product tables and host helpers against golden vectors taken from the reference itself
(tests/golden/make_golden.py)."""
import json
import math
import re
from pathlib import Path

import numpy as np

from conftest import PKG, ROOT

G = Path(__file__).resolve().parent / "golden"


def _inc_tables():
    txt = (PKG / "csrc" / "smear_tables.inc").read_text()
    out = {}
    for nm in ("kSmear20", "kSmear30", "kSmear150"):
        body = re.search(nm + r"\[\d+\] = \{([^}]*)\}", txt).group(1)
        out[nm] = [float(v.strip().rstrip("f")) for v in body.split(",") if v.strip()]
    return out


def test_smear_tables_match_reference():
    g = json.loads((G / "smear_schemes.json").read_text())
    t = _inc_tables()
    assert t["kSmear20"] == g["20"] and t["kSmear30"] == g["30"] and t["kSmear150"] == g["150"]
    # the offsets are rounded standard-normal quantiles (b + 1/2) / N
    from statistics import NormalDist
    for key in ("20", "30", "150"):
        n = int(key)
        q = [NormalDist().inv_cdf((b + 0.5) / n) for b in range(n)]
        assert max(abs(a - b) for a, b in zip(g[key], q)) < 1.5e-3


def test_oracle_tables_match_reference():
    src = (ROOT / "oracle" / "pwa_oracle.cpp").read_text()
    g = json.loads((G / "smear_schemes.json").read_text())
    for nm, key in (("kSmear20", "20"), ("kSmear30", "30"), ("kSmear150", "150")):
        body = re.search(nm + r"\[\d+\] = \{([^}]*)\}", src).group(1)
        assert [float(v.strip().rstrip("f")) for v in body.split(",") if v.strip()] == g[key]


def test_c2_table_and_clebsch():
    from pwa_b200 import model as M
    g = json.loads((G / "cg_c2.json").read_text())["C2"]
    assert [list(r) for r in M.C2] == g
    for s in range(6):
        S = 2 * s + 1
        for li, L in enumerate((S - 1, S + 1)):
            assert abs(M.clebsch(L, 0, S, 1, 1, 1) - g[s][li]) < 1e-13


def test_cg_tables_match_reference_evtgen_tables():
    from pwa_b200 import model as M
    rows = json.loads((G / "cg_ref.json").read_text())
    for j1, j2, J, Mm, m1, m2, v in rows:
        assert M.cg_evtgen(j1, j2, J, Mm, m1, m2) == v, (j1, j2, J, Mm, m1, m2)
        # and within float precision of the exact coefficient
        assert abs(M.clebsch(j1, m1, j2, m2, J, Mm) - v) < 1e-6


def test_dfun_matches_reference():
    from pwa_b200 import basis as B
    rows = json.loads((G / "dfun_ref.json").read_text())
    for b, j, m, n, v in rows:
        got = float(B.dfun(np.array([b]), j, m, n)[0])
        assert abs(got - v) < 1e-13, (b, j, m, n, got, v)


def test_func_format_round_trip():
    from pwa_b200 import model as M
    ref = json.loads((G / "func_example.json").read_text())
    params = {k: M.Param(k, v[0], v[1], bool(v[2]), v[3], v[4]) for k, v in ref.items()}
    back = M.read_func(M.write_func(params))
    assert set(back) == set(ref)
    for k, v in ref.items():
        p = back[k]
        assert math.isclose(p.value, v[0], rel_tol=1e-7, abs_tol=1e-12) and p.constant == bool(v[2])
        assert (p.lo == v[3] or math.isclose(p.lo, v[3], rel_tol=1e-6)) and \
               (p.hi == v[4] or math.isclose(p.hi, v[4], rel_tol=1e-6))
    assert ref["FFB_var"][0] == 3.0 and ref["FFB_var"][2]
