"""Generates the golden fixtures of tests/golden/ from the reference tree, named by the environment
variable PWA_REFERENCE_TREE (run where that tree exists; the fixtures are committed and the tests
never read the reference).

* smear_schemes.json : the three resolution-offset tables (RooTDalitz/Resonances.h:31-54)
* cg_c2.json         : the reference's tabulated <L 0; S 1/2 | 1/2 1/2> (RooDalitzAmplitude.cxx:96-107)
* cg_ref.json        : Clebsch-Gordan values from the reference's EvtCGCoefSingle, built from source
* dfun_ref.json      : Wigner d values from the reference's dfun / dfunhalf / dfunone, built from source
* ref_nll.json       : NLL of seeded small samples from the reference's own likelihood code on host
                       cores (FP32) next to the FP64 oracle
* func_example.json  : a parameter file of the reference parsed by pwa_b200.model.read_func
* swave_knots.json   : the reference's 24-knot S-wave spline (mass, Re, Im) of Fit_Jpsippi/toyr_fine_bin.dat
"""
from __future__ import annotations

import ctypes as C
import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "pwa-xib2jpsilambdak_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
import build_ref  # noqa: E402

REF = build_ref.reference_tree()


def smear():
    src = (REF / "RooTDalitz" / "Resonances.h").read_text()
    out = {}
    for key, nm in (("20", "_smear_bad_binning_scheme"), ("30", "_smear_binning_scheme"),
                    ("150", "_smear_fine_binning_scheme")):
        m = re.search(nm + r"\[\w+\]\s*=\s*\{([^}]*)\}", src)
        out[key] = [float(v) for v in m.group(1).split(",") if v.strip()]
    m = {k: float(re.search(rf"_mres{k}\s*=\s*([-\d.e]+)", src).group(1)) for k in "012"}
    out["mres"] = [m["0"], m["1"], m["2"]]
    (HERE / "smear_schemes.json").write_text(json.dumps(out, indent=0))


def c2():
    src = (REF / "src" / "RooDalitzAmplitude.cxx").read_text()
    m = re.search(r"Double_t C2\[6\]\[2\] = \{([^}]*)\}", src)
    vals = [float(v) for v in m.group(1).split(",") if v.strip()]
    (HERE / "cg_c2.json").write_text(json.dumps({"C2": [vals[2 * i:2 * i + 2] for i in range(6)]}))


def aux():
    import build_ref
    return C.CDLL(str(build_ref.build_aux()))


def cg(L):
    L.ref_cg.restype = C.c_double
    L.ref_cg.argtypes = [C.c_int] * 6
    rows = []
    for j1, j2 in ((1, 2), (3, 2), (5, 2), (7, 2), (9, 2), (2, 1), (4, 1), (0, 3), (2, 3), (4, 3), (6, 3), (0, 2),
                   (2, 2), (4, 2)):
        for J in range(abs(j1 - j2), j1 + j2 + 1, 2):
            for m1 in range(-j1, j1 + 1, 2):
                for m2 in range(-j2, j2 + 1, 2):
                    M = m1 + m2
                    if abs(M) <= J:
                        rows.append([j1, j2, J, M, m1, m2, L.ref_cg(j1, j2, J, M, m1, m2)])
    (HERE / "cg_ref.json").write_text(json.dumps(rows))


def dfun(L):
    L.ref_dfun.restype = C.c_double
    L.ref_dfun.argtypes = [C.c_double] * 4
    rows = []
    betas = [0.0, 1e-12, 0.3, 1.0, 1.5707963267948966, 2.2, 3.0, float(np.float32(np.pi))]
    for j2 in range(1, 10, 2):
        for m2 in range(-j2, j2 + 1, 2):
            for n2 in range(-j2, j2 + 1, 2):
                for b in betas:
                    rows.append([b, j2 / 2, m2 / 2, n2 / 2, L.ref_dfun(b, j2 / 2, m2 / 2, n2 / 2)])
    (HERE / "dfun_ref.json").write_text(json.dumps(rows))


def ref_nll():
    import oracle as O
    from pwa_b200 import configs, dataset as D, model as M
    rows = []
    for name, nd, nm, seed in (("small_kmatrix", 1500, 15000, 21), ("small_bw", 1500, 15000, 22),
                               ("kmatrix", 1000, 10000, 23), ("lstar_only", 1000, 10000, 24),
                               ("full_bw", 1000, 10000, 25), ("lineshapes", 1000, 10000, 26)):
        mdl, vals = configs.MODELS[name]()
        blk = M.build_param_block(mdl, vals)

        def amp2(ang):
            s = D.build_sample({k: v[:0] for k, v in ang.items()}, ang, np.ones(len(ang["mLk"])))
            fx, _ = O.eval_fx(s, blk, -1, 0)
            return fx
        smp = D.make_sample(nd, nm, (0.2, 1.0), seed, amp2)
        v, s, fx, _ = O.nll(smp, blk)
        rv, rs = O.RefHost(smp, blk).store_fx(blk)
        rows.append({"model": name, "n_data": nd, "n_mc": nm, "seed": seed, "nll_oracle": v, "sumint_oracle": s,
                     "nll_reference_fp32": rv, "sumint_reference_fp32": rs,
                     "fx_head_oracle": fx[:8].tolist(), "param_block_sha": _sha(blk.data)})
    (HERE / "ref_nll.json").write_text(json.dumps(rows, indent=1))


def _sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def swave_knots():
    rows = [[float(x) for x in ln.split()] for ln in
            (REF / "Fit_Jpsippi" / "toyr_fine_bin.dat").read_text().splitlines() if ln.strip()]
    (HERE / "swave_knots.json").write_text(json.dumps(rows))


def func_example():
    from pwa_b200 import model as M
    text = (REF / "Fit_Jpsippi" / "func" / "yujie_test.func").read_text()
    ps = M.read_func(text)
    (HERE / "func_example.json").write_text(json.dumps(
        {k: [p.value, p.error, p.constant, p.lo, p.hi] for k, p in ps.items()}, indent=0, allow_nan=True))


if __name__ == "__main__":
    if "--nll-only" not in sys.argv:
        smear()
        c2()
        L = aux()
        cg(L)
        dfun(L)
        func_example()
        swave_knots()
    ref_nll()
    print("fixtures written to", HERE)
