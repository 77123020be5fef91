"""The reference-signature C++ boundary (include/kernel_calEva_compat.h) driven by a ROOT-free
replay of RooDalitzAmplitude's call sequence, against the oracle."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import PKG, ROOT, make_test_sample


def build_harness(tmp: Path) -> Path:
    exe = tmp / "compat_harness"
    lib = PKG / "pwa_b200"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "compat_harness.cpp"),
                    f"-L{lib}", "-lpwa_b200", f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    return exe


def test_harness_links(tmp_path):
    # links against every compat symbol (no GPU needed to link)
    assert build_harness(tmp_path).exists()


@pytest.mark.gpu
def test_host_store_fx_replay(tmp_path, oracle_mod):
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 1500, 15000)
    exe = build_harness(tmp_path)
    smp.pp.tofile(tmp_path / "pp.bin")
    smp.pp1.tofile(tmp_path / "pp1.bin")
    smp.pp2.tofile(tmp_path / "pp2.bin")
    smp.sw.tofile(tmp_path / "sw.bin")
    blk.data.tofile(tmp_path / "para.bin")
    (tmp_path / "meta.txt").write_text(
        f"{smp.n} {smp.n_size} {smp.nda} {smp.nda_smr1} {smp.nda_fine} {blk.para_size} {blk.vamp_size} {blk.NR} "
        f"{blk.NZ} {smp.sum_w_mc!r} {smp.sum_w_data!r} {blk.ffr} {blk.ffb} 2\n")
    subprocess.run([str(exe), str(tmp_path)], check=True)
    nll, sumint = map(float, (tmp_path / "out.txt").read_text().split())
    fx = np.fromfile(tmp_path / "fx.bin", np.float64)
    amp = np.fromfile(tmp_path / "amp2.bin", np.float64)
    v, s, ofx, _ = oracle_mod.nll(smp, blk)
    assert abs(nll - v) < 1e-6
    assert abs(sumint / s - 1) < 1e-12
    assert np.max(np.abs(fx - ofx) / np.abs(ofx)) < 1e-9
    oa = oracle_mod.amp2(smp, blk)
    assert np.max(np.abs(amp - oa) / oa) < 1e-9
