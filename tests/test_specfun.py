"""The special functions of the device matching path (exciting_b200/csrc/specfun.cuh)
against the oracle's restatement of genylm, sbessel/sbesseldm and polynom
(oracle/lapw_math.py, itself pinned to SciPy and to closed forms in
tests/test_oracle.py).  The header's routines are compiled for the host with
nvcc (tests/specfun_harness.cu) and evaluated on the argument ranges the
matching uses: Y_lm over the sphere up to l = 12; d^m j_l(x) for m <= 3,
l <= 12 and x = |G+k| R_MT from 0 to 30; derivatives of the interpolating
polynomials through radial-grid windows of 3 to 6 points.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import lapw_math

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "exciting_b200", "csrc")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("specfun") / "specfun_harness")
    subprocess.run([nvcc, "-x", "cu", "-std=c++17", "-O2", "-I", CSRC,
                    os.path.join(HERE, "specfun_harness.cu"), "-o", exe], check=True)
    return exe


def _run(exe, tmp_path, lines):
    inp, out = tmp_path / "in.txt", tmp_path / "out.bin"
    inp.write_text("\n".join(lines) + "\n")
    subprocess.run([exe, str(inp), str(out)], check=True)
    return np.fromfile(str(out), dtype=np.float64)


def test_ylm_matches_oracle(harness, tmp_path):
    rng = np.random.default_rng(1)
    lmax = 12
    th = np.concatenate([[0.0, np.pi, np.pi / 2, 1e-9], rng.uniform(0, np.pi, 60)])
    ph = np.concatenate([[0.0, 1.0, -2.0, 3.1], rng.uniform(-np.pi, np.pi, 60)])
    got = _run(harness, tmp_path, [f"Y {lmax} {float(t):.17g} {float(p):.17g}" for t, p in zip(th, ph)])
    got = got.view(np.complex128).reshape(len(th), (lmax + 1) ** 2)
    ref = lapw_math.genylm(lmax, th, ph)
    assert np.abs(got - ref).max() < 1e-13


@pytest.mark.parametrize("m", [0, 1, 2, 3])
def test_bessel_derivatives_match_oracle(harness, tmp_path, m):
    lmax = 12
    x = np.concatenate([[0.0, 1e-9, 1e-4, 0.5, 0.999999, 1.0, 1.000001, 11.999, 12.0, 12.5],
                        np.linspace(0.01, 30.0, 157)])
    got = _run(harness, tmp_path, [f"J {m} {lmax} {float(v):.17g}" for v in x]).reshape(len(x), lmax + 1)
    ref = lapw_math.sbesseldm(m, lmax, x)
    # relative to the largest order's magnitude in the row (the matching
    # multiplies each by coefficients of comparable size), and per element
    # where the value itself is not tiny
    scale = np.maximum(np.abs(ref).max(axis=1, keepdims=True), 1e-300)
    assert (np.abs(got - ref) / scale).max() < 1e-13
    big = np.abs(ref) > 1e-6 * scale
    assert (np.abs(got - ref)[big] / np.abs(ref)[big]).max() < 1e-11


@pytest.mark.parametrize("np_", [3, 4, 5, 6])
def test_polynomial_derivatives_match_oracle(harness, tmp_path, np_):
    rng = np.random.default_rng(np_)
    lines, refs = [], []
    for _ in range(40):
        # the last np points of a logarithmic radial mesh ending at R_MT
        rmt = rng.uniform(1.5, 2.5)
        h = rng.uniform(0.01, 0.04)
        xa = rmt * np.exp(-h * np.arange(np_)[::-1])
        ya = rng.standard_normal() * np.sin(1.3 * xa + rng.uniform(0, 3)) + 0.2 * xa ** 2
        for m in range(np_ + 1):
            lines.append(f"P {m} {np_} {float(rmt):.17g} " + " ".join(f"{float(v):.17g}" for v in xa) + " "
                         + " ".join(f"{float(v):.17g}" for v in ya))
            refs.append(lapw_math.polynom(m, xa, ya, rmt))
    got = _run(harness, tmp_path, lines)
    refs = np.array(refs)
    err = np.abs(got - refs) / np.maximum(np.abs(refs), 1.0)
    assert err.max() < 1e-9
