"""The two-stage Householder reduction restated in ``oracle/two_stage.py``.

Checks, on CPU, that each stage is a unitary similarity with the advertised
structure (band of width b after the first stage, real tridiagonal after the
second) and that the tridiagonal has the Hermitian matrix's eigenvalues, on
random complex Hermitian and real symmetric matrices, a matrix with repeated
eigenvalues, and the edge sizes (n <= b + 1, n = 1, 2).
"""
import numpy as np
import pytest

from oracle import two_stage as ts


def _herm(n, rng, real=False):
    X = rng.standard_normal((n, n))
    if not real:
        X = X + 1j * rng.standard_normal((n, n))
    return (X + X.conj().T) / 2


def _check(C, b):
    n = C.shape[0]
    scale = max(1.0, np.abs(C).max())
    B, Q1, panels = ts.he2hb(C, b)
    I = np.eye(n)
    assert np.abs(Q1.conj().T @ Q1 - I).max() < 1e-13
    full = Q1.conj().T @ C @ Q1
    outside = np.abs(np.subtract.outer(np.arange(n), np.arange(n))) > b
    if outside.any():
        assert np.abs(full[outside]).max() < 1e-13 * scale * n
    assert np.abs(full - B).max() < 1e-13 * scale * n
    d, e, Q2, refl = ts.hb2st(B, b)
    assert np.all(e >= 0.0)
    T = np.diag(d) + np.diag(e, -1) + np.diag(e, 1)
    Q = Q1 @ Q2
    assert np.abs(Q.conj().T @ Q - I).max() < 1e-13
    assert np.abs(Q.conj().T @ C @ Q - T).max() < 1e-13 * scale * n
    assert np.abs(np.linalg.eigvalsh(T) - np.linalg.eigvalsh(C)).max() < 1e-13 * scale * n
    return d, e, Q


@pytest.mark.parametrize("n,b", [(37, 2), (37, 8), (64, 16), (100, 32), (130, 5), (50, 48)])
def test_two_stage_random_hermitian(n, b):
    _check(_herm(n, np.random.default_rng(n * 100 + b)), b)


def test_two_stage_real_symmetric():
    _check(_herm(80, np.random.default_rng(7), real=True), 12)


def test_two_stage_repeated_eigenvalues():
    rng = np.random.default_rng(11)
    n = 60
    lam = np.repeat(np.array([-2.0, 0.5, 0.5 + 1e-12, 3.0]), 15)
    U, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    C = (U * lam) @ U.conj().T
    d, e, Q = _check(C, 8)
    w, Z = np.linalg.eigh(np.diag(d) + np.diag(e, -1) + np.diag(e, 1))
    X = Q @ Z  # back-transformed eigenvectors of C
    assert np.abs(C @ X - X * w).max() < 1e-12


@pytest.mark.parametrize("n,b", [(1, 4), (2, 4), (5, 4), (6, 4), (9, 8)])
def test_two_stage_edge_sizes(n, b):
    _check(_herm(n, np.random.default_rng(n)), b)


def test_householder_matches_zlarfg_convention():
    rng = np.random.default_rng(3)
    x = rng.standard_normal(9) + 1j * rng.standard_normal(9)
    v, tau, beta = ts.householder(x)
    H = np.eye(9) - tau * np.outer(v, v.conj())
    y = H.conj().T @ x
    assert v[0] == 1.0
    assert abs(y[0] - beta) < 1e-13 and np.abs(y[1:]).max() < 1e-13
    assert np.abs(H.conj().T @ H - np.eye(9)).max() < 1e-13


@pytest.mark.parametrize("n,b", [(37, 2), (64, 16), (130, 32), (130, 5), (9, 8)])
def test_blocked_band_stage_matches_reflector_by_reflector(n, b):
    """The compact-WY form (panel QR, ZLARFT, X = C22 V T, W = X - V (T^H V^H X)/2,
    C22 -= V W^H + W V^H) gives the same band matrix and Q1."""
    C = _herm(n, np.random.default_rng(n + 7 * b))
    B, Q1, _ = ts.he2hb(C, b)
    Bb, Q1b = ts.he2hb_blocked(C, b)
    scale = np.abs(C).max()
    assert np.abs(B - Bb).max() < 1e-13 * scale * n
    assert np.abs(Q1 - Q1b).max() < 1e-13 * n


def test_apply_q2_is_the_product_of_the_chase_reflectors():
    rng = np.random.default_rng(21)
    n, b = 90, 12
    B, _, _ = ts.he2hb(_herm(n, rng), b)
    _, _, _, refl = ts.hb2st(B, b)
    Qd = np.eye(n, dtype=np.complex128)
    for (_i, lo, v, tau) in refl:
        hi = lo + len(v)
        Qd[:, lo:hi] -= tau * np.outer(Qd[:, lo:hi] @ v, v.conj())
    Z = rng.standard_normal((n, 9)) + 1j * rng.standard_normal((n, 9))
    assert np.abs(ts.apply_q2(refl, Z) - Qd @ Z).max() < 1e-13


@pytest.mark.parametrize("n,b", [(60, 4), (97, 8), (130, 16)])
def test_chase_schedule_lag_three_is_concurrency_safe(n, b):
    """Time slot 3 i + k: each slot's tasks commute (executing them in reverse
    sweep order gives the sweep-by-sweep result); slot 2 i + k does not."""
    B, _, _ = ts.he2hb(_herm(n, np.random.default_rng(n)), b)
    ref = ts.run_chase(B, ts.chase_tasks(n, b))
    scale = np.abs(B).max()
    assert np.abs(ts.run_chase(B, ts.chase_schedule(n, b, lag=3)) - ref).max() < 1e-13 * scale
    assert np.abs(ts.run_chase(B, ts.chase_schedule(n, b, lag=2)) - ref).max() > 1e-3 * scale


def _harness(tmp_path):
    """Builds tests/chase_harness.cu (host code only) with nvcc; skips without nvcc."""
    import os
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    here = os.path.dirname(os.path.abspath(__file__))
    exe = str(tmp_path / "chase_harness")
    subprocess.run([nvcc, "-x", "cu", "-std=c++17", "-O2",
                    "-I", os.path.join(here, "..", "exciting_b200", "csrc"),
                    os.path.join(here, "chase_harness.cu"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("n,b", [(40, 4), (97, 8), (150, 16), (70, 32)])
def test_chase_task_on_band_storage_matches_dense_chase(tmp_path, n, b):
    """exciting_b200/csrc/chase.cuh (compact band storage with bulge room),
    run on the host sweep by sweep, reproduces the dense chase and its
    reflectors."""
    import subprocess
    exe = _harness(tmp_path)
    C = _herm(n, np.random.default_rng(3 * n + b))
    B, _, _ = ts.he2hb(C, b)
    ld = 2 * b + 1
    ab = np.zeros((n, ld), dtype=np.complex128)  # row c = column c of the storage
    for c in range(n):
        for off in range(0, min(b, n - 1 - c) + 1):
            ab[c, off] = B[c + off, c]
    (tmp_path / "band.bin").write_bytes(ab.tobytes())
    subprocess.run([exe, str(n), str(b), str(tmp_path / "band.bin"), str(tmp_path / "out.bin"),
                    str(tmp_path / "refl.bin")], check=True)
    out = np.frombuffer((tmp_path / "out.bin").read_bytes(), dtype=np.complex128).reshape(n, ld)
    dense = ts.run_chase(B, ts.chase_tasks(n, b))
    scale = np.abs(B).max()
    for c in range(n):
        for off in range(0, min(2 * b, n - 1 - c) + 1):
            assert abs(out[c, off] - dense[c + off, c]) < 1e-12 * scale, (c, off)
    # tridiagonal: everything below the subdiagonal is gone
    assert np.abs(out[:, 2:]).max() < 1e-12 * scale
    # the reflectors agree with hb2st's
    _, _, _, refl = ts.hb2st(B, b)
    rec = np.frombuffer((tmp_path / "refl.bin").read_bytes(), dtype=np.complex128)
    pos = 0
    for (i, lo, v, tau) in refl:
        hdr_i, hdr_lo = int(rec[pos].real), int(rec[pos].imag)
        ln = int(rec[pos + 1].real)
        assert (hdr_i, hdr_lo, ln) == (i, lo, len(v))
        assert abs(rec[pos + 2] - tau) < 1e-12
        assert np.abs(rec[pos + 3:pos + 3 + ln] - v).max() < 1e-10
        pos += 3 + ln
    assert pos == len(rec)


@pytest.mark.parametrize("n,b,m", [(60, 4, 4), (97, 8, 8), (150, 16, 8), (130, 32, 16), (40, 8, 1)])
def test_chase_back_transform_in_blocks(n, b, m):
    """Step-ascending, sweep-descending order with m sweeps per block reflector
    reproduces Q2 Z of the chase reflectors."""
    rng = np.random.default_rng(n + b + m)
    B, _, _ = ts.he2hb(_herm(n, rng), b)
    _, _, _, refl = ts.hb2st(B, b)
    Z = rng.standard_normal((n, 11)) + 1j * rng.standard_normal((n, 11))
    assert np.abs(ts.apply_q2_blocked(refl, Z, m) - ts.apply_q2(refl, Z)).max() < 1e-13


def test_chase_task_compiles_for_the_device(tmp_path):
    """chase.cuh's task is __host__ __device__: its sm_100a device build
    compiles (a one-thread wrapper; compile only, nothing runs)."""
    import os
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    here = os.path.dirname(os.path.abspath(__file__))
    src = tmp_path / "chase_device.cu"
    src.write_text('#include "chase.cuh"\n'
                   "__global__ void k_chase_one(BandView B, int col, int lo, int hi, cplx* v, cplx* tau,\n"
                   "                            cplx* work) {\n"
                   "  if (threadIdx.x == 0 && blockIdx.x == 0) chase_task(B, col, lo, hi, v, tau, work);\n"
                   "}\n")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-c",
                    "-I", os.path.join(here, "..", "exciting_b200", "csrc"), str(src),
                    "-o", str(tmp_path / "chase_device.o")], check=True)
