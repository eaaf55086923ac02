"""Tile lists of the grouped GEMM (the host side of zgemm_grouped_kernel in
exciting_b200/csrc/zgemm.cu), built on the CPU by tests/group_tiles_harness.cu:
for products of different sizes and triangular structure (the grouped
Cholesky, inverse factor and two-sided reduction use all of them) every
element of each product's written triangle lies in exactly one listed tile,
no tile lies wholly outside it, each tile's K range is the one its
triangular operands allow, and a launch lists its tiles longest K range
first."""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
NONE, LOWER, UPPER = 0, 1, 2
BN = 64

# (m, n, k, uplo_c, tri_a, tri_b): shapes of the grouped front's products
PRODUCTS = [
    (64, 1900, 64, NONE, LOWER, NONE),      # Cholesky row panel
    (1900, 1900, 64, UPPER, NONE, NONE),    # Cholesky trailing update
    (128, 128, 128, NONE, NONE, UPPER),     # inverse factor: T = U12 X22
    (128, 100, 128, NONE, UPPER, NONE),     # X12 = -X11 T (short second block)
    (2089, 2089, 2089, NONE, NONE, UPPER),  # ZHEGST: T = H U^-1
    (1834, 1834, 1834, UPPER, LOWER, NONE), # ZHEGST: C = U^-H T (upper)
    (70, 33, 5, LOWER, NONE, NONE),
]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    exe = str(tmp_path_factory.mktemp("group_tiles") / "group_tiles_harness")
    subprocess.run([nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(HERE, "..", "exciting_b200", "csrc"),
                    os.path.join(HERE, "group_tiles_harness.cu"), "-o", exe], check=True)
    return exe


def _run(exe, tbm, products):
    inp = "".join(" ".join(map(str, p)) + "\n" for p in products)
    out = subprocess.run([exe, str(tbm)], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    nprob = int(out[0])
    tiles = np.array([list(map(int, l.split())) for l in out[1:] if l.strip()], dtype=np.int64).reshape(-1, 4)
    return nprob, tiles


def _k_range(p, i0, j0, tbm):
    m, n, k, uplo, ta, tb = p
    kbeg, kend = 0, k
    if ta == LOWER:
        kend = min(kend, i0 + tbm)
    if ta == UPPER:
        kbeg = max(kbeg, i0)
    if tb == UPPER:
        kend = min(kend, j0 + BN)
    if tb == LOWER:
        kbeg = max(kbeg, j0)
    return max(0, kend - (kbeg // 8) * 8)


@pytest.mark.parametrize("tbm", [64, 128])
def test_tiles_cover_each_written_triangle_once(harness, tbm):
    nprob, tiles = _run(harness, tbm, PRODUCTS)
    assert nprob == len(PRODUCTS)
    for pi, p in enumerate(PRODUCTS):
        m, n, k, uplo, ta, tb = p
        cover = np.zeros((m, n), dtype=np.int32)
        for _, ti, tj, klen in tiles[tiles[:, 0] == pi]:
            i0, j0 = ti * tbm, tj * BN
            assert 0 <= i0 < m and 0 <= j0 < n
            block = cover[i0:i0 + tbm, j0:j0 + BN]
            block += 1
            r = np.arange(i0, min(m, i0 + tbm))[:, None]
            c = np.arange(j0, min(n, j0 + BN))[None, :]
            if uplo == UPPER:
                assert np.any(r <= c), "tile wholly below the diagonal"
            if uplo == LOWER:
                assert np.any(r >= c), "tile wholly above the diagonal"
            assert klen == _k_range(p, i0, j0, tbm)
        r = np.arange(m)[:, None]
        c = np.arange(n)[None, :]
        need = np.ones((m, n), dtype=bool)
        if uplo == UPPER:
            need = r <= c
        if uplo == LOWER:
            need = r >= c
        assert np.all(cover[need] == 1)
        assert np.all(cover <= 1)


def test_launch_lists_longest_k_range_first(harness):
    _, tiles = _run(harness, 64, PRODUCTS)
    assert np.all(np.diff(tiles[:, 3]) <= 0)
