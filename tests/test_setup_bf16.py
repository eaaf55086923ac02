"""The exact restatement of the split-BF16 setup (oracle/bf16split.py), on the CPU.

- slicing reproduces every entry to the truncation bound 2^-(7 nsl + 1) of
  its column scale, and slices are integers within the BF16-exact range;
- the recombined product approaches the FP64 product as nsl grows, and with
  nsl = 5 its error is below 1e-9 of the largest entry on matching-
  coefficient-like data.
"""
import numpy as np

from oracle import bf16split


def test_slices_are_exact_small_integers():
    rng = np.random.default_rng(1)
    X = (rng.standard_normal((300, 40)) + 1j * rng.standard_normal((300, 40))) * np.exp(rng.uniform(-20, 20, 40))
    sc, sl = bf16split.split(X, 5)
    back = np.zeros_like(X)
    for s, (qr, qi) in enumerate(sl):
        assert np.all(qr == np.rint(qr)) and np.all(qi == np.rint(qi))
        lim = 128 if s == 0 else 64
        assert np.abs(qr).max() <= lim and np.abs(qi).max() <= lim
        back += np.ldexp(1.0, -7 * (s + 1)) * (qr + 1j * qi)
    d = (back * sc[None, :] - X) / sc[None, :]
    assert max(np.abs(d.real).max(), np.abs(d.imag).max()) <= 2.0 ** -(7 * 5 + 1) * 1.0001


def test_product_converges_to_fp64():
    rng = np.random.default_rng(2)
    A = rng.standard_normal((500, 60)) + 1j * rng.standard_normal((500, 60))
    B = rng.standard_normal((500, 50)) + 1j * rng.standard_normal((500, 50))
    exact = A.conj().T @ B
    errs = [np.abs(bf16split.product(A, B, s) - exact).max() / np.abs(exact).max() for s in (3, 4, 5)]
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 1e-9
