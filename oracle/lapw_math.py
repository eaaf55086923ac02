"""Special functions used by ``match``, restated in NumPy (oracle only).

* ``genylm``   -- ``src/src_lib/genylm.f90:13-94`` (Masters & Richards-Dinger
  recursion, Condon-Shortley phase, packed index lm = l(l+1)+m).
* ``sbessel``  -- ``src/src_lib/sbessel.f90`` (series for x<1e-8, Miller
  downward recurrence with rescaling for x<lmax, upward recurrence otherwise).
* ``sbesseldm`` -- ``src/src_lib/sbesseldm.f90:13-140`` (m-th derivative:
  j_l / j_{l+1} polynomial-in-1/x form for x>1, power series for x<=1).
* ``polynom``  -- ``src/src_lib/polynom.f90:11-190`` (m-th derivative at x of
  the polynomial through np points; closed forms for np<=4).

All functions are vectorised over their sample points.
"""
from __future__ import annotations

import math

import numpy as np

Y00 = 0.28209479177387814347


def genylm(lmax: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Y_lm(theta, phi) for l <= lmax; returns (npts, (lmax+1)**2) complex."""
    theta = np.atleast_1d(np.asarray(theta, float))
    phi = np.atleast_1d(np.asarray(phi, float))
    npt = theta.shape[0]
    out = np.zeros((npt, (lmax + 1) ** 2), dtype=np.complex128)
    out[:, 0] = Y00
    if lmax == 0:
        return out
    sn = np.sin(theta)
    cs = np.cos(theta)
    eim = [None] + [np.cos(m * phi) + 1j * np.sin(m * phi) for m in range(1, lmax + 1)]
    for l in range(1, lmax + 1):
        x = np.zeros((l + 1, npt))
        x[l] = 1.0 if l % 2 == 0 else -1.0
        dx = np.zeros(npt)
        for m in range(l, 0, -1):
            t = math.sqrt(float((l + m) * (l - m + 1)))
            x[m - 1] = -(sn * dx + 2.0 * m * cs * x[m]) / t
            dx = sn * x[m] * t
        scale = sn.copy()
        acc = np.zeros(npt)
        for m in range(1, l + 1):
            x[m] = scale * x[m]
            acc += x[m] ** 2
            scale = scale * sn
        acc = 2.0 * acc + x[0] ** 2
        norm = np.sqrt((2 * l + 1) / (4.0 * math.pi * acc))
        c = l * (l + 1)
        out[:, c] = norm * x[0]
        for m in range(1, l + 1):
            v = norm * x[m] * eim[m]
            out[:, c + m] = v
            out[:, c - m] = np.conj(v) * (-1.0 if m % 2 else 1.0)
    return out


def sbessel(lmax: int, x: np.ndarray) -> np.ndarray:
    """j_l(x), l = 0..lmax; returns (npts, lmax+1)."""
    x = np.atleast_1d(np.asarray(x, float))
    out = np.zeros((x.shape[0], lmax + 1))
    for p, xv in enumerate(x):
        out[p] = _sbessel1(lmax, float(xv))
    return out


def _sbessel1(lmax: int, x: float) -> np.ndarray:
    jl = np.zeros(lmax + 1)
    if x < 1e-8:
        jl[0] = 1.0
        t1 = 1.0
        t2 = 1.0
        for l in range(1, lmax + 1):
            t1 /= (2 * l + 1)
            t2 *= x
            jl[l] = t2 * t1
        return jl
    xi = 1.0 / x
    if x < lmax:
        rsc = 1e150
        rsci = 1.0 / rsc
        j0 = 0.6370354636449841609 * rsci
        j1 = 0.3532702964695481204 * rsci
        lst = 25
        for l in range(lmax + lst, lmax, -1):
            jt = j0 * (2 * l + 1) * xi - j1
            j1 = j0
            j0 = jt
            if abs(j0) > rsc:
                jt *= rsci
                j1 *= rsci
                j0 *= rsci
        for l in range(lmax, -1, -1):
            jt = j0 * (2 * l + 1) * xi - j1
            j1 = j0
            j0 = jt
            if abs(j0) > rsc:
                jt *= rsci
                j1 *= rsci
                j0 *= rsci
                jl[l + 1:] *= rsci
            jl[l] = j1
        t1 = 1.0 / ((jl[0] - x * jl[1]) * math.cos(x) + x * jl[0] * math.sin(x))
        return t1 * jl
    jl[0] = math.sin(x) * xi
    if lmax == 0:
        return jl
    jl[1] = (jl[0] - math.cos(x)) * xi
    j0, j1 = jl[0], jl[1]
    for l in range(2, lmax + 1):
        jt = (2 * l - 1) * j1 * xi - j0
        j0, j1 = j1, jt
        jl[l] = j1
    return jl


def _deriv_coeffs(m: int, l: int):
    """Integer coefficients a_i, b_i with d^m j_l = sum_i (a_i j_l + b_i j_{l+1}) / x^i.

    Built by differentiating term by term with j_l' = (l/x) j_l - j_{l+1} and
    j_{l+1}' = j_l - ((l+2)/x) j_{l+1}.
    """
    a = [0] * (m + 2)
    b = [0] * (m + 2)
    a[0] = 1
    for _ in range(m):
        na = [0] * (m + 2)
        nb = [0] * (m + 2)
        for i in range(m + 1):
            if a[i]:
                na[i + 1] += a[i] * (l - i)
                nb[i] -= a[i]
            if b[i]:
                na[i] += b[i]
                nb[i + 1] -= b[i] * (l + 2 + i)
        a, b = na, nb
    return a, b


def sbesseldm(m: int, lmax: int, x: np.ndarray) -> np.ndarray:
    """m-th derivative of j_l(x), l = 0..lmax; returns (npts, lmax+1)."""
    x = np.atleast_1d(np.asarray(x, float))
    if m == 0:
        return sbessel(lmax, x)
    out = np.zeros((x.shape[0], lmax + 1))
    for p, xv in enumerate(x):
        xv = float(xv)
        if xv > 1.0:
            jl = _sbessel1(lmax + 1, xv)
            for l in range(lmax + 1):
                a, b = _deriv_coeffs(m, l)
                acc = a[0] * jl[l] + b[0] * jl[l + 1]
                t = 1.0
                for i in range(1, m + 2):
                    t *= xv
                    acc += (a[i] * jl[l] + b[i] * jl[l + 1]) / t
                out[p, l] = acc
        else:
            x2 = xv * xv
            for l in range(lmax + 1):
                i0 = max((m - l + 1) // 2, 0)
                j = 2 * i0 + l - m
                t = 1.0 if j == 0 else xv ** j
                # (j+m)!/j! / (i0! (2 i0 + 2l + 1)!! (-2)^i0)
                num = math.factorial(j + m) / math.factorial(j)
                dfac = 1.0
                for k in range(2 * i0 + 2 * l + 1, 0, -2):
                    dfac *= k
                t = num * t / (math.factorial(i0) * dfac * float((-2) ** i0))
                acc = t
                for i in range(i0 + 1, 21):
                    jj = 2 * i + l
                    t = -t * float((jj - 1) * jj) * x2 / float((jj - l) * (jj - m - 1) * (jj - m) * (jj + l + 1))
                    if abs(t) <= 1e-40:
                        break
                    acc += t
                out[p, l] = acc
    return out


def polynom(m: int, xa: np.ndarray, ya: np.ndarray, x: float) -> float:
    """m-th derivative (m >= 0) at x of the polynomial through (xa, ya)."""
    xa = np.asarray(xa, float)
    ya = np.asarray(ya, float)
    npnt = xa.shape[0]
    if m >= npnt:
        return 0.0
    if npnt == 1:
        return float(ya[0]) if m == 0 else 0.0
    if npnt == 2:
        c2 = (ya[1] - ya[0]) / (xa[1] - xa[0])
        t1 = x - xa[0]
        return float(c2 * t1 + ya[0]) if m == 0 else float(c2)
    if npnt == 3:
        x1 = xa[1] - xa[0]; x2 = xa[2] - xa[0]
        y1 = ya[1] - ya[0]; y2 = ya[2] - ya[0]
        t1 = 1.0 / (x1 * x2 * (x2 - x1))
        t2 = x1 * y2; t3 = x2 * y1
        c2 = t1 * (x2 * t3 - x1 * t2)
        c3 = t1 * (t2 - t3)
        t1 = x - xa[0]
        return float([ya[0] + t1 * (c2 + c3 * t1), 2.0 * c3 * t1 + c2, 2.0 * c3][m])
    if npnt == 4:
        x1 = xa[1] - xa[0]; x2 = xa[2] - xa[0]; x3 = xa[3] - xa[0]
        y1 = ya[1] - ya[0]; y2 = ya[2] - ya[0]; y3 = ya[3] - ya[0]
        t1 = 1.0 / (x1 * x2 * x3 * (x1 - x2) * (x1 - x3) * (x2 - x3))
        t2 = x1 * x2 * y3; t3 = x2 * x3 * y1; t4 = x3 * x1 * y2
        t5 = x1 * x1; t6 = x2 * x2; t7 = x3 * x3
        c2 = t1 * (t3 * (x3 * t6 - x2 * t7) + t4 * (x1 * t7 - x3 * t5) + t2 * (x2 * t5 - x1 * t6))
        c3 = t1 * (t3 * (t7 - t6) + t4 * (t5 - t7) + t2 * (t6 - t5))
        c4 = t1 * (t3 * (x2 - x3) + t4 * (x3 - x1) + t2 * (x1 - x2))
        t1 = x - xa[0]
        vals = [ya[0] + t1 * (c2 + t1 * (c3 + c4 * t1)),
                c2 + t1 * (2.0 * c3 + 3.0 * c4 * t1),
                6.0 * c4 * t1 + 2.0 * c3,
                6.0 * c4]
        return float(vals[m])
    # general case: Newton divided differences -> monomials about xa[0]
    c = ya.copy()
    for i in range(1, npnt):
        for j in range(npnt - 1, i - 1, -1):
            c[j] = (c[j] - c[j - 1]) / (xa[j] - xa[j - i])
    if m == 0:
        acc = c[0]
        t = 1.0
        for i in range(1, npnt):
            t *= (x - xa[i - 1])
            acc += c[i] * t
        return float(acc)
    x0 = xa[0]
    for j in range(1, npnt):
        for i in range(1, npnt - j + 1):
            k = npnt - i
            c[k - 1] = c[k - 1] + (x0 - xa[k - j]) * c[k]
    for j in range(1, m + 1):
        for i in range(m, npnt):
            c[i] *= (i - j + 1)
    t1 = c[npnt - 1]
    t2 = x - x0
    for i in range(npnt - 2, m - 1, -1):
        t1 = t1 * t2 + c[i]
    return float(t1)
