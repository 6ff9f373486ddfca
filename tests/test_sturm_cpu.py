"""The bisection of the cluster eigensolver counts eigenvalues below x with
the product form of the Sturm recurrence (no division per step; a vanishing
pivot replaced by a tiny one of the opposite sign, the pair rescaled by
powers of two) instead of the pivot form of LAPACK's dlaebz.  Both forms are
restated here in Python, step for step as the kernel (csrc/tridiag_eig.cu,
sturm_count) and dlaebz take them, and must give the same count on random
and adversarial tridiagonal matrices wherever the count is well defined
(probes further than 1e-9 ||T|| from every eigenvalue: between close
eigenvalues, at zeros of the leading minors, at 0, with split (e = 0) blocks
and large norms); at an eigenvalue itself either count is the exact count of
a matrix within rounding, and the two may differ by the eigenvalues there.
"""
import math

import numpy as np
import scipy.linalg as sla

DBL_MIN = 2.2250738585072014e-308


def count_pivot(d, e2, x, pivmin):
    q = d[0] - x
    if abs(q) <= pivmin:
        q = -pivmin
    c = int(q <= 0.0)
    for i in range(1, len(d)):
        q = d[i] - x - e2[i - 1] / q
        if abs(q) <= pivmin:
            q = -pivmin
        c += q <= 0.0
    return c


def count_product(d, e2, x, pivmin):
    pm = 1.0
    p = d[0] - x
    if abs(p) <= pivmin:
        p = -pivmin
    c = int(p <= 0.0)
    for i in range(1, len(d)):
        pn = math.fma((d[i] - x), p, -e2[i - 1] * pm) if hasattr(math, "fma") else (d[i] - x) * p - e2[i - 1] * pm
        if abs(pn) <= pivmin * abs(p):
            pn = -p * 2.0 ** -200
        c += (pn < 0.0) != (p < 0.0)
        a = abs(pn)
        if a > 2.0 ** 400 or a < 2.0 ** -400:
            sc = 2.0 ** (-math.frexp(pn)[1])
            pn *= sc
            p *= sc
        pm, p = p, pn
    return c


def _check(d, e, xs, ev):
    e2 = e * e
    pivmin = DBL_MIN * max(1.0, float(e2.max()) if len(e2) else 1.0)
    tol = 1e-9 * max(1.0, float(np.abs(ev).max()))
    for x in xs:
        a, b = count_pivot(d, e2, x, pivmin), count_product(d, e2, x, pivmin)
        near = int(np.sum(np.abs(ev - x) <= tol))
        if near == 0:
            assert a == b, x
        else:
            assert abs(a - b) <= near, x


def test_density_matrix_spectra():
    rng = np.random.default_rng(0)
    for trial in range(12):
        n = int(rng.integers(5, 200))
        Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        lam = np.exp(-np.linspace(0, np.log(1e14), n)) * rng.uniform(0.5, 1, n)
        if trial % 3 == 0:
            lam[: n // 3] = 1e-3  # a large cluster
        T, _ = sla.hessenberg((Q * lam) @ Q.T, calc_q=True)
        d, e = np.diag(T).copy(), np.diag(T, -1).copy()
        ev = np.linalg.eigvalsh(T)
        mids = list(0.5 * (ev[1:] + ev[:-1]))  # between neighbours, however close
        xs = list(ev) + mids + [0.0, 1e-300, -1e-300, -0.5, 2.0]
        _check(d, e, xs, ev)


def test_splits_exact_hits_and_large_norms():
    rng = np.random.default_rng(1)
    for n, scale in [(400, 1.0), (300, 1e3), (50, 1.0), (7, 1.0)]:
        d = rng.standard_normal(n) * scale
        e = rng.standard_normal(n - 1) * scale
        e[rng.integers(0, n - 1, n // 10)] = 0.0
        ev = np.linalg.eigvalsh(np.diag(d) + np.diag(e, 1) + np.diag(e, -1))
        xs = list(ev[:: max(1, n // 60)]) + list(0.5 * (ev[1:] + ev[:-1])[:: max(1, n // 60)]) + list(d[:20]) + [0.0]
        _check(d, e, xs, ev)


def _bisect_plain(d, e2, j, lo, hi, open_interval, pivmin):
    """One eigenvalue by plain bisection (the reference walk)."""
    it = 0
    while it < 128 and open_interval(lo, hi):
        mid = 0.5 * (lo + hi)
        if count_product(d, e2, mid, pivmin) > j:
            hi = mid
        else:
            lo = mid
        it += 1
    return 0.5 * (lo + hi), it


def _bisect_multisection(d, e2, j, lo, hi, open_interval, pivmin, levels=4):
    """bisect_sectors: per round, counts at the 2^levels - 1 nodes of the
    bisection tree below the current interval (each node's point computed
    by the chain of midpoints that leads to it), then the walk down the tree
    with those counts."""
    root = 1 << (levels - 1)
    it = 0
    work = open_interval(lo, hi)
    while work:
        counts = {}
        for p in range(1, 2 * root):
            a, b, pos, half = lo, hi, root, root >> 1
            while pos != p:
                m = 0.5 * (a + b)
                if p < pos:
                    b, pos = m, pos - half
                else:
                    a, pos = m, pos + half
                half >>= 1
            counts[p] = count_product(d, e2, 0.5 * (a + b), pivmin)
        pos, half, go = root, root >> 1, True
        for _ in range(levels):
            go = go and it < 128 and open_interval(lo, hi)
            if go:
                mid = 0.5 * (lo + hi)
                if counts[pos] > j:
                    hi, pos = mid, pos - half
                else:
                    lo, pos = mid, pos + half
                half >>= 1
                it += 1
        work = it < 128 and open_interval(lo, hi)
    return 0.5 * (lo + hi), it


def test_multisection_walk_is_plain_bisection_bit_for_bit():
    """The GPU-wide bisection advances four halvings per round from counts
    at the 15 tree nodes; its intervals, and so its eigenvalues and halving
    counts, must be exactly those of plain bisection (graded spectra as in a
    density matrix, and a matrix with close eigenvalues)."""
    rng = np.random.default_rng(11)
    eps = np.finfo(float).eps
    cases = []
    n = 24
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.sort(10.0 ** rng.uniform(-14, 0, n))
    A = (Q * lam) @ Q.T
    T = sla.hessenberg(A)  # tridiagonal: A is symmetric
    cases.append((np.diag(T).copy(), np.diag(T, -1).copy()))
    dd = rng.uniform(-1, 1, n)
    ee = rng.uniform(-1e-3, 1e-3, n - 1)
    cases.append((dd, ee))
    for d, e in cases:
        e2 = e * e
        r = np.abs(np.concatenate([[0.0], e])) + np.abs(np.concatenate([e, [0.0]]))
        gl, gu = float(np.min(d - r)), float(np.max(d + r))
        bnorm = max(abs(gl), abs(gu))
        pivmin = DBL_MIN * max(1.0, float(e2.max()))
        atol = 4.0 * eps * bnorm + 2.0 * pivmin

        def open_interval(lo, hi):
            return hi - lo > max(atol, 2.0 * eps * max(abs(lo), abs(hi)))

        for j in range(len(d)):
            a = _bisect_plain(d, e2, j, gl - atol, gu + atol, open_interval, pivmin)
            b = _bisect_multisection(d, e2, j, gl - atol, gu + atol, open_interval, pivmin)
            assert a == b
