"""CPU restatement of tensor-tools' Davidson eigensolvers.

TEST INFRASTRUCTURE ONLY -- the parity oracle; see ``oracle/qtensor.py``.

* ``DIAG`` follows linalg/lapack_wrapper.cpp:40-54 (``dsyev('V','U')`` in place
  on a column-major array); scipy's ``eigh(driver='ev')`` is the same LAPACK
  routine.
* ``tensor_davidsonIT`` follows linalg/tensor_davidson.cpp:193-347 (the QN
  path), including the M/Mnext bookkeeping, the sign flip, the convergence
  rule and the random refill on Gram-Schmidt failure (seeded here; the
  reference uses CTF's unseeded ``fill_random``).
* ``tensor_davidson`` follows linalg/tensor_davidson.cpp:74-184 (the dense
  path) with ``elemWiseDivide`` (:25-36).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla


def DIAG(n: int, M: np.ndarray, evals: np.ndarray) -> None:
    """In-place dsyev on the leading n*n entries of flat column-major ``M``."""
    A = M[: n * n].reshape((n, n), order="F").copy()
    w, v = sla.eigh(A, lower=False, driver="ev")
    evals[:n] = w
    M[: n * n] = v.reshape(-1, order="F")


class DavidsonStats:
    def __init__(self):
        self.matvecs = 0
        self.iters = 0
        self.randomized = 0


def tensor_davidsonIT(A, x, m: int, max_restart: int, tol: float, mode: str = "S",
                      rng: np.random.Generator | None = None,
                      stats: DavidsonStats | None = None) -> float:
    """linalg/tensor_davidson.cpp:193-347.  ``A`` offers product(), size();
    ``x`` offers copy/norm/scale/add/contract/inner_product/set_random."""
    assert m >= 1 and max_restart >= 1 and tol > 0
    if rng is None:
        rng = np.random.default_rng(12345)
    x_norm = x.norm()
    x.scale(1.0 / x_norm)
    maxsize = A.size()
    actual_maxiter = min(max_restart, maxsize - 1)
    nsz = actual_maxiter + 2
    v = [None] * nsz
    va = [None] * nsz
    M = np.zeros(nsz * nsz)
    Mnext = np.zeros(nsz * nsz)
    evals = np.zeros(nsz)
    last_lambda = 1000.0
    Approx0 = 1e-12
    v[0] = x.copy()
    va[0] = A.product(v[0])
    if stats is not None:
        stats.matvecs += 1
    initEn = va[0].inner_product(v[0])
    lam = 0.0
    for ii in range(actual_maxiter + 1):
        ni = ii + 1
        if ii == 0:
            lam = initEn
            for mi in range(ni):
                M[mi] = lam
                Mnext[mi] = lam
            q = va[0].copy()
            q.add(v[0], -lam)
        else:
            for mi in range(ni):
                for mj in range(mi + 1):
                    Mnext[mj + mi * (ni + 1)] = M[mj + mi * ni]
                    Mnext[mi + mj * (ni + 1)] = M[mi + mj * ni]
            DIAG(ni, M, evals)
            lam = float(evals[0])
            xn = v[0].copy()
            xn.scale(M[0])
            q = va[0].copy()
            q.scale(M[0])
            for k in range(1, ii + 1):
                xn.add(v[k], M[k])
                q.add(va[k], M[k])
            q.add(xn, -lam)
            if M[0] < 0.0:
                xn.scale(-1.0)
                q.scale(-1.0)
            x.__dict__.update(xn.copy().__dict__)
        v[ni] = q
        if stats is not None:
            stats.iters = ii
        qnorm = q.norm()
        converged = (qnorm < tol and abs(lam - last_lambda) < tol) or qnorm < max(Approx0, tol * 1e-3)
        last_lambda = lam
        if qnorm < 1e-20 or (converged and ii >= 1) or ii == actual_maxiter:
            break
        Npass = 1
        Vq = [0.0] * ni
        pss = 1
        tot_pass = 0
        done = False
        while pss <= Npass:
            tot_pass += 1
            for k in range(ni):
                Vq[k] = q.contract(v[k])
            for k in range(ni):
                q.add(v[k], -Vq[k])
            qnrm = q.norm()
            if qnrm < 1e-10:
                # orthogonalisation failure: refill with random numbers (:298-316)
                q = v[ni - 1].copy()
                q.set_random(rng)
                v[ni] = q
                if stats is not None:
                    stats.randomized += 1
                qnrm = q.norm()
                pss -= 1
                if ni >= maxsize or tot_pass > Npass * 3:
                    done = True
                    break
            q.scale(1.0 / qnrm)
            pss += 1
        if done:
            break
        va[ni] = A.product(v[ni])
        if stats is not None:
            stats.matvecs += 1
        M, Mnext = Mnext, M
        l = ni
        for k in range(ni + 1):
            M[l + k * (ni + 1)] = va[l].inner_product(v[k])
            M[k + l * (ni + 1)] = M[l + k * (ni + 1)]
    x.normalize()
    return lam


def elem_wise_divide(x, theta: float, D) -> None:
    """elemWiseDivide (linalg/tensor_davidson.cpp:25-36): x /= (D - theta) where D != theta."""
    d = D.data
    mask = d != theta
    x.data[mask] = x.data[mask] / (d[mask] - theta)


def tensor_davidson(A, x, m: int, max_restart: int, tol: float, mode: str = "S",
                    stats: DavidsonStats | None = None) -> float:
    """linalg/tensor_davidson.cpp:74-184 (restarted, diagonal-preconditioned)."""
    assert m >= 1 and max_restart >= 1 and tol > 0
    v = [None] * m
    va = [None] * m
    D = A.diagonal()
    M = np.zeros((m + 1) * (m + 1))
    Mnext = np.zeros((m + 1) * (m + 1))
    evals = np.zeros(m)
    ev = 0.0
    r_norm = 0.0
    u = ua = None
    for i in range(max_restart):
        for j in range(m):
            v[j] = x.copy()
            for k in range(j - 1, -1, -1):
                alpha = v[k].inner_product(v[j])
                v[j].add(v[k], -alpha)
            v[j].normalize()
            va[j] = A.product(v[j])
            if stats is not None:
                stats.matvecs += 1
            l = j
            for k in range(j + 1):
                M[l + k * (j + 1)] = va[l].inner_product(v[k])
                M[k + l * (j + 1)] = M[l + k * (j + 1)]
            for k in range(j + 1):
                for l2 in range(k + 1):
                    Mnext[l2 + k * (j + 2)] = M[l2 + k * (j + 1)]
                    Mnext[k + l2 * (j + 2)] = M[k + l2 * (j + 1)]
            if j > 0:
                DIAG(j + 1, M, evals)
                if mode == "S":
                    ev = float(evals[0])
                    for k in range(j + 1):
                        if k == 0:
                            u = v[k].copy(); u.scale(M[0])
                            ua = va[k].copy(); ua.scale(M[0])
                        else:
                            u.add(v[k], M[k])
                            ua.add(va[k], M[k])
                else:
                    ev = float(evals[j])
                    for k in range(j + 1):
                        if k == 0:
                            u = v[k].copy(); u.scale(M[j * (j + 1)])
                            ua = va[k].copy(); ua.scale(M[j * (j + 1)])
                        else:
                            u.add(v[k], M[k + j * (j + 1)])
                            ua.add(va[k], M[k + j * (j + 1)])
            else:
                ev = float(M[0])
                u = v[0].copy()
                ua = va[0].copy()
            ua.add(u, -ev)
            r = ua.copy()
            r_norm = r.norm()
            if j < m - 1:
                x = _assign(x, r)
                elem_wise_divide(x, ev, D)
                x.normalize()
            M, Mnext = Mnext, M
        x = _assign(x, u)
        if stats is not None:
            stats.iters += 1
        if r_norm < tol:
            break
    return ev


def _assign(dst, src):
    dst.__dict__.update(src.copy().__dict__)
    return dst
