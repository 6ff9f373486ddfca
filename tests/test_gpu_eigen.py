"""The block SVD's two-phase symmetric eigensolver, called directly through the C ABI.

``tt_sym_eigvals_batched`` / ``tt_sym_eigvecs_batched`` diagonalise the
per-QN-sector density matrices of ``svd_bond`` (qtensor/qtensor_op.cpp:1229-1300).
Sectors up to n = 160 run on one CTA with the matrix in shared memory; larger
ones run on a thread-block cluster.  One batch here mixes both kinds, with
density-matrix-like spectra (exponential decay down to 1e-14 of the largest
eigenvalue, so most kept eigenvalues fall into one cluster of close values),
a rank-deficient matrix (exact zero eigenvalues) and a matrix with exactly
degenerate pairs.  The oracle is LAPACK (numpy ``eigh``): eigenvalues within
1e-12 ||G||, eigenvector residuals ||G z - lambda z|| within 1e-10 ||G||,
orthonormality within 1e-10, and the gauge (largest-magnitude entry positive).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class EigProblem(C.Structure):
    _fields_ = [("g_off", C.c_int64), ("w_off", C.c_int64), ("a_off", C.c_int64),
                ("n", C.c_int32), ("flags", C.c_int32)]


def _bind():
    import tt_b200
    lib = tt_b200.lib
    P = C.c_void_p
    lib.tt_sym_eigvals_batched.restype = C.c_int
    lib.tt_sym_eigvals_batched.argtypes = [P, C.POINTER(EigProblem), C.c_int, P, P, P, P]
    lib.tt_sym_eigvecs_batched.restype = C.c_int
    lib.tt_sym_eigvecs_batched.argtypes = [P, C.POINTER(EigProblem), C.c_int, C.POINTER(C.c_int), P, P, P,
                                           P, P, P]
    return tt_b200, lib


def _density_matrix(n, rng, kind):
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    if kind == "decay":
        lam = np.exp(-np.linspace(0.0, np.log(1e14), n)) * rng.uniform(0.5, 1.0, n)
    elif kind == "rank":
        r = n // 3
        lam = np.concatenate([np.exp(-np.linspace(0.0, 20.0, r)), np.zeros(n - r)])
    else:  # exactly degenerate pairs
        base = np.exp(-np.linspace(0.0, 25.0, (n + 1) // 2))
        lam = np.repeat(base, 2)[:n]
    G = (Q * lam) @ Q.T
    return 0.5 * (G + G.T)


@pytest.mark.parametrize("seed", [0, 1])
def test_batched_eigensolver_small_and_cluster_sectors(seed):
    import torch
    tt_b200, lib = _bind()
    rng = np.random.default_rng(seed)
    cases = [(24, "decay"), (161, "decay"), (300, "rank"), (578, "decay"), (140, "degenerate"),
             (700, "degenerate"), (1100, "decay"), (195, "decay"), (1630, "decay")]
    if seed == 1:
        cases.append((2600, "decay"))  # beyond the former 2048 cap; narrower panels
    mats = [_density_matrix(n, rng, kind) for n, kind in cases]
    ns = [m.shape[0] for m in mats]
    g_off = np.concatenate([[0], np.cumsum([n * n for n in ns])[:-1]]).astype(np.int64)
    w_off = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64)
    total = int(sum(n * n for n in ns))
    probs = (EigProblem * len(ns))(*[EigProblem(int(g), int(w), 0, n, 0) for g, w, n in zip(g_off, w_off, ns)])
    nvec = [min(n, 2048, n // 2 + 7) for n in ns]
    nvec_c = (C.c_int * len(ns))(*nvec)
    ctx = tt_b200.Context(0)
    try:
        for repeat in range(2):  # two calls in a row on the same buffers
            G = torch.tensor(np.concatenate([m.reshape(-1, order="F") for m in mats]), dtype=torch.float64,
                             device="cuda")
            T = torch.zeros(3 * sum(ns), dtype=torch.float64, device="cuda")
            w = torch.zeros(sum(ns), dtype=torch.float64, device="cuda")
            Z = torch.full((total,), float("nan"), dtype=torch.float64, device="cuda")
            work = torch.zeros(3 * total, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            rc = lib.tt_sym_eigvals_batched(ctx.h, probs, len(ns), G.data_ptr(), T.data_ptr(), w.data_ptr(), None)
            assert rc == 0, lib.tt_get_last_error()
            rc = lib.tt_sym_eigvecs_batched(ctx.h, probs, len(ns), nvec_c, G.data_ptr(), T.data_ptr(),
                                            w.data_ptr(), Z.data_ptr(), work.data_ptr(), None)
            assert rc == 0, lib.tt_get_last_error()
            ctx.sync()
            wh, Zh = w.cpu().numpy(), Z.cpu().numpy()
            for p, M in enumerate(mats):
                n, k = ns[p], nvec[p]
                gnorm = np.linalg.norm(M, 2)
                ref = np.linalg.eigvalsh(M)[::-1]
                got = wh[w_off[p]:w_off[p] + n]
                assert np.all(np.diff(got) <= 0.0)
                assert np.abs(got - ref).max() <= 1e-12 * gnorm, (n, np.abs(got - ref).max())
                V = Zh[g_off[p]:g_off[p] + n * k].reshape(n, k, order="F")
                resid = np.linalg.norm(M @ V - V * got[:k], axis=0).max()
                assert resid <= 1e-10 * gnorm, (n, resid)
                assert np.abs(V.T @ V - np.eye(k)).max() <= 1e-10, n
                idx = np.argmax(np.abs(V), axis=0)
                assert np.all(V[idx, np.arange(k)] > 0.0)
    finally:
        ctx.close()
