"""Host logic of bench.py that needs no GPU: the reference arm's mid-chain
problem on the J1-J2 cylinder (oracle only, small bond dimension here).

The reference arm times real oracle two-site updates on environments
contracted through a Neel product state with random canonical windows; these
checks pin that construction: the window tensors are isometries, the
effective Hamiltonian built from the environments is symmetric, and an update
runs the oracle's own update_site / update_env and lowers the energy."""
import numpy as np

import bench
from oracle import qdmrg
from oracle.qtensor import contract


def _isometry_error(T, left_canonical):
    """max |A^T A - I| per sector of the new bond (blocks stacked as in the builder)."""
    na = 2 if left_canonical else 0
    err = 0.0
    for q in range(T.idx[na].size()):
        bl = [b for b, qi in enumerate(T.bqi) if qi[na] == q and np.any(T.blocks[b])]
        if not bl:
            continue
        if left_canonical:
            M = np.vstack([T.blocks[b].reshape(-1, T.blocks[b].shape[2], order="F") for b in bl])
        else:
            M = np.vstack([T.blocks[b].reshape(T.blocks[b].shape[0], -1, order="F").T for b in bl])
        err = max(err, np.abs(M.T @ M - np.eye(M.shape[1])).max())
    return err


def test_reference_mid_chain_problem_small():
    om = bench.OracleMidChain(chi=24, max_restart=2, w=5, seed=3)
    m = om.m
    assert om.bond_dims[0] == 24 and om.bond_dims[2] == 24
    for i in range(m - 5, m):
        assert _isometry_error(om.psi.A[i], True) < 1e-12
    for i in range(m + 2, m + 7):
        assert _isometry_error(om.psi.A[i], False) < 1e-12
    # symmetric effective Hamiltonian: <y|H x> = <H y|x>
    A = qdmrg.BigQTensor()
    A.setLeft(om.TL[m])
    A.addMid(om.H.A[m])
    A.addMid(om.H.A[m + 1])
    A.setRight(om.TR[m + 1])
    rng = np.random.default_rng(0)
    x = contract(om.psi.A[m], om.psi.A[m + 1])
    y = x.copy()
    for b in y.blocks:
        b[...] = rng.standard_normal(b.shape)
    lhs = y.inner_product(A.product(x))
    rhs = A.product(y).inner_product(x)
    assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs))
    e0 = A.expec(x) / x.inner_product(x)
    e1 = om.update()
    e2 = om.update()
    assert np.isfinite(e1) and e1 < e0 and e2 <= e1 + 1e-9
