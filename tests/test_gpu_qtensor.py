"""Parity of the CUDA qtensor path with the CPU oracle (FP64).

Random block-sparse tensors with U(1) sectors go through the C ABI
(contraction, vector ops, block SVD, big_qtensor product, Davidson) and are
compared block by block with the oracle's restatement of the reference.
Structure (block keys, sector positions, dims, kept counts) must match
exactly; values within 1e-12 relative to the largest entry.
"""
import numpy as np
import pytest

from oracle import qdmrg, qsvd
from oracle.davidson import tensor_davidsonIT
from oracle.qtensor import QIndex, QTensor, Inward, Outward, Link, Site, contract, qn, to_dense

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    import tt_b200
    c = tt_b200.Context(0)
    yield c
    c.close()


def _index(arrow, name, sectors, typ=Link, level=0):
    ix = QIndex(arrow, name, typ, level)
    for q, d in sectors:
        ix.add_qn(qn(q), d)
    return ix


def _random(idx, rng, drop=0.0):
    T = QTensor(idx)
    T.init_block()
    if drop:
        keep = [i for i in range(len(T.blocks)) if rng.random() >= drop or i == 0]
        R = QTensor(idx)
        R.initted = True
        for i in keep:
            R._append_block(T.bqn[i], T.bqi[i], T.bqd[i], rng.standard_normal(T.bqd[i]))
        return R
    for b in T.blocks:
        b[...] = rng.standard_normal(b.shape)
    return T


def assert_same(gpu, ora, tol=TOL):
    import tt_b200
    assert len(ora.blocks) > 0 and ora.norm() > 0, "vacuous comparison"
    got = gpu.to_oracle() if isinstance(gpu, tt_b200.QTensor) else gpu
    assert [ix.tag() for ix in got.idx] == [ix.tag() for ix in ora.idx]
    assert sorted(got.bid.keys()) == sorted(ora.bid.keys())
    scale = max([1.0] + [float(np.max(np.abs(b))) for b in ora.blocks if b.size])
    for key, i in ora.bid.items():
        j = got.bid[key]
        assert got.bqi[j] == ora.bqi[i] and got.bqd[j] == ora.bqd[i]
        np.testing.assert_allclose(got.blocks[j], ora.blocks[i], rtol=0, atol=tol * scale)


def _two_site(rng, chi=(4, 3, 2)):
    """(a, s1, s2, b) with 2Sz charges: a + s1 + s2 = b for every legal block."""
    sec_l = [(-2, chi[0]), (0, chi[1]), (2, chi[2])]
    sec_r = [(-4, chi[2]), (-2, chi[0]), (0, chi[1]), (2, chi[0]), (4, chi[2])]
    a = _index(Inward, "a", sec_l)
    s1 = _index(Inward, "s1", [(-1, 1), (1, 1)], Site)
    s2 = _index(Inward, "s2", [(-1, 1), (1, 1)], Site)
    b = _index(Outward, "b", sec_r)
    return [a, s1, s2, b]


def test_contract_matches_oracle(ctx):
    import tt_b200
    rng = np.random.default_rng(1)
    idx = _two_site(rng, (17, 33, 9))
    X = _random(idx, rng)
    # environment-like tensor contracting the first index
    ap = _index(Inward, "a", [(-2, 17), (0, 33), (2, 9)], Link, 1)
    w = _index(Outward, "w", [(-2, 1), (0, 3), (2, 1)])
    L = _random([ap, w, idx[0].dagged()], rng)
    want = contract(L, X)
    got = tt_b200.QTensor.from_oracle(L) * tt_b200.QTensor.from_oracle(X)
    assert_same(got, want)


def test_contract_permuted_and_multi_index(ctx):
    import tt_b200
    rng = np.random.default_rng(2)
    idx = _two_site(rng, (5, 7, 3))
    X = _random(idx, rng)
    # contract s1 and b (non-adjacent, permuted) against a tensor holding them in reverse order
    c = _index(Outward, "c", [(-1, 4), (1, 6), (3, 2)])
    Y = _random([idx[3].dagged(), c, idx[1].dagged()], rng)
    want = contract(X, Y)
    got = tt_b200.QTensor.from_oracle(X) * tt_b200.QTensor.from_oracle(Y)
    assert_same(got, want)
    # and the other operand order
    want2 = contract(Y, X)
    got2 = tt_b200.QTensor.from_oracle(Y) * tt_b200.QTensor.from_oracle(X)
    assert_same(got2, want2)


def test_contract_missing_blocks_creates_empty_outputs(ctx):
    """Output blocks exist for every (left, right) tuple pair with matching
    mid-QN, also when no block pair contributes (qtensor.cpp:689-694)."""
    import tt_b200
    rng = np.random.default_rng(3)
    idx = _two_site(rng, (3, 4, 2))
    X = _random(idx, rng, drop=0.5)
    ap = _index(Inward, "a", [(-2, 3), (0, 4), (2, 2)], Link, 1)
    w = _index(Outward, "w", [(-2, 1), (0, 3), (2, 1)])
    L = _random([ap, w, idx[0].dagged()], rng, drop=0.5)
    want = contract(L, X)
    got = tt_b200.QTensor.from_oracle(L) * tt_b200.QTensor.from_oracle(X)
    assert_same(got, want)


def test_vector_ops(ctx):
    import tt_b200
    rng = np.random.default_rng(4)
    idx = _two_site(rng, (6, 8, 5))
    A = _random(idx, rng)
    B = _random(idx, rng, drop=0.4)
    gA, gB = tt_b200.QTensor.from_oracle(A), tt_b200.QTensor.from_oracle(B)
    assert abs(gA.norm() - A.norm()) <= 1e-13 * A.norm()
    assert abs(gA.inner_product(gB) - A.inner_product(B)) <= 1e-12 * A.norm() * B.norm()
    assert abs(gB.inner_product(gA) - B.inner_product(A)) <= 1e-12 * A.norm() * B.norm()
    # add with block insertion (qtensor.cpp:1127-1156)
    C = B.copy()
    C.add(A, -0.75)
    gC = gB.copy()
    gC.add(gA, -0.75)
    assert_same(gC, C)
    gA.scale(2.5)
    A.scale(2.5)
    assert_same(gA, A)


@pytest.mark.parametrize("direction", [qsvd.MoveFromLeft, qsvd.MoveFromRight])
@pytest.mark.parametrize("cutoff,K", [(0.0, 0), (1e-6, 0), (0.0, 12), (1e-3, 20)])
def test_block_svd_matches_oracle(ctx, direction, cutoff, K):
    import tt_b200
    rng = np.random.default_rng(5)
    idx = _two_site(rng, (7, 9, 4))
    X = _random(idx, rng)
    # graded spectrum so the cuts are away from ties
    for b in X.blocks:
        b *= rng.uniform(0.05, 1.0)
    info = qsvd.TruncInfo()
    U, V, S = qsvd.svd(X, X.idx[:2], X.idx[2:], direction, cutoff, K, info)
    assert len(X.blocks) > 10 and info.kept > 0
    gU, gV, gS, te, kept = tt_b200.svd(tt_b200.QTensor.from_oracle(X), [0, 1], direction, cutoff, K)
    assert kept == info.kept
    assert abs(te - info.trunc_err) < 1e-12
    oS = gS.to_oracle()
    assert sorted(oS.bid.keys()) == sorted(S.bid.keys())
    for key, i in S.bid.items():
        np.testing.assert_allclose(oS.blocks[oS.bid[key]], S.blocks[i], rtol=1e-10, atol=1e-13)
    # gauge-invariant check: U*V equals the oracle's U*V
    oU, oV = gU.to_oracle(), gV.to_oracle()
    assert sorted(oU.bid.keys()) == sorted(U.bid.keys())
    assert sorted(oV.bid.keys()) == sorted(V.bid.keys())
    want = to_dense(contract(U, V))
    got = to_dense(contract(oU, oV))
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-11 * np.max(np.abs(want)))
    # the canonical side is orthonormal
    canon = oU if direction == qsvd.MoveFromLeft else oV
    M = to_dense(canon)
    M = M.reshape(-1, M.shape[-1]) if direction == qsvd.MoveFromLeft else M.reshape(M.shape[0], -1).T
    np.testing.assert_allclose(M.T @ M, np.eye(M.shape[1]), atol=1e-12)


def _dmrg_state(L=10, sweeps=2, maxm=16, seed=7, site=0):
    """A converged oracle state with its orthogonality centre on `site`, the
    right environments TR of the right-orthonormal tensors and the left
    environments TL[0..site] of the left-orthonormal ones (so sites `site`
    and `site`+1 see non-trivial environments on both sides)."""
    rng = np.random.default_rng(seed)
    h = list(rng.uniform(-0.1, 0.1, L))
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    H = qdmrg.QMPO(L, dh=h)
    qdmrg.dmrg(psi, H, sweeps, [maxm], [1e-12], [4])
    psi.position(0)
    TR, TL = qdmrg.build_env(psi, H)
    psi.position(site)  # changes A[0..site] only: TR[site+1] stays valid
    for i in range(site):
        TL[i + 1] = qdmrg.env_step(TL[i], psi.A[i], H.A[i])
    return psi, H, TR, TL, h


def _mid_chain_operator(psi, H, TR, TL, site):
    import tt_b200
    A = qdmrg.BigQTensor()
    A.setLeft(TL[site])
    A.addMid(H.A[site])
    A.addMid(H.A[site + 1])
    A.setRight(TR[site + 1])
    op = tt_b200.BigQTensor(tt_b200.QTensor.from_oracle(TL[site]), tt_b200.QTensor.from_oracle(H.A[site]),
                            tt_b200.QTensor.from_oracle(H.A[site + 1]), tt_b200.QTensor.from_oracle(TR[site + 1]))
    return A, op, contract(psi.A[site], psi.A[site + 1])


@pytest.mark.parametrize("site", [0, 4])
def test_heff_product_matches_oracle(ctx, site):
    """H_eff*x at the chain edge (trivial left boundary) and mid-chain (L, R
    with several QN sectors on both sides)."""
    import tt_b200
    psi, H, TR, TL, _ = _dmrg_state(site=site)
    A, op, x = _mid_chain_operator(psi, H, TR, TL, site)
    if site > 0:
        assert len(TL[site].blocks) > 4 and len(TR[site + 1].blocks) > 4
    want = A.product(x)
    got = op.product(tt_b200.QTensor.from_oracle(x))
    assert_same(got, want, tol=1e-11)
    assert op.size() == A.size()


@pytest.mark.parametrize("site", [0, 5])
def test_davidson_matches_oracle(ctx, site):
    import tt_b200
    psi, H, TR, TL, _ = _dmrg_state(L=12, sweeps=1, maxm=12, site=site)
    A, op, x = _mid_chain_operator(psi, H, TR, TL, site)
    gx = tt_b200.QTensor.from_oracle(x)
    xo = x.copy()
    e_ref = tensor_davidsonIT(A, xo, 3, 6, 1e-12)
    e_gpu, mv = op.davidson(gx, 6, 1e-12)
    assert abs(e_gpu - e_ref) <= 1e-10 * abs(e_ref)
    got = gx.to_oracle()
    assert sorted(got.bid.keys()) == sorted(xo.bid.keys())
    sgn = np.sign(got.inner_product(xo))
    for key, i in xo.bid.items():
        np.testing.assert_allclose(sgn * got.blocks[got.bid[key]], xo.blocks[i], atol=1e-9)


@pytest.mark.parametrize("side", ["left", "right"])
def test_env_update_matches_oracle(ctx, side):
    """tt_qtensor_env_update against the oracle's env_step (algos/dmrg/dmrg.cpp:
    491-509): a left environment extended over a left-orthonormal site, and a
    right one over a right-orthonormal site, both mid-chain."""
    import tt_b200
    site = 4
    psi, H, TR, TL, _ = _dmrg_state(site=site)
    k = site - 1 if side == "left" else site + 3
    env = TL[k] if side == "left" else TR[k]
    assert len(env.blocks) > 4
    want = qdmrg.env_step(env, psi.A[k], H.A[k])
    got = tt_b200.env_update(tt_b200.QTensor.from_oracle(env), tt_b200.QTensor.from_oracle(psi.A[k]),
                             tt_b200.QTensor.from_oracle(H.A[k]))
    assert_same(got, want, tol=1e-12)
    if side == "left":
        assert_same(got, TL[k + 1], tol=1e-12)


@pytest.mark.parametrize("direction", [qsvd.MoveFromLeft, qsvd.MoveFromRight])
def test_svd_bond_reports_kept_states_per_sector(ctx, direction):
    """tt_qtensor_svd_bond_sectors: the same factors as svd_bond, with the
    kept count of every mid-QN sector equal to the oracle's truncation log."""
    import tt_b200
    site = 4
    psi, H, TR, TL, _ = _dmrg_state(site=site)
    x = contract(psi.A[site], psi.A[site + 1])
    mid = [ix for ix in psi.A[site].idx if any(ix.tag() == jx.dagged().tag() for jx in psi.A[site + 1].idx)][0]
    info = qsvd.TruncInfo()
    U, V, S = qsvd.svd_bond(x, psi.A[site], psi.A[site + 1], mid, direction, 1e-8, 10, info)
    gl, gr = tt_b200.QTensor.from_oracle(psi.A[site]), tt_b200.QTensor.from_oracle(psi.A[site + 1])
    mid_axis = [ix.tag() for ix in psi.A[site].idx].index(mid.tag())
    gS, te, kept, sectors = tt_b200.svd_bond_sectors(tt_b200.QTensor.from_oracle(x), gl, gr, mid_axis,
                                                      direction, 1e-8, 10)
    assert kept == info.kept and kept <= 10
    assert abs(te - info.trunc_err) < 1e-12
    assert [q for q, _ in sectors] == [tuple(q) for q in info.sector_qn]
    assert [k for _, k in sectors] == list(info.kept_per_sector)
    assert sum(k for _, k in sectors) == kept
    oS = gS.to_oracle()
    for key, i in S.bid.items():
        np.testing.assert_allclose(oS.blocks[oS.bid[key]], S.blocks[i], rtol=1e-10, atol=1e-13)
