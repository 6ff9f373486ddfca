"""Pin the oracle's block SVD with truncation (qtensor/qtensor_op.cpp:1097-1453)
against dense linear algebra on the same two-site tensor.

The two-site tensor x(a, s1, s2, b), reshaped to a (a s1) x (s2 b) matrix, is
block diagonal in the middle U(1) charge, so its singular values are the union
of the per-sector ones.  Checked: without truncation U V reproduces x; with a
rank cap K the kept values are exactly the K largest of that union (with the
per-sector counts they imply) and U V misses exactly the rest, while the
reported truncation error is, as in the reference, relative to the weight of
the per-sector rank-K SVDs; the cutoff rule keeps the fewest values whose
discarded weight is below the cutoff; the 1 x 2 sector special case
(:1247-1267) reproduces its sector exactly.
"""
import numpy as np
import pytest

from oracle import qsvd
from oracle.qtensor import QIndex, QTensor, Inward, Outward, Link, Site, contract, qn, to_dense


def _index(arrow, name, sectors, typ=Link):
    ix = QIndex(arrow, name, typ, 0)
    for q, d in sectors:
        ix.add_qn(qn(q), d)
    return ix


def _two_site(rng, a_secs, b_secs):
    a = _index(Inward, "a", a_secs)
    s1 = _index(Inward, "s1", [(-1, 1), (1, 1)], Site)
    s2 = _index(Inward, "s2", [(-1, 1), (1, 1)], Site)
    b = _index(Outward, "b", b_secs)
    x = QTensor([a, s1, s2, b])
    x.init_block()
    for blk in x.blocks:
        # graded magnitudes so that the global order mixes sectors
        blk[...] = rng.standard_normal(blk.shape) * rng.uniform(0.05, 1.0)
    return x, [a, s1], [s2, b]


def _dense_matrix(x):
    d = to_dense(x)
    return d.reshape(d.shape[0] * d.shape[1], d.shape[2] * d.shape[3])


def _sv(x):
    return np.linalg.svd(_dense_matrix(x), compute_uv=False)


@pytest.mark.parametrize("direction", [qsvd.MoveFromLeft, qsvd.MoveFromRight])
def test_no_truncation_reproduces_the_tensor(direction):
    rng = np.random.default_rng(1)
    x, left, right = _two_site(rng, [(-2, 3), (0, 5), (2, 4)], [(-2, 4), (0, 6), (2, 3)])
    info = qsvd.TruncInfo()
    U, V, S = qsvd.svd(x, left, right, direction, 0.0, 0, info)
    np.testing.assert_allclose(to_dense(contract(U, V)), to_dense(x), rtol=0, atol=1e-12 * np.abs(to_dense(x)).max())
    assert info.trunc_err <= 1e-14


def test_rank_cap_keeps_the_globally_largest_values():
    rng = np.random.default_rng(2)
    x, left, right = _two_site(rng, [(-2, 3), (0, 6), (2, 4)], [(-2, 5), (0, 6), (2, 4)])
    all_sv = _sv(x)
    K = 7
    info = qsvd.TruncInfo()
    U, V, S = qsvd.svd(x, left, right, qsvd.MoveFromLeft, 0.0, K, info)
    kept = np.sort(np.concatenate([np.asarray(b).ravel() for b in S.blocks]))[::-1]
    assert info.kept == K and kept.size == K
    np.testing.assert_allclose(kept, all_sv[:K], rtol=1e-12, atol=0)
    # per-sector counts: how many of the K largest each sector's own values supply
    per = []
    for s in info.svals:
        per.append(int(np.sum(np.asarray(s) >= all_sv[K - 1] * (1 - 1e-12))))
    assert sum(info.kept_per_sector) == K
    assert info.kept_per_sector == per
    # U V misses exactly the discarded singular values
    miss = np.linalg.norm(to_dense(contract(U, V)) - to_dense(x)) ** 2 / np.linalg.norm(to_dense(x)) ** 2
    assert abs(miss - np.sum(all_sv[K:] ** 2) / np.sum(all_sv ** 2)) <= 1e-12
    # the reported error, as in the reference, is relative to the weight of the
    # per-sector rank-K SVDs (each sector is cut to K values before the global sort)
    nm = sum(float(np.sum(np.asarray(v) ** 2)) for v in info.svals)
    assert all(np.asarray(v).size <= K for v in info.svals)
    assert abs(info.trunc_err - (nm - float(np.sum(kept ** 2))) / nm) <= 1e-12


def test_cutoff_keeps_the_fewest_values_below_the_discarded_weight():
    rng = np.random.default_rng(3)
    x, left, right = _two_site(rng, [(-2, 4), (0, 5), (2, 3)], [(-2, 3), (0, 7), (2, 4)])
    w = _sv(x) ** 2
    w = w / w.sum()
    cutoff = 0.05
    discarded = 1.0 - np.cumsum(w)
    expect = int(np.argmax(discarded < cutoff)) + 1  # first k with discarded weight below the cutoff
    info = qsvd.TruncInfo()
    U, V, S = qsvd.svd(x, left, right, qsvd.MoveFromRight, cutoff, 0, info)
    assert info.kept == expect
    assert info.trunc_err < cutoff
    assert abs(info.trunc_err - discarded[expect - 1]) <= 1e-12


def test_one_by_two_sector_is_exact():
    # a sector with one row and two columns takes the ScaLAPACK workaround
    rng = np.random.default_rng(4)
    a = _index(Inward, "a", [(0, 1)])
    s1 = _index(Inward, "s1", [(1, 1)], Site)
    s2 = _index(Inward, "s2", [(-1, 1), (1, 1)], Site)
    b = _index(Outward, "b", [(0, 1), (2, 1)])
    x = QTensor([a, s1, s2, b])
    x.init_block()
    for blk in x.blocks:
        blk[...] = rng.standard_normal(blk.shape)
    assert len(x.blocks) == 2  # one middle sector: 1 row (a s1), 2 columns (s2 b)
    info = qsvd.TruncInfo()
    U, V, S = qsvd.svd(x, [a, s1], [s2, b], qsvd.MoveFromLeft, 0.0, 0, info)
    np.testing.assert_allclose(to_dense(contract(U, V)), to_dense(x), rtol=0, atol=1e-14)
    assert info.kept == 1
