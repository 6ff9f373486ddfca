"""MPS checkpoints (metadata + raw block file) and resuming a DMRG schedule.

A saved and re-loaded MPS is block-for-block identical to the original, its
raw file is exactly the blocks back to back, and resuming the schedule from
the checkpoint reproduces the continuation of the in-memory state.
"""
import os

import numpy as np
import pytest

from oracle import qdmrg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import tt_b200
    c = tt_b200.Context(0)
    yield c
    c.close()


def _blocks(psi):
    out = []
    for i in range(psi.L):
        T = psi.tensor(i).to_oracle()
        out.append(([ix.qns for ix in T.idx], list(T.bqi), [b.copy() for b in T.blocks]))
    return out


def test_qmps_checkpoint_roundtrip_and_resume(ctx, tmp_path):
    import tt_b200
    L = 10
    h = list(np.random.default_rng(17).uniform(-0.1, 0.1, L))
    maxm, cutoff, mr = [8, 16, 32, 32, 32, 32], [1e-10], [6]
    H = tt_b200.QMPO(L, dh=h)
    psi = tt_b200.QMPS(L, qdmrg.neel(L))
    tt_b200.QDMRG(psi, H).run(3, maxm, cutoff, mr)
    fn = str(tmp_path / "psi")
    psi.save(fn)
    assert os.path.exists(fn + ".ttmps") and os.path.exists(fn + "__T.bin")
    loaded = tt_b200.QMPS.load(fn + ".ttmps")
    assert loaded.L == L
    assert loaded.bond_dims() == psi.bond_dims()
    assert loaded.center() == psi.center()
    a, b = _blocks(psi), _blocks(loaded)
    raw = np.fromfile(fn + "__T.bin", dtype=np.float64)
    pos = 0
    for (qa, ia, ba), (qb, ib, bb) in zip(a, b):
        assert qa == qb and ia == ib
        for x, y in zip(ba, bb):
            np.testing.assert_array_equal(x, y)
            n = x.size
            np.testing.assert_array_equal(raw[pos:pos + n], x.reshape(-1, order="F"))
            pos += n
    assert pos == raw.size
    # data_prefix: the recorded raw file name is relative to the prefix
    os.rename(fn + "__T.bin", str(tmp_path / "moved__T.bin"))
    with pytest.raises(tt_b200.TTError):
        tt_b200.QMPS.load(fn + ".ttmps")
    os.rename(str(tmp_path / "moved__T.bin"), fn + "__T.bin")
    # resume sweeps 3..5 from the in-memory state and from the checkpoint
    e_mem = tt_b200.QDMRG(psi, H).run(6, maxm, cutoff, mr, start_sweep=3)
    e_ck = tt_b200.QDMRG(loaded, H).run(6, maxm, cutoff, mr, start_sweep=3)
    # equal up to the random refills of the Krylov basis at the chain ends,
    # which draw from the context's running counter
    assert abs(e_mem - e_ck) <= 1e-12 * abs(e_mem)
    assert loaded.bond_dims() == psi.bond_dims()


def test_dmps_checkpoint_roundtrip(ctx, tmp_path):
    import tt_b200
    L = 10
    psi = tt_b200.DMPS(L, qdmrg.neel(L))
    H = tt_b200.DMPO(L)
    tt_b200.ddmrg_run(psi, H, 2, [8, 16], [1e-10], [4])
    fn = str(tmp_path / "dpsi")
    psi.save(fn)
    loaded = tt_b200.DMPS.load(fn + ".ttmps")
    assert loaded.L == L and loaded.bond_dims() == psi.bond_dims()
    assert abs(loaded.overlap(psi) - psi.overlap()) <= 1e-14 * psi.overlap()
    assert abs(loaded.expectation(H) - psi.expectation(H)) <= 1e-12 * abs(psi.expectation(H))
    raw = np.fromfile(fn + "__T.bin", dtype=np.float64)
    assert raw.size == sum(a * 2 * b for a, b in zip(psi.bond_dims()[:-1], psi.bond_dims()[1:]))
