"""Independent chains solved concurrently on one GPU (one host thread, device
context and CUDA stream per worker) give the same energies as solving them
one after another, and match exact diagonalisation."""
import numpy as np
import pytest

from oracle import ed, qdmrg

pytestmark = pytest.mark.gpu


def _chains(n, seed=3):
    rng = np.random.default_rng(seed)
    return [(int(L), float(d), list(rng.uniform(-0.1, 0.1, int(L))))
            for L, d in zip(rng.integers(8, 13, n), rng.uniform(0.5, 1.5, n))]


def _solve(item):
    import tt_b200
    L, delta, h = item
    a = tt_b200.AutoMPO()
    for i in range(L - 1):
        a.add(0.5, "S+", i, "S-", i + 1).add(0.5, "S-", i, "S+", i + 1).add(delta, "Sz", i, "Sz", i + 1)
    for i in range(L):
        a.add(h[i], "Sz", i)
    psi = tt_b200.QMPS(L, qdmrg.neel(L))
    run = tt_b200.QDMRG(psi, tt_b200.QMPO.from_autompo(a, L))
    e = run.run(8, [8, 16, 32, 64, 64, 64, 64, 64], [1e-12], [6])
    del run, psi
    return e


def test_concurrent_chains_match_sequential_and_ed():
    import tt_b200
    from tt_b200 import replicas
    items = _chains(6)
    conc = replicas.run_chains_concurrent(items, _solve, streams=3)
    ctx = tt_b200.Context(0)
    try:
        seq = [_solve(it) for it in items]
    finally:
        ctx.close()
    for (L, delta, h), ec, es in zip(items, conc, seq):
        assert abs(ec - es) <= 1e-11 * abs(es)
        Eed = ed.ground_energy(L, ed.chain_bonds(L), delta=delta, h=h)
        assert abs(ec - Eed) <= 1e-9 * abs(Eed)
