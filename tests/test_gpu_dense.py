"""Dense (dtensor / big_dtensor) DMRG path on the GPU against the oracle and ED.

Config 1 of the benchmark suite: spin-1/2 Heisenberg chain, L=16, open
boundaries, hand-written D=5 MPO, Neel start (1 on the chosen spin, machine
epsilon elsewhere), 6 sweeps with maxdim 16,32,64,64,64,64, cutoff 1e-10,
restarted Davidson with 3 vectors and 4 restarts.  The exact ground energy of
the Sz=0 sector (12870 states) is the known answer.
"""
import numpy as np
import pytest

from oracle import ddmrg, ed, freefermion, qdmrg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import tt_b200
    c = tt_b200.Context(0)
    yield c
    c.close()


def test_dense_config1_matches_ed_and_oracle(ctx):
    import tt_b200
    L = 16
    maxm, cutoff, mr = [16, 32, 64, 64, 64, 64], [1e-10], [4]
    psi = tt_b200.DMPS(L, qdmrg.neel(L))
    H = tt_b200.DMPO(L)
    e, sweep_e, kept = tt_b200.ddmrg_run(psi, H, 6, maxm, cutoff, mr)
    Eed = ed.ground_energy(L, ed.chain_bonds(L))
    assert abs(e - Eed) <= 1e-10 * abs(Eed)
    opsi = ddmrg.DMPS(L, qdmrg.neel(L))
    oH = ddmrg.DMPO(L)
    logs = []
    e_ref = ddmrg.ddmrg(opsi, oH, 6, maxm, cutoff, mr, sweep_logs=logs)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
    for s, lg in zip(sweep_e, logs):
        assert abs(s - lg.energies[-1]) <= 1e-8 * abs(lg.energies[-1])
    assert psi.bond_dims() == opsi.bond_dims


def test_dense_field_chain_matches_ed(ctx):
    import tt_b200
    L = 10
    h = list(np.random.default_rng(5).uniform(-0.1, 0.1, L))
    psi = tt_b200.DMPS(L, qdmrg.neel(L))
    H = tt_b200.DMPO(L, dh=h)
    e, _, _ = tt_b200.ddmrg_run(psi, H, 6, [8, 16, 32], [1e-12], [4])
    Eed = ed.ground_energy(L, ed.chain_bonds(L), h=h)
    assert abs(e - Eed) <= 1e-9 * abs(Eed)


def test_dense_tfi_chain_L100_matches_free_fermions(ctx):
    """The dense path at chain length 100 against an exact answer: the
    critical transverse-field Ising chain H = -sum Z Z - sum X (free Majorana
    fermions, E0 = -sum of the singular values of the bidiagonal matrix with
    1 on and above the diagonal), AutoMPO MPO, seeded random product start,
    bond dimension ramped to 64 (the CPU oracle, same schedule, lands within
    1e-15)."""
    import tt_b200
    L = 100
    a = tt_b200.AutoMPO()
    for i in range(L - 1):
        a.add(-4.0, "Sz", i, "Sz", i + 1)
    for i in range(L):
        a.add(-2.0, "Sx", i)
    H = tt_b200.DMPO.from_autompo(a, L)
    psi = tt_b200.DMPS(L, list(np.random.default_rng(5).integers(0, 2, L)))
    E, _, _ = tt_b200.ddmrg_run(psi, H, 6, [8, 16, 32, 64, 64, 64], [1e-12], [4])
    Eex = freefermion.tfi_chain_energy(L, 1.0)
    assert abs(E - Eex) <= 1e-11 * abs(Eex)
