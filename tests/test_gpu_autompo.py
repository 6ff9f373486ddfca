"""AutoMPO-built MPOs on the GPU path: the device qMPO / dense MPO equal the
oracle's, and two-site DMRG on them reaches the exact ground energy.

Models (small versions of the benchmark suite's configurations):
* XXZ chain with anisotropy and random site fields, U(1) (the batched-chains
  configuration);
* J1-J2 Heisenberg on a y-periodic cylinder, U(1) (the J1-J2 configuration);
* transverse-field Ising on a y-periodic cylinder, dense (the TFI configuration).
"""
import numpy as np
import pytest

from oracle import autompo as am
from oracle import ddmrg, ed, qdmrg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import tt_b200
    c = tt_b200.Context(0)
    yield c
    c.close()


def _both(terms):
    import tt_b200
    a, o = tt_b200.AutoMPO(), am.AutoMPO()
    for coef, ops in terms:
        args = [coef]
        for i, op in ops:
            args += [op, i]
        a.add(*args)
        o.add(*args)
    return a, o


def _xxz_terms(L, delta, h):
    t = []
    for i in range(L - 1):
        t += [(0.5, ((i, "S+"), (i + 1, "S-"))), (0.5, ((i, "S-"), (i + 1, "S+"))), (delta, ((i, "Sz"), (i + 1, "Sz")))]
    t += [(h[i], ((i, "Sz"),)) for i in range(L)]
    return t


def _j1j2_terms(Nx, Ny, J2):
    t = []
    for s1, s2, typ, *_ in am.square_next_neighbor(Nx, Ny, True):
        J = 1.0 if typ == 1 else J2
        i, j = s1 - 1, s2 - 1
        t += [(0.5 * J, ((i, "S+"), (j, "S-"))), (0.5 * J, ((i, "S-"), (j, "S+"))), (J, ((i, "Sz"), (j, "Sz")))]
    return t


def _tfi_terms(Nx, Ny, g):
    t = [(-4.0, ((s1 - 1, "Sz"), (s2 - 1, "Sz"))) for s1, s2, *_ in am.square_lattice(Nx, Ny, True)]
    return t + [(-2.0 * g, ((i, "Sx"),)) for i in range(Nx * Ny)]


def test_qmpo_from_autompo_equals_oracle(ctx):
    import tt_b200
    a, o = _both(_j1j2_terms(3, 4, 0.5))
    N = 12
    H = tt_b200.QMPO.from_autompo(a, N)
    ref = am.build_qmpo(o, N)
    for i in range(N):
        T = H.tensor(i).to_oracle()
        R = ref.A[i]
        assert [ix.qns for ix in T.idx] == [ix.qns for ix in R.idx]
        assert T.bqi == R.bqi
        for x, y in zip(T.blocks, R.blocks):
            np.testing.assert_array_equal(x, y)


def test_dmpo_from_autompo_equals_oracle(ctx):
    import tt_b200
    a, o = _both(_tfi_terms(3, 4, 3.0))
    N = 12
    H = tt_b200.DMPO.from_autompo(a, N)
    ref = am.build_dmpo(o, N)
    for i in range(N):
        np.testing.assert_array_equal(H.tensor(i), ref.A[i].data)


def test_xxz_field_chain_autompo_dmrg_matches_oracle_and_ed(ctx):
    import tt_b200
    L, delta = 12, 0.75
    h = list(np.random.default_rng(21).uniform(-0.1, 0.1, L))
    a, o = _both(_xxz_terms(L, delta, h))
    # the schedule is cyclic (maxm[sweep % len]): list every sweep
    maxm, cutoff, mr = [8, 16, 32, 64, 64, 64, 64, 64], [1e-10], [6]
    gpsi = tt_b200.QMPS(L, qdmrg.neel(L))
    run = tt_b200.QDMRG(gpsi, tt_b200.QMPO.from_autompo(a, L))
    e = run.run(8, maxm, cutoff, mr)
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    e_ref = qdmrg.dmrg(psi, am.build_qmpo(o, L), 8, maxm, cutoff, mr)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
    Eed = ed.ground_energy(L, ed.chain_bonds(L), delta=delta, h=h)
    assert abs(e - Eed) <= 1e-9 * abs(Eed)
    assert gpsi.bond_dims() == psi.bond_dims


def test_j1j2_cylinder_autompo_dmrg_matches_ed(ctx):
    import tt_b200
    Nx, Ny = 4, 4
    N = Nx * Ny
    terms = _j1j2_terms(Nx, Ny, 0.5)
    a, _ = _both(terms)
    gpsi = tt_b200.QMPS(N, qdmrg.neel(N))
    run = tt_b200.QDMRG(gpsi, tt_b200.QMPO.from_autompo(a, N))
    e = run.run(8, [32, 64, 128, 256, 256, 256, 256, 256], [1e-12], [6])
    Eed = ed.terms_ground_energy(N, terms, N // 2)
    assert abs(e - Eed) <= 1e-8 * abs(Eed)


def test_tfi_cylinder_dense_autompo_dmrg_matches_oracle_and_ed(ctx):
    import tt_b200
    Nx, Ny, g = 3, 4, 3.0
    N = Nx * Ny
    terms = _tfi_terms(Nx, Ny, g)
    a, o = _both(terms)
    state = list(np.random.default_rng(4).integers(0, 2, N))
    maxm, cutoff, mr = [16, 32, 64, 64, 64, 64], [1e-10], [4]
    psi = tt_b200.DMPS(N, state)
    e, sweep_e, _ = tt_b200.ddmrg_run(psi, tt_b200.DMPO.from_autompo(a, N), 6, maxm, cutoff, mr)
    opsi = ddmrg.DMPS(N, state)
    e_ref = ddmrg.ddmrg(opsi, am.build_dmpo(o, N), 6, maxm, cutoff, mr)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
    Eed = ed.terms_ground_energy(N, terms)
    assert abs(e - Eed) <= 1e-9 * abs(Eed)
