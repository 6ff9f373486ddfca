"""Overlaps, MPO expectation values and <Sz_i Sz_j> correlators on the GPU.

The device MPS after DMRG is read back block by block, contracted into its
2^L amplitude vector on the CPU, and the correlators are evaluated exactly on
it (bit-for-bit the same state, so the tolerance is round-off, 1e-12).  The
correlators of the exact ground state (ED) pin the physics at the DMRG
accuracy, and psiHphi / psiphi reproduce the DMRG energy.  A coupling
derivative dE/dJ comes from the same expectation-value contraction
(Hellmann-Feynman) and is checked against ED.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import autompo as am
from oracle import ed, observables, qdmrg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import tt_b200
    c = tt_b200.Context(0)
    yield c
    c.close()


def _ed_ground_state(L, terms, n_up=None):
    H = ed.terms_hamiltonian(L, terms, n_up)
    w, v = np.linalg.eigh(H.toarray()) if H.shape[0] <= 2000 else spla.eigsh(H, k=1, which="SA", tol=1e-14)
    v0 = v[:, 0]
    if n_up is None:
        return w[0], v0
    full = np.zeros(2 ** L)
    full[ed.sector_basis(L, n_up)] = v0
    return w[0], full


def _xxz_terms(L, delta, h):
    t = []
    for i in range(L - 1):
        t += [(0.5, ((i, "S+"), (i + 1, "S-"))), (0.5, ((i, "S-"), (i + 1, "S+"))), (delta, ((i, "Sz"), (i + 1, "Sz")))]
    return t + [(h[i], ((i, "Sz"),)) for i in range(L)]


def test_qmps_correlators_overlap_expectation(ctx):
    import tt_b200
    L, delta = 12, 0.8
    h = list(np.random.default_rng(13).uniform(-0.1, 0.1, L))
    terms = _xxz_terms(L, delta, h)
    a = tt_b200.AutoMPO()
    for coef, ops in terms:
        args = [coef]
        for i, op in ops:
            args += [op, i]
        a.add(*args)
    H = tt_b200.QMPO.from_autompo(a, L)
    psi = tt_b200.QMPS(L, qdmrg.neel(L))
    e = tt_b200.QDMRG(psi, H).run(8, [8, 16, 32, 64, 64, 64, 64, 64], [1e-12], [6])
    sz, szsz = psi.measure_sz()
    # exact evaluation on the same state
    v = observables.qmps_state_vector([psi.tensor(i).to_oracle() for i in range(L)])
    one, two = observables.sz_correlators(v, L)
    np.testing.assert_allclose(sz, one, rtol=0, atol=1e-12)
    np.testing.assert_allclose(szsz, two, rtol=0, atol=1e-12)
    n2 = psi.overlap()
    assert abs(n2 - v @ v) <= 1e-12 * (v @ v)
    Hs = ed.terms_hamiltonian(L, terms)
    assert abs(psi.expectation(H) - v @ (Hs @ v)) <= 1e-11 * abs(e)
    assert abs(psi.expectation(H) / n2 - e) <= 1e-10 * abs(e)
    # physics: the exact ground state of the Sz=0 sector
    E0, v0 = _ed_ground_state(L, terms, L // 2)
    one0, two0 = observables.sz_correlators(v0, L)
    assert abs(e - E0) <= 1e-9 * abs(E0)
    np.testing.assert_allclose(szsz, two0, rtol=0, atol=1e-6)
    np.testing.assert_allclose(sz, one0, rtol=0, atol=1e-6)
    assert abs(sz.sum()) < 1e-10


def test_dense_tfi_correlators_and_energy(ctx):
    import tt_b200
    Nx, Ny, g = 3, 4, 3.0
    N = Nx * Ny
    terms = [(-4.0, ((s1 - 1, "Sz"), (s2 - 1, "Sz"))) for s1, s2, *_ in am.square_lattice(Nx, Ny, True)]
    terms += [(-2.0 * g, ((i, "Sx"),)) for i in range(N)]
    a = tt_b200.AutoMPO()
    for coef, ops in terms:
        args = [coef]
        for i, op in ops:
            args += [op, i]
        a.add(*args)
    H = tt_b200.DMPO.from_autompo(a, N)
    psi = tt_b200.DMPS(N, list(np.random.default_rng(4).integers(0, 2, N)))
    e, _, _ = tt_b200.ddmrg_run(psi, H, 8, [16, 32, 64, 64, 64, 64, 64, 64], [1e-12], [4])
    n2 = psi.overlap()
    assert abs(psi.expectation(H) / n2 - e) <= 1e-10 * abs(e)
    E0, v0 = _ed_ground_state(N, terms)
    assert abs(e - E0) <= 1e-9 * abs(E0)
    one0, two0 = observables.sz_correlators(v0, N)
    sz, szsz = psi.measure_sz()
    np.testing.assert_allclose(szsz, two0, rtol=0, atol=1e-6)
    np.testing.assert_allclose(np.diag(szsz), 0.25)


def test_hellmann_feynman_dE_dJ2_from_expectation(ctx):
    """dE/dJ2 of the J1-J2 model on a 4x4 cylinder, by Hellmann-Feynman: the
    expectation value of the J2 part of H (its own AutoMPO) in the DMRG ground
    state, against the same expectation in the exact ground state (ED, Sz=0)
    and against a central finite difference of ED energies."""
    import tt_b200
    Nx, Ny, J2 = 4, 4, 0.5
    N = Nx * Ny
    bonds = list(am.square_next_neighbor(Nx, Ny, True))

    def part(kind, coef):
        t = []
        for s1, s2, typ, *_ in bonds:
            if typ == kind:
                i, j = s1 - 1, s2 - 1
                t += [(0.5 * coef, ((i, "S+"), (j, "S-"))), (0.5 * coef, ((i, "S-"), (j, "S+"))),
                      (coef, ((i, "Sz"), (j, "Sz")))]
        return t

    def mpo(terms):
        a = tt_b200.AutoMPO()
        for coef, ops in terms:
            args = [coef]
            for i, op in ops:
                args += [op, i]
            a.add(*args)
        return tt_b200.QMPO.from_autompo(a, N)

    h1, h2 = part(1, 1.0), part(2, 1.0)
    psi = tt_b200.QMPS(N, qdmrg.neel(N))
    e = tt_b200.QDMRG(psi, mpo(h1 + part(2, J2))).run(8, [32, 64, 128, 256, 256, 256, 256, 256], [1e-12], [6])
    dE = psi.expectation(mpo(h2)) / psi.overlap()
    E0, v0 = _ed_ground_state(N, h1 + part(2, J2), N // 2)
    full_h2 = ed.terms_hamiltonian(N, h2)
    exact = float(v0 @ (full_h2 @ v0))
    assert abs(e - E0) <= 1e-8 * abs(E0)
    # first order in the state's error (truncation at cutoff 1e-12): ~1e-5 relative
    assert abs(dE - exact) <= 2e-5
    step = 1e-4
    fd = (ed.terms_ground_energy(N, h1 + part(2, J2 + step), N // 2) -
          ed.terms_ground_energy(N, h1 + part(2, J2 - step), N // 2)) / (2 * step)
    assert abs(dE - fd) <= 2e-5
