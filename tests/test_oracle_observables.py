"""The state-vector observables used to check the device correlators, pinned
on the oracle's own DMRG ground state: <psi|H|psi>/<psi|psi> from the
amplitude vector equals the DMRG energy, and <Sz_i Sz_j> agrees with the
exact-diagonalisation ground state."""
import numpy as np

from oracle import ed, freefermion, observables, qdmrg


def test_state_vector_energy_and_correlators():
    L = 10
    h = list(np.random.default_rng(3).uniform(-0.1, 0.1, L))
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    e = qdmrg.dmrg(psi, qdmrg.QMPO(L, dh=h), 8, [8, 16, 32, 32, 32, 32, 32, 32], [1e-12], [6])
    v = observables.qmps_state_vector(psi.A)
    terms = [(0.5, ((i, "S+"), (i + 1, "S-"))) for i in range(L - 1)]
    terms += [(0.5, ((i, "S-"), (i + 1, "S+"))) for i in range(L - 1)]
    terms += [(1.0, ((i, "Sz"), (i + 1, "Sz"))) for i in range(L - 1)]
    terms += [(h[i], ((i, "Sz"),)) for i in range(L)]
    H = ed.terms_hamiltonian(L, terms)
    assert abs(v @ (H @ v) / (v @ v) - e) <= 1e-10 * abs(e)
    Hs = ed.terms_hamiltonian(L, terms, L // 2)
    w, U = np.linalg.eigh(Hs.toarray())
    v0 = np.zeros(2 ** L)
    v0[ed.sector_basis(L, L // 2)] = U[:, 0]
    one, two = observables.sz_correlators(v, L)
    one0, two0 = observables.sz_correlators(v0, L)
    assert np.abs(two - two0).max() < 1e-6
    assert np.abs(one - one0).max() < 1e-6
    assert abs(one.sum()) < 1e-12


def test_free_fermion_correlators_match_ed():
    """<Sz_i Sz_j> of the open XX chain by Wick's theorem (oracle/freefermion.py)
    equal the exact-diagonalisation ground state's; the GPU correlators are
    checked against the same closed form at L = 100."""
    L = 10
    terms = [(0.5, ((i, "S+"), (i + 1, "S-"))) for i in range(L - 1)]
    terms += [(0.5, ((i, "S-"), (i + 1, "S+"))) for i in range(L - 1)]
    Hs = ed.terms_hamiltonian(L, terms, L // 2)
    w, U = np.linalg.eigh(Hs.toarray())
    v0 = np.zeros(2 ** L)
    v0[ed.sector_basis(L, L // 2)] = U[:, 0]
    one, two = observables.sz_correlators(v0, L)
    assert np.abs(two - freefermion.xx_chain_szsz(L)).max() < 1e-12
    assert np.abs(one).max() < 1e-12
