"""Pin the CPU oracle against exact-diagonalisation known answers.

The reference ships no golden vectors for the DMRG path, so the oracle's
restatement of it is pinned by exact ground energies: a converged two-site
DMRG must reproduce the ED energy of the same Hamiltonian in the same
total-Sz sector, and intermediate energies must respect the variational bound.
"""
import numpy as np
import pytest

from oracle import ddmrg, ed, freefermion, qdmrg
from oracle.qtensor import QIndex, QTensor, Inward, Outward, contract, qn, to_dense


def test_qdmrg_heisenberg_matches_ed():
    L = 10
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    H = qdmrg.QMPO(L)
    logs = []
    E = qdmrg.dmrg(psi, H, 8, [16, 32, 64], [1e-12], [6], sweep_logs=logs)
    Eed = ed.ground_energy(L, ed.chain_bonds(L))
    assert abs(E - Eed) < 1e-10 * abs(Eed)
    for lg in logs:
        assert min(lg.energies) >= Eed - 1e-10


def test_qdmrg_xx_chain_matches_free_fermions():
    """A known answer beyond exact diagonalisation: the open XX chain
    H = sum_i (S+_i S-_{i+1} + S-_i S+_{i+1}) / 2 is a chain of free fermions
    with single-particle energies cos(pi k / (L + 1)), k = 1..L (Jordan-Wigner),
    so its ground energy at Sz = 0 is the sum of the L/2 lowest of them.  At
    L = 40 the Sz = 0 sector has 1.4e11 states; the oracle's two-site DMRG
    (AutoMPO MPO) must reach that energy from above."""
    from oracle import autompo as am
    L = 40
    a = am.AutoMPO()
    for i in range(L - 1):
        a.add(0.5, "S+", i, "S-", i + 1)
        a.add(0.5, "S-", i, "S+", i + 1)
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    E = qdmrg.dmrg(psi, am.build_qmpo(a, L), 6, [16, 32, 64, 64, 64, 64], [1e-12], [6])
    Eex = freefermion.xx_chain_energy(L)
    assert -1e-12 * abs(Eex) <= E - Eex <= 1e-9 * abs(Eex)


def test_free_fermion_energies_match_ed():
    """The closed forms the free-fermion tests rely on, against ED."""
    L, g = 8, 0.7
    terms = [(-4.0, ((i, "Sz"), (i + 1, "Sz"))) for i in range(L - 1)]
    terms += [(-2.0 * g, ((i, "Sx"),)) for i in range(L)]
    assert abs(ed.terms_ground_energy(L, terms) - freefermion.tfi_chain_energy(L, g)) < 1e-12 * L
    L = 10
    terms = [(0.5, ((i, "S+"), (i + 1, "S-"))) for i in range(L - 1)]
    terms += [(0.5, ((i, "S-"), (i + 1, "S+"))) for i in range(L - 1)]
    Hs = ed.terms_hamiltonian(L, terms, L // 2)
    assert abs(np.linalg.eigvalsh(Hs.toarray())[0] - freefermion.xx_chain_energy(L)) < 1e-12 * L


def test_ddmrg_tfi_chain_matches_free_fermions():
    """Dense-path known answer beyond exact diagonalisation: the critical
    transverse-field Ising chain (g = 1, L = 40, Z = 2 Sz, X = 2 Sx) from a
    seeded random product state, AutoMPO MPO; the oracle's dense two-site
    DMRG must reach the free-fermion energy."""
    from oracle import autompo as am
    L, g = 40, 1.0
    a = am.AutoMPO()
    for i in range(L - 1):
        a.add(-4.0, "Sz", i, "Sz", i + 1)
    for i in range(L):
        a.add(-2.0 * g, "Sx", i)
    psi = ddmrg.DMPS(L, list(np.random.default_rng(5).integers(0, 2, L)))
    E = ddmrg.ddmrg(psi, am.build_dmpo(a, L), 6, [8, 16, 32, 32, 32, 32], [1e-12], [4])
    Eex = freefermion.tfi_chain_energy(L, g)
    assert -1e-12 * abs(Eex) <= E - Eex <= 1e-12 * abs(Eex)


def test_qdmrg_field_matches_ed():
    L = 8
    rng = np.random.default_rng(3)
    h = list(rng.uniform(-0.1, 0.1, L))
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    H = qdmrg.QMPO(L, dh=h)
    E = qdmrg.dmrg(psi, H, 8, [32], [1e-12], [6])
    Eed = ed.ground_energy(L, ed.chain_bonds(L), h=h)
    assert abs(E - Eed) < 1e-10 * abs(Eed)


def test_ddmrg_config1_matches_ed():
    """Dense L=16 Heisenberg, maxdim 16,32,64x4, cutoff 1e-10, 4 restarts."""
    L = 16
    psi = ddmrg.DMPS(L, qdmrg.neel(L))
    H = ddmrg.DMPO(L)
    E = ddmrg.ddmrg(psi, H, 6, [16, 32, 64, 64, 64, 64], [1e-10], [4])
    Eed = ed.ground_energy(L, ed.chain_bonds(L))
    assert abs(E - Eed) < 1e-10 * abs(Eed)


def test_ed_sector_size():
    assert len(ed.sector_basis(16, 8)) == 12870


def test_contract_matches_dense():
    """Block-sparse contraction agrees with the dense contraction of the scattered blocks."""
    rng = np.random.default_rng(0)
    a = QIndex(Inward, "a")
    for q, d in ((-1, 2), (1, 3), (3, 1)):
        a.add_qn(qn(q), d)
    s = QIndex(Inward, "s", 1)
    for q in (-1, 1):
        s.add_qn(qn(q), 1)
    b = QIndex(Outward, "b")
    for q, d in ((-2, 2), (0, 4), (2, 3), (4, 1)):
        b.add_qn(qn(q), d)
    T1 = QTensor([a, s, b])
    T1.init_block()
    for blk in T1.blocks:
        blk[...] = rng.standard_normal(blk.shape)
    c = QIndex(Outward, "c")
    for q, d in ((-3, 1), (-1, 2), (1, 2), (3, 2), (5, 1)):
        c.add_qn(qn(q), d)
    t = QIndex(Inward, "t", 1)
    for q in (-1, 1):
        t.add_qn(qn(q), 1)
    T2 = QTensor([b.dagged(), t, c])
    T2.init_block()
    for blk in T2.blocks:
        blk[...] = rng.standard_normal(blk.shape)
    C = contract(T1, T2)
    assert [ix.name for ix in C.idx] == ["a", "s", "t", "c"]
    ref = np.tensordot(to_dense(T1), to_dense(T2), axes=([2], [0]))
    np.testing.assert_allclose(to_dense(C), ref, rtol=0, atol=1e-13)


def test_qdmrg_on_autompo_xxz_chain_matches_ed():
    """U(1) oracle DMRG on an AutoMPO-built XXZ chain (anisotropy, site fields)."""
    from oracle import autompo as am
    L, delta = 10, 0.7
    h = np.random.default_rng(8).uniform(-0.1, 0.1, L)
    a = am.AutoMPO()
    for i in range(L - 1):
        a.add(0.5, "S+", i, "S-", i + 1)
        a.add(0.5, "S-", i, "S+", i + 1)
        a.add(delta, "Sz", i, "Sz", i + 1)
    for i in range(L):
        a.add(float(h[i]), "Sz", i)
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    E = qdmrg.dmrg(psi, am.build_qmpo(a, L), 8, [8, 16, 32, 32, 32, 32, 32, 32], [1e-12], [6])
    Eed = ed.terms_ground_energy(L, a.terms(), L // 2)
    assert abs(E - Eed) < 1e-10 * abs(Eed)


def test_ddmrg_on_autompo_tfi_cylinder_matches_ed():
    """Dense oracle DMRG on an AutoMPO-built transverse-field Ising 2x4 cylinder."""
    from oracle import autompo as am
    Nx, Ny, g = 2, 4, 3.0
    N = Nx * Ny
    a = am.AutoMPO()
    for s1, s2, *_ in am.square_lattice(Nx, Ny, True):
        a.add(-4.0, "Sz", s1 - 1, "Sz", s2 - 1)
    for i in range(N):
        a.add(-2.0 * g, "Sx", i)
    state = list(np.random.default_rng(4).integers(0, 2, N))
    psi = ddmrg.DMPS(N, state)
    E = ddmrg.ddmrg(psi, am.build_dmpo(a, N), 6, [8, 16, 16, 16, 16, 16], [1e-12], [4])
    Eed = ed.terms_ground_energy(N, a.terms())
    assert abs(E - Eed) < 1e-9 * abs(Eed)
