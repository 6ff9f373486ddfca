"""AutoMPO, lattices and the AutoMPO -> MPO builders on the CPU.

* The oracle's finite-state MPOs (dense and U(1)) contracted to a full matrix
  equal the Hamiltonian assembled term by term, for an XXZ chain with site
  fields, a J1-J2 cylinder and a transverse-field Ising cylinder.
* The C ABI's host logic (term accumulator, lattices, MPO link dimensions)
  equals the oracle's; no device is touched.
"""
import numpy as np
import pytest

from oracle import autompo as am
from oracle import ed
from oracle.qtensor import to_dense


def xxz_chain(L, delta, h):
    a = am.AutoMPO()
    for i in range(L - 1):
        a.add(0.5, "S+", i, "S-", i + 1)
        a.add(0.5, "S-", i, "S+", i + 1)
        a.add(delta, "Sz", i, "Sz", i + 1)
    for i in range(L):
        a.add(h[i], "Sz", i)
    return a


def j1j2(Nx, Ny, J2, lattice=am.square_next_neighbor):
    a = am.AutoMPO()
    for s1, s2, t, *_ in lattice(Nx, Ny, True):
        J = 1.0 if t == 1 else J2
        a.add(0.5 * J, "S+", s1 - 1, "S-", s2 - 1)
        a.add(0.5 * J, "S-", s1 - 1, "S+", s2 - 1)
        a.add(J, "Sz", s1 - 1, "Sz", s2 - 1)
    return a


def tfi(Nx, Ny, g):
    a = am.AutoMPO()
    for s1, s2, *_ in am.square_lattice(Nx, Ny, True):
        a.add(-4.0, "Sz", s1 - 1, "Sz", s2 - 1)
    for i in range(Nx * Ny):
        a.add(-2.0 * g, "Sx", i)
    return a


@pytest.mark.parametrize("case", ["xxz", "j1j2", "tfi"])
def test_oracle_mpo_equals_term_sum(case):
    rng = np.random.default_rng(5)
    if case == "xxz":
        N = 7
        a = xxz_chain(N, 0.7, rng.uniform(-0.1, 0.1, N))
    elif case == "j1j2":
        N = 8
        a = j1j2(2, 4, 0.5)
    else:
        N = 8
        a = tfi(2, 4, 3.0)
    T = am.term_matrix(N, a.terms())
    D = am.build_dmpo(a, N)
    assert np.abs(am.mpo_matrix([A.data for A in D.A]) - T).max() < 1e-13
    if case != "tfi":
        Q = am.build_qmpo(a, N)
        assert np.abs(am.mpo_matrix([to_dense(A) for A in Q.A]) - T).max() < 1e-13
        # the dense and U(1) layouts agree on the link dimensions
        assert [A.idx[0].dim() for A in Q.A] == [A.data.shape[0] for A in D.A]


def test_xxz_terms_match_ed_hamiltonian():
    L = 8
    h = np.random.default_rng(2).uniform(-0.1, 0.1, L)
    a = xxz_chain(L, 1.3, h)
    e1 = ed.terms_ground_energy(L, a.terms(), L // 2)
    e2 = ed.ground_energy(L, ed.chain_bonds(L), delta=1.3, h=h)
    assert abs(e1 - e2) < 1e-12


def test_accumulator_semantics():
    a = am.AutoMPO()
    a.add(0.5, "S-", 3, "S+", 1)        # stored in site order
    a.add(2, 0.25, "S-", 3, "S+", 1)    # numbers multiply, repeated list sums
    a.add(0.0, "Sz", 0)                 # zero coefficient dropped
    a.add(1.0, "Sz", 2)
    assert a.terms() == [(1.0, ((2, "Sz"),)), (1.0, ((1, "S+"), (3, "S-")))]
    with pytest.raises(ValueError):
        a.add(1.0, "Sz", "Sz", 1)
    with pytest.raises(ValueError):
        a.add(1.0, "Sz")


def test_capi_accumulator_and_lattices_match_oracle():
    import tt_b200 as tt
    for f, g in [(tt.square_lattice, am.square_lattice), (tt.square_next_neighbor, am.square_next_neighbor),
                 (tt.triangular_lattice, am.triangular_lattice)]:
        for Nx, Ny, yp in [(6, 12, True), (6, 16, True), (3, 4, False), (4, 2, True), (1, 5, False)]:
            ours = [tuple(b) for b in f(Nx, Ny, yp)]
            ref = [tuple(float(v) if k > 2 else v for k, v in enumerate(b)) for b in g(Nx, Ny, yp)]
            assert ours == ref
    rng = np.random.default_rng(3)
    a, o = tt.AutoMPO(), am.AutoMPO()
    for _ in range(300):
        i, j = (int(v) for v in rng.integers(0, 12, 2))
        c = float(rng.choice([0.0, 0.5, 1.0, -2.0, 0.1]))
        op1, op2 = (str(v) for v in rng.choice(["Sz", "S+", "S-"], 2))
        args = (c, op1, i) if rng.random() < 0.3 else (c, op1, i, op2, j)
        a.add(*args)
        o.add(*args)
    assert a.terms() == o.terms()
    a += (1.0, "Sz", 1)
    assert len(a) == len(o.terms()) + (0 if (1, "Sz") in [t[1][0] for t in o.terms() if len(t[1]) == 1] else 1)


@pytest.mark.parametrize("case", ["xxz", "j1j2", "tfi"])
def test_capi_link_dims_match_oracle(case):
    import tt_b200 as tt
    rng = np.random.default_rng(9)
    if case == "xxz":
        N, terms = 20, xxz_chain(20, 0.9, rng.uniform(-0.1, 0.1, 20)).terms()
    elif case == "j1j2":
        N, terms = 96, j1j2(16, 6, 0.5).terms()
    else:
        N, terms = 72, tfi(12, 6, 3.0).terms()
    a = tt.AutoMPO()
    for coef, ops in terms:
        args = [coef]
        for i, op in ops:
            args += [op, i]
        a.add(*args)
    charges = case != "tfi"
    oa = am.AutoMPO()
    for coef, ops in terms:
        args = [coef]
        for i, op in ops:
            args += [op, i]
        oa.add(*args)
    ref = [len(l) for l in am.links(oa, N, charges)]
    assert a.link_dims(N, charges) == ref
    assert ref[0] == 1 and ref[-1] == 1


def test_capi_rejects_unsupported_terms():
    import tt_b200 as tt
    a = tt.AutoMPO()
    a.add(1.0, "Sx", 0, "Sx", 1)
    with pytest.raises(tt.TTError):
        a.link_dims(3, True)       # Sx carries no definite U(1) charge
    assert a.link_dims(3, False) == [1, 3, 2, 1]
    b = tt.AutoMPO()
    b.add(1.0, "Sz", 0, "Sz", 1)
    b.add(1.0, "Sz", 1)
    b.add(1.0, "Sz", 0, "Sz", 0)
    with pytest.raises(tt.TTError):
        b.link_dims(3, True)       # two operators on one site
    c = tt.AutoMPO()
    c.add(1.0, "Sz", 0, "Sz", 5)
    with pytest.raises(tt.TTError):
        c.link_dims(4, True)       # site out of range


def test_snake_order_relabels_the_same_bonds():
    """Snake order: the same bonds (types, coordinates) under the site map
    n(x, y) = (x-1) Ny + (y if x odd else Ny+1-y); consecutive chain sites are
    nearest neighbours; the C ABI's relabelling equals the oracle's; and the
    J1-J2 spectrum does not depend on the order (term matrices are similar)."""
    import tt_b200 as tt
    for Nx, Ny, yp in [(6, 16, True), (16, 6, True), (3, 4, False), (4, 2, True)]:
        col = am.square_next_neighbor(Nx, Ny, yp)
        sn = am.snake_relabel(col, Nx, Ny)
        ours = [tuple(b) for b in tt.square_next_neighbor(Nx, Ny, yp, snake=True)]
        assert ours == [tuple(float(v) if k > 2 else v for k, v in enumerate(b)) for b in sn]
        assert [tuple(b) for b in tt.square_lattice(Nx, Ny, yp, snake=True)] == \
            [tuple(float(v) if k > 2 else v for k, v in enumerate(b))
             for b in am.snake_relabel(am.square_lattice(Nx, Ny, yp), Nx, Ny)]
        def snake(n):
            x, y = (n - 1) // Ny + 1, (n - 1) % Ny + 1
            return (x - 1) * Ny + (y if x % 2 == 1 else Ny + 1 - y)
        assert sorted(snake(n) for n in range(1, Nx * Ny + 1)) == list(range(1, Nx * Ny + 1))
        for (s1, s2, t, *_), (c1, c2, ct, *_) in zip(sn, col):
            assert s1 < s2 and t == ct and {s1, s2} == {snake(c1), snake(c2)}
        nn = {(s1, s2) for s1, s2, t, *_ in sn if t == 1}
        assert all((n, n + 1) in nn for n in range(1, Nx * Ny)) or Ny == 1
    with pytest.raises(RuntimeError):
        tt._lattice(tt.TT_LATTICE_TRIANGULAR | tt.TT_LATTICE_SNAKE, 3, 4, True)

    def j1j2_terms(bonds):
        a = am.AutoMPO()
        for s1, s2, t, *_ in bonds:
            J = 1.0 if t == 1 else 0.5
            a.add(0.5 * J, "S+", s1 - 1, "S-", s2 - 1)
            a.add(0.5 * J, "S-", s1 - 1, "S+", s2 - 1)
            a.add(J, "Sz", s1 - 1, "Sz", s2 - 1)
        return a.terms()

    Hc = am.term_matrix(8, j1j2_terms(am.square_next_neighbor(4, 2, True)))
    Hs = am.term_matrix(8, j1j2_terms(am.snake_relabel(am.square_next_neighbor(4, 2, True), 4, 2)))
    assert np.allclose(np.linalg.eigvalsh(Hc), np.linalg.eigvalsh(Hs), atol=1e-10)
