"""The mixed-precision (tcgen05 kind::tf32) contraction path.

* Grouped block-sparse contractions in TF32 and in split 3xTF32 against the
  FP64 oracle: relative Frobenius error below 5e-3 (TF32: 10-bit mantissa
  products, FP32 accumulation) and below 2e-6 (3xTF32: hi*hi + hi*lo + lo*hi,
  FP32 accumulation), on QN-blocked tensors with ragged sector sizes (tile
  edges in m, n and k); on a single 700 x 513 x 450 block the FP32
  accumulation over k = 513 dominates (about sqrt(k) * 2^-24), bound 1e-5.
* The automatic form ("tf32x3-auto") keeps bandwidth-bound contractions in
  FP64 (bit-identical to the FP64 path) and sends large blocks to the tensor
  cores.
* Two-site DMRG with H_eff*x and the environment updates in 3xTF32 (GS,
  Rayleigh-Ritz and the SVD in FP64; the sweep energy <psi|H|psi> contracted
  in FP64, because mixed-precision environments bias the Ritz value to first
  order while the state keeps FP64 quality) ends within |dE|/N <= 1e-8 of the
  FP64 run and of exact diagonalisation, on the U(1) and the dense path.
"""
import numpy as np
import pytest

from oracle import ed, qdmrg
from oracle.qtensor import QIndex, QTensor, Inward, Outward, Link, Site, contract, qn, to_dense

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import tt_b200
    c = tt_b200.Context(0)
    yield c
    tt_b200.set_precision()
    c.close()


def _index(arrow, name, sectors, typ=Link, level=0):
    ix = QIndex(arrow, name, typ, level)
    for q, d in sectors:
        ix.add_qn(qn(q), d)
    return ix


def _random(idx, rng):
    T = QTensor(idx)
    T.init_block()
    for b in T.blocks:
        b[...] = rng.standard_normal(b.shape)
    return T


def _rel_err(got, want):
    return np.linalg.norm(to_dense(got) - to_dense(want)) / np.linalg.norm(to_dense(want))


@pytest.mark.parametrize("prec,tol", [("tf32", 5e-3), ("tf32x3", 2e-6)])
def test_blocked_contraction_tf32(ctx, prec, tol):
    import tt_b200
    rng = np.random.default_rng(31)
    # ragged sectors: m, n and k cross the 128 x 64 x 32 tile edges
    a = _index(Inward, "a", [(-2, 37), (0, 161), (2, 70)])
    s1 = _index(Inward, "s1", [(-1, 1), (1, 1)], Site)
    s2 = _index(Inward, "s2", [(-1, 1), (1, 1)], Site)
    b = _index(Outward, "b", [(-4, 19), (-2, 133), (0, 150), (2, 40), (4, 65)])
    X = _random([a, s1, s2, b], rng)
    ap = _index(Inward, "a", [(-2, 37), (0, 161), (2, 70)], Link, 1)
    w = _index(Outward, "w", [(-2, 1), (0, 3), (2, 1)])
    L = _random([ap, w, a.dagged()], rng)
    want = contract(L, X)
    gL, gX = tt_b200.QTensor.from_oracle(L), tt_b200.QTensor.from_oracle(X)
    tt_b200.set_precision(op=prec)
    try:
        got = (gL * gX).to_oracle()
        # the other operand order gives the transposed GEMMs (other gather paths)
        got2 = (gX * gL).to_oracle()
    finally:
        tt_b200.set_precision()
    assert sorted(got.bid) == sorted(want.bid)
    assert _rel_err(got, want) < tol
    assert _rel_err(got2, contract(X, L)) < tol
    ref = (gL * gX).to_oracle()  # FP64 again: the precision switch is scoped
    assert _rel_err(ref, want) < 1e-14


def test_large_single_block_tf32x3(ctx):
    import tt_b200
    rng = np.random.default_rng(5)
    i = _index(Inward, "i", [(0, 700)])
    k = _index(Outward, "k", [(0, 513)])
    j = _index(Inward, "j", [(0, 450)])
    A = _random([i, k], rng)
    B = _random([k.dagged(), j], rng)
    want = contract(A, B)
    gA, gB = tt_b200.QTensor.from_oracle(A), tt_b200.QTensor.from_oracle(B)
    tt_b200.set_precision(op="tf32x3")
    try:
        got = (gA * gB).to_oracle()
    finally:
        tt_b200.set_precision()
    assert _rel_err(got, want) < 1e-5


def test_mixed_precision_dmrg_energy(ctx):
    import tt_b200
    L = 16
    h = list(np.random.default_rng(41).uniform(-0.1, 0.1, L))
    sched = ([16, 32, 64, 64, 64, 64, 64, 64], [1e-12], [6])
    p64 = tt_b200.QMPS(L, qdmrg.neel(L))
    e64 = tt_b200.QDMRG(p64, tt_b200.QMPO(L, dh=h)).run(8, *sched)
    tt_b200.set_precision(heff="tf32x3", env="tf32x3")
    try:
        pmx = tt_b200.QMPS(L, qdmrg.neel(L))
        emx = tt_b200.QDMRG(pmx, tt_b200.QMPO(L, dh=h)).run(8, *sched)
    finally:
        tt_b200.set_precision()
    Eed = ed.ground_energy(L, ed.chain_bonds(L), h=h)
    assert abs(e64 - Eed) / L <= 1e-10
    assert abs(emx - e64) / L <= 1e-8
    assert abs(emx - Eed) / L <= 1e-8


def test_mixed_precision_dense_tfi(ctx):
    import tt_b200
    from oracle import autompo as am
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
    state = list(np.random.default_rng(4).integers(0, 2, N))
    sched = ([16, 32, 64, 64, 64, 64, 64, 64], [1e-12], [4])
    e64, _, _ = tt_b200.ddmrg_run(tt_b200.DMPS(N, state), H, 8, *sched)
    tt_b200.set_precision(heff="tf32x3", env="tf32x3")
    try:
        emx, _, _ = tt_b200.ddmrg_run(tt_b200.DMPS(N, state), H, 8, *sched)
    finally:
        tt_b200.set_precision()
    Eed = ed.terms_ground_energy(N, terms)
    assert abs(e64 - Eed) / N <= 1e-10
    assert abs(emx - e64) / N <= 1e-8


def test_mixed_precision_dense_tfi_cylinder_6x12(ctx):
    """The dense transverse-field Ising configuration at its geometry: the
    6 x 12 cylinder (periodic around the 6-site circumference, 72 sites in
    snake order), H = -sum ZZ - 3 sum X (Z = 2 Sz, X = 2 Sx), a seeded random
    product state, the MPO from the AutoMPO (uncompressed basis of
    models/hams/AutoMPO.cpp: the identity states plus one string state per
    ZZ term open across a link, at most 8 here -- the configuration quotes
    14 for its MPO); the bond dimension is ramped to 128 instead of 1024 so
    the test takes seconds.  The mixed
    form (3xTF32 tensor-core H_eff*x and environment contractions, FP64 SVD)
    must hold |dE|/N <= 1e-8 against the FP64 GPU form, with the same bond
    dimensions."""
    import tt_b200
    from oracle import autompo as am
    Nx, Ny, g = 12, 6, 3.0
    N = Nx * Ny
    bonds = am.snake_relabel(am.square_lattice(Nx, Ny, True), Nx, Ny)
    a = tt_b200.AutoMPO()
    for s1, s2, *_ in bonds:
        a.add(-4.0, "Sz", s1 - 1, "Sz", s2 - 1)
    for i in range(N):
        a.add(-2.0 * g, "Sx", i)
    assert max(a.link_dims(N, with_charges=False)) == 8
    H = tt_b200.DMPO.from_autompo(a, N)
    state = list(np.random.default_rng(12).integers(0, 2, N))
    sched = ([16, 32, 64, 128, 128, 128], [1e-10], [4])
    p64 = tt_b200.DMPS(N, state)
    e64, s64, _ = tt_b200.ddmrg_run(p64, H, 6, *sched)
    tt_b200.set_precision(heff="tf32x3", env="tf32x3")
    try:
        pmx = tt_b200.DMPS(N, state)
        emx, smx, _ = tt_b200.ddmrg_run(pmx, H, 6, *sched)
    finally:
        tt_b200.set_precision()
    assert max(p64.bond_dims()) == 128
    assert pmx.bond_dims() == p64.bond_dims()
    assert abs(emx - e64) / N <= 1e-8
    # variational and converging: the last sweeps agree to well below the gap
    assert abs(s64[-1] - s64[-2]) / N <= 1e-6


def test_auto_precision_picks_per_contraction(ctx):
    """'tf32x3-auto' resolves per contraction: a contraction over a small MPO
    link (k = 5, bandwidth-bound) stays FP64 and is bit-identical to the FP64
    result; a 2048^3 block goes to the tensor cores (differs from FP64, within
    the 3xTF32 bound of the oracle, 5e-5 for FP32 accumulation over k = 2048)."""
    import tt_b200
    rng = np.random.default_rng(17)
    a = _index(Inward, "a", [(-2, 300), (0, 400), (2, 300)])
    w = _index(Outward, "w", [(-2, 1), (0, 3), (2, 1)])
    b = _index(Outward, "b", [(-2, 200), (0, 250), (2, 200)])
    X = _random([a, w.dagged(), b], rng)        # contract over w (k <= 3 per block pair)
    wp = _index(Inward, "w", [(-2, 1), (0, 3), (2, 1)], Link, 1)
    W = _random([w, wp.dagged()], rng)
    gX, gW = tt_b200.QTensor.from_oracle(X), tt_b200.QTensor.from_oracle(W)
    ref64 = (gX * gW).to_oracle()
    tt_b200.set_precision(op="tf32x3-auto")
    try:
        got = (gX * gW).to_oracle()
    finally:
        tt_b200.set_precision()
    for x, y in zip(got.blocks, ref64.blocks):
        np.testing.assert_array_equal(x, y)
    i = _index(Inward, "i", [(0, 2048)])
    k = _index(Outward, "k", [(0, 2048)])
    j = _index(Inward, "j", [(0, 2048)])
    A = _random([i, k], rng)
    B = _random([k.dagged(), j], rng)
    gA, gB = tt_b200.QTensor.from_oracle(A), tt_b200.QTensor.from_oracle(B)
    big64 = (gA * gB).to_oracle()
    tt_b200.set_precision(op="tf32x3-auto")
    try:
        big = (gA * gB).to_oracle()
    finally:
        tt_b200.set_precision()
    assert not np.array_equal(big.blocks[0], big64.blocks[0])
    # FP32 accumulation over k = 2048 (about sqrt(k) * 2^-24 per element): measured 1.4e-5
    assert _rel_err(big, contract(A, B)) < 5e-5


def test_forced_tf32x3_every_sweep_matches_fp64(ctx):
    """Forced 3xTF32 products everywhere (no automatic choice) on a J1-J2
    cylinder: EVERY sweep energy -- not only the last -- stays within 1e-8
    per site of the FP64 run's.  The two-site problems at the chain ends are
    small enough for the Krylov vectors to exhaust them, where product noise
    must not enter the Ritz vector (those problems run their products in FP64)."""
    import tt_b200
    Nx, Ny = 6, 4
    N = Nx * Ny
    a = tt_b200.AutoMPO()
    for s1, s2, typ, *_ in tt_b200.square_next_neighbor(Nx, Ny, True):
        J = 1.0 if typ == 1 else 0.5
        a.add(0.5 * J, "S+", s1 - 1, "S-", s2 - 1).add(0.5 * J, "S-", s1 - 1, "S+", s2 - 1).add(J, "Sz", s1 - 1, "Sz", s2 - 1)
    H = tt_b200.QMPO.from_autompo(a, N)
    sched = [32, 64, 128, 128, 128, 128, 128, 128]
    run64 = tt_b200.QDMRG(tt_b200.QMPS(N, qdmrg.neel(N)), H)
    e64 = [run64.sweep(m, 1e-10, 6) for m in sched]
    tt_b200.set_precision(heff="tf32x3", env="tf32x3")
    try:
        runmx = tt_b200.QDMRG(tt_b200.QMPS(N, qdmrg.neel(N)), H)
        emx = [runmx.sweep(m, 1e-10, 6) for m in sched]
    finally:
        tt_b200.set_precision()
    # the first sweeps differ in their path (truncation ties, noise); from the
    # third sweep on both runs sit at the same fixed bond dimension
    for s in range(3, len(sched)):
        assert abs(emx[s] - e64[s]) / N <= 1e-8, (s, emx[s], e64[s])
