"""Parity of the CUDA path with the CPU oracle at the benchmark configurations'
own sizes (the oracle runs on the host cores; each case takes one to two
minutes of oracle time).

* The L = 100 Heisenberg chain (the U(1) chain configuration): ramp 32, 64,
  128, 256 and two sweeps at 512, cutoff 1e-12, Davidson 6 iterations --
  final energy within 1e-10 relative of the oracle's.
  The same chain with small random fields (no singular-value ties): the kept
  states per QN sector at every one of the 1188 two-site steps and every
  step's energy.
* The J1-J2 6 x 16 cylinder in snake order (the J1-J2 configuration's
  lattice) to bond dimension 256, with small random fields so that SU(2)
  multiplets do not tie at the truncation: every step's energy and kept
  states per sector.
* The transverse-field Ising 6 x 12 cylinder, dense path (the TFI
  configuration's lattice) to bond dimension 128 from a seeded random product
  state: every sweep's energy and the bond dimensions.
"""
import numpy as np
import pytest

from oracle import autompo as am
from oracle import ddmrg, qdmrg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import tt_b200
    c = tt_b200.Context(0)
    yield c
    c.close()


def _compare_steps(run, logs, tol_e=1e-9):
    steps = run.steps()
    ref_steps = [t for lg in logs for t in lg.trunc]
    ref_e = [e for lg in logs for e in lg.energies]
    assert len(steps) == len(ref_steps)
    for k, (s, (te, kept, per)) in enumerate(zip(steps, ref_steps)):
        assert s["kept"] == kept, k
        assert tuple(c for (_, c) in s["sectors"]) == tuple(per), k
    for s, e in zip(steps, ref_e):
        assert abs(s["energy"] - e) <= tol_e * abs(e)


@pytest.mark.parametrize("fields", [False, True])
def test_heisenberg_chain_L100_to_maxdim_512(ctx, fields):
    import tt_b200
    L = 100
    h = list(np.random.default_rng(17).uniform(-1e-2, 1e-2, L)) if fields else None
    maxm, cutoff, mr = [32, 64, 128, 256, 512, 512], [1e-12], [6]
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    logs = []
    e_ref = qdmrg.dmrg(psi, qdmrg.QMPO(L, dh=h), len(maxm), maxm, cutoff, mr, sweep_logs=logs)
    gpsi = tt_b200.QMPS(L, qdmrg.neel(L))
    run = tt_b200.QDMRG(gpsi, tt_b200.QMPO(L, dh=h))
    e = run.run(len(maxm), maxm, cutoff, mr)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
    if fields:
        _compare_steps(run, logs)
        assert gpsi.bond_dims() == psi.bond_dims
    # without fields SU(2) multiplets tie at the cut, where the reference's
    # std::sort leaves the choice open: kept counts (and bond dimensions) may
    # differ by members of a multiplet, the energy may not


def _j1j2_snake(Nx, Ny, J2, h):
    terms = []
    for s1, s2, t, *_ in am.snake_relabel(am.square_next_neighbor(Nx, Ny, True), Nx, Ny):
        J = 1.0 if t == 1 else J2
        i, j = s1 - 1, s2 - 1
        terms += [(0.5 * J, ("S+", i, "S-", j)), (0.5 * J, ("S-", i, "S+", j)), (J, ("Sz", i, "Sz", j))]
    terms += [(float(h[i]), ("Sz", i)) for i in range(Nx * Ny)]
    return terms


def test_j1j2_6x16_snake_to_maxdim_256_step_by_step(ctx):
    import tt_b200
    Nx, Ny = 16, 6
    N = Nx * Ny
    h = np.random.default_rng(1).uniform(-1e-2, 1e-2, N)
    a, o = tt_b200.AutoMPO(), am.AutoMPO()
    for coef, ops in _j1j2_snake(Nx, Ny, 0.5, h):
        a.add(coef, *ops)
        o.add(coef, *ops)
    maxm, cutoff, mr = [64, 128, 256], [1e-10], [4]
    psi = qdmrg.QMPS(N, qdmrg.neel(N))
    logs = []
    e_ref = qdmrg.dmrg(psi, am.build_qmpo(o, N), 3, maxm, cutoff, mr, sweep_logs=logs)
    gpsi = tt_b200.QMPS(N, qdmrg.neel(N))
    run = tt_b200.QDMRG(gpsi, tt_b200.QMPO.from_autompo(a, N))
    e = run.run(3, maxm, cutoff, mr)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
    _compare_steps(run, logs)
    assert gpsi.bond_dims() == psi.bond_dims


def test_tfi_6x12_dense_to_maxdim_128(ctx):
    import tt_b200
    Nx, Ny, g = 12, 6, 3.0
    N = Nx * Ny
    a, o = tt_b200.AutoMPO(), am.AutoMPO()
    for s1, s2, *_ in am.snake_relabel(am.square_lattice(Nx, Ny, True), Nx, Ny):
        a.add(-4.0, "Sz", s1 - 1, "Sz", s2 - 1)
        o.add(-4.0, "Sz", s1 - 1, "Sz", s2 - 1)
    for i in range(N):
        a.add(-2.0 * g, "Sx", i)
        o.add(-2.0 * g, "Sx", i)
    state = list(np.random.default_rng(4).integers(0, 2, N))
    maxm, cutoff, mr = [16, 32, 64, 128, 128], [1e-10], [4]
    psi = tt_b200.DMPS(N, state)
    e, sweep_e, _ = tt_b200.ddmrg_run(psi, tt_b200.DMPO.from_autompo(a, N), len(maxm), maxm, cutoff, mr)
    opsi = ddmrg.DMPS(N, state)
    logs = []
    e_ref = ddmrg.ddmrg(opsi, am.build_dmpo(o, N), len(maxm), maxm, cutoff, mr, sweep_logs=logs)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
    for s, lg in zip(sweep_e, logs):
        assert abs(s - lg.energies[-1]) <= 1e-9 * abs(lg.energies[-1])
    assert psi.bond_dims() == opsi.bond_dims
