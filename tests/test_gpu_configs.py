"""Parity of the CUDA path with the CPU oracle at the benchmark configurations'
own sizes (the oracle runs on the host cores; each case takes one to two
minutes of oracle time).

* The L = 100 Heisenberg chain (the U(1) chain configuration): ramp 32, 64,
  128, 256 and two sweeps at 512, cutoff 1e-12, Davidson 6 iterations --
  final energy within 1e-10 relative of the oracle's.
  The same chain with small random fields (no singular-value ties): the kept
  states per QN sector and the energy of every two-site step, and the final
  bond dimensions.
* The J1-J2 6 x 16 cylinder in snake order (the J1-J2 configuration's
  lattice) to bond dimension 256, with small random fields so that SU(2)
  multiplets do not tie at the truncation: the same step-by-step comparison.
* The transverse-field Ising 6 x 12 cylinder, dense path (the TFI
  configuration's lattice) to bond dimension 128 from a seeded random product
  state: every sweep's energy and the bond dimensions.

Step by step, a DMRG run from a product state is not a smooth function of
its rounding: in the first sweeps (few Davidson iterations, heavy
truncation) a change in the last bit grows by orders of magnitude within a
few dozen steps.  The CUDA path run twice, with the Davidson decisions on the
device and on the host (the same arithmetic summed in different orders),
shows where that starts for each run: up to there the CUDA path must match
the oracle step for step (energies to 1e-9, kept states per sector exactly);
after it, the two CUDA runs themselves drift apart, and the final energy must
agree with the oracle's to 1e-10 relative or to within 20 times the spread
of the two CUDA runs, whichever is larger, and the final bond dimensions to
one state on at most one bond in twenty.
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


def _rounding_onset(steps_a, steps_b, tol=1e-11):
    """First step at which two runs of the same schedule differ in energy by
    more than tol (relative)."""
    for k, (a, b) in enumerate(zip(steps_a, steps_b)):
        if abs(a["energy"] - b["energy"]) > tol * abs(b["energy"]):
            return k
    return min(len(steps_a), len(steps_b))


def _compare_steps(steps, logs, upto, tol_e=1e-9):
    ref_steps = [t for lg in logs for t in lg.trunc]
    ref_e = [e for lg in logs for e in lg.energies]
    assert len(steps) == len(ref_steps)
    for k in range(upto):
        te, kept, per = ref_steps[k]
        s = steps[k]
        assert s["kept"] == kept, k
        assert tuple(c for (_, c) in s["sectors"]) == tuple(per), k
        assert abs(s["energy"] - ref_e[k]) <= tol_e * abs(ref_e[k]), k


def _run_twice(make, nsweeps, maxm, cutoff, mr):
    """The CUDA path with the Davidson decisions on the device, then on the
    host: (energy, steps, bond dims) of each."""
    import tt_b200
    out = []
    try:
        for device in (True, False):
            tt_b200.set_davidson_control(device)
            psi, H = make()
            run = tt_b200.QDMRG(psi, H)
            e = run.run(nsweeps, maxm, cutoff, mr)
            out.append((e, run.steps(), psi.bond_dims()))
    finally:
        tt_b200.set_davidson_control(True)
    return out


def _check_trajectory(runs, logs, e_ref, ref_bonds, min_onset):
    (e, steps, bonds), (e_h, steps_h, _) = runs
    onset = _rounding_onset(steps, steps_h)
    assert onset >= min_onset, onset
    _compare_steps(steps, logs, onset)
    assert abs(e - e_ref) <= max(1e-10 * abs(e_ref), 20.0 * abs(e - e_h)), (e, e_h, e_ref)
    # the cutoff decides the last state of a bond on eigenvalues of the order of
    # the cutoff, which the rounding-sensitive stretch moves: a bond may end one
    # state apart, no more, and few may
    diff = [abs(a - b) for a, b in zip(bonds, ref_bonds)]
    assert len(bonds) == len(ref_bonds) and max(diff) <= 1 and sum(d > 0 for d in diff) <= len(diff) // 20, diff


@pytest.mark.parametrize("fields", [False, True])
def test_heisenberg_chain_L100_to_maxdim_512(ctx, fields):
    import tt_b200
    L = 100
    h = list(np.random.default_rng(17).uniform(-1e-2, 1e-2, L)) if fields else None
    maxm, cutoff, mr = [32, 64, 128, 256, 512, 512], [1e-12], [6]
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    logs = []
    e_ref = qdmrg.dmrg(psi, qdmrg.QMPO(L, dh=h), len(maxm), maxm, cutoff, mr, sweep_logs=logs)
    if not fields:
        # without fields SU(2) multiplets tie at the cut, where the reference's
        # std::sort leaves the choice open: kept counts (and bond dimensions)
        # may differ by members of a multiplet, the converged energy may not
        gpsi = tt_b200.QMPS(L, qdmrg.neel(L))
        e = tt_b200.QDMRG(gpsi, tt_b200.QMPO(L, dh=h)).run(len(maxm), maxm, cutoff, mr)
        assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
        return
    runs = _run_twice(lambda: (tt_b200.QMPS(L, qdmrg.neel(L)), tt_b200.QMPO(L, dh=h)), len(maxm), maxm, cutoff, mr)
    # converged at bond dimension 512: the final energies agree to 1e-10 whatever the path
    assert abs(runs[0][0] - e_ref) <= 1e-10 * abs(e_ref)
    _check_trajectory(runs, logs, e_ref, psi.bond_dims, min_onset=60)


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
    o = am.AutoMPO()
    for coef, ops in _j1j2_snake(Nx, Ny, 0.5, h):
        o.add(coef, *ops)

    def make():
        a = tt_b200.AutoMPO()
        for coef, ops in _j1j2_snake(Nx, Ny, 0.5, h):
            a.add(coef, *ops)
        return tt_b200.QMPS(N, qdmrg.neel(N)), tt_b200.QMPO.from_autompo(a, N)

    maxm, cutoff, mr = [64, 128, 256], [1e-10], [4]
    psi = qdmrg.QMPS(N, qdmrg.neel(N))
    logs = []
    e_ref = qdmrg.dmrg(psi, am.build_qmpo(o, N), 3, maxm, cutoff, mr, sweep_logs=logs)
    runs = _run_twice(make, 3, maxm, cutoff, mr)
    _check_trajectory(runs, logs, e_ref, psi.bond_dims, min_onset=120)


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
