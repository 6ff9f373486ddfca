"""End-to-end parity of the CUDA U(1) two-site DMRG with the CPU oracle and ED.

The chains carry small random site fields so that SU(2) multiplets are split
and the truncation has no singular-value ties: then every two-site step must
keep the same number of states in every QN sector as the oracle, and the
energies must agree to 1e-10 relative (FP64 path).
"""
import numpy as np
import pytest

from oracle import ed, freefermion, qdmrg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import tt_b200
    c = tt_b200.Context(0)
    yield c
    c.close()


def _run_both(L, maxm, cutoff, mr, nsweeps, h=None):
    import tt_b200
    psi = qdmrg.QMPS(L, qdmrg.neel(L))
    H = qdmrg.QMPO(L, dh=h)
    logs = []
    e_ref = qdmrg.dmrg(psi, H, nsweeps, maxm, cutoff, mr, sweep_logs=logs)
    gpsi = tt_b200.QMPS(L, qdmrg.neel(L))
    gH = tt_b200.QMPO(L, dh=h)
    run = tt_b200.QDMRG(gpsi, gH)
    e_gpu = run.run(nsweeps, maxm, cutoff, mr)
    return e_ref, e_gpu, logs, run, gpsi, psi


def test_dmrg_field_chain_matches_oracle_step_by_step(ctx):
    L = 10
    h = list(np.random.default_rng(11).uniform(-0.1, 0.1, L))
    e_ref, e_gpu, logs, run, gpsi, psi = _run_both(L, [8, 16, 32, 32, 32], [1e-10], [6], 5, h)
    assert abs(e_gpu - e_ref) <= 1e-10 * abs(e_ref)
    steps = run.steps()
    ref_steps = [t for lg in logs for t in lg.trunc]
    ref_e = [e for lg in logs for e in lg.energies]
    assert len(steps) == len(ref_steps)
    for s, (te, kept, per) in zip(steps, ref_steps):
        assert s["kept"] == kept
        assert tuple(k for (_, k) in s["sectors"]) == tuple(per)
    for s, e in zip(steps, ref_e):
        assert abs(s["energy"] - e) <= 1e-9 * abs(e)
    assert gpsi.bond_dims() == psi.bond_dims
    Eed = ed.ground_energy(L, ed.chain_bonds(L), h=h)
    assert abs(e_gpu - Eed) <= 1e-9 * abs(Eed)


def test_dmrg_heisenberg_matches_ed(ctx):
    import tt_b200
    L = 16
    gpsi = tt_b200.QMPS(L, qdmrg.neel(L))
    gH = tt_b200.QMPO(L)
    run = tt_b200.QDMRG(gpsi, gH)
    e = run.run(6, [16, 32, 64], [1e-12], [6])
    Eed = ed.ground_energy(L, ed.chain_bonds(L))
    assert abs(e - Eed) <= 1e-10 * abs(Eed)
    assert gpsi.center() == 0
    st = run.stats()
    assert st["heff_flops"] > 0 and st["heff_seconds"] > 0


def test_device_and_host_davidson_control_agree(ctx):
    """The device-resident Davidson control (one synchronisation per call) and
    the host loop run the same algorithm: same kept states per sector at every
    step, energies within round-off."""
    import tt_b200
    L = 12
    h = list(np.random.default_rng(23).uniform(-0.1, 0.1, L))
    sched = ([8, 16, 32, 32, 32], [1e-10], [6])
    out = {}
    for mode in (False, True):
        tt_b200.set_davidson_control(mode)
        try:
            psi = tt_b200.QMPS(L, qdmrg.neel(L))
            run = tt_b200.QDMRG(psi, tt_b200.QMPO(L, dh=h))
            e = run.run(5, *sched)
            out[mode] = (e, [(s["kept"], s["sectors"]) for s in run.steps()], [s["energy"] for s in run.steps()])
        finally:
            tt_b200.set_davidson_control(True)
    (eh, kh, sh), (ed_, kd, sd) = out[False], out[True]
    assert abs(eh - ed_) <= 1e-12 * abs(eh)
    assert kh == kd
    for a, b in zip(sh, sd):
        assert abs(a - b) <= 1e-10 * abs(a)


def test_noise_schedule_converges_to_the_noise_free_ground_state(ctx):
    """Density-matrix noise decaying to zero (as in the J1-J2 configuration)
    on a small J1-J2 cylinder: the final energy equals exact diagonalisation
    and the noise-free oracle's, every noisy sweep stays variational, and the
    noise changes the kept bases while it is on."""
    import tt_b200
    from oracle import autompo as am
    Nx, Ny, J2 = 4, 4, 0.5
    N = Nx * Ny
    terms = []
    for s1, s2, typ, *_ in am.square_next_neighbor(Nx, Ny, True):
        J = 1.0 if typ == 1 else J2
        i, j = s1 - 1, s2 - 1
        terms += [(0.5 * J, ((i, "S+"), (j, "S-"))), (0.5 * J, ((i, "S-"), (j, "S+"))), (J, ((i, "Sz"), (j, "Sz")))]
    a, o = tt_b200.AutoMPO(), am.AutoMPO()
    for coef, ops in terms:
        args = [coef]
        for i, op in ops:
            args += [op, i]
        a.add(*args)
        o.add(*args)
    maxm, cutoff, mr = [16, 32, 64, 128, 256, 256, 256, 256, 256], [1e-12], [6]
    noise = [1e-4, 1e-5, 1e-6, 1e-8, 0.0]
    Eed = ed.terms_ground_energy(N, terms, N // 2)
    psi = tt_b200.QMPS(N, qdmrg.neel(N))
    run = tt_b200.QDMRG(psi, tt_b200.QMPO.from_autompo(a, N))
    e = run.run(9, maxm, cutoff, mr, noise=noise)
    for se, _ in run.sweeps():
        assert se >= Eed - 1e-9 * abs(Eed)
    assert abs(e - Eed) <= 1e-8 * abs(Eed)
    # the noise-free path through the same sweeps ends at the same state
    psi0 = tt_b200.QMPS(N, qdmrg.neel(N))
    run0 = tt_b200.QDMRG(psi0, tt_b200.QMPO.from_autompo(a, N))
    e0 = run0.run(9, maxm, cutoff, mr)
    assert abs(e - e0) <= 1e-8 * abs(Eed)
    # while on, noise changes the kept bases, hence the early sweep energies
    early = [abs(x[0] - y[0]) for x, y in zip(run.sweeps()[:3], run0.sweeps()[:3])]
    assert max(early) > 1e-12


def test_gram_schmidt_failures_are_refilled_on_the_device(ctx):
    """Near convergence the residual's projection falls below 1e-10 and the
    reference refills the new vector at random (linalg/tensor_davidson.cpp:
    298-316).  The device-resident loop does this itself: refills happen, no
    call is handed to the host loop, and the result is the ED ground state."""
    import tt_b200
    from oracle import autompo as am
    Nx, Ny, J2 = 4, 4, 0.5
    N = Nx * Ny
    terms, a = [], tt_b200.AutoMPO()
    for s1, s2, typ, *_ in am.square_next_neighbor(Nx, Ny, True):
        J = 1.0 if typ == 1 else J2
        i, j = s1 - 1, s2 - 1
        terms += [(0.5 * J, ((i, "S+"), (j, "S-"))), (0.5 * J, ((i, "S-"), (j, "S+"))), (J, ((i, "Sz"), (j, "Sz")))]
        a.add(0.5 * J, "S+", i, "S-", j).add(0.5 * J, "S-", i, "S+", j).add(J, "Sz", i, "Sz", j)
    r0, f0 = tt_b200.davidson_refills(), tt_b200.davidson_fallbacks()
    psi = tt_b200.QMPS(N, qdmrg.neel(N))
    run = tt_b200.QDMRG(psi, tt_b200.QMPO.from_autompo(a, N))
    e = run.run(8, [32, 64, 128, 256, 256, 256, 256, 256], [1e-12], [6])
    assert tt_b200.davidson_refills() > r0
    assert tt_b200.davidson_fallbacks() == f0
    Eed = ed.terms_ground_energy(N, terms, N // 2)
    assert abs(e - Eed) <= 1e-8 * abs(Eed)


def test_xx_chain_L100_matches_free_fermions(ctx):
    """A known answer at the chain length of the L = 100 configuration, far
    beyond exact diagonalisation: the open XX chain (S+S- + S-S+) / 2 is free
    fermions with single-particle energies cos(pi k / 101), so its Sz = 0
    ground energy is the sum of the 50 lowest.  The MPO comes from the
    library's AutoMPO; the sweep ramps to bond dimension 128 (the CPU oracle,
    same schedule, lands 6.6e-11 above the exact energy); the correlators
    of the state follow from Wick's theorem."""
    import tt_b200
    L = 100
    a = tt_b200.AutoMPO()
    for i in range(L - 1):
        a.add(0.5, "S+", i, "S-", i + 1)
        a.add(0.5, "S-", i, "S+", i + 1)
    H = tt_b200.QMPO.from_autompo(a, L)
    psi = tt_b200.QMPS(L, qdmrg.neel(L))
    E = tt_b200.QDMRG(psi, H).run(6, [16, 32, 64, 128, 128, 128], [1e-12], [6])
    Eex = freefermion.xx_chain_energy(L)
    assert -1e-12 * abs(Eex) <= E - Eex <= 1e-9 * abs(Eex)
    assert max(psi.bond_dims()) == 128
    # <Sz_i> and <Sz_i Sz_j> of the DMRG state against Wick's theorem
    sz, szsz = psi.measure_sz()
    err = np.abs(szsz - freefermion.xx_chain_szsz(L)).max()
    assert np.abs(sz).max() < 1e-6, np.abs(sz).max()
    assert err < 1e-6, err
