"""Parity of the CUDA path (through the C ABI) with the oracle and the
reference's golden vectors.  FP64 bar: 1e-10 relative on G1 trajectories and
the dipole (RHS terms: 1e-12)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, dipole_err, load_golden, rand_c, rel_err
from oracle import REF_EXE, Config

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
RUN_TOL = 1e-10


def params_of(g12, cfg: Config):
    return g12.make_params(Ns=cfg.Ns, Nb=cfg.Nb, Nq=cfg.Nq, time_steps=cfg.time_steps, HF=cfg.HF, EHM=cfg.EHM,
                           q_type=cfg.q_type, v_law=cfg.vlaw, t1=cfg.t1, t2=cfg.t2, t3=cfg.t3, U=cfg.U, dt=cfg.dt,
                           quench_strength=cfg.quench_strength, AS_rate=cfg.AS_rate, AS_midpoint=cfg.AS_midpoint,
                           quench_rate=cfg.quench_rate, quench_on_midpoint=cfg.quench_on_midpoint,
                           quench_off_midpoint=cfg.quench_off_midpoint)


def oracle_rhs(oracle, cfg, G1, XX, XY, U, w, Nq):
    Ns, Nb = cfg.Ns, cfg.Nb
    V = cfg.vvec(U)
    h = oracle.h_hf(G1, Ns, Nb, U, cfg.t1, cfg.t2, w, V, Nq)
    comm1 = oracle.hG_comm(G1, h)
    n = Ns * Nb
    gate = cfg.U != 0 and not cfg.HF
    out = {"h": h, "comm1": comm1}
    if gate:
        Ix = oracle.collision(XY, XX, Ns, Nb, U, V)
        out["Ix"] = Ix
        for tag, X, psi_xy, A, B in (("xx", XX, 0, XY, XX), ("xy", XY, 1, XX, XY)):
            C = oracle.h2_comm(X, h, Ns, Nb)
            psi = oracle.psi(G1, Ns, Nb, U, V, psi_xy)
            pi = oracle.pi(G1, A, B, U, Ns, Nb, V)
            out["K2" + tag], _ = oracle.G2_step(C, psi, pi, np.zeros(n ** 4, complex), 1.0, Ns, Nb)
    else:
        Ix = np.zeros((n, n), complex)
        out["Ix"] = Ix
        out["K2xx"] = out["K2xy"] = np.zeros(n ** 4, complex)
    out["K1"], _ = oracle.G1_step(comm1, Ix, np.zeros((n, n), complex), 1.0, Ns, Nb)
    return out


RHS_CASES = [
    Config(Ns=2, Nb=1, U=1.1), Config(Ns=3, Nb=1, U=0.7, EHM=True), Config(Ns=4, Nb=1, U=1.0, EHM=True, vlaw="inv"),
    Config(Ns=2, Nb=2, U=1.3, t2=0.4), Config(Ns=3, Nb=2, U=2.0, t2=0.5, EHM=True, vlaw="inv"),
    Config(Ns=5, Nb=1, U=0.9, EHM=True), Config(Ns=3, Nb=3, U=1.2, t2=0.2, EHM=True), Config(Ns=1, Nb=2, U=0.6, t2=0.7),
    Config(Ns=6, Nb=2, U=1.5, t2=0.3, EHM=True, vlaw="inv"), Config(Ns=4, Nb=1, U=0.0),
    Config(Ns=3, Nb=2, U=1.0, HF=True),
    # n >= 16: the FP64 tensor-core (DMMA) halves; n = 24 and 20 pad to 32
    Config(Ns=8, Nb=2, U=2.0, t2=0.5, EHM=True, vlaw="inv"), Config(Ns=12, Nb=2, U=1.2, t2=0.4, EHM=True),
    Config(Ns=20, Nb=1, U=0.9, EHM=True, vlaw="inv"), Config(Ns=16, Nb=2, U=1.5, t2=0.3, EHM=True, vlaw="inv"),
]


@pytest.mark.parametrize("cfg", RHS_CASES, ids=lambda c: f"{c.Ns}x{c.Nb}-U{c.U}-E{int(c.EHM)}-{c.vlaw}-HF{int(c.HF)}")
def test_rhs_terms_vs_oracle(g12, oracle, cfg):
    rng = np.random.default_rng(cfg.Ns * 100 + cfg.Nb)
    n = cfg.n
    G1, XX, XY = rand_c(rng, n, n), rand_c(rng, n ** 4), rand_c(rng, n ** 4)
    U, w, Nq = cfg.U * 0.83, 0.37, min(2, cfg.Ns)
    with g12.Context(params_of(g12, cfg)) as ctx:
        got = ctx.rhs(G1, XX, XY, U, w, Nq)
    ref = oracle_rhs(oracle, cfg, G1, XX, XY, U, w, Nq)
    for k in ("h", "comm1", "Ix", "K1", "K2xx", "K2xy"):
        if np.max(np.abs(ref[k])) == 0:
            assert np.max(np.abs(got[k])) == 0, k
        else:
            assert rel_err(got[k], ref[k]) <= RHS_TOL, (k, rel_err(got[k], ref[k]))


def _cfg_from(g):
    return Config(**{k[4:]: g[k].item() for k in g.files if k.startswith("cfg_")})


@pytest.mark.parametrize("name", ["run_c1_short", "run_ehm_nb2", "run_quench_on", "run_hf", "run_guard"])
def test_full_run_vs_reference_golden(g12, name):
    g = load_golden(name + ".npz")
    cfg = _cfg_from(g)
    p = params_of(g12, cfg)
    T = int(g["T"])
    with g12.Context(p) as ctx:
        ctx.set_state(g["g0"])
        nas = ctx.adiabatic_switch()
        G1as, XXas, XYas = ctx.get_state()
        traj, rc = ctx.propagate(g12.rk_iterations(p))
        G1, XX, XY = ctx.get_state()
    assert nas == g12.as_steps(p)
    assert traj.shape[0] == T
    if name == "run_guard":
        assert rc == g12.G12_GUARD_TRIPPED
        ref = g["traj"]
        # the offending snapshot is recorded; the run is unstable, so compare
        # the prefix and require the same finite trip on the last snapshot
        assert rel_err(traj[:-1], ref[:-1]) <= RUN_TOL
        assert np.isfinite(traj[-1]).all() and abs(2 * traj[-1, 0, 0].imag) > 3
        return
    assert rc == 0
    assert rel_err(G1as, g["g1_as"]) <= RUN_TOL
    if np.max(np.abs(g["g2xx_as"])) > 0:
        assert rel_err(XXas, g["g2xx_as"]) <= RUN_TOL and rel_err(XYas, g["g2xy_as"]) <= RUN_TOL
    if "traj" in g.files:
        assert rel_err(traj, g["traj"]) <= RUN_TOL
    else:
        assert rel_err(traj[::10], g["traj_every10"]) <= RUN_TOL
        assert rel_err(traj[-1], g["traj_last"]) <= RUN_TOL
    if np.max(np.abs(g["g2xx"])) > 0:
        assert rel_err(XX, g["g2xx"]) <= RUN_TOL and rel_err(XY, g["g2xy"]) <= RUN_TOL
    else:
        assert np.max(np.abs(XX)) == 0 and np.max(np.abs(XY)) == 0
    assert dipole_err(g12.dipole(traj), g["dipole"], traj) <= RUN_TOL


def _g2_projections(G2):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(ROOT, "tests", "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.g2_projections(G2)


def _running_dev(a, b):
    d = np.max(np.abs(a - b).reshape(a.shape[0], -1), axis=1) / np.max(np.abs(b))
    return np.maximum.accumulate(d)


def test_config2_full_run_within_the_references_own_roundoff_sensitivity(g12):
    """Config 2 (n = 16, EHM U/(1+r), 5001 iterations after 1373 switching
    steps) against the compiled reference.  On this model the reference's
    algorithm amplifies round-off: the reference itself, started from G0
    moved by one ulp in half of its entries (run_c2_full_ulp.npz, made by
    tests/golden/make_golden.py), ends 5e-5 away from its own unperturbed run
    (9e-9 after the switching).  Two correct FP64 implementations (different
    summation orders) can differ by as much, so the bar here is that curve:
    at every compared snapshot the GPU's running deviation from the reference
    stays within 10x the reference's own one-ulp running deviation."""
    g, u = load_golden("run_c2_full.npz"), load_golden("run_c2_full_ulp.npz")
    cfg = _cfg_from(g)
    p = params_of(g12, cfg)
    every = int(g["every"])
    with g12.Context(p) as ctx:
        ctx.set_state(g["g0"])
        ctx.adiabatic_switch()
        G1as, _, _ = ctx.get_state()
        traj, rc = ctx.propagate(g12.rk_iterations(p))
        _, XX, XY = ctx.get_state()
    assert rc == 0 and traj.shape[0] == int(g["T"])
    ref_as = np.max(np.abs(u["g1_as"] - g["g1_as"])) / np.max(np.abs(g["g1_as"]))
    assert rel_err(G1as, g["g1_as"]) <= 10 * ref_as + 1e-12
    ours = _running_dev(traj[::every], g["traj_sub"])
    theirs = _running_dev(u["traj_sub"], g["traj_sub"])
    assert np.all(ours <= 10 * theirs + 1e-12), float(np.max(ours / (theirs + 1e-30)))
    # the final G2, by its checksums
    for X, key in ((XX, "g2xx_proj"), (XY, "g2xy_proj")):
        pr = _g2_projections(X)
        assert np.max(np.abs(pr - g[key])) <= 10 * np.max(np.abs(u[key] - g[key])) + 1e-12 * np.max(np.abs(g[key]))


@pytest.mark.parametrize("name", ["run_c1_full", "run_c3_20"])
def test_benchmark_config_vs_reference_golden(g12, name):
    """The benchmark configurations at their stated lengths against the
    compiled reference (RK_solver.h:96-216 after AS.h:63-214): config 1
    (n = 4, 2000 steps), config 2 (n = 16, EHM U/(1+r), 5001 iterations) and
    config 3 (n = 32, 20 steps after a shortened switching phase).  G1 every
    25th snapshot and the last, the dipole, and the G2 state after switching
    and at the end (in full for n <= 16, by seeded projections for n = 32)."""
    g = load_golden(name + ".npz")
    cfg = _cfg_from(g)
    p = params_of(g12, cfg)
    T = int(g["T"])
    every = int(g["every"])
    with g12.Context(p) as ctx:
        ctx.set_state(g["g0"])
        ctx.adiabatic_switch()
        G1as, XXas, XYas = ctx.get_state()
        traj, rc = ctx.propagate(g12.rk_iterations(p))
        G1, XX, XY = ctx.get_state()
    assert rc == 0 and traj.shape[0] == T
    assert rel_err(G1as, g["g1_as"]) <= RUN_TOL
    assert rel_err(traj[::every], g["traj_sub"]) <= RUN_TOL
    assert rel_err(traj[-1], g["traj_last"]) <= RUN_TOL
    assert dipole_err(g12.dipole(traj), g["dipole"], traj) <= RUN_TOL
    norms = g["g2_norms"]
    for i, (X, key) in enumerate(((XXas, "g2xx_as_proj"), (XYas, "g2xy_as_proj"), (XX, "g2xx_proj"),
                                  (XY, "g2xy_proj"))):
        assert abs(np.linalg.norm(X) - norms[i]) <= RUN_TOL * norms[i]
        pr = _g2_projections(X)
        assert np.max(np.abs(pr - g[key])) <= RUN_TOL * norms[i] * np.sqrt(X.size), key
    if "g2xx" in g.files:
        assert rel_err(XX, g["g2xx"]) <= RUN_TOL and rel_err(XY, g["g2xy"]) <= RUN_TOL


def test_device_dipole_and_chunked_clock(g12):
    g = load_golden("run_quench_on.npz")
    cfg = _cfg_from(g)
    p = params_of(g12, cfg)
    T = g12.rk_iterations(p)
    with g12.Context(p) as ctx:
        ctx.set_state(g["g0"])
        ctx.adiabatic_switch()
        d1, rc1 = ctx.propagate_dipole(400)
        d2, rc2 = ctx.propagate_dipole(T - 400)
    dip = np.concatenate([d1, d2])
    assert rc1 == 0 and rc2 == 0 and dip.shape[0] == T
    # quench switches on at t >= 50 (RK_solver.h:141): a real signal
    assert np.max(np.abs(g["dipole"])) > 1e-3
    assert rel_err(dip, g["dipole"]) <= RUN_TOL


def test_snapshot_ring_halves_split_calls_bitwise(g12):
    """One call over several halves of the snapshot ring (copies overlapped with
    the next half's steps) equals the same steps taken in uneven calls."""
    p = g12.make_params(Ns=4, Nb=2, Nq=2, time_steps=10000, U=1.0, t2=0.2, EHM=True, dt=0.02)
    G0 = g12.make_G0(p)
    with g12.Context(p) as ctx:
        ctx.set_state(G0)
        ctx.adiabatic_switch()
        S = ctx.get_state()
        traj, rc = ctx.propagate(5000)
        end = ctx.get_state()
    assert rc == 0 and traj.shape[0] == 5000
    parts = []
    with g12.Context(p) as ctx:
        ctx.set_state(*S)
        for m in (1, 2047, 2050, 902):
            t, rc = ctx.propagate(m)
            assert rc == 0
            parts.append(t)
        end2 = ctx.get_state()
    assert np.array_equal(traj, np.concatenate(parts))
    for a, b in zip(end, end2):
        assert np.array_equal(a, b)


def test_guard_trip_with_a_later_half_queued(g12):
    """The guard trips in the first half of a call that spans several halves:
    the call stops there, the queued half leaves the state alone."""
    g = load_golden("run_guard.npz")
    cfg = _cfg_from(g)
    p = params_of(g12, cfg)
    p.time_steps = 6000  # same schedule for the first steps, several ring halves
    T = int(g["T"])
    with g12.Context(p) as ctx:
        ctx.set_state(g["g0"])
        ctx.adiabatic_switch()
        traj, rc = ctx.propagate(g12.rk_iterations(p))
        G1 = ctx.get_state()[0]
    assert g12.rk_iterations(p) > 4100
    assert rc == g12.G12_GUARD_TRIPPED and traj.shape[0] == T
    assert rel_err(traj[:-1], g["traj"][:-1]) <= RUN_TOL
    # the state stays at the recorded offending snapshot: the queued half did not advance it
    assert np.array_equal(G1, traj[-1])


def test_deterministic(g12):
    g = load_golden("run_ehm_nb2.npz")
    p = params_of(g12, _cfg_from(g))
    outs = []
    for _ in range(2):
        with g12.Context(p) as ctx:
            ctx.set_state(g["g0"])
            ctx.adiabatic_switch()
            traj, _ = ctx.propagate(30)
            outs.append((traj, ctx.get_state()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1][1], outs[1][1][1])


def test_n16_steps_vs_oracle(g12, oracle):
    # the extended model (Ns=8, Nb=2, EHM, U/(1+r), pulse quench) from a correlated state
    cfg = Config(Ns=8, Nb=2, Nq=3, time_steps=6, U=2.0, t1=1.0, t2=0.5, dt=0.01, EHM=True, vlaw="inv",
                 q_type="pulse", quench_strength=2.0, quench_rate=2, quench_on_midpoint=15, quench_off_midpoint=25)
    p = params_of(g12, cfg)
    n = cfg.n
    rng = np.random.default_rng(3)
    G0 = g12.make_G0(p)
    XX = 1e-2 * rand_c(rng, n ** 4)
    XY = 1e-2 * rand_c(rng, n ** 4)
    G1 = G0.copy()
    XXo, XYo = XX.copy(), XY.copy()
    ref = []
    tt = 0.0
    for s in range(cfg.time_steps):
        ref.append(G1.copy())
        tt = oracle.step(cfg, 1, s * cfg.dt, tt, G1, XXo, XYo)
    with g12.Context(p) as ctx:
        ctx.set_state(G0, XX, XY)
        traj, rc = ctx.propagate(cfg.time_steps)
        _, XXg, XYg = ctx.get_state()
    assert rc == 0
    assert rel_err(traj, np.array(ref)) <= RUN_TOL
    assert rel_err(XXg, XXo) <= RUN_TOL and rel_err(XYg, XYo) <= RUN_TOL


def test_n32_rhs_vs_oracle(g12, oracle):
    # the n=32 system (Ns=16, Nb=2): one full right-hand side against the oracle
    cfg = Config(Ns=16, Nb=2, Nq=4, U=1.5, t2=0.3, EHM=True, vlaw="inv")
    rng = np.random.default_rng(11)
    n = cfg.n
    G1, XX, XY = rand_c(rng, n, n), 1e-2 * rand_c(rng, n ** 4), 1e-2 * rand_c(rng, n ** 4)
    with g12.Context(params_of(g12, cfg)) as ctx:
        got = ctx.rhs(G1, XX, XY, 1.5, 0.8, 4)
    ref = oracle_rhs(oracle, cfg, G1, XX, XY, 1.5, 0.8, 4)
    for k in ("h", "comm1", "Ix", "K1", "K2xx", "K2xy"):
        assert rel_err(got[k], ref[k]) <= RHS_TOL, k


def test_cli_drop_in(g12):
    """bin/g12kba on the reference's input format writes the reference's files."""
    g = load_golden("run_c1_short.npz")
    cfg = _cfg_from(g)
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "input"), "w") as f:
            f.write(cfg.input_text())
        r = subprocess.run([g12.CLI_PATH], cwd=d, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        assert "Execution Succesful" in r.stdout
        re_ = np.loadtxt(os.path.join(d, "real_G1.txt"))
        im_ = np.loadtxt(os.path.join(d, "imag_G1.txt"))
        dip = np.loadtxt(os.path.join(d, "dipole.txt"))
        ref = g["traj"].reshape(g["traj"].shape[0], -1).T
        # 6 significant digits (write_to_file.h default ostream precision)
        assert np.allclose(re_, ref.real, rtol=1e-5, atol=1e-7 * np.max(np.abs(ref)))
        assert np.allclose(im_, ref.imag, rtol=1e-5, atol=1e-7 * np.max(np.abs(ref)))
        assert dip.shape[0] == ref.shape[1]
        if os.path.exists(REF_EXE):
            rd = os.path.join(d, "ref")
            os.makedirs(rd)
            with open(os.path.join(rd, "input"), "w") as f:
                f.write(cfg.input_text())
            subprocess.run([REF_EXE], cwd=rd, check=True, stdout=subprocess.DEVNULL, timeout=600)
            scale = float(np.max(np.abs(ref)))
            for name in ("real_G1.txt", "imag_G1.txt", "dipole.txt", "progress.txt"):
                a = open(os.path.join(d, name)).read().split()
                b = open(os.path.join(rd, name)).read().split()
                assert len(a) == len(b), name
                fa, fb = np.array(a, dtype=float), np.array(b, dtype=float)
                # entries that are round-off (e.g. Re G1 of i*rho) print as noise
                big = np.abs(fb) > 1e-9 * scale
                assert np.all(np.abs(fa[~big] - fb[~big]) <= 1e-12 * scale), name
                same = np.mean([x == y for x, y, k in zip(a, b, big) if k]) if big.any() else 1.0
                # identical text except where a ~1e-15 difference straddles a 6th-digit rounding
                assert same >= 0.99, (name, same)
