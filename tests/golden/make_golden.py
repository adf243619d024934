"""Generates the golden vectors in tests/golden/ from the compiled reference.

The reference (VlcekGroup/G12KBA) ships no tests or golden data, so these
fixtures are outputs of its own routines, compiled from its headers by
oracle/build_ref.sh (oracle/_ref/libg12ref.so for per-routine cases,
oracle/_ref/g12_ref for full Main.cpp runs).  Inputs are seeded random
complex arrays or the physics configurations listed below.

Run from the repository root:  python tests/golden/make_golden.py
(``python tests/golden/make_golden.py energy`` writes energy_pin.npz alone;
``... baseline [name ...]`` the full-length benchmark-configuration runs).
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import Config, Reference, run_reference_exe  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (Ns, Nb) shapes for per-routine vectors: odd Ns, Nb = 1..3, Ns = 1 edge
SHAPES = [(1, 2), (2, 1), (3, 1), (2, 2), (3, 2), (2, 3), (4, 2), (5, 1)]

RUNS = {
    # the Ns=4, Nb=1 chain (U=1, t1=1, dt=0.02), shortened to 200 of its 2000 steps
    "run_c1_short": Config(Ns=4, Nb=1, Nq=2, time_steps=200, U=1.0, t1=1.0, t2=0.0, dt=0.02,
                           AS_rate=0.5, AS_midpoint=10, q_type="full", quench_strength=1.0),
    # extended model, Nb = 2, U/(1+r) law, pulse quench (masked by the t < 50 gate)
    "run_ehm_nb2": Config(Ns=3, Nb=2, Nq=1, time_steps=60, U=2.0, t1=1.0, t2=0.5, dt=0.01, EHM=True,
                          vlaw="inv", q_type="pulse", quench_strength=2.0, quench_rate=2,
                          quench_on_midpoint=15, quench_off_midpoint=25, AS_rate=0.5, AS_midpoint=2),
    # quench switched on at t >= 50: dt = 0.05, 1100 steps, exp law
    "run_quench_on": Config(Ns=4, Nb=1, Nq=2, time_steps=1100, U=1.0, t1=1.0, dt=0.05, EHM=True,
                            q_type="full", quench_strength=1.0, quench_rate=0.2, quench_on_midpoint=52,
                            AS_rate=0.5, AS_midpoint=3),
    # HF-only propagation (G2 frozen at zero, RK_solver.h:154)
    "run_hf": Config(Ns=5, Nb=1, Nq=2, time_steps=300, U=1.5, t1=1.0, dt=0.02, HF=True,
                     AS_rate=1.0, AS_midpoint=5),
    # unstable step size: the site-0 density jumps past |2 Im G1_00| = 3 while
    # still finite, and the guard stops RK4 (RK_solver.h:101-110)
    "run_guard": Config(Ns=3, Nb=1, Nq=1, time_steps=200, U=4.0, t1=1.0, dt=0.35,
                        AS_rate=0.5, AS_midpoint=2),
}


def per_routine(ref):
    rng = np.random.default_rng(20261203)
    out = {}
    for Ns, Nb in SHAPES:
        n = Ns * Nb
        tag = f"{Ns}x{Nb}"
        G1 = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        G2a = rng.standard_normal(n ** 4) + 1j * rng.standard_normal(n ** 4)
        G2b = rng.standard_normal(n ** 4) + 1j * rng.standard_normal(n ** 4)
        V = rng.random(max(Ns - 1, 0))
        U, t1, t2, w, Nq = 0.8, 1.0, 0.4, 0.3, min(2, Ns)
        h = ref.h_hf(G1, Ns, Nb, U, t1, t2, w, V, Nq)
        RK1 = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        RK2 = rng.standard_normal(n ** 4) + 1j * rng.standard_normal(n ** 4)
        comm1 = ref.hG_comm(G1, h)
        C2 = ref.h2_comm(G2a, h, Ns, Nb)
        psi_xx = ref.psi(G1, Ns, Nb, U, V, 0)
        psi_xy = ref.psi(G1, Ns, Nb, U, V, 1)
        pi_ab = ref.pi(G1, G2a, G2b, U, Ns, Nb, V)
        coll = ref.collision(G2a, G2b, Ns, Nb, U, V)
        K1, RK1o = ref.G1_step(comm1, coll, RK1, 2.0, Ns, Nb)
        K2, RK2o = ref.G2_step(C2, psi_xy, pi_ab, RK2, 2.0, Ns, Nb)
        g0 = ref.make_G0(Ns, Nb, Ns // 2, t1, t2)
        tr = rng.standard_normal((7, n, n)) + 1j * rng.standard_normal((7, n, n))
        dip = ref.dipole(tr)
        for k, v in dict(G1=G1, G2a=G2a, G2b=G2b, V=V, h=h, comm1=comm1, C2=C2, psi_xx=psi_xx,
                         psi_xy=psi_xy, pi_ab=pi_ab, coll=coll, RK1=RK1, RK2=RK2, K1=K1, RK1o=RK1o,
                         K2=K2, RK2o=RK2o, g0=g0, traj=tr, dipole=dip).items():
            out[f"{tag}/{k}"] = v
        out[f"{tag}/scalars"] = np.array([U, t1, t2, w, Nq], dtype=np.float64)
    np.savez_compressed(os.path.join(OUT, "routines.npz"), **out)


def full_runs():
    for name, cfg in RUNS.items():
        with tempfile.TemporaryDirectory() as d:
            r = run_reference_exe(cfg, d)
        traj = r["traj"]
        keep = {
            "g0": r["g0"], "g1_as": r["g1_as"], "g2xx_as": r["g2xx_as"], "g2xy_as": r["g2xy_as"],
            "g2xx": r["g2xx"], "g2xy": r["g2xy"], "dipole": r["dipole"],
            "T": np.array(traj.shape[0]),
        }
        if traj.shape[0] > 300:
            keep["traj_every10"] = traj[::10]
            keep["traj_last"] = traj[-1]
        else:
            keep["traj"] = traj
        for k, v in cfg.__dict__.items():
            keep["cfg_" + k] = np.array(v)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **keep)
        print(name, "T =", traj.shape[0], "max|G2| =", float(np.max(np.abs(r["g2xx"]))))


# The benchmark configurations at their stated lengths (the reference's own
# RK_solver.h:96 loop, AS.h:63 switching first).  Config 2 leaves the switching
# parameters at the reference defaults (AS_rate 3, AS_midpoint 25: 1373
# switching steps); config 3 (n = 32) uses a shortened switching phase
# (AS_rate 0.5, AS_midpoint 3: 234 steps) so that the compiled reference
# finishes it in minutes, then 20 RK4 steps.  The pulse of config 2 and the
# quench of config 3 stay masked by the reference's t < 50 gate.
BASELINE_RUNS = {
    "run_c1_full": Config(Ns=4, Nb=1, Nq=2, time_steps=2000, U=1.0, t1=1.0, t2=0.0, dt=0.02,
                          AS_rate=0.5, AS_midpoint=10, q_type="full", quench_strength=1.0),
    "run_c2_full": Config(Ns=8, Nb=2, Nq=3, time_steps=5000, U=2.0, t1=1.0, t2=0.5, dt=0.01, EHM=True,
                          vlaw="inv", q_type="pulse", quench_strength=2.0, quench_rate=2,
                          quench_on_midpoint=15, quench_off_midpoint=25),
    "run_c3_20": Config(Ns=16, Nb=2, Nq=4, time_steps=20, U=1.5, t1=1.0, t2=0.3, dt=0.01, EHM=True,
                        vlaw="inv", q_type="full", quench_strength=1.5, AS_rate=0.5, AS_midpoint=3),
}
# seeded complex test vectors for the G2 checksums (projections) of large runs
N_PROJ = 8


def g2_projections(G2, seed=7):
    """N_PROJ linear functionals of a G2 tensor (reference layout): a checksum
    of the full state that stays small for n = 16 and 32."""
    rng = np.random.default_rng(seed)
    P = rng.standard_normal((N_PROJ, G2.size)) + 1j * rng.standard_normal((N_PROJ, G2.size))
    return P @ G2.reshape(-1)


def baseline_runs(names=None):
    for name, cfg in BASELINE_RUNS.items():
        if names and name not in names:
            continue
        with tempfile.TemporaryDirectory() as d:
            r = run_reference_exe(cfg, d, timeout=4 * 3600)
        traj = r["traj"]
        T = traj.shape[0]
        every = 1 if T <= 40 else 25
        keep = {"g0": r["g0"], "g1_as": r["g1_as"], "dipole": r["dipole"], "T": np.array(T),
                "every": np.array(every), "traj_sub": traj[::every], "traj_last": traj[-1],
                "g2xx_as_proj": g2_projections(r["g2xx_as"]), "g2xy_as_proj": g2_projections(r["g2xy_as"]),
                "g2xx_proj": g2_projections(r["g2xx"]), "g2xy_proj": g2_projections(r["g2xy"]),
                "g2_norms": np.array([np.linalg.norm(r[k]) for k in ("g2xx_as", "g2xy_as", "g2xx", "g2xy")])}
        if cfg.n <= 16:
            keep["g2xx"], keep["g2xy"] = r["g2xx"], r["g2xy"]
        for k, v in cfg.__dict__.items():
            keep["cfg_" + k] = np.array(v)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **keep)
        print(name, "T =", T, "max|G2| =", float(np.max(np.abs(r["g2xx"]))), flush=True)


def roundoff_sensitivity(name="run_c2_full"):
    """The reference's own sensitivity to round-off on a benchmark run: the same
    input with G0 moved by one ulp in a seeded half of its (nonzero imaginary)
    entries.  Stores the
    perturbed run's G1 (every 25th snapshot and the last), its dipole and its
    final G2 checksums; the deviation from the unperturbed golden run is what
    two correct FP64 implementations of these equations can differ by."""
    cfg = BASELINE_RUNS[name]
    g = np.load(os.path.join(OUT, f"{name}.npz"))
    g0 = g["g0"].copy()
    rng = np.random.default_rng(11)
    mask = rng.random(g0.shape) < 0.5
    # G0 = i rho with rho real here: move the imaginary parts (the real parts are zero)
    g0 = np.where(mask & (g0.imag != 0), g0.real + 1j * np.nextafter(g0.imag, np.inf), g0)
    with tempfile.TemporaryDirectory() as d:
        r = run_reference_exe(cfg, d, g0=g0, timeout=4 * 3600)
    traj = r["traj"]
    every = int(g["every"])
    keep = {"g0": g0, "traj_sub": traj[::every], "traj_last": traj[-1], "dipole": r["dipole"],
            "g1_as": r["g1_as"], "g2xx_proj": g2_projections(r["g2xx"]), "g2xy_proj": g2_projections(r["g2xy"])}
    np.savez_compressed(os.path.join(OUT, f"{name}_ulp.npz"), **keep)
    dev = np.max(np.abs(traj[::every] - g["traj_sub"])) / np.max(np.abs(g["traj_sub"]))
    print(name, "one-ulp G0 perturbation: max G1 deviation", dev, flush=True)


# total-energy pin: the state after adiabatic switching and the state after the
# T RK4 iterations of a run (constant U, quench masked by the t < 50 gate), at
# two step sizes over the same simulated time
ENERGY_PIN = {
    "dt02": Config(Ns=4, Nb=2, Nq=1, time_steps=150, U=1.5, t1=1.0, t2=0.3, dt=0.02, EHM=True,
                    vlaw="inv", q_type="full", quench_strength=1.0, AS_rate=0.5, AS_midpoint=3),
    "dt01": Config(Ns=4, Nb=2, Nq=1, time_steps=300, U=1.5, t1=1.0, t2=0.3, dt=0.01, EHM=True,
                    vlaw="inv", q_type="full", quench_strength=1.0, AS_rate=0.5, AS_midpoint=3),
}


def energy_pin():
    """G1 and both G2 at the same time: the final G2 of a run of T steps and
    G1 at index T of a longer run of the same input (both runs take the same
    steps up to T)."""
    import dataclasses
    out = {}
    for tag, cfg in ENERGY_PIN.items():
        with tempfile.TemporaryDirectory() as d:
            a = run_reference_exe(cfg, d)
        T = a["traj"].shape[0]  # while (t < tmax) iterations (RK_solver.h:96)
        longer = dataclasses.replace(cfg, time_steps=cfg.time_steps + 3)
        with tempfile.TemporaryDirectory() as d:
            b = run_reference_exe(longer, d)
        assert np.array_equal(a["traj"], b["traj"][:T])
        out[f"{tag}/g1_0"], out[f"{tag}/g2xx_0"], out[f"{tag}/g2xy_0"] = a["g1_as"], a["g2xx_as"], a["g2xy_as"]
        out[f"{tag}/g1_T"], out[f"{tag}/g2xx_T"], out[f"{tag}/g2xy_T"] = b["traj"][T], a["g2xx"], a["g2xy"]
        out[f"{tag}/T"] = np.array(T)
        for k, v in cfg.__dict__.items():
            out[f"{tag}/cfg_{k}"] = np.array(v)
    np.savez_compressed(os.path.join(OUT, "energy_pin.npz"), **out)


def sample_input():
    """The reference's only fixture (G12KBA-GW/input), kept verbatim as test
    data for the input reader."""
    root = os.environ.get("G12_REFERENCE")
    if not root:
        sys.exit("set G12_REFERENCE to the reference checkout (the directory holding G12KBA-GW/)")
    src = os.path.join(root, "G12KBA-GW", "input")
    with open(src, "rb") as f, open(os.path.join(OUT, "sample_input"), "wb") as g:
        g.write(f.read())


if __name__ == "__main__":
    if not Reference.available():
        sys.exit("build the compiled reference first: oracle/build_ref.sh")
    if sys.argv[1:] == ["energy"]:
        energy_pin()
        sys.exit(0)
    if sys.argv[1:2] == ["baseline"]:
        baseline_runs(sys.argv[2:])
        sys.exit(0)
    if sys.argv[1:] == ["sensitivity"]:
        roundoff_sensitivity()
        sys.exit(0)
    per_routine(Reference())
    full_runs()
    baseline_runs()
    roundoff_sensitivity()
    energy_pin()
    sample_input()
