"""Host-side logic of libg12kba.so (no GPU needed): the C ABI loads and exports
every symbol of include/g12kba.h, the input reader reproduces read_input.h's
quirks, schedule counts, G0, dipole and the text writers."""
import ctypes
import json
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, load_golden, rel_err
from oracle import REF_EXE, Config, Reference


def header_symbols():
    src = open(os.path.join(ROOT, "include", "g12kba.h")).read()
    return sorted(set(re.findall(r"\b(g12_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol(g12):
    lib = ctypes.CDLL(g12.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_no_device_fails_loudly(g12):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    p = g12.make_params(Ns=2, Nb=1)
    with pytest.raises(g12.G12Error):
        g12.Context(p)


def test_defaults_match_reference(g12):
    p = g12.default_params()
    assert (p.Ns, p.Nb, p.Nq, p.time_steps) == (2, 1, 0, 1000)
    assert (p.U, p.dt, p.t1, p.AS_rate, p.AS_midpoint) == (0.5, 0.02, 1.0, 3.0, 25.0)
    assert (p.quench_gate, p.as_dt, p.decay_rate) == (50.0, 0.1, 0.7)


INPUTS = {
    "sample": open(os.path.join(ROOT, "tests", "golden", "sample_input")).read()
    if os.path.exists(os.path.join(ROOT, "tests", "golden", "sample_input")) else None,
    "missing_keys": "HF\nfalse\nU\n2\nNs\n3\n",
    # every numeric key present, EHM missing: past the end std::getline keeps
    # the last line ("pulse"), which is neither true nor false
    "no_trailing_newline": "t1\n1\nt2\n.2\nt3\n0\nU\n1.5\ntime_steps\n10\ndt\n.01\nquench_strength\n1\n"
                           "Ns\n5\nNb\n2\nNq\n1\nAS_rate\n1\nAS_midpoint\n2\nquench_on_midpoint\n3\n"
                           "quench_off_midpoint\n4\nquench_rate\n.5\nHF\ntrue\nq_type\npulse",
    "bad_bool_and_none": "HF\nmaybe\nEHM\nyes\nq_type\nnone\nNq\n3\nquench_strength\n2\nNs\n4\n",
    "invalid_qtype": "q_type\nhalf\nNq\n2\nquench_strength\n2.5\nNs\n6\nU\n1\n",
    "crlf": "HF\r\nfalse\r\nNs\r\n4\r\nU\r\n0.75\r\n",
    "substring": "U_x\n7\nU\n3\nNs\n4\ntime_steps\n12abc\ndt\n 2e-2\n",
}


def _reader_cases():
    return [k for k, v in INPUTS.items() if v is not None]


@pytest.mark.parametrize("case", _reader_cases())
def test_read_input_matches_restatement(g12, oracle, case):
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "input")
        with open(path, "w", newline="") as f:
            f.write(INPUTS[case])
        p, log = g12.read_input(path)
        rc, q, qlog = oracle.read_input(path)
    assert rc == 0
    assert log == qlog
    for k in ("Ns", "Nb", "Nq", "time_steps", "HF", "EHM", "t1", "t2", "t3", "U", "dt", "quench_strength",
              "AS_rate", "AS_midpoint", "quench_rate", "quench_on_midpoint", "quench_off_midpoint"):
        assert getattr(p, k) == q[k], k
    assert p.q_type == q["q_pulse"]


@pytest.mark.parametrize("case", _reader_cases())
def test_read_input_matches_reference_binary(g12, case):
    if not os.path.exists(REF_EXE):
        pytest.skip("compiled reference not built here")
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "input"), "w", newline="") as f:
            f.write(INPUTS[case])
        out = subprocess.run([REF_EXE, "--print-params"], cwd=d, capture_output=True, text=True, check=True).stdout
        p, log = g12.read_input(os.path.join(d, "input"))
    lines = out.splitlines()
    ref = json.loads(lines[-1])
    assert "\n".join(lines[:-1]) + ("\n" if len(lines) > 1 else "") == log
    for k, v in ref.items():
        if k == "q_type":
            assert ("pulse" if p.q_type == 1 else "full") == v
        else:
            assert getattr(p, k) == v, k


def test_unparseable_value_is_rejected(g12):
    # a missing numeric key on a file without a final newline reads the last
    # line ("pulse"): std::stod throws and the reference terminates
    text = "HF\ntrue\nNs\n5\nq_type\npulse"
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "input")
        with open(path, "w") as f:
            f.write(text)
        with pytest.raises(g12.G12Error):
            g12.read_input(path)
        if os.path.exists(REF_EXE):
            r = subprocess.run([REF_EXE, "--print-params"], cwd=d, capture_output=True, text=True)
            assert r.returncode != 0


def test_schedule_counts(g12, oracle):
    for kw in [dict(U=1.0, AS_rate=0.5, AS_midpoint=10, dt=0.02, time_steps=2000),
               dict(U=0.5, AS_rate=3, AS_midpoint=25, dt=0.07, time_steps=15000),
               dict(U=2.0, AS_rate=0.5, AS_midpoint=10, dt=0.01, time_steps=5000),
               dict(U=0.0, AS_rate=0.5, AS_midpoint=10, dt=0.01, time_steps=6000)]:
        p = g12.make_params(Ns=4, Nb=1, **kw)
        c = Config(Ns=4, Nb=1, **kw)
        assert g12.as_steps(p) == oracle.as_steps(c)
        assert g12.rk_iterations(p) == oracle.rk_iterations(c)


@pytest.mark.parametrize("Ns,Nb,t2", [(4, 1, 0.0), (8, 2, 0.5), (16, 2, 0.3), (5, 3, 0.2), (1, 2, 0.7), (12, 2, 0.41)])
def test_make_G0_bit_identical(g12, oracle, Ns, Nb, t2):
    p = g12.make_params(Ns=Ns, Nb=Nb, t2=t2)
    mine = g12.make_G0(p)
    ref = oracle.make_G0(Ns, Nb, Ns // 2, 1.0, t2)
    assert np.array_equal(mine, ref)
    # a rank-(Ns/2) projector times i, to complex64 accuracy
    rho = -1j * mine
    assert np.allclose(rho @ rho, rho, atol=2e-6)
    assert abs(np.trace(rho).real - Ns // 2) < 1e-5


def test_dipole_matches_golden(g12):
    g = load_golden("routines.npz")
    for tag in ("3x2", "5x1", "4x2"):
        assert rel_err(g12.dipole(g[tag + "/traj"]), g[tag + "/dipole"]) <= 1e-14


def test_writers_match_reference_text(g12):
    if not os.path.exists(REF_EXE):
        pytest.skip("compiled reference not built here")
    cfg = Config(Ns=3, Nb=1, Nq=1, time_steps=25, U=1.0, dt=0.02, AS_rate=0.5, AS_midpoint=2)
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "input"), "w") as f:
            f.write(cfg.input_text())
        dump = os.path.join(d, "dump")
        os.makedirs(dump)
        subprocess.run([REF_EXE, "--dump", dump], cwd=d, check=True, stdout=subprocess.DEVNULL)
        traj = np.fromfile(os.path.join(dump, "traj.bin"), np.complex128).reshape(-1, 3, 3)
        p = np.fromfile(os.path.join(dump, "dipole.bin"))
        mine = os.path.join(d, "mine")
        os.makedirs(mine)
        cwd = os.getcwd()
        os.chdir(mine)
        try:
            g12.lib().g12_write_cfile2D(b"G1.txt", traj.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        traj.shape[0], 9)
            g12.lib().g12_write_rfile(b"dipole.txt", p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), p.size)
        finally:
            os.chdir(cwd)
        for name in ("real_G1.txt", "imag_G1.txt", "dipole.txt"):
            assert open(os.path.join(d, name)).read() == open(os.path.join(mine, name)).read(), name


def test_writers_g_format_wide_range(g12, tmp_path):
    """The text writers format every value as the reference's streams do
    (default precision 6, i.e. printf %g): values over the whole exponent range,
    ties at the sixth significant digit, signed zeros, subnormals and integers;
    and a 2-D file with more rows than one pass of the multithreaded writer (16
    threads x 64-row blocks) and a ragged last pass, rows in order."""
    rng = np.random.default_rng(11)
    vals = np.concatenate([
        rng.standard_normal(4000) * 10.0 ** rng.integers(-300, 300, 4000),
        np.array([0.0, -0.0, 1.0, -1.0, 123456.5, 1234565.0, 0.1234565, 1e-5, 9.999995e-5, 1e16, 5e-324,
                  1.7976931348623157e308]),
        np.round(rng.standard_normal(500) * 1e6),
    ])
    rfile = tmp_path / "dipole.txt"
    assert g12.lib().g12_write_rfile(str(rfile).encode(), vals.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     vals.size) == 0
    assert rfile.read_text() == "".join("%g\n" % v for v in vals)
    T, n2 = 7, 2 * 16 * 64 + 5
    z = (rng.standard_normal((T, n2)) + 1j * rng.standard_normal((T, n2))) * 10.0 ** rng.integers(-8, 8, (T, n2))
    z = np.ascontiguousarray(z)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rc = g12.lib().g12_write_cfile2D(b"G1.txt", z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), T, n2)
    finally:
        os.chdir(cwd)
    assert rc == 0
    for part, name in ((z.real, "real_G1.txt"), (z.imag, "imag_G1.txt")):
        want = "".join("".join("%g " % part[i, j] for i in range(T)) + "\n" for j in range(n2))
        assert (tmp_path / name).read_text() == want, name


def test_ensemble_generator_is_seeded(g12):
    a = g12.ensemble_params(16)
    b = g12.ensemble_params(16)
    assert [p.as_dict() for p in a] == [p.as_dict() for p in b]
    for p in a:
        assert p.Ns in (4, 6, 8, 10, 12) and p.Nb in (1, 2)
        assert 0.5 <= p.U <= 2.5 and 0.5 <= p.quench_strength <= 3.0 and p.Nq == p.Ns // 3
        assert p.EHM == 1 and p.v_law == 1 and p.dt == 0.01
