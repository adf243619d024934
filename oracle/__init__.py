"""Oracle test infrastructure: ctypes bindings for the CPU checkers.

Two checkers live here, both used only by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg:

* ``libg12oracle.so`` - the plain-C FP64 restatement of the reference algorithm
  (``g12_oracle.c``; each routine cites the reference file:line it restates);
* ``_ref/libg12ref.so`` and ``_ref/g12_ref`` - the reference's own headers
  compiled against a self-written MKL shim (``build_ref.sh``), present where
  the reference tree was available at build time.

Arrays are numpy complex128.  G1 is (n, n) row-major with orbital index
``site + band*Ns``; G2 arrays use the reference's flat IDX_8D layout
(``commutators.h:60``) of length n**4.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libg12oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "libg12ref.so")
REF_EXE = os.path.join(REF_DIR, "g12_ref")

_dp = C.POINTER(C.c_double)


class OracleParams(C.Structure):
    """Mirror of ``oracle_params`` (g12_oracle.h)."""

    _fields_ = [
        ("Ns", C.c_int), ("Nb", C.c_int), ("Nq", C.c_int), ("time_steps", C.c_int),
        ("HF", C.c_int), ("EHM", C.c_int), ("q_pulse", C.c_int), ("vlaw", C.c_int),
        ("t1", C.c_double), ("t2", C.c_double), ("t3", C.c_double), ("U", C.c_double),
        ("dt", C.c_double), ("quench_strength", C.c_double),
        ("AS_rate", C.c_double), ("AS_midpoint", C.c_double), ("quench_rate", C.c_double),
        ("quench_on_midpoint", C.c_double), ("quench_off_midpoint", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


@dataclasses.dataclass
class Config:
    """A reference ``input`` file's contents (read_input.h:27-49 defaults)."""

    Ns: int = 2
    Nb: int = 1
    Nq: int = 0
    time_steps: int = 1000
    HF: bool = False
    EHM: bool = False
    q_type: str = "full"
    vlaw: str = "exp"
    t1: float = 1.0
    t2: float = 0.0
    t3: float = 0.0
    U: float = 0.5
    dt: float = 0.02
    quench_strength: float = 1.0
    AS_rate: float = 3.0
    AS_midpoint: float = 25.0
    quench_rate: float = 0.2
    quench_on_midpoint: float = 50.0
    quench_off_midpoint: float = 55.0

    @property
    def n(self):
        return self.Ns * self.Nb

    def to_c(self) -> OracleParams:
        p = OracleParams()
        for f in ("Ns", "Nb", "Nq", "time_steps"):
            setattr(p, f, int(getattr(self, f)))
        p.HF, p.EHM = int(self.HF), int(self.EHM)
        qs, nq, pulse = self.quench_strength, self.Nq, 0
        if self.q_type == "pulse":
            pulse = 1
        elif self.q_type == "none":
            qs, nq = 0.0, 0
        p.q_pulse, p.quench_strength, p.Nq = pulse, float(qs), int(nq)
        p.vlaw = 1 if self.vlaw == "inv" else 0
        for f in ("t1", "t2", "t3", "U", "dt", "AS_rate", "AS_midpoint", "quench_rate",
                  "quench_on_midpoint", "quench_off_midpoint"):
            setattr(p, f, float(getattr(self, f)))
        return p

    def input_text(self, extra: dict | None = None) -> str:
        """The reference's alternating key/value-line ``input`` format."""
        def fmt(v):
            if isinstance(v, bool):
                return "true" if v else "false"
            return repr(v) if isinstance(v, float) else str(v)
        keys = ["HF", "EHM", "t1", "t2", "t3", "U", "time_steps", "dt", "quench_strength", "Ns",
                "Nq", "Nb", "q_type", "AS_rate", "AS_midpoint", "quench_rate",
                "quench_on_midpoint", "quench_off_midpoint"]
        lines = []
        for k in keys:
            lines += [k, fmt(getattr(self, k))]
        if self.vlaw != "exp":
            lines += ["V_law", self.vlaw]
        for k, v in (extra or {}).items():
            lines += [k, fmt(v)]
        return "\n".join(lines) + "\n"

    def vvec(self, u=None):
        """The long-range V(r), r = 1..Ns-1 (AS.h:136-140) for EHM, else empty."""
        u = self.U if u is None else u
        if not self.EHM:
            return np.zeros(0)
        r = np.arange(1, self.Ns, dtype=np.float64)
        law = 1.0 / (1.0 + r) if self.vlaw == "inv" else np.exp(-0.7 * r)
        return u * law


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _c(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a if shape is None else a.reshape(shape)


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE, "libg12oracle.so"], check=True)


class _Lib:
    """Per-function numpy wrappers shared by the restatement and the compiled reference."""

    def __init__(self, path, prefix):
        self.lib = C.CDLL(path)
        self.p = prefix
        self.path = path

    def fn(self, name):
        return getattr(self.lib, self.p + name)

    def fermi(self, t, t0, tau):
        f = self.fn("fermi")
        f.restype = C.c_double
        return f(C.c_double(t), C.c_double(t0), C.c_double(tau))

    def h_hf(self, G1, Ns, Nb, U, t1, t2, w, V, Nq):
        n = Ns * Nb
        G1 = _c(G1)
        V = np.ascontiguousarray(V, dtype=np.float64)
        h = np.zeros((n, n), np.complex128)
        self.fn("h_HFx_quench")(_ptr(h), _ptr(G1), Ns, Nb, C.c_double(U), C.c_double(t1),
                                C.c_double(t2), C.c_double(w), _ptr(V), len(V), Nq)
        return h

    def hG_comm(self, G, h):
        G, h = _c(G), _c(h)
        out = np.zeros_like(G)
        self.fn("hG_commutator")(_ptr(G), _ptr(h), _ptr(out), G.shape[0])
        return out

    def h2_comm(self, G2, h, Ns, Nb):
        G2, h = _c(G2), _c(h)
        out = np.zeros_like(G2)
        self.fn("h2_commutator")(_ptr(G2), _ptr(h), _ptr(out), Ns, Nb)
        return out

    def psi(self, G1, Ns, Nb, U, V, xy):
        n = Ns * Nb
        G1 = _c(G1)
        V = np.ascontiguousarray(V, dtype=np.float64)
        out = np.zeros(n ** 4, np.complex128)
        self.fn("psi_xyxy" if xy else "psi_xxxx")(_ptr(out), _ptr(G1), Ns, Nb, C.c_double(U),
                                                 _ptr(V), len(V))
        return out

    def pi(self, G1, G2a, G2b, U, Ns, Nb, V):
        G1, G2a, G2b = _c(G1), _c(G2a), _c(G2b)
        V = np.ascontiguousarray(V, dtype=np.float64)
        out = np.zeros_like(G2a)
        self.fn("pi")(_ptr(out), _ptr(G1), _ptr(G2a), _ptr(G2b), C.c_double(U), Ns, Nb, _ptr(V), len(V))
        return out

    def collision(self, G2xy, G2xx, Ns, Nb, U, V):
        n = Ns * Nb
        G2xy, G2xx = _c(G2xy), _c(G2xx)
        V = np.ascontiguousarray(V, dtype=np.float64)
        out = np.zeros((n, n), np.complex128)
        self.fn("collision")(_ptr(out), _ptr(G2xy), _ptr(G2xx), Ns, Nb, C.c_double(U), _ptr(V), len(V))
        return out

    def G1_step(self, comm, Ix, RK, w, Ns, Nb):
        comm, Ix = _c(comm), _c(Ix)
        RK = _c(RK).copy()
        K = np.zeros_like(comm)
        last = Ns * Nb if self.p == "oracle_" else None
        if last is None:
            self.fn("G1_step")(_ptr(comm), _ptr(Ix), _ptr(K), _ptr(RK), C.c_double(w), Ns, Nb)
        else:
            self.fn("G1_step")(_ptr(comm), _ptr(Ix), _ptr(K), _ptr(RK), C.c_double(w), last)
        return K, RK

    def G2_step(self, comm, psi, pi, RK, w, Ns, Nb):
        comm, psi, pi = _c(comm), _c(psi), _c(pi)
        RK = _c(RK).copy()
        K = np.zeros_like(comm)
        self.fn("G2_step")(_ptr(comm), _ptr(psi), _ptr(pi), _ptr(K), _ptr(RK), C.c_double(w), Ns, Nb)
        return K, RK

    def make_G0(self, Ns, Nb, p_number, t1, t2):
        n = Ns * Nb
        out = np.zeros((n, n), np.complex128)
        self.fn("make_G0")(_ptr(out), Ns, Nb, p_number, C.c_double(t1), C.c_double(t2))
        return out

    def dipole(self, traj):
        traj = _c(traj)
        T = traj.shape[0]
        n = int(round(np.sqrt(traj[0].size)))
        p = np.zeros(T)
        if self.p == "oracle_":
            self.fn("dipole")(_ptr(p), _ptr(traj), C.c_int64(T), n)
        else:
            self.fn("dipole")(_ptr(p), _ptr(traj), T, n * n)
        return p


class Oracle(_Lib):
    """The plain-C restatement (g12_oracle.c)."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        super().__init__(ORACLE_SO, "oracle_")
        L = self.lib
        L.oracle_as_steps.restype = C.c_int64
        L.oracle_rk_iterations.restype = C.c_int64
        L.oracle_run.restype = C.c_int64
        L.oracle_run.argtypes = [C.POINTER(OracleParams), _dp, C.c_int, _dp, C.c_int64, _dp, _dp, _dp]
        L.oracle_step.argtypes = [C.POINTER(OracleParams), C.c_int, C.c_double, _dp, _dp, _dp, _dp]
        L.oracle_read_input.argtypes = [C.c_char_p, C.POINTER(OracleParams), C.c_char_p, C.c_int]

    def as_steps(self, cfg: Config) -> int:
        p = cfg.to_c()
        return int(self.lib.oracle_as_steps(C.byref(p)))

    def rk_iterations(self, cfg: Config) -> int:
        p = cfg.to_c()
        return int(self.lib.oracle_rk_iterations(C.byref(p)))

    def step(self, cfg: Config, phase, t, t_temp, G1, G2xx, G2xy):
        """One RK4 step in place (phase 0 = adiabatic switching, 1 = propagation)."""
        p = cfg.to_c()
        tt = C.c_double(t_temp)
        self.lib.oracle_step(C.byref(p), phase, C.c_double(t), C.byref(tt), _ptr(G1), _ptr(G2xx), _ptr(G2xy))
        return tt.value

    def run(self, cfg: Config, G0, skip_as=False, max_T=None):
        """AS then RK4 from G0: returns (traj[T, n, n], G1, G2xx, G2xy)."""
        n = cfg.n
        p = cfg.to_c()
        if max_T is None:
            max_T = self.rk_iterations(cfg)
        traj = np.zeros((max(max_T, 1), n, n), np.complex128)
        G1 = np.zeros((n, n), np.complex128)
        XX = np.zeros(n ** 4, np.complex128)
        XY = np.zeros(n ** 4, np.complex128)
        G0 = _c(G0, (n, n))
        T = self.lib.oracle_run(C.byref(p), _ptr(G0), int(skip_as), _ptr(traj), max_T, _ptr(G1), _ptr(XX), _ptr(XY))
        return traj[:T], G1, XX, XY

    def read_input(self, path):
        p = OracleParams()
        log = C.create_string_buffer(1 << 16)
        rc = self.lib.oracle_read_input(path.encode(), C.byref(p), log, len(log))
        return rc, p.as_dict(), log.value.decode()


class Reference(_Lib):
    """The reference's headers compiled against the MKL shim (oracle/_ref)."""

    def __init__(self):
        super().__init__(REF_SO, "ref_")
        self.lib.ref_fermi.restype = C.c_double

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO) and os.path.exists(REF_EXE)


def run_reference_exe(cfg: Config, workdir, g0=None, skip_as=False, no_text=True, timeout=3600):
    """Runs oracle/_ref/g12_ref on ``cfg`` in ``workdir``; returns the dumps."""
    os.makedirs(workdir, exist_ok=True)
    with open(os.path.join(workdir, "input"), "w") as f:
        f.write(cfg.input_text())
    dump = os.path.join(workdir, "dump")
    os.makedirs(dump, exist_ok=True)
    cmd = [REF_EXE, "--vlaw", cfg.vlaw, "--dump", dump]
    if g0 is not None:
        g0p = os.path.join(workdir, "g0_in.bin")
        _c(g0).tofile(g0p)
        cmd += ["--g0", g0p]
    if skip_as:
        cmd.append("--skip-as")
    if no_text:
        cmd.append("--no-text")
    subprocess.run(cmd, cwd=workdir, check=True, stdout=subprocess.DEVNULL, timeout=timeout)
    n = cfg.n
    rd = lambda name: np.fromfile(os.path.join(dump, name), dtype=np.complex128)
    out = {
        "g0": rd("g0.bin").reshape(n, n),
        "g1_as": rd("g1_as.bin").reshape(n, n),
        "g2xx_as": rd("g2xx_as.bin"),
        "g2xy_as": rd("g2xy_as.bin"),
        "traj": rd("traj.bin").reshape(-1, n, n),
        "g2xx": rd("g2xx.bin"),
        "g2xy": rd("g2xy.bin"),
        "dipole": np.fromfile(os.path.join(dump, "dipole.bin"), dtype=np.float64),
    }
    return out


def pair_index(Ns, Nb):
    """[p, q] -> IDX_8D position of G2[p q; p q] (commutators.h:60 with
    mu1 = nu1 = p = (i, a), mu2 = nu2 = q = (j, b))."""
    n = Ns * Nb
    mu = np.arange(n)
    s, b = mu % Ns, mu // Ns
    i, a = s[:, None], b[:, None]
    j, bb = s[None, :], b[None, :]
    Ns2, Nb2 = Ns * Ns, Nb * Nb
    return (i + j * Ns) + (a + bb * Nb) * Ns2 + (i + j * Ns) * Ns2 * Nb2 + (a + bb * Nb) * Ns2 * Ns2 * Nb2


def pair_weights(cfg: Config, U):
    """Pair interaction (w_xx, w_xy)[p, q] of the collision integral
    (collision_integral.h:41-62): on one site U (w_xx: different bands only),
    between sites m apart V_m (AS.h:136-140 law at U)."""
    n, Ns = cfg.n, cfg.Ns
    mu = np.arange(n)
    s, b = mu % Ns, mu // Ns
    d = np.abs(s[:, None] - s[None, :])
    V = cfg.vvec(U)
    Vd = np.zeros((n, n))
    for m in range(1, len(V) + 1):
        Vd[d == m] = V[m - 1]
    wxy = np.where(d == 0, U, Vd)
    wxx = np.where(d == 0, np.where(b[:, None] != b[None, :], U, 0.0), Vd)
    return wxx, wxy


def total_energy(o: "_Lib", cfg: Config, G1, G2xx, G2xy, U=None, w_quench=0.0, Nq=0):
    """Total energy [E, 2 Tr[h0 rho], Tr[(h - h0) rho], correlation part] of a
    state (G2 in the IDX_8D layout).  The reference computes none: this is the
    energy its equations conserve while h0 and U are constant, with h from the
    restated HF.h:57-104 (h0: the same at G1 = 0) and the pair weights of
    collision_integral.h:41-62:
        E = 2 Tr[h0 rho] + Tr[(h - h0) rho] - Re sum w_xx G2xx[pq;pq] + w_xy G2xy[pq;pq]."""
    U = cfg.U if U is None else U
    n = cfg.n
    G1 = _c(G1, (n, n))
    V = cfg.vvec(U)
    h = o.h_hf(G1, cfg.Ns, cfg.Nb, U, cfg.t1, cfg.t2, w_quench, V, Nq)
    h0 = o.h_hf(np.zeros((n, n), np.complex128), cfg.Ns, cfg.Nb, U, cfg.t1, cfg.t2, w_quench, V, Nq)
    rho = -1j * G1
    e0 = 2.0 * np.trace(h0 @ rho).real
    eh = np.trace((h - h0) @ rho).real
    wxx, wxy = pair_weights(cfg, U)
    I = pair_index(cfg.Ns, cfg.Nb)
    ec = -float(np.sum(wxx * np.asarray(G2xx)[I].real + wxy * np.asarray(G2xy)[I].real))
    return np.array([e0 + eh + ec, e0, eh, ec])


def idx8_to_orbital(Ns, Nb):
    """Permutation p with orbital_flat = ref_flat[p] where orbital_flat is
    indexed nu1 + n*nu2 + n^2*mu1 + n^3*mu2 (mu = site + band*Ns)."""
    n = Ns * Nb
    mu = np.arange(n)
    s, b = mu % Ns, mu // Ns
    # reference IDX_8D(k,l,g,d,i,j,a,b)
    nu1 = mu[None, None, None, :]
    nu2 = mu[None, None, :, None]
    mu1 = mu[None, :, None, None]
    mu2 = mu[:, None, None, None]
    Ns2, Nb2 = Ns * Ns, Nb * Nb
    ref = (s[nu1] + s[nu2] * Ns + (b[nu1] + b[nu2] * Nb) * Ns2
           + (s[mu1] + s[mu2] * Ns) * Ns2 * Nb2 + (b[mu1] + b[mu2] * Nb) * Ns2 * Ns2 * Nb2)
    return ref.reshape(-1)
