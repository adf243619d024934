"""g12kba_b200: B200-native HF-GKBA G1-G2 propagation with GW self-energy.

Python bindings (ctypes) over the C ABI of ``libg12kba.so`` declared in
``include/g12kba.h``.  The library is the CUDA implementation; there is no CPU
fallback: loading fails loudly when the shared object has not been built, and
``Context`` creation fails when no B200 is visible.

Arrays are numpy complex128.  G1 is (n, n) with orbital index ``site +
band*Ns``; G2 tensors use the reference's flat IDX_8D layout (length n**4).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libg12kba.so")
CLI_PATH = os.path.join(PKG, "bin", "g12kba")
HEADER = os.path.join(os.path.dirname(PKG), "include", "g12kba.h")

G12_OK = 0
G12_GUARD_TRIPPED = 1
PREC = {"fp64": 0, "tf32x3": 1, "bf16oz": 2, "fp32": 3, "tf32x6": 4, "fp64sym": 5}
QUENCH = {"full": 0, "pulse": 1}
VLAW = {"exp": 0, "inv": 1}

_dp = C.POINTER(C.c_double)


class Params(C.Structure):
    """``g12_params`` (include/g12kba.h)."""

    _fields_ = [
        ("Ns", C.c_int32), ("Nb", C.c_int32), ("Nq", C.c_int32), ("time_steps", C.c_int32),
        ("HF", C.c_int32), ("EHM", C.c_int32), ("q_type", C.c_int32), ("v_law", C.c_int32),
        ("t1", C.c_double), ("t2", C.c_double), ("t3", C.c_double), ("U", C.c_double),
        ("dt", C.c_double), ("quench_strength", C.c_double),
        ("AS_rate", C.c_double), ("AS_midpoint", C.c_double), ("quench_rate", C.c_double),
        ("quench_on_midpoint", C.c_double), ("quench_off_midpoint", C.c_double),
        ("quench_gate", C.c_double), ("as_dt", C.c_double), ("decay_rate", C.c_double),
    ]

    @property
    def n(self):
        return self.Ns * self.Nb

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class G12Error(RuntimeError):
    pass


_lib = None


def build(force: bool = False):
    """Compiles libg12kba.so and bin/g12kba for sm_100a (nvcc; no GPU needed)."""
    args = ["make", "-s", "-C", os.path.join(PKG, "csrc"), "-j8"]
    if force:
        subprocess.run(args[:4] + ["clean"], check=True)
    subprocess.run(args, check=True)


def lib():
    """The loaded libg12kba.so.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise G12Error(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                           "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        L.g12_params_default.argtypes = [C.POINTER(Params)]
        L.g12_read_input.argtypes = [C.c_char_p, C.POINTER(Params), C.c_char_p, C.c_int32]
        L.g12_as_steps.restype = C.c_int64
        L.g12_as_steps.argtypes = [C.POINTER(Params)]
        L.g12_rk_iterations.restype = C.c_int64
        L.g12_rk_iterations.argtypes = [C.POINTER(Params)]
        L.g12_make_G0.argtypes = [C.POINTER(Params), C.c_int32, _dp]
        L.g12_dipole.argtypes = [_dp, C.c_int64, C.c_int32, _dp]
        L.g12_particle_number.argtypes = [_dp, C.c_int64, C.c_int32, _dp]
        L.g12_write_cfile2D.argtypes = [C.c_char_p, _dp, C.c_int64, C.c_int32]
        L.g12_write_rfile.argtypes = [C.c_char_p, _dp, C.c_int64]
        L.g12_create.argtypes = [C.POINTER(Params), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
        L.g12_destroy.argtypes = [C.c_void_p]
        L.g12_last_error.restype = C.c_char_p
        L.g12_last_error.argtypes = [C.c_void_p]
        L.g12_set_state.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.g12_get_state.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.g12_adiabatic_switch.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        L.g12_propagate.argtypes = [C.c_void_p, C.c_int64, _dp, C.POINTER(C.c_int64)]
        L.g12_propagate_dipole.argtypes = [C.c_void_p, C.c_int64, _dp, C.POINTER(C.c_int64)]
        L.g12_rhs.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_double, C.c_double, C.c_int32,
                              _dp, _dp, _dp, _dp, _dp, _dp]
        L.g12_last_device_ms.restype = C.c_double
        L.g12_last_device_ms.argtypes = [C.c_void_p]
        L.g12_total_energy.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int32, _dp]
        L.g12_launches_per_step.restype = C.c_int32
        L.g12_launches_per_step.argtypes = [C.c_void_p]
        L.g12_kernel_times.restype = C.c_int32
        L.g12_kernel_times.argtypes = [C.c_void_p, C.c_int32, _dp, C.POINTER(C.c_int32), C.c_int32]
        L.g12_kernel_name.restype = C.c_char_p
        L.g12_kernel_name.argtypes = [C.c_void_p, C.c_int32]
        L.g12_set_l2_eviction.restype = C.c_int32
        L.g12_set_l2_eviction.argtypes = [C.c_void_p, C.c_int64]
        L.g12_fp64_peak_tflops.restype = C.c_double
        L.g12_fp64_peak_tflops.argtypes = [C.c_int32]
        L.g12_batch_create.argtypes = [C.POINTER(Params), C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
        L.g12_batch_destroy.argtypes = [C.c_void_p]
        L.g12_batch_last_error.restype = C.c_char_p
        L.g12_batch_last_error.argtypes = [C.c_void_p]
        L.g12_batch_set_state.argtypes = [C.c_void_p, C.c_int32, _dp, _dp, _dp]
        L.g12_batch_get_state.argtypes = [C.c_void_p, C.c_int32, _dp, _dp, _dp]
        L.g12_batch_adiabatic_switch.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        L.g12_batch_propagate.argtypes = [C.c_void_p, C.c_int64, _dp, C.POINTER(C.c_int64)]
        L.g12_batch_last_device_ms.restype = C.c_double
        L.g12_batch_last_device_ms.argtypes = [C.c_void_p]
        L.g12_batch_tile.restype = C.c_int32
        L.g12_batch_tile.argtypes = [C.c_void_p, C.c_int32]
        L.g12_rhs_noalloc.argtypes = [C.POINTER(Params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                      C.c_double, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_char_p, C.c_int32]
        _vp, _fp, _i64p = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_int64)
        L.g12_batch_propagate_features.argtypes = [_vp, C.c_int64, C.c_int32, _vp, _dp, _i64p]
        L.g12_mlp_create.argtypes = [C.POINTER(C.c_int32), C.c_int32, C.c_uint64, C.c_int32, C.POINTER(C.c_void_p)]
        L.g12_mlp_destroy.argtypes = [_vp]
        L.g12_mlp_last_error.restype = C.c_char_p
        L.g12_mlp_last_error.argtypes = [_vp]
        L.g12_mlp_param_count.restype = C.c_int64
        L.g12_mlp_param_count.argtypes = [_vp]
        L.g12_mlp_set_params.argtypes = [_vp, _fp]
        L.g12_mlp_get_params.argtypes = [_vp, _fp]
        L.g12_mlp_get_grads.argtypes = [_vp, _fp]
        L.g12_mlp_forward.argtypes = [_vp, _vp, C.c_int32, _vp]
        L.g12_mlp_loss_grad.argtypes = [_vp, _vp, _vp, C.c_int32, _dp]
        L.g12_mlp_adam.argtypes = [_vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float]
        L.g12_mlp_set_norm.argtypes = [_vp, C.c_int32, C.c_int32, C.c_int32, _fp, C.c_float, C.c_float, C.c_float]
        L.g12_mlp_windows.argtypes = [_vp, _vp, C.c_int32, C.c_int64, _i64p, C.c_int32, _vp, _vp]
        L.g12_mlp_grad_windows.argtypes = [_vp, _vp, C.c_int32, C.c_int64, _i64p, C.c_int32, _dp]
        L.g12_mlp_grad_buffer.argtypes = [_vp, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]
        L.g12_mlp_train_windows.argtypes = [_vp, _vp, C.c_int32, C.c_int64, _i64p, C.c_int32, C.c_float, C.c_float,
                                            _dp]
        L.g12_mlp_train_pushforward.argtypes = [_vp, _vp, C.c_int32, C.c_int64, _i64p, C.c_int32, C.c_int32,
                                                C.c_float, C.c_float, C.c_float, _dp]
        L.g12_mlp_rollout.argtypes = [_vp, _vp, C.c_int32, C.c_int64, C.c_int64, _fp]
        L.g12_mlp_judge.argtypes = [_vp, _vp, _vp, C.c_int32, C.c_int64, C.c_int64, C.c_int32, C.c_double,
                                    C.POINTER(C.c_int64)]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _cx(a, size=None):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if size is not None and a.size != size:
        raise ValueError(f"expected {size} complex entries, got {a.size}")
    return a


def default_params() -> Params:
    p = Params()
    lib().g12_params_default(C.byref(p))
    return p


def make_params(**kw) -> Params:
    """Params from keyword overrides of the reference defaults.  ``q_type`` and
    ``v_law`` take the input-file strings; q_type "none" sets qs = Nq = 0."""
    p = default_params()
    q = kw.pop("q_type", "full")
    if q == "none":
        kw["quench_strength"], kw["Nq"] = 0.0, 0
        q = "full"
    p.q_type = QUENCH[q]
    p.v_law = VLAW[kw.pop("v_law", kw.pop("vlaw", "exp"))]
    for k, v in kw.items():
        if k in ("HF", "EHM"):
            v = int(bool(v))
        setattr(p, k, v)
    return p


def read_input(path):
    """read_input.h:53-146 semantics; returns (Params, log text)."""
    p = Params()
    log = C.create_string_buffer(1 << 16)
    rc = lib().g12_read_input(path.encode(), C.byref(p), log, len(log))
    if rc:
        raise G12Error(f"g12_read_input failed ({rc}): {log.value.decode()}")
    return p, log.value.decode()


def as_steps(p: Params) -> int:
    return int(lib().g12_as_steps(C.byref(p)))


def rk_iterations(p: Params) -> int:
    return int(lib().g12_rk_iterations(C.byref(p)))


def make_G0(p: Params, p_number=None):
    n = p.n
    out = np.zeros((n, n), np.complex128)
    pn = p.Ns // 2 if p_number is None else p_number
    _check(lib().g12_make_G0(C.byref(p), pn, _ptr(out)))
    return out


def dipole(traj):
    traj = _cx(traj)
    T = traj.shape[0]
    n = int(round(np.sqrt(traj[0].size)))
    out = np.zeros(T)
    _check(lib().g12_dipole(_ptr(traj), T, n, _ptr(out)))
    return out


def particle_number(traj):
    """N = 2 Tr Im G1 per snapshot of traj [T, n, n] (conserved by the equations)."""
    traj = np.ascontiguousarray(traj, np.complex128)
    if traj.ndim == 2:
        traj = traj[None]
    out = np.zeros(traj.shape[0])
    _check(lib().g12_particle_number(_ptr(traj), traj.shape[0], traj.shape[-1], _ptr(out)))
    return out


def _check(rc, ctx=None):
    if rc < 0:
        msg = lib().g12_last_error(ctx).decode() if ctx is not None else lib().g12_last_error(None).decode()
        raise G12Error(f"libg12kba error {rc}: {msg}")
    return rc


class Context:
    """One system on one GPU (``g12_ctx``)."""

    def __init__(self, p: Params, precision="fp64", device=0):
        self.p = p
        self.n = p.n
        h = C.c_void_p()
        rc = lib().g12_create(C.byref(p), PREC[precision], device, C.byref(h))
        if rc:
            raise G12Error(f"g12_create failed ({rc}): {lib().g12_last_error(None).decode()}")
        self.h = h

    def close(self):
        if self.h:
            lib().g12_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, G1, G2xx=None, G2xy=None):
        n = self.n
        G1 = _cx(G1, n * n)
        G2xx = None if G2xx is None else _cx(G2xx, n ** 4)
        G2xy = None if G2xy is None else _cx(G2xy, n ** 4)
        _check(lib().g12_set_state(self.h, _ptr(G1), _ptr(G2xx), _ptr(G2xy)), self.h)

    def get_state(self):
        n = self.n
        G1 = np.zeros((n, n), np.complex128)
        XX = np.zeros(n ** 4, np.complex128)
        XY = np.zeros(n ** 4, np.complex128)
        _check(lib().g12_get_state(self.h, _ptr(G1), _ptr(XX), _ptr(XY)), self.h)
        return G1, XX, XY

    def adiabatic_switch(self) -> int:
        done = C.c_int64()
        _check(lib().g12_adiabatic_switch(self.h, C.byref(done)), self.h)
        return done.value

    def propagate(self, nsteps, record=True):
        """RK4 steps; returns (traj[T, n, n] or None, status)."""
        n = self.n
        traj = np.zeros((max(nsteps, 1), n, n), np.complex128) if record else None
        done = C.c_int64()
        rc = _check(lib().g12_propagate(self.h, nsteps, _ptr(traj), C.byref(done)), self.h)
        return (traj[: done.value] if record else None), rc

    def propagate_dipole(self, nsteps):
        p = np.zeros(max(nsteps, 1))
        done = C.c_int64()
        rc = _check(lib().g12_propagate_dipole(self.h, nsteps, _ptr(p), C.byref(done)), self.h)
        return p[: done.value], rc

    def total_energy(self, U_eff=None, w_quench=0.0, Nq_eff=0):
        """Total energy of the current state (``g12_total_energy``):
        array [E, 2 Tr[h0 rho], Tr[(h - h0) rho], correlation part].
        U_eff defaults to the parameters' U (the value after adiabatic switching)."""
        out = np.zeros(4)
        U = self.p.U if U_eff is None else U_eff
        _check(lib().g12_total_energy(self.h, float(U), float(w_quench), int(Nq_eff), _ptr(out)), self.h)
        return out

    def rhs(self, G1, G2xx, G2xy, U_eff, w_quench=0.0, Nq_eff=0):
        """One RHS evaluation: dict of h, comm1, Ix, K1, K2xx, K2xy (replaces the state)."""
        n = self.n
        G1 = _cx(G1, n * n)
        G2xx = None if G2xx is None else _cx(G2xx, n ** 4)
        G2xy = None if G2xy is None else _cx(G2xy, n ** 4)
        out = {k: np.zeros((n, n), np.complex128) for k in ("h", "comm1", "Ix", "K1")}
        out["K2xx"] = np.zeros(n ** 4, np.complex128)
        out["K2xy"] = np.zeros(n ** 4, np.complex128)
        _check(lib().g12_rhs(self.h, _ptr(G1), _ptr(G2xx), _ptr(G2xy), U_eff, w_quench, Nq_eff,
                             _ptr(out["h"]), _ptr(out["comm1"]), _ptr(out["Ix"]), _ptr(out["K1"]),
                             _ptr(out["K2xx"]), _ptr(out["K2xy"])), self.h)
        return out

    @property
    def last_device_ms(self) -> float:
        return float(lib().g12_last_device_ms(self.h))

    @property
    def launches_per_step(self) -> int:
        return int(lib().g12_launches_per_step(self.h))

    def set_l2_eviction(self, nbytes):
        """Write ``nbytes`` of a scratch buffer after every step (0 = off), so
        each step starts with the state evicted from L2."""
        _check(lib().g12_set_l2_eviction(self.h, int(nbytes)), self.h)

    def kernel_times(self, nsteps=2):
        """{kernel name: (mean ms per launch, launches per step)} measured with
        CUDA events around each launch (advances the state by nsteps)."""
        avg = np.zeros(16)
        calls = (C.c_int32 * 16)()
        nk = _check(lib().g12_kernel_times(self.h, nsteps, _ptr(avg), calls, 16), self.h)
        return {lib().g12_kernel_name(self.h, i).decode(): (float(avg[i]), int(calls[i]))
                for i in range(nk) if calls[i]}


class Batch:
    """An ensemble of independent systems advanced together (``g12_batch``)."""

    def __init__(self, params, precision="fp64", device=0):
        arr = (Params * len(params))(*params)
        self.params = list(params)
        self.nsys = len(params)
        h = C.c_void_p()
        rc = lib().g12_batch_create(arr, self.nsys, PREC[precision], device, C.byref(h))
        if rc:
            raise G12Error(f"g12_batch_create failed ({rc}): {lib().g12_batch_last_error(None).decode()}")
        self.h = h

    def close(self):
        if self.h:
            lib().g12_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc < 0:
            raise G12Error(f"libg12kba batch error {rc}: {lib().g12_batch_last_error(self.h).decode()}")
        return rc

    def set_state(self, i, G1, G2xx=None, G2xy=None):
        n = self.params[i].n
        G1 = _cx(G1, n * n)
        G2xx = None if G2xx is None else _cx(G2xx, n ** 4)
        G2xy = None if G2xy is None else _cx(G2xy, n ** 4)
        self._chk(lib().g12_batch_set_state(self.h, i, _ptr(G1), _ptr(G2xx), _ptr(G2xy)))

    def get_state(self, i):
        n = self.params[i].n
        G1 = np.zeros((n, n), np.complex128)
        XX = np.zeros(n ** 4, np.complex128)
        XY = np.zeros(n ** 4, np.complex128)
        self._chk(lib().g12_batch_get_state(self.h, i, _ptr(G1), _ptr(XX), _ptr(XY)))
        return G1, XX, XY

    def adiabatic_switch(self):
        done = C.c_int64()
        self._chk(lib().g12_batch_adiabatic_switch(self.h, C.byref(done)))
        return done.value

    def propagate(self, nsteps):
        """nsteps RK4 steps of every system; returns the dipoles (nsys, nsteps)."""
        dip = np.zeros((self.nsys, max(nsteps, 1)))
        done = C.c_int64()
        self._chk(lib().g12_batch_propagate(self.h, nsteps, _ptr(dip), C.byref(done)))
        return dip[:, :nsteps]

    def propagate_features(self, nsteps, every, feat_ptr):
        """nsteps RK4 steps recording snapshot features (rho = -i G1, upper
        triangle, real then imaginary parts) every `every` steps into the device
        buffer at feat_ptr [nsys][nsteps // every][n(n+1)] (float32); returns
        the dipoles (nsys, nsteps)."""
        dip = np.zeros((self.nsys, max(nsteps, 1)))
        done = C.c_int64()
        self._chk(lib().g12_batch_propagate_features(self.h, nsteps, every, C.c_void_p(feat_ptr), _ptr(dip),
                                                     C.byref(done)))
        return dip[:, :nsteps]

    @property
    def last_device_ms(self):
        return float(lib().g12_batch_last_device_ms(self.h))

    def tile(self, i):
        return int(lib().g12_batch_tile(self.h, i))


def ensemble_params(nsys=256, seed=20261203, time_steps=4000):
    """The batched-ensemble configuration: Ns in {4,6,8,10,12}, Nb in {1,2},
    U ~ U[0.5,2.5], t2 ~ U[0,0.5], quench strength ~ U[0.5,3] on Nq = Ns//3
    sites; t1 = 1, EHM with w(r) = U/(1+r), dt = 0.01 (seeded MT19937)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    out = []
    for _ in range(nsys):
        Ns = int(rng.choice([4, 6, 8, 10, 12]))
        Nb = int(rng.choice([1, 2]))
        U = float(rng.uniform(0.5, 2.5))
        t2 = float(rng.uniform(0.0, 0.5))
        qs = float(rng.uniform(0.5, 3.0))
        out.append(make_params(Ns=Ns, Nb=Nb, Nq=Ns // 3, U=U, t1=1.0, t2=t2 if Nb > 1 else 0.0,
                               quench_strength=qs, EHM=True, v_law="inv", dt=0.01, time_steps=time_steps,
                               q_type="full"))
    return out


def fp64_peak_tflops(device=0) -> float:
    return float(lib().g12_fp64_peak_tflops(device))


def run(p: Params, precision="fp64", device=0, G0=None):
    """Main.cpp:47-58 through the library: G0, AS, RK4; returns (traj, dipole, status)."""
    G1 = make_G0(p) if G0 is None else _cx(G0, p.n ** 2)
    with Context(p, precision, device) as ctx:
        ctx.set_state(G1)
        ctx.adiabatic_switch()
        traj, rc = ctx.propagate(rk_iterations(p))
    return traj, dipole(traj), rc
