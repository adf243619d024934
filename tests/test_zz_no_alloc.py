"""g12_rhs_noalloc: the allocation-free right-hand side.

Some callers cannot call cudaMalloc - their device memory belongs to another
allocator that has already reserved it, or they run latency-critical loops
that cannot absorb cudaMalloc's implicit synchronisation.  For them the library
keeps the scratch of one right-hand-side evaluation in a static device array
and the caller passes only input and output device buffers.  This test calls
that entry point through the C ABI (the test itself allocates the buffers, with
torch) and checks it against g12_rhs, the context-based entry point, on two
calls in a row with different systems and inputs, so that contents the first
call leaves in the shared array cannot leak into the second.
"""
import ctypes

import numpy as np
import pytest

from conftest import rand_c, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the RHS tolerance of tests/test_gpu_parity.py


def _call_noalloc(g12, torch, p, G1, XX, XY, U, w, Nq, stream=None):
    n = p.Ns * p.Nb
    dev = torch.device("cuda:0")
    as_dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.complex128).reshape(-1)).to(dev)
    g1, xx, xy = as_dev(G1), as_dev(XX), as_dev(XY)
    k1 = torch.full((n * n,), complex(7.0, -3.0), dtype=torch.complex128, device=dev)
    k2xx = torch.full((n ** 4,), complex(7.0, -3.0), dtype=torch.complex128, device=dev)
    k2xy = torch.full((n ** 4,), complex(7.0, -3.0), dtype=torch.complex128, device=dev)
    torch.cuda.synchronize()
    err = ctypes.create_string_buffer(512)
    handle = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    rc = g12.lib().g12_rhs_noalloc(ctypes.byref(p), g1.data_ptr(), xx.data_ptr(), xy.data_ptr(), U, w, Nq,
                                   k1.data_ptr(), k2xx.data_ptr(), k2xy.data_ptr(), handle, err, len(err))
    assert rc == 0, err.value.decode()
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize()
    return k1.cpu().numpy().reshape(n, n), k2xx.cpu().numpy(), k2xy.cpu().numpy()


CASES = [
    dict(Ns=4, Nb=2, U=1.5, t2=0.3, EHM=True, v_law="inv", seed=1, Uf=1.2, w=0.4, Nq=2),
    dict(Ns=3, Nb=1, U=0.8, t2=0.0, EHM=False, v_law="exp", seed=2, Uf=0.8, w=0.0, Nq=0),
    # n = G12_NOALLOC_MAX_N: the largest system the scratch array is carved for
    dict(Ns=8, Nb=2, U=2.0, t2=0.5, EHM=True, v_law="inv", seed=3, Uf=2.0, w=0.7, Nq=3),
]


def test_noalloc_matches_rhs_two_calls_in_a_row(g12):
    torch = pytest.importorskip("torch")
    for c in CASES:
        p = g12.make_params(Ns=c["Ns"], Nb=c["Nb"], U=c["U"], t2=c["t2"], EHM=c["EHM"], v_law=c["v_law"])
        n = p.Ns * p.Nb
        rng = np.random.default_rng(c["seed"])
        G1, XX, XY = rand_c(rng, n, n), rand_c(rng, n ** 4), rand_c(rng, n ** 4)
        k1, k2xx, k2xy = _call_noalloc(g12, torch, p, G1, XX, XY, c["Uf"], c["w"], c["Nq"])
        with g12.Context(p) as ctx:
            ref = ctx.rhs(G1, XX, XY, c["Uf"], c["w"], c["Nq"])
        assert rel_err(k1, ref["K1"]) <= TOL
        assert rel_err(k2xx, ref["K2xx"]) <= TOL
        assert rel_err(k2xy, ref["K2xy"]) <= TOL


def test_noalloc_rejects_oversized_system(g12):
    torch = pytest.importorskip("torch")
    p = g12.make_params(Ns=17, Nb=1, U=1.0)
    buf = torch.zeros(4, dtype=torch.complex128, device="cuda:0")
    err = ctypes.create_string_buffer(512)
    rc = g12.lib().g12_rhs_noalloc(ctypes.byref(p), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 1.0, 0.0, 0,
                                   buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None, err, len(err))
    assert rc < 0 and b"G12_NOALLOC_MAX_N" in err.value


def test_noalloc_without_two_body_terms_gives_zero_K2(g12):
    """U = 0 or HF: no two-body terms (RK_solver.h:154), K2 is cleared."""
    torch = pytest.importorskip("torch")
    for kw in (dict(U=0.0), dict(U=1.0, HF=True)):
        p = g12.make_params(Ns=4, Nb=1, **kw)
        rng = np.random.default_rng(4)
        G1, XX, XY = rand_c(rng, 4, 4), rand_c(rng, 4 ** 4), rand_c(rng, 4 ** 4)
        k1, k2xx, k2xy = _call_noalloc(g12, torch, p, G1, XX, XY, p.U, 0.3, 1)
        with g12.Context(p) as ctx:
            ref = ctx.rhs(G1, XX, XY, p.U, 0.3, 1)
        assert rel_err(k1, ref["K1"]) <= TOL
        assert np.all(k2xx == 0) and np.all(k2xy == 0)
        assert np.all(ref["K2xx"] == 0) and np.all(ref["K2xy"] == 0)


def test_noalloc_on_a_side_stream(g12):
    torch = pytest.importorskip("torch")
    c = CASES[0]
    p = g12.make_params(Ns=c["Ns"], Nb=c["Nb"], U=c["U"], t2=c["t2"], EHM=c["EHM"], v_law=c["v_law"])
    n = p.Ns * p.Nb
    rng = np.random.default_rng(5)
    G1, XX, XY = rand_c(rng, n, n), rand_c(rng, n ** 4), rand_c(rng, n ** 4)
    side = torch.cuda.Stream(device="cuda:0")
    k1, k2xx, k2xy = _call_noalloc(g12, torch, p, G1, XX, XY, c["Uf"], c["w"], c["Nq"], stream=side)
    with g12.Context(p) as ctx:
        ref = ctx.rhs(G1, XX, XY, c["Uf"], c["w"], c["Nq"])
    assert rel_err(k1, ref["K1"]) <= TOL
    assert rel_err(k2xx, ref["K2xx"]) <= TOL
    assert rel_err(k2xy, ref["K2xy"]) <= TOL


def test_noalloc_rejects_empty_system_with_its_own_message(g12):
    torch = pytest.importorskip("torch")
    p = g12.make_params(Ns=4, Nb=1, U=1.0)
    p.Nb = 0
    buf = torch.zeros(4, dtype=torch.complex128, device="cuda:0")
    err = ctypes.create_string_buffer(512)
    rc = g12.lib().g12_rhs_noalloc(ctypes.byref(p), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 1.0, 0.0, 0,
                                   buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None, err, len(err))
    assert rc < 0 and b"invalid Ns" in err.value and b"G12_NOALLOC_MAX_N" not in err.value
