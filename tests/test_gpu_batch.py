"""Batched ensembles: every system of a heterogeneous batch reproduces, bit for
bit, what a single-system context computes (same device code per system), and
the single-system path is itself pinned to the reference."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(g12):
    kw = dict(t1=1.0, dt=0.02, time_steps=60, AS_rate=0.5, AS_midpoint=1.5)
    return [
        g12.make_params(Ns=4, Nb=1, Nq=1, U=1.0, **kw),
        g12.make_params(Ns=3, Nb=2, Nq=1, U=1.5, t2=0.4, EHM=True, v_law="inv", **kw),
        g12.make_params(Ns=6, Nb=1, Nq=2, U=0.8, EHM=True, q_type="pulse", quench_strength=2.0, **kw),
        g12.make_params(Ns=4, Nb=2, Nq=1, U=2.0, t2=0.3, EHM=True, v_law="inv", **kw),
        g12.make_params(Ns=5, Nb=1, Nq=2, U=1.2, HF=True, **kw),
        g12.make_params(Ns=4, Nb=1, Nq=1, U=0.0, **kw),
        g12.make_params(Ns=8, Nb=2, Nq=2, U=1.3, t2=0.2, EHM=True, v_law="inv", **kw),
    ]


def test_batch_matches_single_contexts(g12):
    ps = _systems(g12)
    G0 = [g12.make_G0(p) for p in ps]
    nsteps = 60
    with g12.Batch(ps) as b:
        for i, g in enumerate(G0):
            b.set_state(i, g)
        b.adiabatic_switch()
        dip = b.propagate(nsteps)
        states = [b.get_state(i) for i in range(len(ps))]
        tiles = [b.tile(i) for i in range(len(ps))]
    assert all(t >= 1 for t in tiles)
    for i, p in enumerate(ps):
        with g12.Context(p) as ctx:
            ctx.set_state(G0[i])
            ctx.adiabatic_switch()
            d1, rc = ctx.propagate_dipole(nsteps)
            st = ctx.get_state()
        assert rc == 0
        assert np.array_equal(dip[i], d1), i
        for a, b_ in zip(states[i], st):
            assert np.array_equal(a, b_), i


def test_batch_propagation_continues(g12):
    ps = _systems(g12)[:3]
    G0 = [g12.make_G0(p) for p in ps]
    with g12.Batch(ps) as b:
        for i, g in enumerate(G0):
            b.set_state(i, g)
        d_a = np.concatenate([b.propagate(20), b.propagate(30)], axis=1)
    with g12.Batch(ps) as b:
        for i, g in enumerate(G0):
            b.set_state(i, g)
        d_b = b.propagate(50)
    assert np.array_equal(d_a, d_b)
