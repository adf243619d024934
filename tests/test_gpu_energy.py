"""Total energy on the GPU (g12_total_energy) against the oracle's functional
on the reference's own states (tests/golden/energy_pin.npz), and its
conservation by both engines.  Bars: 1e-12 relative for the functional on a
given state (FP64 reduction of the same terms); drift over the run 1e-9
(FP64 engine, RK4 truncation) and 1e-7 (mixed engine) relative."""
import numpy as np
import pytest

from oracle import Config, total_energy
from test_gpu_parity import params_of
from test_oracle import energy_pin_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["dt02", "dt01"])
def test_energy_vs_oracle_on_reference_states(g12, oracle, tag):
    cfg, s0, sT, _ = energy_pin_case(tag)
    p = params_of(g12, cfg)
    with g12.Context(p, "fp64") as ctx:
        for s in (s0, sT):
            ctx.set_state(*s)
            got = ctx.total_energy()
            want = total_energy(oracle, cfg, *s)
            assert np.max(np.abs(got - want)) <= 1e-12 * abs(want[0]), (got, want)


def test_energy_after_propagation_matches_reference(g12, oracle):
    """FP64 engine from the reference's post-switching state: after the same T
    iterations the energy equals the reference's final state's."""
    cfg, s0, sT, T = energy_pin_case("dt02")
    p = params_of(g12, cfg)
    with g12.Context(p, "fp64") as ctx:
        ctx.set_state(*s0)
        _, rc = ctx.propagate(T, record=False)
        assert rc == 0
        got = ctx.total_energy()
    want = total_energy(oracle, cfg, *sT)
    assert np.max(np.abs(got - want)) <= 1e-11 * abs(want[0]), (got, want)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("bf16oz", 1e-7)])
@pytest.mark.parametrize("Ns", [8, 16])
def test_energy_conserved(g12, prec, tol, Ns):
    """Extended model (Nb = 2, U/(1+r)) after adiabatic switching, 400 RK4
    steps at constant U with the quench masked: the energy stays put while
    its correlation part moves."""
    cfg = Config(Ns=Ns, Nb=2, Nq=3, time_steps=400, U=1.5, t1=1.0, t2=0.3, dt=0.01, EHM=True, vlaw="inv",
                 q_type="full", quench_strength=1.0, AS_rate=0.5, AS_midpoint=3.0)
    p = params_of(g12, cfg)
    with g12.Context(p, prec) as ctx:
        ctx.set_state(g12.make_G0(p))
        ctx.adiabatic_switch()
        E0 = ctx.total_energy()
        _, rc = ctx.propagate(400, record=False)
        assert rc == 0
        E1 = ctx.total_energy()
    assert abs(E1[0] - E0[0]) <= tol * abs(E0[0]), (E0, E1)
    assert abs(E1[3] - E0[3]) > 1e-3 * abs(E0[3]), (E0, E1)
