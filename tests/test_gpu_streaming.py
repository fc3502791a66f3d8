"""The streaming kernel's side paths on the GPU.

* A stored J^-1 that differs from 1 / J (set by the caller) is read as
  stored: the step matches the oracle, which always reads the stored rows.
* The bounded wait for the bulk copies: with the debug bound of one
  non-blocking poll every CTA's first wait runs out; the kernel records the
  timeout, waits for the copies it issued and returns.  The host reports the
  status, no fault occurs, and the context stays usable.
"""
import numpy as np
import pytest

import elasticapp_b200 as eb
from elasticapp_b200 import _lib as L
from elasticapp_b200 import workloads as W
from oracle_bridge import max_rel_error_per_rod, oracle_from_workload, state_slots

pytestmark = pytest.mark.gpu


def _modified_oracle(wl, r, jinv):
    orc = oracle_from_workload(wl)
    orc.set_rod("inv_inertia", r, jinv)
    return orc


@pytest.mark.parametrize("window", [0, 128])
def test_stored_inverse_inertia_is_read_when_it_differs(window):
    wl = W.uneven_batch(n_rods=24, seed=77, n_range=(8, 200))
    sim = wl.build(step_mode="streaming", window=window)
    # rod 3: a stored J^-1 1.5 times 1 / J (no longer its inverse)
    r = 3
    jinv = sim.rods[r].get("InvMassSecondMomentOfInertia") * 1.5
    sim.rods[r].set("InvMassSecondMomentOfInertia", jinv)
    steps = 200
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, steps)
    orc = _modified_oracle(wl, r, jinv)
    orc.step(wl.dt, steps)
    # the FP64 parity rule: 1e-10, or 10x the oracle's own one-ulp envelope
    spread = {}
    for key in ("x", "Q"):
        p = _modified_oracle(wl, r, jinv)
        p.arrays[key] = np.nextafter(p.arrays[key], np.inf)
        p.step(wl.dt, steps)
        for name, k, place in (("Position", "x", 0), ("AngularVelocity", "w", 1)):
            e = max_rel_error_per_rod(p.comp(k), orc.comp(k), wl.n_elements, place)
            spread[name] = max(spread.get(name, 0.0), e)
    want = state_slots(orc)
    for name, place in (("Position", 0), ("AngularVelocity", 1)):
        err = max_rel_error_per_rod(sim.get_slots(name), want[name], wl.n_elements, place)
        assert err <= max(1e-10, 10.0 * spread[name]), (name, err, spread[name])
    # the modified rod really moves differently from an unmodified run
    ref = wl.build(step_mode="streaming")
    ref.step(eb.PositionVerlet(), 0.0, wl.dt, 200)
    assert not np.array_equal(ref.rods[r].get("AngularVelocity"), sim.rods[r].get("AngularVelocity"))
    ref.close()
    sim.close()


@pytest.mark.parametrize("window", [0, 256])
def test_bounded_wait_timeout_is_reported_without_fault(window):
    wl = W.uneven_batch(n_rods=64, seed=78, n_range=(32, 300))
    sim = wl.build(step_mode="streaming", window=window)
    L.call("eb_debug_set_wait_bound", sim._h, 1)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1)
    with pytest.raises(L.EbError) as ex:
        sim.synchronize()
        sim.rods[0].get("Position")
    assert "bounded wait" in str(ex.value)
    sim.close()
    # the context is intact: a fresh simulator steps and matches the oracle
    ok = wl.build(step_mode="streaming")
    ok.step(eb.PositionVerlet(), 0.0, wl.dt, 20)
    orc = oracle_from_workload(wl)
    orc.step(wl.dt, 20)
    err = max_rel_error_per_rod(ok.get_slots("Position"), state_slots(orc)["Position"], wl.n_elements, 0)
    assert err <= 1e-12
    ok.close()
