"""Snapshots (checkpoint / restart) on the GPU: a restored simulator
continues bit for bit as the original did, in the same or in an identically
built simulator; mismatched configurations and malformed buffers are
rejected; the case study's checkpoint carries its clock; rod dumps hold the
per-rod arrays."""
import numpy as np
import pytest

import elasticapp_b200 as eb
from elasticapp_b200 import _lib as L
from elasticapp_b200 import case_study as C
from elasticapp_b200 import workloads as W

pytestmark = pytest.mark.gpu

STATE = ("Position", "Velocity", "Director", "AngularVelocity")


def state(sim):
    return {k: sim.get_slots(k) for k in STATE}


@pytest.mark.parametrize("step_mode", ["streaming", "resident"])
def test_restore_continues_bit_for_bit(step_mode):
    wl = W.uneven_batch(n_rods=12, seed=3, n_range=(20, 300))
    cfg = 2 if step_mode == "resident" else 0  # one fixed configuration for both simulators
    a = wl.build(step_mode=step_mode, resident_config=cfg)
    t = a.step(eb.PositionVerlet(), 0.0, wl.dt, 100)
    snap = a.snapshot()
    a.step(eb.PositionVerlet(), t, wl.dt, 150)
    want = state(a)
    a.restore(snap)
    a.step(eb.PositionVerlet(), t, wl.dt, 150)
    got = state(a)
    for k in STATE:
        assert np.array_equal(want[k], got[k]), k
    b = wl.build(step_mode=step_mode, resident_config=cfg)  # a fresh, identically built simulator
    b.restore(snap)
    b.step(eb.PositionVerlet(), t, wl.dt, 150)
    for k in STATE:
        assert np.array_equal(want[k], b.get_slots(k)), k


def test_snapshot_rejects_mismatches(tmp_path):
    wl = W.uneven_batch(n_rods=4, seed=1, n_range=(10, 30))
    a = wl.build()
    snap = a.snapshot()
    other = W.uneven_batch(n_rods=4, seed=2, n_range=(10, 30)).build()
    with pytest.raises(L.EbError) as e:
        other.restore(snap)
    assert e.value.status == 1
    with pytest.raises(L.EbError) as e:
        a.restore(b"not a snapshot" * 10)
    assert e.value.status == 1
    with pytest.raises(L.EbError) as e:
        a.restore(snap[:-8])
    assert e.value.status == 1
    fresh = eb.Simulator()
    fresh.emplace_back(eb.CosseratRodWithoutDamping, wl.rods[0])
    with pytest.raises(L.EbError) as e:
        fresh.snapshot()
    assert e.value.status == 2  # not finalized
    # file round trip
    a.save(tmp_path / "sim.snap")
    a.step(eb.PositionVerlet(), 0.0, wl.dt, 10)
    a.load(tmp_path / "sim.snap")
    np.testing.assert_array_equal(a.rods[0].get("Position"), wl.build().rods[0].get("Position"))


def test_case_study_checkpoint(tmp_path):
    cs = C.DynamicCantileverCaseStudy(n_elements=30)
    rod = cs.communicate()
    rod.loc[rod.Velocity][2, :] = 1e-3 * np.linspace(0.0, 1.0, 31) ** 2
    cs.run_for(n_iterations=120)
    cs.save(tmp_path / "cs.npz")
    t, it = cs.current_time(), cs.current_iteration()
    cs.run_for(n_iterations=80)
    want = rod.get_position().copy()
    cs.run_for(n_iterations=50)  # move on, then go back
    cs.load(tmp_path / "cs.npz")
    assert cs.current_time() == t and cs.current_iteration() == it
    cs.run_for(n_iterations=80)
    assert np.array_equal(cs.communicate().get_position(), want)
    cs.close()


def test_dump_rods(tmp_path):
    wl = W.uneven_batch(n_rods=3, seed=4, n_range=(5, 12))
    sim = wl.build()
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 5)
    sim.dump_rods(tmp_path / "rods.npz")
    with np.load(tmp_path / "rods.npz") as z:
        assert sorted(z.files) == sorted(f"rod{k}/{f}" for k in range(3) for f in STATE)
        for k, ref in enumerate(sim.rods):
            np.testing.assert_array_equal(z[f"rod{k}/Director"], ref.get("Director"))
