"""Collision system on the GPU against the oracle (rows a23-a27).

* Candidate pairs (capsule-capsule and capsule-plane) of a step are the
  oracle's exhaustive search of the same state, bit for bit (the reference
  requires its hash grids to equal the exhaustive search, Test_HashGrids.cpp).
* Capsule loads of a step equal the oracle's (the contact kernels round
  every operation as written, like the oracle), and the state after a few
  steps with contact meets the FP64 parity rule.
* Edge cases: rods without contact, planes only, a pile-up whose pair count
  overflows the initial buffer, determinism, error paths; and the pair set
  of the full 8,192-rod contact batch.
"""
import numpy as np
import pytest

from oracle_bridge import (contact_spec, max_rel_error_per_rod, oracle_from_workload, oracle_spread_contact,
                           parity_bounds, state_slots)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eb():
    import elasticapp_b200
    return elasticapp_b200


@pytest.fixture(scope="module")
def W():
    from elasticapp_b200 import workloads
    return workloads


def _sync_oracle_state(sim, rods):
    """Copy the simulator's state into the oracle's arrays (slot layout)."""
    for name, key in (("Position", "x"), ("Velocity", "v"), ("Director", "Q"), ("AngularVelocity", "w")):
        rods.arrays[key][:] = sim.get_slots(name).reshape(-1)


def _pairs_from_oracle(oracle_mod, rods, spec, half_dt, exhaustive=True):
    return oracle_mod.contact_pairs(rods, spec, half_dt, exhaustive=exhaustive)


def test_pairs_first_step_bit_exact(eb, W, oracle_mod):
    wl = W.contact_batch(n_rods=96, seed=5, box=0.3)
    sim = wl.build()
    rods = oracle_from_workload(wl)
    spec = contact_spec(wl)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1)
    got = sim.contact_pairs()
    want = _pairs_from_oracle(oracle_mod, rods, spec, 0.5 * wl.dt)
    assert want.shape[0] > 96 * 63  # adjacent capsules at least
    assert np.array_equal(got, want)
    # plane pairs are present and encoded after the capsules
    assert (got[:, 1] >= sim.n_slots()).any()
    sim.close()


def test_pairs_after_evolution_bit_exact(eb, W, oracle_mod):
    wl = W.contact_batch(n_rods=64, seed=6, box=0.25, dt=1e-7)
    sim = wl.build()
    rods = oracle_from_workload(wl)
    spec = contact_spec(wl)
    t = sim.step(eb.PositionVerlet(), 0.0, wl.dt, 7)
    _sync_oracle_state(sim, rods)
    sim.step(eb.PositionVerlet(), t, wl.dt, 1)
    want = _pairs_from_oracle(oracle_mod, rods, spec, 0.5 * wl.dt)
    assert np.array_equal(sim.contact_pairs(), want)
    sim.close()


def test_capsule_loads_equal_oracle(eb, W, oracle_mod):
    wl = W.contact_batch(n_rods=64, seed=7, box=0.25)
    sim = wl.build()
    rods = oracle_from_workload(wl)
    spec = contact_spec(wl)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1)
    oracle_mod.contact_step(rods, spec, wl.dt, 1)
    want_f = spec.capsule_force.reshape(3, -1)
    want_t = spec.capsule_torque.reshape(3, -1)
    assert np.abs(want_f).max() > 0.0
    offs = sim.slot_offsets()
    for r, ref in enumerate(sim.rods):
        o, n = int(offs[r]), ref.n_elements
        np.testing.assert_array_equal(ref.get("ContactForce"), want_f[:, o:o + n])
        np.testing.assert_array_equal(ref.get("ContactTorque"), want_t[:, o:o + n])
    sim.close()


@pytest.mark.parametrize("reference_rounding", [False, True])
def test_state_parity_with_contact(eb, W, oracle_mod, reference_rounding):
    # a short horizon at a small step: the contact dynamics of these thin
    # rods diverges within tens of microseconds in the reference model
    wl = W.contact_batch(n_rods=48, seed=8, box=0.25, dt=1e-7)
    sim = wl.build(reference_rounding=reference_rounding)
    steps = 10
    base, spread = oracle_spread_contact(wl, steps)
    bounds = parity_bounds(spread)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, steps)
    want = state_slots(base)
    n_el = wl.n_elements
    for name, place in (("Position", 0), ("Velocity", 0), ("Director", 1), ("AngularVelocity", 1)):
        err = max_rel_error_per_rod(sim.get_slots(name), want[name], n_el, place)
        assert err <= bounds[name], (name, float(err), bounds[name])
    sim.close()


def test_rods_without_contact_and_no_planes(eb, W, oracle_mod):
    wl = W.contact_batch(n_rods=40, seed=9, box=0.2)
    wl.planes = []
    wl.contact_rod_material = [0 if k % 3 else -1 for k in range(40)]
    sim = wl.build()
    rods = oracle_from_workload(wl)
    spec = contact_spec(wl)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1)
    got = sim.contact_pairs()
    want = _pairs_from_oracle(oracle_mod, rods, spec, 0.5 * wl.dt)
    assert np.array_equal(got, want)
    offs = sim.slot_offsets()
    for r in range(0, 40, 3):  # no capsule of a rod without contact
        assert not ((got >= offs[r]) & (got < offs[r + 1])).any()
        assert not sim.rods[r].get("ContactForce").any()
    assert got.max() < sim.n_slots()
    sim.close()


def test_pile_up_regrows_pair_buffer(eb, W, oracle_mod):
    # every capsule of 40 rods inside a 1 cm cube: every pair overlaps, far
    # more candidate pairs than the initial buffer holds
    wl = W.contact_batch(n_rods=40, seed=10, box=0.01, length=0.01, dt=1e-8)
    sim = wl.build()
    rods = oracle_from_workload(wl)
    spec = contact_spec(wl)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1)
    got = sim.contact_pairs()
    want = _pairs_from_oracle(oracle_mod, rods, spec, 0.5 * wl.dt)
    n_caps = 40 * 64
    assert want.shape[0] > 24 * n_caps // 2
    assert np.array_equal(got, want)
    sim.close()


def test_contact_is_deterministic(eb, W):
    wl = W.contact_batch(n_rods=64, seed=11, box=0.25, dt=1e-7)
    out = []
    for _ in range(2):
        sim = wl.build()
        sim.step(eb.PositionVerlet(), 0.0, wl.dt, 5)
        out.append((sim.get_slots("Position").copy(), sim.rods[3].get("ContactForce").copy(), sim.contact_pairs()))
        sim.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


def test_contact_error_paths(eb, W):
    from elasticapp_b200._lib import EbError
    wl = W.contact_batch(n_rods=4, seed=12, box=0.3)
    sim = wl.build()
    with pytest.raises(EbError):
        sim.contact_pairs()  # no evaluation yet
    with pytest.raises(EbError):
        sim.rods[0].set("ContactForce", np.zeros((3, 64)))
    sim.close()
    with pytest.raises(EbError):
        wl.build(precision="mixed")
    s2 = eb.Simulator()
    with pytest.raises(EbError):
        s2.create_material(eb.ContactMaterial(0.0, 1.0, 1.0, 0.1, 0.1))
    with pytest.raises(EbError):
        s2.create_material(eb.ContactMaterial(1.0, -1.0, 1.0, 0.1, 0.1))
    m = s2.create_material(eb.ContactMaterial(1.0, 1.0, 1.0, 0.1, 0.1))
    with pytest.raises(EbError):
        s2.emplace_plane((0, 0, 0), (0, 0, 0), m)
    with pytest.raises(EbError):
        s2.emplace_plane((0, 0, 0), (0, 0, 1), m + 1)
    s2.close()


def test_full_contact_batch_pairs(eb, W, oracle_mod):
    wl = W.contact_batch()
    sim = wl.build()
    rods = oracle_from_workload(wl)
    spec = contact_spec(wl)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1)
    got = sim.contact_pairs()
    want = _pairs_from_oracle(oracle_mod, rods, spec, 0.5 * wl.dt, exhaustive=False)
    assert want.shape[0] > 8192 * 63
    assert np.array_equal(got, want)
    sim.close()
