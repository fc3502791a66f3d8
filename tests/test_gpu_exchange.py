"""Host-state exchange (GPU): eb_step_host_state.

One call sets the state from host arrays, steps and reads the state back.
Under a resident plan the rods are cut into contiguous slot groups and each
group's copies overlap the other groups' launches.  The result must be the
same, bit for bit and in every slot entry, as eb_set_field_batch, eb_step and
eb_get_field_batch in sequence, for one and several resident chunks, an
output that is its own input, inputs or outputs left out, and both
precisions and for the whole-batch and per-size-bucket resident plans; plans
the overlap does not cover take the sequential path."""
import numpy as np
import pytest
import torch

import elasticapp_b200 as eb
from elasticapp_b200 import workloads as W

pytestmark = pytest.mark.gpu

STATE = ("Position", "Velocity", "Director", "AngularVelocity")
NCOMP = {"Position": 3, "Velocity": 3, "Director": 9, "AngularVelocity": 3}


def pinned(shape):
    return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()


@pytest.fixture(scope="module")
def batch():
    # about 1.6 M slots, 21 waves of 512-slot CTAs on 148 SMs: groups of
    # 1, 2, about 4 ... 4, 2 and 1 waves
    return W.uneven_batch(n_rods=6000, seed=41, n_range=(32, 512), n_steps=200)


def perturbed_state(sim, seed):
    rng = np.random.default_rng(seed)
    host = {}
    for name in STATE:
        a = pinned((NCOMP[name], sim.n_slots()))
        sim.get_slots(name, out=a)
        if name in ("Velocity", "AngularVelocity"):
            a += 1e-4 * rng.standard_normal(a.shape)
        host[name] = a
    return host


def planned(wl, **kw):
    sim = wl.build(**kw)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 8)  # chooses the plan
    return sim


@pytest.mark.parametrize("precision,config", [("fp64", 1), ("fp64", 2), ("mixed", 1)])
@pytest.mark.parametrize("n_steps", [200, 128, 1])
def test_exchange_equals_sequential_calls(batch, precision, config, n_steps):
    seq = planned(batch, precision=precision, step_mode="resident", resident_config=config)
    xch = planned(batch, precision=precision, step_mode="resident", resident_config=config)
    assert seq.step_plan()["mode"] == "resident" and xch.step_plan()["mode"] == "resident"
    host = perturbed_state(seq, seed=n_steps)
    for name in STATE:
        seq.set_slots(name, host[name])
    t_seq = seq.step(eb.PositionVerlet(), 0.5, batch.dt, n_steps)
    want = {name: seq.get_slots(name) for name in STATE}
    out = {name: pinned(host[name].shape) for name in STATE}
    before = xch.launch_count()
    t_x = xch.step_host_state(eb.PositionVerlet(), 0.5, batch.dt, n_steps, inputs=host, outputs=out)
    chunks = -(-n_steps // 128)
    assert xch.launch_count() - before >= 2 * chunks  # more than one slot group
    assert t_x == t_seq
    for name in STATE:
        assert np.array_equal(out[name], want[name]), name
        assert np.array_equal(xch.get_slots(name), want[name]), name
    # the next plain step continues from the same state on both
    seq.step(eb.PositionVerlet(), t_seq, batch.dt, 3)
    xch.step(eb.PositionVerlet(), t_x, batch.dt, 3)
    for name in STATE:
        assert np.array_equal(xch.get_slots(name), seq.get_slots(name)), name


def test_exchange_equal_groups_equals_sequential_calls():
    """A batch of fewer than twelve waves of 512-slot CTAs (about 440 k
    slots on 148 SMs) is cut into equal groups instead of the tapered ones;
    the result is the same bit for bit."""
    wl = W.uneven_batch(n_rods=1600, seed=47, n_range=(32, 512), n_steps=200)
    seq = planned(wl, step_mode="resident", resident_config=1)
    xch = planned(wl, step_mode="resident", resident_config=1)
    host = perturbed_state(seq, seed=7)
    for name in STATE:
        seq.set_slots(name, host[name])
    t_seq = seq.step(eb.PositionVerlet(), 0.5, wl.dt, 200)
    want = {name: seq.get_slots(name) for name in STATE}
    out = {name: pinned(host[name].shape) for name in STATE}
    before = xch.launch_count()
    t_x = xch.step_host_state(eb.PositionVerlet(), 0.5, wl.dt, 200, inputs=host, outputs=out)
    assert xch.launch_count() - before >= 2 * 2  # two chunks in each of at least two groups
    assert t_x == t_seq
    for name in STATE:
        assert np.array_equal(out[name], want[name]), name


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_exchange_bucketed_plan(precision):
    # rods of all three size buckets (pairs of CTAs for 520-1039 elements),
    # about 1.6 M slots; the sequential calls and the exchange run on the same
    # simulator (same bucket configurations) from the same snapshot
    wl = W.uneven_batch(n_rods=3100, seed=45, n_range=(32, 1000), n_steps=200)
    sim = planned(wl, precision=precision, step_mode="bucketed")
    assert sim.step_plan()["mode"] == "bucketed"
    host = perturbed_state(sim, seed=11)
    snap = sim.snapshot()
    for name in STATE:
        sim.set_slots(name, host[name])
    t_seq = sim.step(eb.PositionVerlet(), 0.25, wl.dt, 200)
    want = {name: sim.get_slots(name) for name in STATE}
    sim.restore(snap)
    out = {name: pinned(host[name].shape) for name in STATE}
    before = sim.launch_count()
    t_x = sim.step_host_state(eb.PositionVerlet(), 0.25, wl.dt, 200, inputs=host, outputs=out)
    assert sim.launch_count() - before > 2 * 3  # two chunks of at most three bucket launches, per group
    assert t_x == t_seq
    for name in STATE:
        assert np.array_equal(out[name], want[name]), name


def test_exchange_pefrl(batch):
    # four force evaluations a step on the resident kernel, per slot group
    seq = batch.build(step_mode="resident", resident_config=1, stepper=eb.PEFRL)
    xch = batch.build(step_mode="resident", resident_config=1, stepper=eb.PEFRL)
    for sim in (seq, xch):
        sim.step(eb.PEFRL(), 0.0, batch.dt, 8)
        assert sim.step_plan()["mode"] == "resident"
    host = perturbed_state(seq, seed=5)
    for name in STATE:
        seq.set_slots(name, host[name])
    t_seq = seq.step(eb.PEFRL(), 0.0, batch.dt, 130)
    out = {name: pinned(host[name].shape) for name in STATE}
    t_x = xch.step_host_state(eb.PEFRL(), 0.0, batch.dt, 130, inputs=host, outputs=out)
    assert t_x == t_seq
    for name in STATE:
        assert np.array_equal(out[name], seq.get_slots(name)), name


def test_exchange_in_place_and_partial_fields(batch):
    seq = planned(batch, step_mode="resident", resident_config=1)
    xch = planned(batch, step_mode="resident", resident_config=1)
    host = perturbed_state(seq, seed=7)
    # inputs only for the velocities; outputs only for positions and directors,
    # the velocity array also its own output
    for name in ("Velocity", "AngularVelocity"):
        seq.set_slots(name, host[name])
    seq.step(eb.PositionVerlet(), 0.0, batch.dt, 130)
    want = {name: seq.get_slots(name) for name in STATE}
    buf = {name: host[name].copy() for name in STATE}
    ins = {"Velocity": buf["Velocity"], "AngularVelocity": buf["AngularVelocity"]}
    outs = {"Velocity": buf["Velocity"], "Position": pinned(host["Position"].shape),
            "Director": pinned(host["Director"].shape)}
    xch.step_host_state(eb.PositionVerlet(), 0.0, batch.dt, 130, inputs=ins, outputs=outs)
    for name in ("Velocity", "Position", "Director"):
        assert np.array_equal(outs[name], want[name]), name
    for name in STATE:
        assert np.array_equal(xch.get_slots(name), want[name]), name
    # no outputs: asynchronous, the state is read afterwards
    seq.step(eb.PositionVerlet(), 0.0, batch.dt, 5)
    xch.step_host_state(eb.PositionVerlet(), 0.0, batch.dt, 5)
    for name in STATE:
        assert np.array_equal(xch.get_slots(name), seq.get_slots(name)), name


def test_exchange_sequential_plans_and_first_call():
    # a streaming plan, and a first call that still has to choose the plan,
    # take the sequential path with the same result
    wl = W.uneven_batch(n_rods=64, seed=43, n_range=(16, 300), n_steps=20)
    for kw in ({"step_mode": "streaming"}, {}):
        seq, xch = wl.build(**kw), wl.build(**kw)
        host = perturbed_state(seq, seed=3)
        for name in STATE:
            seq.set_slots(name, host[name])
        seq.step(eb.PositionVerlet(), 0.0, wl.dt, 20)
        out = {name: pinned(host[name].shape) for name in STATE}
        xch.step_host_state(eb.PositionVerlet(), 0.0, wl.dt, 20, inputs=host, outputs=out)
        assert xch.step_plan()["mode"] == seq.step_plan()["mode"] or not kw
        for name in STATE:
            got, want = out[name], seq.get_slots(name)
            if kw:
                assert np.array_equal(got, want), name
            else:
                # both plans chosen by timing, perhaps differently: the FP64
                # parity bound between them
                assert np.max(np.abs(got - want)) <= 1e-10 * max(1.0, np.max(np.abs(want))), name


def test_exchange_rejects_bad_arrays(batch):
    sim = W.uneven_batch(n_rods=8, seed=44, n_range=(16, 40), n_steps=2).build()
    S = sim.n_slots()
    with pytest.raises(ValueError):
        sim.step_host_state(eb.PositionVerlet(), 0.0, 1e-6, 1, inputs={"Position": np.zeros((3, S + 1))})
    with pytest.raises(ValueError):
        sim.step_host_state(eb.PositionVerlet(), 0.0, 1e-6, 1, outputs={"Director": np.zeros((3, S))})
    with pytest.raises(KeyError):
        sim.step_host_state(eb.PositionVerlet(), 0.0, 1e-6, 1, inputs={"Mass": np.zeros((1, S))})
