"""Mixed-precision resident kernel against the FP64 drop-in (GPU).

The mixed path keeps the state (x, v, Q, w) and the cancellation-prone
quantities in FP64 and the element-local arithmetic in FP32.  Its accuracy
requirement: tip positions within 1e-5 of the FP64 path after 10^4 steps,
relative to the rod length, on rods shaped like the 65,536-rod mixed batch
(n ~ U{64..256}, helical rest curvature up to 10 1/m, end torque 1e-3 N m),
at the batch's step dt = 0.5 min(l^2 / (r c)), about 4.6e-7 s: at 1e-5 s
these rods are unstable in FP64 as well."""
import numpy as np
import pytest

import elasticapp_b200 as eb
from elasticapp_b200 import workloads as W

pytestmark = pytest.mark.gpu

TIP_TOL = 1e-5


def tips(sim):
    return np.stack([r.get("Position")[:, -1] for r in sim.rods])


def run(wl, n_steps, **kw):
    sim = wl.build(**kw)
    e0 = sim.energy().sum(axis=1)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, n_steps)
    e1 = sim.energy().sum(axis=1)
    return sim, e0, e1


def test_mixed_tip_error_after_1e4_steps():
    wl = W.mixed_batch(n_rods=64, seed=1003)
    ref, e0r, e1r = run(wl, 10_000, step_mode="streaming")
    mix, e0m, e1m = run(wl, 10_000, precision="mixed")
    assert mix.step_plan()["mode"] == "resident"
    lengths = np.array([r.length for r in wl.rods])
    err = np.linalg.norm(tips(mix) - tips(ref), axis=1) / lengths
    assert np.all(np.isfinite(err))
    assert err.max() <= TIP_TOL, err.max()
    # the energies of the two paths stay together
    np.testing.assert_allclose(e1m, e1r, rtol=1e-4, atol=1e-12 * np.abs(e0r).max())


def test_mixed_with_damper_clamp_gravity_short_run():
    wl = W.uneven_batch(n_rods=32, seed=21, n_range=(40, 300))
    ref, _, _ = run(wl, 2000, step_mode="streaming")
    mix, _, _ = run(wl, 2000, precision="mixed")
    lengths = np.array([r.length for r in wl.rods])
    err = np.linalg.norm(tips(mix) - tips(ref), axis=1) / lengths
    assert err.max() <= TIP_TOL, err.max()


def test_mixed_rods_too_long_fall_back_to_fp64_streaming():
    # longer than a CTA pair holds (1039 elements)
    wl = W.uneven_batch(n_rods=3, seed=5, n_range=(1100, 1200))
    sim = wl.build(precision="mixed")
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 4)
    assert sim.step_plan()["mode"] == "streaming"


def test_full_mixed_batch_stays_within_tip_tolerance():
    """The whole 65,536-rod mixed batch (10.5 M elements), 10^4 steps on both
    paths: every tip within 1e-5 of the FP64 drop-in, relative to the rod
    length, and no non-finite state."""
    wl = W.mixed_batch()
    ref, _, e1r = run(wl, 10_000, step_mode="streaming")
    ref_tips = tips(ref)
    ref.close()
    mix, _, e1m = run(wl, 10_000, precision="mixed")
    mix_tips = tips(mix)
    lengths = np.array([r.length for r in wl.rods])
    err = np.linalg.norm(mix_tips - ref_tips, axis=1) / lengths
    assert np.all(np.isfinite(mix_tips))
    assert err.max() <= TIP_TOL, (err.max(), int(np.argmax(err)))
