"""GPU parity of the fused FP64 step (through the C-ABI) against the reference's
golden vectors and against the CPU oracle."""
import numpy as np
import pytest

import elasticapp_b200 as eb
from elasticapp_b200 import _lib as L
from elasticapp_b200 import workloads as W

import goldens as G
import oracle_bridge as B

pytestmark = pytest.mark.gpu

# Parity of the FP64 drop-in against the oracle after many steps: every
# state field within 1e-10 per-rod normwise relative error, or within 10x the
# oracle's own one-ulp conditioning envelope where that is wider
# (oracle_bridge.parity_bounds).  Positions and directors always meet 1e-10;
# velocities and angular velocities of stiff rods carry high-frequency
# content that amplifies rounding (tests/test_conditioning.py).


def within(errs, bounds):
    return all(errs[k] <= bounds[k] for k in errs)


def golden_sim(case, damped, reference_rounding, step_mode="streaming", resident_config=0):
    sim = eb.Simulator(record_diagnostics=True, reference_rounding=reference_rounding, step_mode=step_mode,
                       resident_config=resident_config)
    s = G.ROD_SETUP
    init = eb.StraightRod(n_elements=s["n"], material=eb.Material(s["density"], s["youngs"], s["shear"]),
                          radius=s["radius"], length=s["length"], origin=s["origin"],
                          direction=s["direction"], normal=s["normal"],
                          force_damping_rate=s["damping"] if damped else 0.0,
                          torque_damping_rate=s["damping"] if damped else 0.0)
    model = eb.CosseratRod if damped else eb.CosseratRodWithoutDamping
    refs = sim.emplace_back_many(model, [init] * case["n_rods"])
    sim.finalize()
    kinds = {**G.STATE_FIELDS, **G.PARAM_FIELDS, **G.DIAG_FIELDS}
    for r in range(case["n_rods"]):
        for field, entry in case["inject"][str(r)].items():
            if field not in kinds:
                continue  # ExternalLoads/Torques are rebuilt from zero every step
            kind = kinds[field][1]
            vals = G.values(entry) if kind == "tensor" else G.as_component_major(entry, kind)
            refs[r].set(field, vals.reshape(refs[r].shape(field)))
    return sim, refs


def compare_golden(refs, case, sec):
    kinds = {**G.STATE_FIELDS, **G.PARAM_FIELDS, **G.DIAG_FIELDS}
    worst = {}
    for r in range(case["n_rods"]):
        for field, entry in sec["expected"][str(r)].items():
            kind = kinds[field][1]
            want = G.as_component_major(entry, kind)
            got = refs[r].get(field).reshape(want.shape)
            worst[(r, field)] = G.catch_violation(got, want, sec["epsilon"])
    return worst


@pytest.mark.parametrize("name,case,sec,damped", list(G.step_cases()),
                         ids=lambda v: v if isinstance(v, str) else (
                             v.get("name", "").split(".")[-1] if isinstance(v, dict) else str(v)))
def test_golden_reference_rounding(name, case, sec, damped):
    """Reference-rounding FP64 build vs the reference's goldens at the
    reference's own epsilon (Catch semantics)."""
    sim, refs = golden_sim(case, damped, reference_rounding=True)
    if sec["steps"]:
        sim.step(eb.PositionVerlet(), 0.0, G.ROD_SETUP["dt"], sec["steps"])
    worst = compare_golden(refs, case, sec)
    bad = {k: v for k, v in worst.items() if v > 1.0}
    assert not bad, bad


@pytest.mark.parametrize("name,case,sec,damped", list(G.step_cases()),
                         ids=lambda v: v if isinstance(v, str) else (
                             v.get("name", "").split(".")[-1] if isinstance(v, dict) else str(v)))
def test_golden_resident(name, case, sec, damped):
    """The resident multi-step kernel vs the goldens (diagnostics of the last
    step come from the streaming kernel, so the state after steps-1 resident
    steps is what this checks), at 4x the reference's epsilon."""
    sim, refs = golden_sim(case, damped, reference_rounding=False, step_mode="resident", resident_config=1)
    if sec["steps"]:
        sim.step(eb.PositionVerlet(), 0.0, G.ROD_SETUP["dt"], sec["steps"])
    worst = compare_golden(refs, case, sec)
    bad = {k: v for k, v in worst.items() if v > 4.0}
    assert not bad, bad


@pytest.mark.parametrize("name,case,sec,damped", list(G.step_cases()),
                         ids=lambda v: v if isinstance(v, str) else (
                             v.get("name", "").split(".")[-1] if isinstance(v, dict) else str(v)))
def test_golden_default(name, case, sec, damped):
    """Default FP64 build (FMA contraction, rounding-level reformulations) vs
    the goldens.  These change rounding by ~1 ulp per operation, so the bound
    is 4x the reference's epsilon (the reference's own tolerances leave under
    2% headroom for its non-FMA arithmetic, see test_oracle_golden)."""
    sim, refs = golden_sim(case, damped, reference_rounding=False)
    if sec["steps"]:
        sim.step(eb.PositionVerlet(), 0.0, G.ROD_SETUP["dt"], sec["steps"])
    worst = compare_golden(refs, case, sec)
    bad = {k: v for k, v in worst.items() if v > 4.0}
    assert not bad, bad


def test_state_injection_roundtrip_exact():
    """Test_PerturbedRod.cpp WithDynamicAndExternal / FullWithDirector: every
    injected variable reads back bit-exactly (epsilon 1e-16 / 1e-20)."""
    doc = G.load("perturbed_rod")
    for case in doc["cases"]:
        if case["name"].split(".")[-1] not in ("WithDynamicAndExternal", "FullWithDirector"):
            continue
        sim, refs = golden_sim(case, damped=True, reference_rounding=False)
        kinds = {**G.STATE_FIELDS, **G.PARAM_FIELDS, **G.DIAG_FIELDS}
        n_checked = 0
        for r in range(case["n_rods"]):
            for field, entry in case["expected"][str(r)].items():
                if field not in kinds:
                    continue
                kind = kinds[field][1]
                want = G.as_component_major(entry, kind)
                got = refs[r].get(field).reshape(want.shape)
                assert np.array_equal(got, want), (case["name"], r, field)
                n_checked += 1
        assert n_checked >= 2 * 26
        sim.close()


def _run_pair(wl, n_steps, reference_rounding=False, damped=False, window=0, step_mode="streaming"):
    """Run the workload on the GPU and in the oracle; return the simulator,
    the oracle run, the per-field errors and the parity bounds."""
    sim = wl.build(record_diagnostics=False, reference_rounding=reference_rounding, window=window,
                   step_mode=step_mode)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, n_steps)
    orc, spread = B.oracle_spread(wl, n_steps, damped=damped)
    want = B.state_slots(orc)
    errs = {}
    for name, place in (("Position", 0), ("Velocity", 0), ("Director", 1), ("AngularVelocity", 1)):
        got = sim.get_slots(name)
        errs[name] = B.max_rel_error_per_rod(got, want[name], wl.n_elements, place)
    bounds = B.parity_bounds(spread)
    assert errs["Position"] <= B.PARITY_FLOOR and errs["Director"] <= B.PARITY_FLOOR, errs
    return sim, orc, errs, bounds


def small_uneven(n_rods=48, seed=7, n_range=(2, 40)):
    wl = W.uneven_batch(n_rods=n_rods, seed=seed, n_range=n_range)
    return wl


@pytest.mark.parametrize("window,step_mode", [(0, "streaming"), (128, "streaming"), (256, "streaming"),
                                              (0, "resident")])
def test_uneven_batch_1000_steps_vs_oracle(window, step_mode):
    """Clamped rods of uneven length with gravity and the analytical damper:
    the FP64 drop-in matches the oracle after 1000 steps."""
    wl = small_uneven()
    sim, orc, errs, bounds = _run_pair(wl, 1000, window=window, step_mode=step_mode)
    assert within(errs, bounds), (errs, bounds)
    assert sim.step_plan()["mode"] == step_mode
    assert sim.launch_count() >= (1000 if step_mode == "streaming" else 8)


@pytest.mark.parametrize("window", [0, 256])
def test_reference_rounding_build_vs_oracle(window):
    wl = small_uneven(n_rods=16, seed=11)
    _, _, errs, bounds = _run_pair(wl, 1000, reference_rounding=True, window=window)
    assert within(errs, bounds), (errs, bounds)


@pytest.mark.parametrize("step_mode", ["streaming", "resident"])
def test_rest_curvature_end_torque_vs_oracle(step_mode):
    wl = W.mixed_batch(n_rods=24, seed=5, n_range=(3, 60), n_steps=500, dt=2e-6)
    _, _, errs, bounds = _run_pair(wl, 500, step_mode=step_mode)
    assert within(errs, bounds), (errs, bounds)


@pytest.mark.parametrize("step_mode", ["streaming", "resident"])
def test_explicitly_damped_rods_vs_oracle(step_mode):
    wl = small_uneven(n_rods=20, seed=3)
    wl.model = eb.CosseratRod
    for r in wl.rods:
        r.force_damping_rate = 0.3
        r.torque_damping_rate = 0.2
    wl.damper = None
    _, _, errs, bounds = _run_pair(wl, 1000, damped=True, step_mode=step_mode)
    assert within(errs, bounds), (errs, bounds)


@pytest.mark.parametrize("lengths", [[1000], [255, 1, 300], [2, 2, 2, 2, 2], [254], [255], [256], [600, 2, 511],
                                     [511, 512, 519, 2, 7, 250, 261]])
def test_tile_and_rod_boundaries(lengths):
    """Rods that span several 256-slot tiles, end exactly on tile edges, or
    are minimal (2 elements); rods that fill a resident CTA's 512-slot packing
    limit exactly (511 elements), pass it (512) or fill its 520-slot capacity
    (519), beside short rods the packing puts into the remainders.  A length
    of 1 in the list is replaced by 2."""
    lengths = [max(2, n) for n in lengths]
    rng = np.random.default_rng(len(lengths) * 1000 + sum(lengths))
    rods = []
    for n in lengths:
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        c = rng.standard_normal(3)
        c -= c.dot(d) * d
        c /= np.linalg.norm(c)
        rods.append(eb.StraightRod(n_elements=n, material=eb.Material(1000.0, 1e6, 1e6 / 3), radius=0.01,
                                   length=float(0.05 * n), origin=tuple(rng.uniform(-1, 1, 3)),
                                   direction=tuple(d), normal=tuple(c)))
    wl = W.Workload("boundaries", 0, rods, velocities=[rng.normal(0, 1e-2, (3, n + 1)) for n in lengths],
                    dt=2e-6, n_steps=200)
    _, _, errs, bounds = _run_pair(wl, 200)
    assert within(errs, bounds), (errs, bounds)
    _, _, errs, bounds = _run_pair(wl, 200, reference_rounding=True, window=256)
    assert within(errs, bounds), (errs, bounds)
    # resident kernel where every rod fits one CTA; rods of 520 to 1039
    # elements run on CTA pairs in the per-size-bucket plan
    sim, _, errs, bounds = _run_pair(wl, 200, step_mode="resident")
    assert within(errs, bounds), (errs, bounds)
    assert sim.step_plan()["mode"] == ("resident" if max(lengths) + 1 <= 520 else "bucketed")


def test_energy_matches_oracle():
    wl = small_uneven(n_rods=12, seed=2)
    sim, orc, _, _ = _run_pair(wl, 50)
    e_gpu = sim.energy()
    e_cpu = orc.energy()
    np.testing.assert_allclose(e_gpu, e_cpu, rtol=1e-9, atol=1e-300)


@pytest.mark.parametrize("step_mode", ["streaming", "resident"])
def test_determinism_bitwise(step_mode):
    wl = small_uneven(n_rods=10, seed=4)
    a = wl.build(step_mode=step_mode)
    b = wl.build(step_mode=step_mode)
    a.step(eb.PositionVerlet(), 0.0, wl.dt, 100)
    b.step(eb.PositionVerlet(), 0.0, wl.dt, 100)
    for name in ("Position", "Velocity", "Director", "AngularVelocity"):
        assert np.array_equal(a.get_slots(name), b.get_slots(name)), name


def test_batch_layouts_agree():
    wl = small_uneven(n_rods=5, seed=9)
    sim = wl.build()
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 3)
    flat = sim.get_batch("Director")
    per = np.concatenate([r.get("Director").ravel() for r in sim.rods])
    assert np.array_equal(flat, per)
    # write through the per-rod batch layout, read back per rod
    v = np.arange(flat.size, dtype=np.float64)
    sim.set_batch("AngularVelocity", np.arange(sum(3 * r.n_elements for r in sim.rods), dtype=np.float64))
    got = np.concatenate([r.get("AngularVelocity").ravel() for r in sim.rods])
    assert np.array_equal(got, np.arange(got.size, dtype=np.float64))
    assert v.size == flat.size


def test_error_paths():
    wl = small_uneven(n_rods=2, seed=1)
    sim = wl.build()
    with pytest.raises(L.EbError) as e:
        sim.emplace_back(eb.CosseratRodWithoutDamping, wl.rods[0])
    assert e.value.status == 2  # EB_ERR_INVALID_STATE
    with pytest.raises(L.EbError) as e:
        L.call("eb_set_field", sim._h, 0, L.FIELD_ID["Position"],
               np.zeros(3).ctypes.data_as(L.ctypes.POINTER(L.ctypes.c_double)), 3)
    assert e.value.status == 1  # EB_ERR_INVALID_ARGUMENT
    with pytest.raises(L.EbError) as e:
        sim.rods[0].get("Curvature")
    assert e.value.status == 3  # EB_ERR_UNSUPPORTED without diagnostics
    with pytest.raises(L.EbError) as e:
        sim.rods[0].get.__self__.sim.step(eb.PositionVerlet(), 0.0, -1.0)
    assert e.value.status == 1
    with pytest.raises(L.EbError) as e:
        L.call("eb_get_field", sim._h, 99, 0, np.zeros(3).ctypes.data_as(L.ctypes.POINTER(L.ctypes.c_double)), 3)
    assert e.value.status == 6  # EB_ERR_NOT_FOUND


@pytest.mark.parametrize("step_mode", ["streaming", "resident"])
def test_full_size_uneven_batch_sampled_parity(step_mode):
    """The full uneven batch (16,384 rods, ~4.4 M elements) for 1000 steps on
    the GPU; rods are independent, so the oracle checks a seeded sample of 48
    of them run on their own."""
    wl = W.uneven_batch()
    sim = wl.build(step_mode=step_mode)
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1000)
    rng = np.random.default_rng(2024)
    pick = np.sort(rng.choice(len(wl.rods), size=48, replace=False))
    sub = W.Workload(wl.name, wl.seed, [wl.rods[k] for k in pick],
                     velocities=[wl.velocities[k] for k in pick], dt=wl.dt, n_steps=1000)
    orc, spread = B.oracle_spread(sub, 1000)
    bounds = B.parity_bounds(spread)
    offs = sim.slot_offsets()
    margins = {}
    for name, key, place in B.STATE_FIELDS:
        full = sim.get_slots(name)
        got = np.concatenate([full[:, offs[k]:offs[k + 1]] for k in pick], axis=1)
        err = B.max_rel_error_per_rod(got, orc.comp(key), sub.n_elements, place)
        # the margin: the error against the oracle's own one-ulp envelope
        margins[name] = {"error": err, "envelope": spread[name], "ratio": err / spread[name] if spread[name] else None,
                         "bound": bounds[name]}
        assert err <= bounds[name], (name, err, bounds[name])
    print(f"full-size parity margins ({step_mode}): {margins}")


def test_step_planner_times_every_candidate():
    wl = small_uneven(n_rods=64, seed=12, n_range=(20, 200))
    sim = wl.build()
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 4)
    plan = sim.step_plan()
    assert plan["mode"] in ("streaming", "resident")
    assert plan["probe_ms"][0] > 0.0  # streaming probe
    assert any(t > 0.0 for t in plan["probe_ms"][1:])  # at least one resident probe
