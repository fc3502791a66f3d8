"""Build the oracle's view of a workload from the workload's own parameters
(the oracle's straight-rod initializer, not the product's), so the product and
the checker share only the numbers a user would pass in."""
from __future__ import annotations

import numpy as np

import oracle


def oracle_from_workload(wl, damped: bool = False, diagnostics: bool = False):
    rods = oracle.RodArrays(wl.n_elements, damped=damped)
    for r, p in enumerate(wl.rods):
        n = int(p.n_elements)
        init = oracle.straight_rod(n, p.origin, p.direction, p.normal, p.length, p.radius,
                                   p.material.density, p.material.youngs_modulus, p.material.shear_modulus)
        rods.set_rod("x", r, init["x"])
        rods.set_rod("Q", r, init["Q"].reshape(9, n))
        rods.set_rod("mass", r, init["mass"])
        rods.set_rod("rest_length", r, init["l0"])
        rods.set_rod("rest_voronoi", r, init["D0"])
        rods.set_rod("volume", r, init["V"])
        rods.set_rod("shear_diag", r, init["S"])
        rods.set_rod("bend_diag", r, init["B"])
        rods.set_rod("inertia_diag", r, init["J"])
        rods.set_rod("inv_inertia", r, init["Jinv"])
        if damped:
            rods.set_rod("nu_force", r, np.full(n + 1, p.force_damping_rate))
            rods.set_rod("nu_torque", r, np.full(n, p.torque_damping_rate))
        if wl.velocities is not None:
            rods.set_rod("v", r, wl.velocities[r])
        if wl.rest_curvature is not None:
            rods.set_rod("rest_kappa", r, wl.rest_curvature[r])
        if wl.clamp if isinstance(wl.clamp, bool) else wl.clamp[r]:
            rods.clamp[r] = 1
            at = list(wl.clamp_at[r]) if getattr(wl, "clamp_at", None) is not None else [0]
            rods.clamp_index[2 * r:2 * r + 2] = (at + [-1, -1])[:2]
            # the targets: the initial state at those indices, as the clamp captures it
            for c, k in enumerate(at[:2]):
                tx, tq = (rods.clamp_x, rods.clamp_Q) if c == 0 else (rods.clamp2_x, rods.clamp2_Q)
                tx[3 * r:3 * r + 3] = init["x"][:, k]
                tq[9 * r:9 * r + 9] = init["Q"][:, :, min(k, n - 1)].ravel()
        if getattr(wl, "torque_element", None) is not None:
            rods.torque_index[r] = int(wl.torque_element[r])
        if wl.damper is not None:
            rods.damper_nu[2 * r:2 * r + 2] = wl.damper
        if wl.end_torque is not None:
            rods.end_torque[3 * r:3 * r + 3] = wl.end_torque[r]
    if wl.gravity is not None:
        rods.gravity[:] = wl.gravity
    if diagnostics:
        rods.enable_diagnostics()
    return rods


def contact_spec(wl):
    """The oracle's collision-system description of a workload (None if the
    workload has no contact)."""
    if not wl.contact_materials:
        return None
    mats = [[m.stiffness, m.normal_damping, m.tangential_damping, m.static_friction, m.dynamic_friction]
            for m in wl.contact_materials]
    rod_mat = wl.contact_rod_material if wl.contact_rod_material is not None else [0] * len(wl.rods)
    return oracle.ContactSpec(mats, rod_mat, list(wl.planes or []))


STATE_MAP = {"Position": "x", "Velocity": "v", "Director": "Q", "AngularVelocity": "w"}


def state_slots(rods):
    """Oracle state as {field: (ncomp, n_slots)} in the product's slot layout."""
    return {name: rods.comp(key) for name, key in STATE_MAP.items()}


def valid_mask(n_elems, place):
    """Boolean mask over slots of the entries that exist for a stagger."""
    out = []
    for n in n_elems:
        n = int(n)
        m = np.zeros(n + 1, dtype=bool)
        cnt = n + 1 if place == 0 else (n if place == 1 else n - 1)
        m[:cnt] = True
        out.append(m)
    return np.concatenate(out)


def max_rel_error(got, want, mask):
    """Normwise relative error: max |got - want| / max |want| over the valid
    entries of one field (all components)."""
    g = np.asarray(got)[:, mask]
    w = np.asarray(want)[:, mask]
    scale = np.max(np.abs(w))
    if scale == 0.0:
        return float(np.max(np.abs(g)))
    return float(np.max(np.abs(g - w)) / scale)


def max_rel_error_per_rod(got, want, n_elems, place):
    """Largest per-rod normwise relative error of one field:
    max over rods of max|got - want| / max|want| (entries of that rod's
    stagger only)."""
    worst = 0.0
    o = 0
    for n in n_elems:
        n = int(n)
        cnt = n + 1 if place == 0 else (n if place == 1 else n - 1)
        g = np.asarray(got)[:, o:o + cnt]
        w = np.asarray(want)[:, o:o + cnt]
        scale = np.max(np.abs(w))
        err = np.max(np.abs(g - w))
        rel = err / scale if scale > 0 else err
        worst = max(worst, float(rel))
        o += n + 1
    return worst


STATE_FIELDS = (("Position", "x", 0), ("Velocity", "v", 0), ("Director", "Q", 1), ("AngularVelocity", "w", 1))


def oracle_spread(wl, n_steps, damped=False, stepper="position_verlet"):
    """Conditioning envelope of a workload: the largest per-rod normwise
    relative change of each state field after n_steps when every initial
    position, or every initial director entry, of the oracle is moved by one
    ulp.  Returns (reference_run, {field: spread})."""
    base = oracle_from_workload(wl, damped=damped)
    base.step(wl.dt, n_steps, stepper=stepper)
    spread = {name: 0.0 for name, _, _ in STATE_FIELDS}
    for key in ("x", "Q"):
        p = oracle_from_workload(wl, damped=damped)
        p.arrays[key] = np.nextafter(p.arrays[key], np.inf)
        p.step(wl.dt, n_steps, stepper=stepper)
        for name, k, place in STATE_FIELDS:
            spread[name] = max(spread[name], max_rel_error_per_rod(p.comp(k), base.comp(k), wl.n_elements, place))
    return base, spread


def oracle_spread_contact(wl, n_steps):
    """oracle_spread for a workload with a collision system (orc_step_contact)."""
    base = oracle_from_workload(wl)
    oracle.contact_step(base, contact_spec(wl), wl.dt, n_steps)
    spread = {name: 0.0 for name, _, _ in STATE_FIELDS}
    for key in ("x", "Q"):
        p = oracle_from_workload(wl)
        p.arrays[key] = np.nextafter(p.arrays[key], np.inf)
        oracle.contact_step(p, contact_spec(wl), wl.dt, n_steps)
        for name, k, place in STATE_FIELDS:
            spread[name] = max(spread[name], max_rel_error_per_rod(p.comp(k), base.comp(k), wl.n_elements, place))
    return base, spread


def connection_spec(wl):
    """The oracle's description of a workload's connections (None if none)."""
    from elasticapp_b200.simulator import HingeJoint
    if not wl.connections:
        return None
    rows = []
    for ra, ia, rb, ib, j in wl.connections:
        hinge = isinstance(j, HingeJoint)
        rows.append((ra, ia, rb, ib, 1 if hinge else 0, j.stiffness, j.damping,
                     j.rotational_stiffness if hinge else 0.0, j.normal if hinge else (0.0, 0.0, 0.0)))
    return oracle.ConnectionSpec(rows)


def loads_step(rods, wl, n_steps):
    oracle.loads_step(rods, contact_spec(wl), connection_spec(wl), wl.dt, n_steps)


def oracle_spread_loads(wl, n_steps):
    """oracle_spread for a workload with connections and/or contact
    (orc_step_loads)."""
    from elasticapp_b200.simulator import CosseratRod
    damped = wl.model is CosseratRod
    base = oracle_from_workload(wl, damped=damped)
    loads_step(base, wl, n_steps)
    spread = {name: 0.0 for name, _, _ in STATE_FIELDS}
    for key in ("x", "Q"):
        p = oracle_from_workload(wl, damped=damped)
        p.arrays[key] = np.nextafter(p.arrays[key], np.inf)
        loads_step(p, wl, n_steps)
        for name, k, place in STATE_FIELDS:
            spread[name] = max(spread[name], max_rel_error_per_rod(p.comp(k), base.comp(k), wl.n_elements, place))
    return base, spread


# Parity rule of the FP64 step: every state field within 1e-10 (per-rod
# normwise relative error), or within 10x the one-ulp conditioning envelope
# of the oracle itself where that envelope is wider.
PARITY_FLOOR = 1e-10
PARITY_ENVELOPE_FACTOR = 10.0


def parity_bounds(spread):
    return {k: max(PARITY_FLOOR, PARITY_ENVELOPE_FACTOR * v) for k, v in spread.items()}
