"""Conditioning of the rod step (CPU, oracle only).

The parity bound of the GPU step against the oracle has to sit above the
spread that rounding alone produces.  This test measures that spread with the
oracle itself: it moves every initial position by one ulp and runs the same
1000 steps.  Positions, velocities and directors stay within 1e-10 of the
unperturbed run, but the angular velocity moves by more than 1e-10, which is
why the angular-velocity bound of the GPU parity tests is 1e-9.
"""
import numpy as np

from elasticapp_b200 import workloads as W

import oracle_bridge as B


def test_one_ulp_position_perturbation_spread(oracle_mod):
    wl = W.uneven_batch(n_rods=48, seed=7, n_range=(2, 40))
    base = B.oracle_from_workload(wl)
    base.step(wl.dt, 1000)
    pert = B.oracle_from_workload(wl)
    pert.arrays["x"] = np.nextafter(pert.arrays["x"], np.inf)
    pert.step(wl.dt, 1000)
    errs = {}
    for name, key, place in (("Position", "x", 0), ("Velocity", "v", 0), ("Director", "Q", 1),
                             ("AngularVelocity", "w", 1)):
        errs[name] = B.max_rel_error_per_rod(pert.comp(key), base.comp(key), wl.n_elements, place)
    assert errs["Position"] < 1e-10 and errs["Velocity"] < 1e-10 and errs["Director"] < 1e-10, errs
    assert 1e-10 < errs["AngularVelocity"] < 1e-9, errs
