"""The oracle's clamps at any index and the torque at any element
(Simulator/Constraints/MakeConstraint.hpp:130-151: a constraint applied
.at(index) receives that index; the clamp generator of
examples/dynamic_cantilever/DynamicCantileverCaseStudy.cpp:73-89 fixes
position(index) and director(index) and zeroes their rates)."""
import numpy as np
import pytest

from oracle_bridge import oracle_from_workload


@pytest.fixture(scope="module")
def W():
    from elasticapp_b200 import workloads
    return workloads


def _batch(W, **kw):
    wl = W.uneven_batch(n_rods=6, seed=21, n_range=(20, 60))
    for k, v in kw.items():
        setattr(wl, k, v)
    return wl


def test_default_clamp_index_is_the_legacy_clamp(W, oracle_mod):
    wl = _batch(W)
    a = oracle_from_workload(wl)
    b = oracle_from_workload(wl)
    b.clamp_index[:] = np.tile([0, -1], len(wl.rods))
    a.step(wl.dt, 50)
    b.step(wl.dt, 50)
    for k in ("x", "v", "Q", "w"):
        np.testing.assert_array_equal(a.comp(k), b.comp(k))


def test_clamps_at_both_ends_and_inside_hold_their_slots(W, oracle_mod):
    wl = _batch(W)
    n = wl.n_elements
    # rod r: clamps at node 0 and node n (a beam held at both ends), except
    # rod 2: node n // 2 alone (a clamp inside the rod)
    wl.clamp_at = [[0, int(m)] for m in n]
    wl.clamp_at[2] = [int(n[2]) // 2]
    orc = oracle_from_workload(wl)
    x0 = {r: orc.get_rod("x", r, int(n[r]) + 1) for r in range(len(n))}
    q0 = {r: orc.get_rod("Q", r, int(n[r])) for r in range(len(n))}
    orc.step(wl.dt, 400)
    for r in range(len(n)):
        m = int(n[r])
        x, v = orc.get_rod("x", r, m + 1), orc.get_rod("v", r, m + 1)
        q, w = orc.get_rod("Q", r, m), orc.get_rod("w", r, m)
        for k in wl.clamp_at[r]:
            np.testing.assert_array_equal(x[:, k], x0[r][:, k])
            assert np.all(v[:, k] == 0.0)
            if k < m:  # the element at the index is held too
                np.testing.assert_array_equal(q[:, k], q0[r][:, k])
                assert np.all(w[:, k] == 0.0)
        if m in wl.clamp_at[r]:
            # node n has no element: the last element still turns (a pin)
            assert np.any(q[:, m - 1] != q0[r][:, m - 1])
        # the free parts of the rod move under gravity
        free = [j for j in range(m + 1) if j not in wl.clamp_at[r]]
        assert np.max(np.abs(x[:, free] - x0[r][:, free])) > 0.0


def test_torque_at_an_inner_element_acts_there(W, oracle_mod):
    wl = _batch(W, gravity=None, damper=None)
    n = wl.n_elements
    wl.end_torque = np.tile([0.0, 0.0, 1e-4], (len(n), 1))
    wl.torque_element = [int(m) // 3 for m in n]
    base = _batch(W, gravity=None, damper=None)
    a, b = oracle_from_workload(wl), oracle_from_workload(base)
    a.step(wl.dt, 1)
    b.step(wl.dt, 1)
    for r in range(len(n)):
        m = int(n[r])
        dw = np.abs(a.get_rod("w", r, m) - b.get_rod("w", r, m)).max(axis=0)
        # after one step only the loaded element has turned differently
        assert np.argmax(dw) == wl.torque_element[r]
        others = np.delete(dw, wl.torque_element[r])
        assert np.all(others == 0.0)
