"""eb_box_pairs_noalloc: the collision system's candidate-pair search for
callers that cannot allocate device memory (operators inside a host framework
that owns the whole GPU memory pool, loops that cannot take the device-wide
synchronisation of cudaMalloc / cudaFree).  Its working memory is a fixed
array inside the library.

Checked through the C-ABI against the existing entry point, eb_contact_pairs
of a simulator stepped once, on two calls in a row with different box counts
(the second call must not see the first call's leftovers in the shared
array): the capsule-capsule pairs must be identical.  The boxes handed to the
new entry point are the capsules' bounding boxes from the CPU oracle, which
builds them with the same rounding as the simulator's kernels.  The input
and output buffers here come from torch; the entry point itself allocates
nothing.

This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

import oracle
from oracle_bridge import contact_spec, oracle_from_workload

pytestmark = pytest.mark.gpu


def _noalloc_call(boxes, cap):
    """(status, count, pairs (count, 2) or None) of eb_box_pairs_noalloc on
    boxes (n, 6) with a pair buffer of cap pairs."""
    import torch

    from elasticapp_b200 import _lib as L

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    b = torch.from_numpy(np.ascontiguousarray(boxes, dtype=np.float64)).to(dev)
    n = boxes.shape[0]
    out = torch.full((max(cap, 1), 2), -1, dtype=torch.int64, device=dev)
    count = ctypes.c_int64()
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = L.load().eb_box_pairs_noalloc(ctypes.c_void_p(b.data_ptr()), n, ctypes.c_void_p(out.data_ptr()), cap,
                                       ctypes.byref(count), ctypes.c_void_p(stream))
    pairs = out[:count.value].cpu().numpy() if st == 0 else None
    return st, count.value, pairs


def _noalloc_pairs(boxes):
    """Candidate pairs (k, 2) of boxes (n, 6) through eb_box_pairs_noalloc."""
    from elasticapp_b200 import _lib as L

    st, _, pairs = _noalloc_call(boxes, 32 * boxes.shape[0])
    assert st == 0, L.load().eb_last_error().decode()
    return pairs


def _all_pairs(boxes):
    """Every overlapping pair (i < j) of closed boxes, sorted: the plain
    all-pairs test, independent of any grid."""
    lo, hi = boxes[:, :3], boxes[:, 3:]
    n = boxes.shape[0]
    i, j = np.triu_indices(n, 1)
    ok = np.all((lo[j] <= hi[i]) & (lo[i] <= hi[j]), axis=1)
    return np.stack([i[ok], j[ok]], axis=1).astype(np.int64)


def _lattice_boxes(n, seed):
    """Boxes on a 1/8 lattice: many touch exactly (a hi equal to another's
    lo) and about one in five has zero width along some axis."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lo = rng.integers(0, 96, size=(n, 3)) * 0.125
    ext = rng.integers(0, 5, size=(n, 3)) * 0.125
    return np.concatenate([lo, lo + ext], axis=1)


def _existing_and_boxes(W, eb, **kw):
    """Capsule-capsule pairs from eb_contact_pairs after one step, and the
    bounding boxes of those capsules (slot order) with their slots."""
    wl = W.contact_batch(**kw)
    sim = wl.build()
    sim.step(eb.PositionVerlet(), 0.0, wl.dt, 1)
    pairs = sim.contact_pairs()
    n_slots = sim.n_slots()
    sim.close()
    pairs = pairs[pairs[:, 1] < n_slots]
    rods = oracle_from_workload(wl)
    caps = oracle.contact_capsules(rods, contact_spec(wl), 0.5 * wl.dt)
    slots = np.flatnonzero(~np.isnan(caps[0]))
    boxes = caps[8:14, slots].T  # lo x, lo y, lo z, hi x, hi y, hi z
    return pairs, boxes, slots


def test_noalloc_pairs_match_contact_pairs_two_calls():
    import elasticapp_b200 as eb
    from elasticapp_b200 import workloads as W

    for kw in (dict(n_rods=96, seed=5, box=0.3), dict(n_rods=40, seed=9, box=0.2)):
        want, boxes, slots = _existing_and_boxes(W, eb, **kw)
        got = _noalloc_pairs(boxes)
        assert got.shape[0] > 0
        assert np.array_equal(slots[got], want), kw


def test_noalloc_pairs_match_all_pairs_on_touching_and_flat_boxes():
    """A few thousand lattice boxes (touching faces, zero-width boxes, all
    boxes with zero extent in the last case, which takes the unit-cell
    fallback) against the all-pairs overlap test; two calls in a row."""
    for n, seed in ((3000, 1), (2500, 2)):
        boxes = _lattice_boxes(n, seed)
        want = _all_pairs(boxes)
        assert want.shape[0] > 0
        np.testing.assert_array_equal(_noalloc_pairs(boxes), want)
    pts = _lattice_boxes(2000, 3)
    pts[:, 3:] = pts[:, :3]  # points: only coincident ones overlap
    np.testing.assert_array_equal(_noalloc_pairs(pts), _all_pairs(pts))


def test_noalloc_too_small_buffer_reports_the_count():
    from elasticapp_b200 import _lib as L

    boxes = _lattice_boxes(1500, 4)
    total = _all_pairs(boxes).shape[0]
    st, count, _ = _noalloc_call(boxes, total - 1)
    assert st == L.EB_ERR_INVALID_ARGUMENT
    assert count == total
    assert "too small" in L.load().eb_last_error().decode()
    st, count, pairs = _noalloc_call(boxes, total)  # exactly enough
    assert st == 0 and count == total
    np.testing.assert_array_equal(pairs, _all_pairs(boxes))


def test_noalloc_rejects_inverted_and_non_finite_boxes():
    from elasticapp_b200 import _lib as L

    for bad in ("inverted", "nan", "inf"):
        boxes = _lattice_boxes(300, 5)
        if bad == "inverted":
            boxes[17, 4] = boxes[17, 1] - 0.5  # hi y < lo y
        elif bad == "nan":
            boxes[40, 2] = np.nan
        else:
            boxes[99, 3] = np.inf
        st, count, _ = _noalloc_call(boxes, 10 * 300)
        assert st == L.EB_ERR_INVALID_ARGUMENT, bad
        assert count == 0
        assert "not finite" in L.load().eb_last_error().decode()
    # a good call after the rejected ones still gives the exact pairs
    boxes = _lattice_boxes(800, 6)
    np.testing.assert_array_equal(_noalloc_pairs(boxes), _all_pairs(boxes))


def test_noalloc_rejects_more_boxes_than_its_array_holds():
    from elasticapp_b200 import _lib as L

    count = ctypes.c_int64()
    with pytest.raises(L.EbError, match="at most 131072"):
        L.call("eb_box_pairs_noalloc", None, 131073, None, 0, ctypes.byref(count), None)
