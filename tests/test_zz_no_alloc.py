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


def _noalloc_pairs(boxes):
    """Candidate pairs (k, 2) of boxes (n, 6) through eb_box_pairs_noalloc."""
    import torch

    from elasticapp_b200 import _lib as L

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    b = torch.from_numpy(np.ascontiguousarray(boxes, dtype=np.float64)).to(dev)
    n = boxes.shape[0]
    cap = 32 * n
    out = torch.full((cap, 2), -1, dtype=torch.int64, device=dev)
    count = ctypes.c_int64()
    stream = torch.cuda.current_stream(dev).cuda_stream
    L.call("eb_box_pairs_noalloc", ctypes.c_void_p(b.data_ptr()), n, ctypes.c_void_p(out.data_ptr()), cap,
           ctypes.byref(count), ctypes.c_void_p(stream))
    return out[:count.value].cpu().numpy()


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


def test_noalloc_rejects_more_boxes_than_its_array_holds():
    from elasticapp_b200 import _lib as L

    count = ctypes.c_int64()
    with pytest.raises(L.EbError, match="at most 131072"):
        L.call("eb_box_pairs_noalloc", None, 131073, None, 0, ctypes.byref(count), None)
