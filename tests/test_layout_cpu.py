"""CPU checks of the step kernel's window arithmetic (csrc/rod_step_fp64.cu).

A CTA of window W stores the W - 4 interior slots of [b (W-4) - 2, b (W-4) - 2 + W)
and stages each input field of the window with one bulk copy.  The copies
need 16-byte aligned source and destination and a byte count that is a
multiple of 16, and every interior slot's stencil must stay inside the
window.  These are checked here for many slot counts, including the batch
sizes used by the benchmark, so no launch shape reaches the GPU unchecked."""
import pytest


def windows(n_slots, W):
    T = W - 4
    S = (n_slots + 31) // 32 * 32
    grid = (n_slots + T - 1) // T
    for b in range(grid):
        g0 = b * T - 2
        lo, hi = max(g0, 0), min(g0 + W, S)
        yield b, g0, lo, hi, S, T


@pytest.mark.parametrize("W", [64, 96, 128, 256])
def test_window_copies_aligned_and_cover_every_slot(W):
    for n_slots in list(range(3, 2000, 7)) + [4458875, 10_517_000 + 3]:
        covered = 0
        last = -1
        for b, g0, lo, hi, S, T in windows(n_slots, W):
            assert hi > lo
            off = lo - g0
            assert (lo * 8) % 16 == 0 and (off * 8) % 16 == 0 and ((hi - lo) * 8) % 16 == 0
            assert 0 <= off and off + (hi - lo) <= W
            first, stop = g0 + 2, min(g0 + 2 + T, n_slots)
            assert first == last + 1
            covered += stop - first
            last = stop - 1
            # stencil reach of an interior slot: one left, two right
            assert 2 - 1 >= 0 and (2 + T - 1) + 2 < W
        assert covered == n_slots


def test_rod_table_index_width():
    # meta word: 5 flag bits, rod index in the remaining 27 bits
    assert (1 << (32 - 5)) > 65536 * 1024


def window_rows(damped, diag):
    """Rows of a window's shared memory (RowMap): 18 state rows and every
    parameter row the variant reads."""
    return 18 + 24 - (0 if damped else 2) - (0 if diag else 1)


@pytest.mark.parametrize("W,per_sm", [(64, 10), (96, 6), (128, 5), (256, 2)])
@pytest.mark.parametrize("damped", [False, True])
@pytest.mark.parametrize("diag", [False, True])
def test_window_shared_memory(W, per_sm, damped, diag):
    """Bytes of a window's rows plus its two mbarriers; the plain variant
    (undamped, no diagnostics) fits the CTAs an SM its launch bound asks for
    (228 KB an SM, 1 KB reserved a CTA)."""
    total = window_rows(damped, diag) * W * 8 + 16
    assert (W * 8) % 16 == 0  # every row starts 16-byte aligned
    assert total <= 227 * 1024
    if not (damped or diag):
        assert per_sm * (total + 1024) <= 228 * 1024
