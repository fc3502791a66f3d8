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


@pytest.mark.parametrize("W", [128, 256])
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


def stage_rows(damped, diag, stored_jinv):
    """Rows of one stage buffer of the persistent kernel (StageMap): 18 state
    rows and every parameter row the variant reads."""
    params = 24 - (0 if damped else 2) - (0 if diag else 1) - (0 if stored_jinv else 3)
    return 18 + params


@pytest.mark.parametrize("sms,per_sm", [(148, 3), (148, 2), (1, 1), (7, 3)])
def test_persistent_schedule_visits_every_window_once(sms, per_sm):
    """CTA c walks windows c, c + G, ... (G = its grid), alternating its two
    stage buffers; every window is computed by exactly one CTA, and the bulk
    copies of window i + 1 go to the buffer window i does not use."""
    W, T = 128, 124
    for n_slots in list(range(3, 3000, 37)) + [4458875]:
        n_win = (n_slots + T - 1) // T
        G = min(n_win, sms * per_sm)
        seen = [0] * n_win
        for c in range(G):
            it, w = 0, c
            while w < n_win:
                seen[w] += 1
                buf, parity = it & 1, (it >> 1) & 1
                nxt = w + G
                if nxt < n_win:
                    # the next window lands in the other buffer, whose
                    # previous window (it - 1) finished before this one began
                    assert ((it + 1) & 1) != buf
                assert parity in (0, 1)
                it, w = it + 1, nxt
        assert all(k == 1 for k in seen)


@pytest.mark.parametrize("damped", [False, True])
@pytest.mark.parametrize("diag", [False, True])
@pytest.mark.parametrize("stored", [False, True])
def test_persistent_shared_memory_fits(damped, diag, stored):
    W = 128
    rows = stage_rows(damped, diag, stored)
    stage_bytes = rows * W * 8
    total = 2 * stage_bytes + 16  # two stage buffers and two mbarriers
    assert stage_bytes % 16 == 0  # the second buffer and every row start 16-byte aligned
    assert (2 * stage_bytes) % 8 == 0  # the mbarriers are 8-byte aligned
    assert total <= 227 * 1024
    # CTAs an SM by shared memory (228 KB an SM, 1 KB reserved a CTA)
    per_sm = 228 * 1024 // (total + 1024)
    assert per_sm >= (2 if (diag or damped or stored) else 3)
