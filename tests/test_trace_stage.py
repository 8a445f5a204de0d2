"""The staged trace store of the packed banded-SW sweep (csrc/bsw16.cuh: TraceStage in
bsw16_group_sweep), restated on the CPU. A group keeps its current interleave block of
R rows in a shared-memory strip and copies the whole strip to the item's trace slot when
the block's last row is done (stored or skipped) and when the sweep ends (last row or
an early abort). Over random row counts, skipped rows (rows whose band lies outside the
window) and abort rows, for several items in a row through the same strip (which keeps
the previous item's contents), this checks that every row the sweep stored reaches the
slot with its own contents, that a block is only ever copied whole, and that the strip
is never written while a copy of it is still pending."""
import random

import pytest


def sweep(q, skipped, abort_at, R, strip, slot, item):
    """One item's sweep; returns the rows it stored and their contents."""
    dirty = False
    inflight = False
    blk = 0
    stored = {}

    def flush():
        nonlocal dirty, inflight
        slot.setdefault(blk, None)
        slot[blk] = list(strip)  # the bulk copy takes the whole strip
        inflight = True
        dirty = False

    def ready():
        nonlocal inflight
        inflight = False  # wait_group.read before the strip is written again

    for i in range(1, q + 1):
        if i in skipped:
            if dirty and (i & (R - 1)) == R - 1:
                flush()
            continue
        ready()
        assert not inflight
        blk = i // R
        strip[i & (R - 1)] = (item, i)
        stored[i] = (item, i)
        dirty = True
        if (i & (R - 1)) == R - 1:
            flush()
        if i == abort_at:
            break
    if dirty:
        flush()
    ready()
    return stored


@pytest.mark.parametrize("R", [1, 2, 4, 8, 16, 32])
def test_every_stored_row_reaches_the_slot(R):
    rng = random.Random(0x57A6 + R)
    strip = [("garbage", -1)] * R
    for item in range(200):
        q = rng.randint(1, 4 * R + 7)
        skipped = {i for i in range(1, q + 1) if rng.random() < 0.2}
        abort_at = rng.randint(1, q) if rng.random() < 0.3 else -1
        slot = {}
        stored = sweep(q, skipped, abort_at, R, strip, slot, item)
        for i, v in stored.items():
            assert slot[i // R][i % R] == v, (R, item, i)
        # the slot holds whole blocks only, inside the item's rows 0..q rounded up to R
        rows = (q + 1 + R - 1) // R * R
        assert all(0 <= b * R < rows and len(v) == R for b, v in slot.items())
