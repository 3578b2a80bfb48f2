"""The write/read rule of the epoch kernel's segment markers, restated on
the CPU and checked on random offspring counts (no GPU).

Phase 4 gives slots [F(i-1), F(i)) to particle i.  A run of up to 128
slots is written slot by slot, plus the marker of the segment whose first
slot it holds (the ancestor when the run covers that segment, else -1); a
longer run writes one marker per segment that starts inside it and the
slots of the (at most two) segments it covers in part.  A reader takes a
segment's marker when it is >= 0 and the slot otherwise.  The rule must
write every segment's marker exactly once and make every slot read back as
its ancestor, whatever the slots held before.
"""
import numpy as np
import pytest

SEG = 128
LIGHT = 128


def write_runs(counts, anc_prev, mk_prev):
    n = len(counts)
    anc = anc_prev.copy()
    mk = mk_prev.copy()
    writes = np.zeros(len(mk), np.int64)
    ends = np.cumsum(counts)
    for i in range(n):
        lo, hi = int(ends[i] - counts[i]), int(ends[i])
        if hi <= lo:
            continue
        s_first, s_last = (lo + SEG - 1) // SEG, (hi - 1) // SEG
        if hi - lo <= LIGHT:
            anc[lo:hi] = i
            if s_first <= s_last:  # at most one segment starts inside a light run
                assert s_first == s_last
                mk[s_first] = i if min((s_first + 1) * SEG, n) <= hi else -1
                writes[s_first] += 1
            continue
        last_full = s_first <= s_last and min((s_last + 1) * SEG, n) <= hi
        for sg in range(s_first, s_last + 1):
            mk[sg] = i if (sg < s_last or last_full) else -1
            writes[sg] += 1
        anc[lo:min(hi, s_first * SEG)] = i
        if s_first <= s_last and not last_full:
            anc[s_last * SEG:hi] = i
    return anc, mk, writes


def read(anc, mk):
    seg = np.arange(len(anc)) // SEG
    return np.where(mk[seg] >= 0, mk[seg], anc)


def _counts(rng, n, kind):
    if kind == "peaked":  # a few heavy particles
        w = np.zeros(n)
        k = min(7, n)
        w[rng.choice(n, k, replace=False)] = rng.exponential(1.0, k)
    elif kind == "classes":  # runs around the segment and light-run sizes
        w = np.zeros(n)
        sizes = [1, 63, 127, 128, 129, 255, 256, 257, 4095]
        idx = rng.choice(n, len(sizes) + 1, replace=False)
        w[idx[:-1]] = sizes
        w[idx[-1]] = max(n - sum(sizes), 1)
    else:  # wide: every particle a few slots
        w = rng.exponential(1.0, n)
    c = np.floor(w / w.sum() * n).astype(np.int64)
    c[np.argmax(w)] += n - c.sum()
    return c


CASES = ([(n, k) for n in (1, 5, 127, 128, 129, 1000, 4099, 70_001) for k in ("peaked", "wide")]
         + [(n, "classes") for n in (5_250, 70_001, 131_075)])  # the size classes need > 5,100 slots


@pytest.mark.parametrize("n,kind", CASES)
def test_marker_rule_reads_back_every_ancestor(n, kind):
    rng = np.random.default_rng(n * 7 + len(kind))
    counts = _counts(rng, n, kind)
    assert counts.sum() == n
    want = np.repeat(np.arange(n), counts)
    # stale contents from an earlier step must not matter
    nseg = (n + SEG - 1) // SEG
    anc0 = rng.integers(0, n, n)
    mk0 = rng.integers(-1, n, nseg)
    anc, mk, writes = write_runs(counts, anc0, mk0)
    assert np.all(writes == 1)  # every marker exactly once
    assert np.array_equal(read(anc, mk), want)
