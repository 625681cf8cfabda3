"""The index logic of the doubling rehash (rehash_double_kernel,
mcdfci_b200/csrc/gpu_solver.cu), restated on the CPU.

When a linear-probing table of C slots doubles, an entry with home p moves to
home p or p + C.  CTA b of the kernel owns the run of whole clusters from the
first empty slot at or after b * kRehashChunk to the first at or after
(b + 1) * kRehashChunk (or the last empty slot of the table), places its
entries in [e0, e1) and [e0 + C, e1 + C) of the new table in any order, and
writes both ranges whole; one extra CTA takes the cluster that wraps from slot
C-1 to slot 0 and the regions [Z, C + W) and [Z + C, 2C) + [0, W).  Runs
longer than kRehashRange are inserted slot by slot inside their ranges.

The checks: every slot of the new table is written exactly once, no probe
leaves its range, and every key is found again by linear probing from its new
home, on random tables at loads up to 0.97, with clusters forced through the
table's last and first slots, and in both the shared-memory and the global
mode.  The same kernel runs on the GPU in tests/test_gpu_growth.py.
"""
import os
import random
import re

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "mcdfci_b200", "csrc", "gpu_solver.cu")


def _constant(name):
    text = open(SRC).read()
    m = re.search(r"constexpr int %s = (\d+);" % name, text)
    assert m, name
    return int(m.group(1))


CHUNK = _constant("kRehashChunk")
RANGE = _constant("kRehashRange")


def _old_table(C, load, rng, wrap):
    t = [None] * C
    keys = {}
    for k in range(int(load * C)):
        h = rng.getrandbits(40)
        if wrap and k < 40:
            h = (h & ~(C - 1)) | (C - 1 - k % 5)  # homes in the last slots
        i = h & (C - 1)
        while t[i] is not None:
            i = (i + 1) & (C - 1)
        t[i] = (k, h)
        keys[k] = h
    return t, keys


def _first_empty(src, lo, hi):
    for i in range(lo, hi):
        if src[i] is None:
            return i
    return hi


def _last_empty(src, lo, hi):
    for i in range(hi - 1, lo - 1, -1):
        if src[i] is None:
            return i
    return -1


def _rehash(src, C, force_global, rng, planted=None):
    N = 2 * C
    dst = ["unwritten"] * N
    writes = [0] * N
    errors = []

    def write(i, v):
        assert 0 <= i < N
        writes[i] += 1
        dst[i] = v

    def insert_global(entry, limit):
        i = entry[1] & (N - 1)
        for _ in range(limit):
            assert dst[i] != "unwritten", "a probe reached a slot no CTA had written"
            if dst[i] is None:
                dst[i] = entry
                return True
            i = (i + 1) & (N - 1)
        return False

    blocks = list(range(C // CHUNK + 1))
    rng.shuffle(blocks)  # CTAs in any order: their regions are disjoint
    for b in blocks:
        if b == C // CHUNK:
            if planted == "no_wrap":
                continue
            W, Z = _first_empty(src, 0, C), _last_empty(src, 0, C)
            n = C - Z + W
            for i in range(n):
                write(Z + i, None)
                write((Z + C + i) & (N - 1), None)
            for i in range(1, n):
                e = src[(Z + i) & (C - 1)]
                if e is not None and not insert_global(e, n):
                    errors.append(("wrap", i))
            continue
        s = b * CHUNK
        e0 = _first_empty(src, s, C)
        e1 = _first_empty(src, s + CHUNK, C)
        if e1 == C:
            e1 = _last_empty(src, s, s + CHUNK)
        if planted == "chunk_cut":  # runs cut at the chunk bounds, not at empty slots
            e0, e1 = max(s - 1, 0), min(s + CHUNK - 1, C - 1)
        if e0 >= C or e1 <= e0:
            continue
        L = e1 - e0
        if L > RANGE or force_global:
            for i in range(L):
                write(e0 + i, None)
                write(e0 + C + i, None)
            for i in range(1, L):
                e = src[e0 + i]
                if e is not None and not insert_global(e, L):
                    errors.append(("run", e0 + i))
            continue
        lo, hi = [-1] * L, [-1] * L
        order = list(range(1, L))
        rng.shuffle(order)  # shared-memory placement in any order
        for i in order:
            e = src[e0 + i]
            if e is None:
                continue
            arr = hi if e[1] & C else lo
            home = e[1] & (C - 1)
            p = home - e0
            if home <= e0 or p > i:
                errors.append(("home", e0 + i))
                continue
            while p < L and arr[p] != -1:
                p += 1
            if p >= L:
                errors.append(("range", e0 + i))
                continue
            arr[p] = i
        for i in range(L):
            write(e0 + i, src[e0 + lo[i]] if lo[i] >= 0 else None)
            write(e0 + C + i, src[e0 + hi[i]] if hi[i] >= 0 else None)
    return dst, writes, errors


@pytest.mark.parametrize("load", [0.3, 0.75, 0.97])
@pytest.mark.parametrize("force_global", [False, True])
@pytest.mark.parametrize("wrap", [False, True])
def test_doubling_rehash_runs(load, force_global, wrap):
    C = 1 << 12
    rng = random.Random(int(load * 100) + 2 * force_global + wrap)
    src, keys = _old_table(C, load, rng, wrap)
    dst, writes, errors = _rehash(src, C, force_global, rng)
    assert not errors
    assert all(w == 1 for w in writes)
    N = 2 * C
    for k, h in keys.items():
        i = h & (N - 1)
        while True:
            assert dst[i] is not None, "key lost"
            if dst[i][0] == k:
                break
            i = (i + 1) & (N - 1)
    assert sum(e is not None for e in dst) == len(keys)
    if wrap:
        assert src[0] is not None and src[C - 1] is not None


@pytest.mark.parametrize("planted", ["chunk_cut", "no_wrap"])
def test_planted_mistakes_are_caught(planted):
    """The checks above catch a rehash that cuts runs at the chunk bounds
    (entries whose home lies in the previous chunk) or leaves out the
    wrapping cluster."""
    C = 1 << 12
    rng = random.Random(7)
    src, keys = _old_table(C, 0.75, rng, True)
    try:
        dst, writes, errors = _rehash(src, C, False, rng, planted)
    except AssertionError:
        return  # a probe reached a slot that no CTA wrote
    N = 2 * C
    lost = 0
    for k, h in keys.items():
        i = h & (N - 1)
        while dst[i] not in (None, "unwritten") and dst[i][0] != k:
            i = (i + 1) & (N - 1)
        lost += dst[i] in (None, "unwritten")
    assert errors or lost or any(w != 1 for w in writes)
