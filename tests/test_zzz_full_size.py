"""Parity at the benchmark's full sizes through properties that do not need
the whole input on the CPU: the result is strictly increasing in (offset, id)
(sorted and unique, as ngap.cu:1890-1932 leaves it), every offset lies inside
the input, and the reports of sampled segments equal the oracle's on those
segments alone (segments are matched independently; the oracle's
first_segment gives a sampled segment the start-of-data rule of its place,
ngap_buffer.cu:613-631). The helper is checked on the CPU first, against the
oracle's own full result and against planted mistakes."""
import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200 import workloads as W
from oracle import oracle

M32 = np.uint64(0xFFFFFFFF)
S32 = np.uint64(32)


def sampled_parity(got, views, data, num_seg, seg_len, sample):
    got = np.asarray(got, dtype=np.uint64)
    off, ids = got & M32, got >> S32
    key = (off << S32) | ids
    assert np.all(key[1:] > key[:-1]), "not sorted by (offset, id) or not unique"
    assert got.size == 0 or int(off.max()) < num_seg * seg_len
    for s in sample:
        lo = s * seg_len
        want, _ = oracle.match(views, data[lo:lo + seg_len], 1, seg_len, first_segment=s)
        want = np.asarray(want, dtype=np.uint64)
        want = (want & ~M32) | ((want & M32) + np.uint64(lo))
        mine = got[(off >= lo) & (off < lo + seg_len)]
        assert np.array_equal(mine, want), f"segment {s}: {len(mine)} reports, oracle {len(want)}"


def test_sampled_parity_helper_catches_planted_mistakes():
    anml, data = W.hamming_set(seed=8, n_patterns=30, input_len=1 << 16, plant_every=1 << 11)
    views = nb.Groups(nb.Nfa.from_string(anml), group_num=3).views()
    full, _ = oracle.match(views, data, 8, 1 << 13)
    assert len(full) > 20
    sampled_parity(full, views, data, 8, 1 << 13, (0, 5))
    off = (full & M32).astype(np.int64)
    k = int(np.nonzero(off >= 5 << 13)[0][0])  # first report of segment 5
    planted = [np.delete(full, k),                      # a report missing
               full.copy(),                             # an offset moved
               np.concatenate([full[:1], full[1:][::-1]])]  # out of order
    planted[1][k] += np.uint64(1)
    for bad in planted:
        with pytest.raises(AssertionError):
            sampled_parity(bad, views, data, 8, 1 << 13, (0, 5))


CONFIGS = {  # the benchmark's workloads at full size
    "hamming_set": (lambda: W.hamming_set(seed=2), 10, 1 << 20, (11,)),
    "high_frontier": (lambda: W.high_frontier(seed=3), 10, 1 << 20, (3, 20)),
    "literal_set": (lambda: W.literal_set(seed=1), 1, 1 << 20, (0,)),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONFIGS))
def test_full_size_sampled_parity(engine, name):
    gen, group_num, seg_len, sample = CONFIGS[name]
    anml, data = gen()
    groups = nb.Groups(nb.Nfa.from_string(anml), group_num=group_num)
    tables = nb.Tables(groups, precompute_depth=-1)
    num_seg = len(data) // seg_len
    got = engine.match(tables, data, num_seg, seg_len, algorithm="nonblockingpcgroups")
    raw, uniq = engine.counts()
    assert uniq == len(got) and raw >= uniq and uniq > 0
    sampled_parity(got, groups.views(), data, num_seg, seg_len, sample)
