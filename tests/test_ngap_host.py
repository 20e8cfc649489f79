"""The Python mirror of the reference's `class ngap` on the host (no GPU):
the main.cu flow up to the launch — input slicing (main.cu:48-51),
duplication and segmentation (main.cu:81-102), the duplicated-stream rule
(ngap_buffer.cu:479-484) — and validation with the library's CPU checker
(ngap.cu:2171-2344) on the apple example (README.md:156-186)."""
import os

import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200.engine import as_u8, cpu_validate

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KAT = np.array([0x400000005, 0x40000002F, 0x400000040, 0x40000004B], dtype=np.uint64)


def _apple(**kw):
    opt = nb.NgapOption(group_num=1, **kw)
    pl = nb.Ngap(nb.Nfa.from_file(os.path.join(GOLD, "apple.anml")), opt)
    pl.preprocessing()
    return pl


def test_bytes_input_and_validation(built):
    pl = _apple()
    raw = open(os.path.join(GOLD, "apple_input.txt"), "rb").read()
    assert pl.prepare_segments(raw) == (1, 81)  # bytes accepted, whole stream = one segment
    assert len(pl.original) == 81 and not pl.is_dup()
    assert pl.automata_validation(KAT)
    assert not pl.automata_validation(KAT[1:]) and not pl.automata_validation(KAT[::-1])


def test_slicing_duplication_segments(built):
    raw = bytearray(open(os.path.join(GOLD, "apple_input.txt"), "rb").read())
    pl = _apple(input_start_pos=40, input_len=30, duplicate_input_stream=3, split_chunk_size=30)
    assert pl.prepare_segments(raw) == (3, 30)
    assert all(np.array_equal(s, np.frombuffer(raw[40:70], np.uint8)) for s in pl.streams)
    assert pl.is_dup()  # split == input_len: start-of-data states in every segment
    pl = _apple(input_start_pos=70, input_len=50)  # shorter input: slice to the end
    assert pl.prepare_segments(raw) == (1, 11)
    pl = _apple(duplicate_input_stream=2, split_chunk_size=50)
    assert pl.prepare_segments(raw) == (3, 50) and not pl.is_dup()
    # matches end at 5, 47, 64, 75 and, in the second copy, 86, 128, 145, 156;
    # every one lies inside one 50-byte segment except 156 (past the third)
    want = cpu_validate(pl.groups, np.concatenate(pl.streams), 3, 50)
    assert [int(x & 0xFFFFFFFF) for x in want] == [5, 47, 64, 75, 86, 128, 145]


def test_sizes_are_checked(built):
    pl = _apple()
    with pytest.raises(nb.NgapError):
        cpu_validate(pl.groups, np.zeros(10, np.uint8), 2, 8)
    assert as_u8(memoryview(b"ab")).tolist() == [97, 98]
    assert as_u8([1, 2, 3]).dtype == np.uint8
