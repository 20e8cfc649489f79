"""Sharding of segments across GPUs (one process per GPU).

Segments never exchange state (code/src/ngap/ngap.cu:2201-2210: every segment
starts from its own frontier), so a stream of S segments splits into
contiguous per-rank blocks with no data-path communication. Each rank matches
its block with offsets local to the block; the only exchange is the final
gather of reports, shifted by the block's first byte, followed by the same
sort + unique as on one GPU.
"""
import numpy as np


def rank_segments(num_seg, rank, world):
    """[first, count) of the contiguous block of segments owned by `rank`."""
    base, extra = divmod(num_seg, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def shift_offsets(reports, byte_base):
    """Moves block-local report offsets (the low 32 bits) to stream offsets.
    The reference's offsets are 32-bit (code/src/ngap/ngap.cu:1899-1905), so a
    shifted offset past 2^32 - 1 is an error rather than a carry into the id."""
    r = np.asarray(reports, dtype=np.uint64)
    off = (r & np.uint64(0xFFFFFFFF)) + np.uint64(byte_base)
    if off.size and int(off.max()) > 0xFFFFFFFF:
        raise ValueError(f"stream offset {int(off.max())} exceeds the 32-bit report offsets")
    return (r & ~np.uint64(0xFFFFFFFF)) | off


def merge_reports(parts):
    """Concatenates per-rank reports and sorts them by (offset, id), unique."""
    allr = np.concatenate([np.asarray(p, dtype=np.uint64) for p in parts]) if parts else \
        np.zeros(0, np.uint64)
    key = ((allr & np.uint64(0xFFFFFFFF)) << np.uint64(32)) | (allr >> np.uint64(32))
    key = np.unique(key)
    return (key << np.uint64(32)) | (key >> np.uint64(32))


def match_shard(engine, tables, data, num_seg, seg_len, rank, world, **kw):
    """Matches this rank's block of a stream of num_seg segments and returns
    its reports with stream offsets."""
    first, count = rank_segments(num_seg, rank, world)
    if count == 0:
        return np.zeros(0, np.uint64)
    block = data[first * seg_len:(first + count) * seg_len]
    rep = engine.match(tables, block, count, seg_len, first_segment=first, **kw)
    return shift_offsets(rep, first * seg_len)
