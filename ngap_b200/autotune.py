"""Autotuner for the batched engine.

The reference tunes by brute force over fetch size, active threshold and AAS
interval, rerunning the whole input for each point (code/src/ngap/ngap.cu:
1995-2056). Here the knobs are the engine's own: worklist window, chunk
length of acyclic tiles, algorithm variant (with or without privatization)
and whether --unique is worth it. Each candidate runs on a sample of the
streams (a few percent of the bytes, whole streams so that per-stream costs
are represented) and the fastest one is kept; results do not depend on the
choice.
"""
import itertools

import numpy as np

from .engine import batch_match_async

DEFAULT_GRID = {
    "window": [512, 1024, 2048],
    "chunk": [0, 4096, 16384],
    "algorithm": ["nonblockingpcgroups", "nonblockingallgroups"],
}


def sample_streams(lengths, frac=0.05, seed=0, min_streams=32):
    """Sorted indices of a random sample of whole streams: streams in a seeded
    random order until they hold `frac` of the bytes and number at least
    min_streams (or all of them)."""
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(lengths))
    total, budget, pick = 0, max(1, int(frac * int(np.sum(lengths)))), []
    for i in order:
        pick.append(int(i))
        total += int(lengths[i])
        if total >= budget and len(pick) >= min(min_streams, len(lengths)):
            break
    return np.array(sorted(pick), dtype=np.int64)


def autotune(engine, tableset, data, offsets, lengths, nfa_of, grid=None, frac=0.05, reps=2,
             stream=None):
    """Returns (best_params, table of (params, ms)) for batched matching."""
    grid = grid or DEFAULT_GRID
    idx = sample_streams(lengths, frac)
    # compact the sample into its own buffer
    lens = lengths[idx]
    offs = np.zeros(len(idx), dtype=np.int64)
    offs[1:] = np.cumsum(lens)[:-1]
    buf = np.concatenate([data[offsets[i]:offsets[i] + lengths[i]] for i in idx]) \
        if len(idx) else np.zeros(0, np.uint8)
    nf = nfa_of[idx]
    keys = list(grid)
    results = []
    for combo in itertools.product(*[grid[k] for k in keys]):
        params = dict(zip(keys, combo))
        best = None
        for r in range(reps + 1):
            batch_match_async(engine, tableset, buf, offs, lens, nf, stream=stream, **params)
            engine.sync()
            ms = engine.times_ms()
            dev = ms[0] + ms[1]
            if r > 0:  # first run warms the plan and buffers
                best = dev if best is None else min(best, dev)
        results.append((params, best))
    results.sort(key=lambda x: x[1])
    return results[0][0], results
