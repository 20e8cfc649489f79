"""Autotuner for the batched engine.

The reference tunes by brute force over fetch size, active threshold and AAS
interval, rerunning the whole input for each point (code/src/ngap/ngap.cu:
1995-2056). Here the knobs are the engine's own: worklist window, chunk
length of acyclic tiles, algorithm variant (with or without
privatization) and CUDA-graph replay of the whole step by default; queue capacity (`queue_capacity` in the grid: a
candidate whose overflow stacks run out on the sample is skipped) and the
tile partition (`tile_grid`: table options per candidate, one tableset built
for each) on request. Each candidate runs on a sample of the streams (a few
percent of the bytes, whole streams so that per-stream costs are
represented) and the fastest one is kept; results do not depend on the
choice.
"""
import itertools

import numpy as np

from .engine import NgapError, batch_match_async

DEFAULT_GRID = {
    "window": [512, 1024, 2048],
    "chunk": [0, 4096, 16384],
    "algorithm": ["nonblockingpcgroups", "nonblockingallgroups"],
    "use_graph": [False, True],
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


def _run_on_device(engine, tableset, buf, offs, lens, nf, stream, params):
    """One batched launch of the sample: device milliseconds (match + sort)."""
    batch_match_async(engine, tableset, buf, offs, lens, nf, stream=stream, **params)
    engine.sync()
    ms = engine.times_ms()
    return ms[0] + ms[1]


def tableset_for(groups, device=0, **table_opts):
    """A tableset of the given NFAs' groups built with one set of table options
    (automatic prefix depth unless precompute_depth is given)."""
    from .engine import Tables, TableSet
    table_opts.setdefault("precompute_depth", -1)
    return TableSet([Tables(g, device=device, **table_opts) for g in groups])


def autotune(engine, tableset, data, offsets, lengths, nfa_of, grid=None, frac=0.05, reps=2,
             stream=None, groups=None, tile_grid=None, run=None, make_tableset=None):
    """Returns (best_params, table of (params, ms)) for batched matching; ms is
    None for a candidate that overflowed its queue. With tile_grid (a list of
    Tables option dicts, e.g. {"tile_mode": "global"}) and groups, every
    candidate is also tried on a tableset built with each option, and
    best_params["tiles"] names the winning option (build it with
    tableset_for). run and make_tableset replace the device launch and the
    tableset builder (tests)."""
    if tile_grid and groups is None and make_tableset is None:
        raise ValueError("tile_grid needs the NFAs' groups")
    grid = grid or DEFAULT_GRID
    run = run or _run_on_device
    make_tableset = make_tableset or (lambda opts: tableset_for(groups, **opts))
    idx = sample_streams(lengths, frac)
    # compact the sample into its own buffer
    lens = np.asarray(lengths)[idx]
    offs = np.zeros(len(idx), dtype=np.int64)
    offs[1:] = np.cumsum(lens)[:-1]
    buf = np.concatenate([data[offsets[i]:offsets[i] + lengths[i]] for i in idx]) \
        if len(idx) else np.zeros(0, np.uint8)
    nf = np.asarray(nfa_of)[idx]
    if run is _run_on_device:  # the sample on the device: a captured graph replays its copy
        import torch
        buf = torch.from_numpy(buf).to(f"cuda:{engine.device}")
    tilesets = [(None, tableset)]
    if tile_grid:
        tilesets = [(dict(opts), make_tableset(dict(opts))) for opts in tile_grid]
    keys = list(grid)
    results = []
    for tiles, ts in tilesets:
        for combo in itertools.product(*[grid[k] for k in keys]):
            params = dict(zip(keys, combo))
            best = None
            try:
                for r in range(reps + 1):
                    dev = run(engine, ts, buf, offs, lens, nf, stream, params)
                    if r > 0:  # the first run warms the plan and buffers
                        best = dev if best is None else min(best, dev)
            except NgapError as ex:
                if ex.status != 6:  # only a queue that ran out disqualifies a candidate
                    raise
                best = None
            if tiles is not None:
                params = dict(params, tiles=tiles)
            results.append((params, best))
    timed = [r for r in results if r[1] is not None]
    if not timed:
        raise NgapError(6, "every candidate overflowed its queue on the sample")
    timed.sort(key=lambda x: x[1])
    return timed[0][0], results
