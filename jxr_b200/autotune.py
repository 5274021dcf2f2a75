"""Launch-shape autotuner for resident sets.

The tile kernels are persistent: each launch starts (SMs x CTAs per SM) CTAs
that claim tiles from the work list until it is empty.  How many CTAs per SM
pay off depends on the mix of tiles (interior tiles with 1..4 planes, edge
tiles, subsampled chroma), and so does whether the edge-tile kernel should
run on a second stream beside the interior kernels.  The autotuner times
every candidate shape on the resident set itself with CUDA events, keeps the
fastest, and caches the choice by device and by a signature of the set's
plans (`JXRB_TUNING_CACHE`, default ~/.cache/jxr_b200/tuning.json).
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os
from pathlib import Path
from typing import Dict, List, Optional, Sequence, Tuple

INTERIOR_CTAS = (1, 2, 3)   # the interior kernels fit 3 CTAs an SM
OTHER_CTAS = (1, 2)         # the general kernel fits 2


def candidates() -> List[Tuple[Tuple[int, ...], bool]]:
    out = []
    for inner, other, side in itertools.product(INTERIOR_CTAS, OTHER_CTAS, (True, False)):
        out.append(((inner, inner, inner, inner, other), side))
    return out


def signature(plans: Sequence) -> str:
    h = hashlib.sha256()
    for p in plans:
        g, o = p.geometry, p.output
        h.update(repr((g.macroblocks_x, g.macroblocks_y, g.color_format, g.overlap, g.alpha_mode, g.hard_tiles,
                       len(g.tile_column_widths or ()), len(g.tile_row_heights or ()), o.storage, o.layout,
                       o.nchw, o.crop_width, o.crop_height)).encode())
    return h.hexdigest()[:24]


def _cache_path() -> Path:
    return Path(os.environ.get("JXRB_TUNING_CACHE", Path.home() / ".cache" / "jxr_b200" / "tuning.json"))


def _load() -> Dict:
    try:
        return json.loads(_cache_path().read_text())
    except (OSError, ValueError):
        return {}


def _store(cache: Dict) -> None:
    path = _cache_path()
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(cache, indent=1, sort_keys=True))
    except OSError:
        pass


def time_shape(res, device_ptr: int, nbytes: int, stream, batched: bool, reps: int) -> float:
    """Median milliseconds of one run of the resident set under its current shape."""
    import torch
    times = []
    res.run(device_ptr, nbytes, batched, stream.cuda_stream)
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        res.run(device_ptr, nbytes, batched, stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    times.sort()
    return times[len(times) // 2]


def tune(res, plans: Sequence, device_ptr: int, nbytes: int, stream, batched: bool = True, reps: int = 7,
         use_cache: bool = True) -> Dict:
    """Choose and apply the fastest launch shape for `res`; returns the choice
    (`blocks_per_sm`, `side_stream`, `ms`, `source`)."""
    import torch
    key = f"{torch.cuda.get_device_name(stream.device)}|{signature(plans)}|{int(batched)}"
    cache = _load() if use_cache else {}
    hit: Optional[Dict] = cache.get(key)
    if hit:
        res.set_tuning(hit["blocks_per_sm"], hit["side_stream"])
        return dict(hit, source="cache")
    best = None
    trials = []
    for blocks, side in candidates():
        res.set_tuning(blocks, side)
        ms = time_shape(res, device_ptr, nbytes, stream, batched, reps)
        trials.append((ms, blocks, side))
        if best is None or ms < best[0]:
            best = (ms, blocks, side)
    ms, blocks, side = best
    res.set_tuning(blocks, side)
    choice = {"blocks_per_sm": list(blocks), "side_stream": bool(side), "ms": round(ms, 4),
              "candidates": len(trials)}
    if use_cache:
        cache[key] = choice
        _store(cache)
    return dict(choice, source="measured")
