"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No codestreams or corpora exist in this environment, so each workload is a set
of coefficient arenas produced by the forward analysis (`jxr_b200.synth`) from
seeded content, with the configuration's sizes, colour formats, quality,
overlap and tiling.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import List

import numpy as np

from . import api as J


@dataclass
class BatchItem:
    kind: str              # "rgb420", "gray16", "rgba"
    image: J.SynthImage
    output: J.OutputFormat

    @property
    def pixels(self) -> int:
        return self.output.crop_width * self.output.crop_height


def log_uniform_size(rng, lo: int, hi: int, multiple: int = 16) -> int:
    v = math.exp(rng.uniform(math.log(lo), math.log(hi)))
    return int(min(hi, max(lo, round(v / multiple) * multiple)))


def mixed_item(rng, lo: int, hi: int, seed: int, threads: int) -> BatchItem:
    """One image of the mixed batch: 50 % RGB8 4:2:0 q75 one-level overlap,
    30 % 16-bit grayscale lossless without overlap, 20 % RGBA8 q85 two-level
    overlap with integrated alpha; tiles 128..512 samples."""
    C_, D, S, L, A = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT, J.ALPHA
    w, h = log_uniform_size(rng, lo, hi), log_uniform_size(rng, lo, hi)
    tw, th = (int(rng.integers(8, 33)) for _ in range(2))   # tile size in macroblocks (128..512 samples)
    r = rng.random()
    if r < 0.5:
        img = J.synth(w, h, color_format=C_["YUV420"], quality=75, overlap=1, tile_width=tw, tile_height=th,
                      seed=seed, threads=threads)
        return BatchItem("rgb420", img, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], w, h))
    if r < 0.8:
        img = J.synth(w, h, content=J.CONTENT["GRAY16"], color_format=C_["LUMA"], quality=100, scaled=0,
                      overlap=0, tile_width=tw, tile_height=th, seed=seed, threads=threads)
        return BatchItem("gray16", img, J.OutputFormat(C_["LUMA"], D["U16"], S["U16"], L["LUMA"], w, h))
    img = J.synth(w, h, alpha_mode=A["INTEGRATED"], quality=85, overlap=2, alpha_overlap=2, alpha_qp=(8, 8, 8),
                  tile_width=tw, tile_height=th, seed=seed, threads=threads)
    return BatchItem("rgba", img, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGBA"], w, h,
                                                 alpha_bit_depth=D["U8"]))


def mixed_batch(count: int = 256, seed: int = 4, lo: int = 64, hi: int = 2048,
                threads: int | None = None) -> List[BatchItem]:
    """The 256-image mixed batch: sizes log-uniform in [64, 2048], multiples of 16."""
    threads = threads or os.cpu_count() or 8
    rng = np.random.default_rng(seed)
    return [mixed_item(rng, lo, hi, seed * 100003 + i, threads) for i in range(count)]


def plans_of(items: List[BatchItem]) -> List[J.CudaDecodePlan]:
    return [J.CudaDecodePlan(it.image.arena, it.image.geometry, it.output, it.image.alpha_arena) for it in items]


def single_image(name: str, seed_offset: int = 0, threads: int | None = None):
    """The single-image configurations as (image, output format):
    c2: 4096x4096 8-bit RGB, quality 90, two-level overlap, 256x256 soft
        tiles, to U8 RGB;
    c3: 8192x8192 half-float RGB (QP 4/8/16) with a separate 8-bit alpha plane
        coded losslessly, two-level overlap, 512x512 tiles, to F32 RGBA NCHW;
    c3_4096: the same at 4096x4096 (a small case for profiling captures).
    `seed_offset` shifts the seed (one image per replica)."""
    threads = threads or os.cpu_count() or 8
    C_, D, S, L, A = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT, J.ALPHA
    if name == "c2":
        img = J.synth(4096, 4096, quality=90, overlap=2, tile_width=16, tile_height=16, hard_tiles=0,
                      seed=2 + seed_offset, threads=threads)
        return img, J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 4096, 4096)
    if name in ("c3", "c3_4096"):
        side = 8192 if name == "c3" else 4096
        img = J.synth(side, side, content=J.CONTENT["HDR_HALF"], alpha_mode=A["SEPARATE"], scaled=0, quality=0,
                      qp=(4, 8, 16), overlap=2, alpha_overlap=0, tile_width=32, tile_height=32, hard_tiles=0,
                      seed=3 + seed_offset, threads=threads)
        return img, J.OutputFormat(C_["RGB"], D["F16"], S["F16"], L["RGBA"], side, side, alpha_bit_depth=D["F16"],
                                   nchw=1, widen_f16=1)
    raise ValueError(f"unknown single-image workload {name}")


def export(items, path: str) -> None:
    """Write a workload's (image, output) pairs to `path` (a pickle of the
    arenas, geometries and output formats; the generated source pixels are
    dropped).  A process that only reads them never maps the generator."""
    import dataclasses
    import pickle
    slim = [(dataclasses.replace(img, source=np.zeros(0, np.uint8)), out) for img, out in items]
    with open(path, "wb") as f:
        pickle.dump(slim, f, protocol=pickle.HIGHEST_PROTOCOL)


def load(path: str):
    import pickle
    with open(path, "rb") as f:
        return pickle.load(f)
