"""Runs the CPU oracle on the engine's input descriptors (test infrastructure)."""
from __future__ import annotations

import numpy as np

from jxr_b200 import COLOR
from jxr_b200.api import Arena, Geometry, OutputFormat, SynthImage
from tests import _oracle as O


def oracle_planes(arena: Arena, geom: Geometry, alpha_arena=None):
    planes = []
    ncomp = 1 if geom.color_format == COLOR["LUMA"] else (4 if geom.color_format == COLOR["YUVK"] else
                                                         (geom.components if geom.color_format == COLOR["NCOMPONENT"] else 3))
    origin = (geom.macroblock_origin_x, geom.macroblock_origin_y)
    cols, rows = geom.column_boundaries(), geom.row_boundaries()
    for c in range(ncomp):
        mb = arena.plane_macroblocks(c, geom.macroblocks_x, geom.macroblocks_y, origin)
        planes.append(dict(coefficients=arena.coefficients, macroblocks_x=geom.macroblocks_x,
                           macroblocks_y=geom.macroblocks_y, scale_after_first_transform=int(geom.scaled and c != 0),
                           overlap=geom.overlap, hard_tiles=geom.hard_tiles, column_boundaries=cols,
                           row_boundaries=rows, **mb))
    alpha = None
    if geom.alpha_mode:
        src, idx = (arena, ncomp) if geom.alpha_mode == 1 else (alpha_arena, 0)
        mb = src.plane_macroblocks(idx, geom.macroblocks_x, geom.macroblocks_y, origin)
        alpha = dict(coefficients=src.coefficients, macroblocks_x=geom.macroblocks_x,
                     macroblocks_y=geom.macroblocks_y, scale_after_first_transform=0, overlap=geom.alpha_overlap,
                     hard_tiles=geom.hard_tiles, column_boundaries=cols, row_boundaries=rows, **mb)
    return planes, alpha


def oracle_output(geom: Geometry, out: OutputFormat) -> O.JoOutput:
    internal = geom.color_format
    if internal in (COLOR["YUV420"], COLOR["YUV422"]) and out.output_color != internal:
        internal = COLOR["YUV444"]
    return O.make_output(
        internal_color=internal, output_color=out.output_color, depth=out.bit_depth, shift_bits=out.shift_bits,
        mantissa_length=out.mantissa_length, exponent_bias=out.exponent_bias, storage=out.storage,
        layout=out.layout, ncomponents=geom.components, scaled=geom.scaled, alpha_depth=out.alpha_bit_depth,
        alpha_shift_bits=out.alpha_shift_bits, alpha_mantissa_length=out.alpha_mantissa_length,
        alpha_exponent_bias=out.alpha_exponent_bias, alpha_scaled=geom.alpha_scaled,
        red_blue_not_swapped=out.red_blue_not_swapped, premultiply=out.premultiply_alpha, crop_x=out.crop_x,
        crop_y=out.crop_y, crop_width=out.crop_width, crop_height=out.crop_height, nchw=out.nchw,
        widen_f16=out.widen_f16)


def oracle_decode(arena: Arena, geom: Geometry, out: OutputFormat, alpha_arena=None, threads: int = 1,
                  denominator: int = 1):
    """(status, output bytes) of the oracle for the engine's inputs, at
    1/denominator resolution (the crop then in reduced coordinates)."""
    planes, alpha = oracle_planes(arena, geom, alpha_arena)
    return O.decode_image(planes, alpha, geom.color_format, (geom.chroma_centering_x, geom.chroma_centering_y),
                          oracle_output(geom, out), threads, denominator)


def decode_synth(img: SynthImage, out: OutputFormat, threads: int = 1, denominator: int = 1):
    return oracle_decode(img.arena, img.geometry, out, img.alpha_arena, threads, denominator)
