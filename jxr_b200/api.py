"""Python host mirror of the reference's CUDA reconstruction API over the C ABI.

Names and argument meaning follow `jxr_cuda` (crates/jxr-cuda/src/lib.rs:26-39):
`CudaDecoderSession`, `CudaDecodePlan`, `CudaSubmission`, `CudaError`.  The
engine itself is libjxr_b200.so (include/jxr_b200.h); this module only binds it.
There is no CPU fallback: without the library or a B200 every call raises.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, Optional, Sequence

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libjxr_b200.so"
SYNTH_LIB_PATH = PKG / "libjxr_synth.so"

# jxrb_status (crates/jxr-cuda/src/error.rs:8-92)
STATUS_NAMES = {
    0: "Ok", 1: "Unavailable", 2: "UnsupportedDevice", 3: "UnsupportedBackend", 4: "InvalidPlan",
    5: "InvalidDestination", 6: "UnsupportedOutputFormat", 7: "RuntimeInitialization",
    8: "KernelArithmetic", 9: "InvalidSubmissionState", 10: "ResourceLimit", 11: "StateInvariant",
    12: "Driver", 13: "Timeout", 14: "ResidentOutputRequiresCuda",
}

COLOR = dict(LUMA=0, YUV420=1, YUV422=2, YUV444=3, RGB=4, CMYK=5, CMYK_DIRECT=6, YUVK=7, RGBE=8, NCOMPONENT=9)
DEPTH = dict(BIT1_WHITE=0, BIT1_BLACK=1, U8=2, U10=3, U16=4, I16=5, F16=6, I32=7, F32=8, RGB555=9,
             RGB101010=10, RGB565=11)
STORE = dict(BITS=0, U8=1, U16=2, I16=3, I32=4, F16=5, F32=6, RGB555=7, RGB565=8, RGB101010=9, RGBE=10)
LAYOUT = dict(LUMA=0, LUMA_ALPHA=1, YUV=2, YUVA=3, RGB=4, RGBX=5, RGBA=6, BGR=7, BGRX=8, BGRA=9, CMYK=10,
              CMYKA=11, NCOMPONENT=12, NCOMPONENT_ALPHA=13)
ALPHA = dict(NONE=0, INTEGRATED=1, SEPARATE=2)
CONTENT = dict(PHOTO_RGB8=0, HDR_HALF=1, GRAY16=2, RANDOM=3)


class CudaError(RuntimeError):
    """A failed engine call: `kind` is the reference's CudaError variant name."""

    def __init__(self, status: int, message: str, stage: int = 0):
        self.status = status
        self.kind = STATUS_NAMES.get(status, f"Status{status}")
        self.stage = stage
        super().__init__(f"{self.kind}: {message}" + (f" (stage {stage})" if stage else ""))


class LaunchTuningC(C.Structure):
    _fields_ = [("blocks_per_sm", C.c_uint32 * 5), ("side_stream", C.c_int32)]


class TileKindsC(C.Structure):
    _fields_ = [("interior", C.c_uint32), ("interior_420", C.c_uint32), ("edge", C.c_uint32),
                ("edge_420", C.c_uint32), ("general", C.c_uint32)]


class CoefficientPlane(C.Structure):
    _fields_ = [("coefficient_offset", C.c_uint64), ("coefficient_count", C.c_uint64),
                ("macroblock_offset", C.c_uint64), ("macroblock_count", C.c_uint64),
                ("block_columns", C.c_uint32), ("block_rows", C.c_uint32)]


class ArenaC(C.Structure):
    _fields_ = [("coefficients", C.c_void_p), ("coefficient_count", C.c_uint64),
                ("coefficient_offsets", C.c_void_p), ("quantizers", C.c_void_p), ("bands", C.c_void_p),
                ("hp_predictions", C.c_void_p), ("coded_x", C.c_void_p), ("coded_y", C.c_void_p),
                ("macroblock_count", C.c_uint64), ("planes", C.POINTER(CoefficientPlane)),
                ("plane_count", C.c_uint32)]


class GeometryC(C.Structure):
    _fields_ = [("macroblock_origin_x", C.c_uint32), ("macroblock_origin_y", C.c_uint32),
                ("macroblocks_x", C.c_uint32), ("macroblocks_y", C.c_uint32),
                ("tile_column_widths", C.c_void_p), ("tile_columns", C.c_uint32),
                ("tile_row_heights", C.c_void_p), ("tile_rows", C.c_uint32),
                ("hard_tiles", C.c_int32), ("color_format", C.c_int32), ("components", C.c_int32),
                ("overlap", C.c_int32), ("scaled", C.c_int32), ("alpha_mode", C.c_int32),
                ("alpha_overlap", C.c_int32), ("alpha_scaled", C.c_int32),
                ("chroma_centering_x", C.c_int32), ("chroma_centering_y", C.c_int32)]


class OutputFormatC(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "output_color", "bit_depth", "shift_bits", "mantissa_length", "exponent_bias", "storage", "layout",
        "alpha_bit_depth", "alpha_shift_bits", "alpha_mantissa_length", "alpha_exponent_bias",
        "red_blue_not_swapped", "premultiply_alpha")] + [
        ("crop_x", C.c_uint32), ("crop_y", C.c_uint32), ("crop_width", C.c_uint32), ("crop_height", C.c_uint32),
        ("nchw", C.c_int32), ("widen_f16", C.c_int32)]


class SessionOptionsC(C.Structure):
    _fields_ = [("streams", C.c_uint32), ("scratch_bytes", C.c_uint64)]


class DiagnosticsC(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submissions", "bytes_uploaded", "bytes_read_back",
                                           "device_bytes_held", "kernel_launches", "bytes_staged")]


class SurfacePlaneC(C.Structure):
    _fields_ = [("byte_offset", C.c_uint64), ("row_stride_bytes", C.c_uint64), ("width", C.c_uint32),
                ("height", C.c_uint32), ("channels", C.c_uint32)]


class SurfaceLayoutC(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("byte_len", C.c_uint64),
                ("element_bytes", C.c_uint32), ("plane_count", C.c_uint32), ("planes", SurfacePlaneC * 6)]


class StageReportC(C.Structure):
    _fields_ = [("stage", C.c_int32), ("executor", C.c_int32)]


class DecodeReportC(C.Structure):
    _fields_ = [("requested_backend", C.c_int32), ("selected_backend", C.c_int32), ("fallback", C.c_int32),
                ("stage_count", C.c_uint32), ("stages", StageReportC * 16), ("upload_ms", C.c_float),
                ("reconstruct_ms", C.c_float), ("readback_ms", C.c_float)]


class AnalysisPlaneC(C.Structure):
    _fields_ = [("samples", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32),
                ("block_columns", C.c_uint32), ("block_rows", C.c_uint32), ("scaled", C.c_int32),
                ("overlap", C.c_int32), ("steps", C.c_uint32 * 3), ("column_boundaries", C.c_void_p),
                ("column_count", C.c_uint32), ("row_boundaries", C.c_void_p), ("row_count", C.c_uint32),
                ("hard_tiles", C.c_int32), ("low_scratch", C.c_void_p), ("low_q", C.c_void_p), ("high_q", C.c_void_p)]


class SynthRequestC(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("content", C.c_int32),
                ("color_format", C.c_int32), ("alpha_mode", C.c_int32), ("overlap", C.c_int32),
                ("alpha_overlap", C.c_int32), ("scaled", C.c_int32), ("quality", C.c_int32),
                ("qp", C.c_int32 * 3), ("alpha_qp", C.c_int32 * 3), ("tile_width", C.c_uint32),
                ("tile_height", C.c_uint32), ("hard_tiles", C.c_int32), ("bands", C.c_int32),
                ("seed", C.c_uint64)]


class SynthArenaViewC(C.Structure):
    _fields_ = [("coefficients", C.c_void_p), ("coefficient_count", C.c_uint64),
                ("coefficient_offsets", C.c_void_p), ("quantizers", C.c_void_p), ("coded_x", C.c_void_p),
                ("coded_y", C.c_void_p), ("bands", C.c_void_p), ("hp_predictions", C.c_void_p),
                ("macroblock_count", C.c_uint64), ("plane_words", C.c_void_p), ("plane_count", C.c_uint32)]


# every entry point of include/jxr_b200.h, with its signature
_vp, _u32, _u64, _i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32
EXPORTS = {
    "jxrb_available": (C.c_int, []),
    "jxrb_last_error": (C.c_char_p, []),
    "jxrb_last_stage": (_u32, []),
    "jxrb_session_create": (C.c_int, [C.c_int, C.POINTER(SessionOptionsC), C.POINTER(_vp)]),
    "jxrb_session_destroy": (None, [_vp]),
    "jxrb_session_diagnostics": (C.c_int, [_vp, C.POINTER(DiagnosticsC)]),
    "jxrb_plan_create": (C.c_int, [C.POINTER(ArenaC), C.POINTER(ArenaC), C.POINTER(GeometryC),
                                   C.POINTER(OutputFormatC), C.POINTER(_vp)]),
    "jxrb_plan_destroy": (None, [_vp]),
    "jxrb_plan_output_bytes": (_u64, [_vp]),
    "jxrb_plan_traffic_bytes": (_u64, [_vp]),
    "jxrb_plan_tile_kinds": (C.c_int, [_vp, C.POINTER(TileKindsC)]),
    "jxrb_submit": (C.c_int, [_vp, _vp, C.POINTER(_vp)]),
    "jxrb_submit_into": (C.c_int, [_vp, _vp, _vp, _u64, C.POINTER(_vp)]),
    "jxrb_submit_batch": (C.c_int, [_vp, C.POINTER(_vp), _u32, _vp, _u64, C.POINTER(_vp)]),
    "jxrb_wait": (C.c_int, [_vp, C.c_int64]),
    "jxrb_is_complete": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "jxrb_enqueue_consumer_wait": (C.c_int, [_vp, _vp]),
    "jxrb_submission_device_ptr": (_vp, [_vp, _u32]),
    "jxrb_readback": (C.c_int, [_vp, _u32, _vp, _u64]),
    "jxrb_readback_all": (C.c_int, [_vp, _vp, _u64]),
    "jxrb_submission_destroy": (None, [_vp]),
    "jxrb_decode_to_host": (C.c_int, [_vp, _vp, _vp, _u64]),
    "jxrb_resident_create": (C.c_int, [_vp, C.POINTER(_vp), _u32, C.POINTER(_vp)]),
    "jxrb_resident_run": (C.c_int, [_vp, _vp, _u64, C.c_int, _vp]),
    "jxrb_resident_status": (C.c_int, [_vp, C.POINTER(_u32)]),
    "jxrb_resident_output_bytes": (_u64, [_vp]),
    "jxrb_resident_launches": (_u32, [_vp, C.c_int]),
    "jxrb_resident_destroy": (None, [_vp]),
    "jxrb_decode_static": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp, _u64, _vp]),
    "jxrb_resident_set_tuning": (C.c_int, [_vp, C.POINTER(LaunchTuningC)]),
    "jxrb_resident_capture": (C.c_int, [_vp, _vp, _u64, C.c_int]),
    "jxrb_resident_replay": (C.c_int, [_vp, _vp]),
    "jxrb_image_create": (C.c_int, [_vp, C.POINTER(ArenaC), C.POINTER(ArenaC), C.POINTER(GeometryC), C.POINTER(_vp)]),
    "jxrb_image_device_bytes": (_u64, [_vp]),
    "jxrb_image_destroy": (None, [_vp]),
    "jxrb_request_create": (C.c_int, [_vp, C.POINTER(OutputFormatC), C.POINTER(_vp)]),
    "jxrb_request_create_scaled": (C.c_int, [_vp, C.POINTER(OutputFormatC), C.c_int, C.POINTER(_vp)]),
    "jxrb_request_destroy": (None, [_vp]),
    "jxrb_request_output_bytes": (_u64, [_vp]),
    "jxrb_request_traffic_bytes": (_u64, [_vp]),
    "jxrb_request_window": (C.c_int, [_vp, C.POINTER(_u32)]),
    "jxrb_submit_requests": (C.c_int, [_vp, C.POINTER(_vp), _u32, _vp, _u64, C.POINTER(_vp)]),
    "jxrb_oriented_bytes": (_u64, [_u32, _u32, _u32, C.c_int]),
    "jxrb_plan_route": (C.c_int, [C.c_int, _u64, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "jxrb_session_create_default": (C.c_int, [C.POINTER(_vp)]),
    "jxrb_plan_reconstructed_coefficients": (_u64, [_vp]),
    "jxrb_plan_output_layout": (C.c_int, [_vp, C.POINTER(SurfaceLayoutC)]),
    "jxrb_decode_batch_to_host": (C.c_int, [_vp, C.POINTER(_vp), _u32, C.POINTER(_vp), C.POINTER(_u64)]),
    "jxrb_allocate_destination": (C.c_int, [_vp, _u64, C.POINTER(_vp)]),
    "jxrb_batch_layout": (C.c_int, [C.POINTER(_vp), _u32, C.POINTER(_u64), C.POINTER(_u64)]),
    "jxrb_allocate_batch_destination": (C.c_int, [_vp, C.POINTER(_vp), _u32, C.POINTER(_vp), C.POINTER(_u64)]),
    "jxrb_free_destination": (C.c_int, [_vp, _vp]),
    "jxrb_submission_report": (C.c_int, [_vp, C.POINTER(DecodeReportC)]),
    "jxrb_analyze_planes": (C.c_int, [C.POINTER(AnalysisPlaneC), _u32, _vp]),
    "jxrb_orient": (C.c_int, [_vp, _vp, _u32, _u32, _u32, C.c_int, _vp]),
}

# the generator's entry points (csrc/synth.h), in libjxr_synth.so
SYNTH_EXPORTS = {
    "jxrb_synth_create": (C.c_int, [C.POINTER(SynthRequestC), C.c_int, C.POINTER(_vp)]),
    "jxrb_synth_destroy": (None, [_vp]),
    "jxrb_synth_arena": (C.c_int, [_vp, C.c_int, C.POINTER(SynthArenaViewC)]),
    "jxrb_synth_geometry": (C.c_int, [_vp, C.POINTER(_u32), C.POINTER(_u32), C.POINTER(_vp), C.POINTER(_u32),
                                      C.POINTER(_vp), C.POINTER(_u32)]),
    "jxrb_synth_source": (_vp, [_vp, C.POINTER(_u32), C.POINTER(_u32)]),
    "jxrb_forward_core_transform": (C.c_int, [_vp]),
    "jxrb_forward_overlap_4x4": (C.c_int, [_vp]),
    "jxrb_forward_overlap_4": (C.c_int, [_vp]),
    "jxrb_forward_overlap_2x2": (C.c_int, [_vp]),
    "jxrb_forward_overlap_2": (C.c_int, [_vp]),
    "jxrb_forward_chroma_420": (C.c_int, [_vp]),
    "jxrb_forward_chroma_422": (C.c_int, [_vp]),
    "jxrb_quant_step": (_u32, [_i32, _i32, _i32, _i32]),
    "jxrb_analyze_plane_cpu": (C.c_int, [_vp, _u32, _u32, _u32, _u32, _i32, _i32, _vp, _vp, _u32, _vp, _u32, _i32,
                                         _vp, _vp]),
}

_lib: Optional[C.CDLL] = None
_synth_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """The engine library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise CudaError(1, f"engine library {LIB_PATH.name} is not built (python -m jxr_b200.build)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in EXPORTS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def synth_lib() -> C.CDLL:
    """The synthetic-input generator (host code only, no engine); raises when
    it has not been built."""
    global _synth_lib
    if _synth_lib is None:
        if not SYNTH_LIB_PATH.exists():
            raise CudaError(1, f"generator library {SYNTH_LIB_PATH.name} is not built (python -m jxr_b200.build)")
        L = C.CDLL(str(SYNTH_LIB_PATH))
        for name, (res, args) in SYNTH_EXPORTS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _synth_lib = L
    return _synth_lib


def _check_synth(status: int, what: str) -> None:
    if status != 0:
        raise CudaError(status, f"synthetic input generator: {what} failed")


def _check(status: int) -> None:
    if status != 0:
        L = lib()
        raise CudaError(status, (L.jxrb_last_error() or b"").decode(), int(L.jxrb_last_stage()) if status == 8 else 0)


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------
@dataclass
class Arena:
    """CoefficientArena (crates/jxr-core/src/plan.rs:62-142) as numpy arrays.

    planes: rows of (coefficient_offset, coefficient_count, macroblock_offset,
    macroblock_count, block_columns, block_rows)."""
    coefficients: np.ndarray
    coefficient_offsets: np.ndarray
    quantizers: np.ndarray      # (n, 3) uint32
    bands: np.ndarray
    hp_predictions: np.ndarray
    coded_x: np.ndarray
    coded_y: np.ndarray
    planes: np.ndarray          # (p, 6) uint64

    def __post_init__(self):
        self.coefficients = np.ascontiguousarray(self.coefficients, np.int32)
        self.coefficient_offsets = np.ascontiguousarray(self.coefficient_offsets, np.uint32)
        self.quantizers = np.ascontiguousarray(self.quantizers, np.uint32).reshape(-1, 3)
        self.bands = np.ascontiguousarray(self.bands, np.uint8)
        self.hp_predictions = np.ascontiguousarray(self.hp_predictions, np.uint8)
        self.coded_x = np.ascontiguousarray(self.coded_x, np.uint32)
        self.coded_y = np.ascontiguousarray(self.coded_y, np.uint32)
        self.planes = np.ascontiguousarray(self.planes, np.uint64).reshape(-1, 6)

    def to_c(self, coefficients: Optional[np.ndarray] = None):
        planes = (CoefficientPlane * len(self.planes))(*[CoefficientPlane(*map(int, p)) for p in self.planes])
        co = self.coefficients if coefficients is None else coefficients
        c = ArenaC(_ptr(co), co.size, _ptr(self.coefficient_offsets), _ptr(self.quantizers), _ptr(self.bands),
                   _ptr(self.hp_predictions), _ptr(self.coded_x), _ptr(self.coded_y), self.coefficient_offsets.size,
                   planes, len(self.planes))
        return c, planes

    def plane_macroblocks(self, index: int, mbs_x: int, mbs_y: int, origin=(0, 0)):
        """Per-plane metadata in raster order over the window (the oracle's input)."""
        off, cnt, mb0, mbn, bc, br = map(int, self.planes[index])
        sl = slice(mb0, mb0 + mbn)
        x = self.coded_x[sl].astype(np.int64) - origin[0]
        y = self.coded_y[sl].astype(np.int64) - origin[1]
        keep = (x >= 0) & (y >= 0) & (x < mbs_x) & (y < mbs_y)
        order = np.full(mbs_x * mbs_y, -1, np.int64)
        order[(y[keep] * mbs_x + x[keep])] = np.nonzero(keep)[0] + mb0
        assert (order >= 0).all(), "window position without a macroblock"
        return dict(offsets=self.coefficient_offsets[order], quantizers=self.quantizers[order].reshape(-1),
                    bands=self.bands[order], hp_prediction=self.hp_predictions[order], block_columns=bc,
                    block_rows=br)


@dataclass
class Geometry:
    """ImageInfo / PreparedPlan fields of the path (jxrb_image_geometry)."""
    macroblocks_x: int
    macroblocks_y: int
    color_format: int = COLOR["YUV444"]
    components: int = 3
    overlap: int = 1
    scaled: int = 1
    tile_column_widths: Sequence[int] = ()
    tile_row_heights: Sequence[int] = ()
    hard_tiles: int = 0
    alpha_mode: int = 0
    alpha_overlap: int = 0
    alpha_scaled: int = 0
    chroma_centering_x: int = 0
    chroma_centering_y: int = 0
    macroblock_origin_x: int = 0
    macroblock_origin_y: int = 0

    def to_c(self):
        tw = np.asarray(self.tile_column_widths or [self.macroblocks_x], np.uint32)
        th = np.asarray(self.tile_row_heights or [self.macroblocks_y], np.uint32)
        g = GeometryC(self.macroblock_origin_x, self.macroblock_origin_y, self.macroblocks_x, self.macroblocks_y,
                      _ptr(tw), tw.size, _ptr(th), th.size, self.hard_tiles, self.color_format, self.components,
                      self.overlap, self.scaled, self.alpha_mode, self.alpha_overlap, self.alpha_scaled,
                      self.chroma_centering_x, self.chroma_centering_y)
        return g, (tw, th)

    def column_boundaries(self):
        return _window_boundaries(self.tile_column_widths or [self.macroblock_origin_x + self.macroblocks_x],
                                  self.macroblock_origin_x, self.macroblocks_x)

    def row_boundaries(self):
        return _window_boundaries(self.tile_row_heights or [self.macroblock_origin_y + self.macroblocks_y],
                                  self.macroblock_origin_y, self.macroblocks_y)


def _window_boundaries(sizes, origin, extent):
    out, pos = [0], 0
    for s in sizes:
        pos += int(s)
        if origin < pos < origin + extent:
            out.append(pos - origin)
    out.append(extent)
    return out


@dataclass
class OutputFormat:
    """OutputFormatRequest (crates/jxr-core/src/output_policy.rs) + extensions."""
    output_color: int
    bit_depth: int
    storage: int
    layout: int
    crop_width: int
    crop_height: int
    crop_x: int = 0
    crop_y: int = 0
    shift_bits: int = 0
    mantissa_length: int = 0
    exponent_bias: int = 0
    alpha_bit_depth: int = 0
    alpha_shift_bits: int = 0
    alpha_mantissa_length: int = 0
    alpha_exponent_bias: int = 0
    red_blue_not_swapped: int = 0
    premultiply_alpha: int = 0
    nchw: int = 0
    widen_f16: int = 0

    def to_c(self):
        return OutputFormatC(self.output_color, self.bit_depth, self.shift_bits, self.mantissa_length,
                             self.exponent_bias, self.storage, self.layout, self.alpha_bit_depth,
                             self.alpha_shift_bits, self.alpha_mantissa_length, self.alpha_exponent_bias,
                             self.red_blue_not_swapped, self.premultiply_alpha, self.crop_x, self.crop_y,
                             self.crop_width, self.crop_height, self.nchw, self.widen_f16)


# ---------------------------------------------------------------------------
# plans, sessions, submissions
# ---------------------------------------------------------------------------
class CudaDecodePlan:
    """CudaDecodePlan::from_prepared (crates/jxr-cuda/src/plan.rs:91-148).

    Keeps the arenas alive: their coefficients are read at submission."""

    def __init__(self, arena: Arena, geometry: Geometry, output: OutputFormat, alpha_arena: Optional[Arena] = None):
        self.arena, self.alpha_arena, self.geometry, self.output = arena, alpha_arena, geometry, output
        self._handle = C.c_void_p()
        a, ap = arena.to_c()
        b, bp = alpha_arena.to_c() if alpha_arena is not None else (None, None)
        g, keep = geometry.to_c()
        o = output.to_c()
        _check(lib().jxrb_plan_create(C.byref(a), C.byref(b) if b is not None else None, C.byref(g), C.byref(o),
                                      C.byref(self._handle)))
        self._keep = (ap, bp, keep)

    @property
    def handle(self):
        return self._handle

    def output_bytes(self) -> int:
        return int(lib().jxrb_plan_output_bytes(self._handle))

    def traffic_bytes(self) -> int:
        return int(lib().jxrb_plan_traffic_bytes(self._handle))

    def reconstructed_coefficients(self) -> int:
        return int(lib().jxrb_plan_reconstructed_coefficients(self._handle))

    def output_layout(self) -> dict:
        """SurfaceLayout of the output (crates/jxr-core/src/surface.rs)."""
        l = SurfaceLayoutC()
        _check(lib().jxrb_plan_output_layout(self._handle, C.byref(l)))
        return {"width": l.width, "height": l.height, "byte_len": int(l.byte_len), "element_bytes": l.element_bytes,
                "planes": [dict(byte_offset=int(p.byte_offset), row_stride_bytes=int(p.row_stride_bytes),
                                width=p.width, height=p.height, channels=p.channels)
                           for p in l.planes[:l.plane_count]]}

    def tile_kinds(self) -> Dict[str, int]:
        """How the plan's tiles split between the tile kernels (interior,
        interior_420, edge, edge_420, general)."""
        k = TileKindsC()
        _check(lib().jxrb_plan_tile_kinds(self._handle, C.byref(k)))
        return {name: int(getattr(k, name)) for name, _ in TileKindsC._fields_}

    def close(self):
        if self._handle:
            lib().jxrb_plan_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceDestination:
    """A caller-owned device output (CudaDestination, crates/jxr-cuda/src/destination.rs)."""

    def __init__(self, session, ptr: int, nbytes: int):
        self.session, self.ptr, self.nbytes = session, ptr, nbytes

    def free(self):
        if self.ptr:
            _check(lib().jxrb_free_destination(self.session._handle, self.ptr))
            self.ptr = 0


def batch_layout(plans: Sequence["CudaDecodePlan"]):
    """(offsets, total bytes) of the dense batch layout of `plans`."""
    arr = (C.c_void_p * len(plans))(*[p.handle.value for p in plans])
    offs = (C.c_uint64 * len(plans))()
    n = C.c_uint64()
    _check(lib().jxrb_batch_layout(arr, len(plans), offs, C.byref(n)))
    return list(offs), int(n.value)


BACKEND = {"AUTO": 0, "CPU": 1, "CUDA": 2, "METAL": 3}
ROUTE = {0: "Cpu", 1: "Cuda"}
STAGES = ["Parse", "EntropyDecode", "InverseScan", "CoefficientRemap", "DcLowPassPrediction",
          "DequantizeAndFirstInverseTransform", "FirstOverlap", "HighPassPrediction", "SecondInverseTransform",
          "SecondOverlap", "ChromaReconstruction", "ColorAndAlphaConversion", "CropClipAndPack", "HostReadback"]
EXECUTORS = ["CpuScalar", "CpuSimd", "Metal", "Cuda"]


def plan_cuda_route(request: int, reconstructed_coefficients: int, cuda_usable: bool, resident_output: bool) -> str:
    """plan_cuda_route (crates/jxr-cuda/src/route.rs:23-49): "Cpu" or "Cuda",
    or a CudaError."""
    d = C.c_int(-1)
    _check(lib().jxrb_plan_route(request, reconstructed_coefficients, int(cuda_usable), int(resident_output),
                                 C.byref(d)))
    return ROUTE[d.value]


class CudaSubmission:
    """CudaSubmission (crates/jxr-cuda/src/submission.rs:31-337)."""

    def __init__(self, handle: C.c_void_p, count: int, plans):
        self._handle, self.count, self._plans = handle, count, plans

    def wait(self, timeout_ns: int = -1) -> None:
        _check(lib().jxrb_wait(self._handle, timeout_ns))

    def is_complete(self) -> bool:
        done = C.c_int()
        _check(lib().jxrb_is_complete(self._handle, C.byref(done)))
        return bool(done.value)

    def device_ptr(self, index: int = 0) -> int:
        return int(lib().jxrb_submission_device_ptr(self._handle, index) or 0)

    def enqueue_consumer_wait(self, stream_handle: int) -> None:
        _check(lib().jxrb_enqueue_consumer_wait(self._handle, stream_handle))

    def report(self) -> dict:
        """The decode report (stages and their executors, timings in ms)."""
        r = DecodeReportC()
        _check(lib().jxrb_submission_report(self._handle, C.byref(r)))
        return {"requested": r.requested_backend, "selected": ROUTE[r.selected_backend],
                "fallback": None if r.fallback == 0 else r.fallback,
                "stages": [(STAGES[r.stages[i].stage], EXECUTORS[r.stages[i].executor]) for i in range(r.stage_count)],
                "upload_ms": r.upload_ms, "reconstruct_ms": r.reconstruct_ms, "readback_ms": r.readback_ms}

    def readback(self, index: int = 0) -> np.ndarray:
        n = self._plans[index].output_bytes()
        out = np.empty(n, np.uint8)
        _check(lib().jxrb_readback(self._handle, index, out.ctypes.data, n))
        return out

    def output_offsets(self) -> list:
        """Each image's byte offset in the submission's output region."""
        base = self.device_ptr(0)
        return [self.device_ptr(i) - base for i in range(self.count)]

    def readback_all(self, host_ptr: int, nbytes: int) -> None:
        """The first `nbytes` of the output region, every image at its
        output_offsets() entry, in one copy into host memory at `host_ptr`."""
        _check(lib().jxrb_readback_all(self._handle, host_ptr, nbytes))

    def close(self):
        if self._handle:
            lib().jxrb_submission_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


ORIENTATION = {n: i for i, n in enumerate(["IDENTITY", "MIRROR_HORIZONTAL", "ROTATE180", "MIRROR_VERTICAL",
                                           "TRANSPOSE", "ROTATE90", "TRANSVERSE", "ROTATE270"])}


def oriented_bytes(width: int, height: int, pixel_bytes: int, orientation: int) -> int:
    return int(lib().jxrb_oriented_bytes(width, height, pixel_bytes, orientation))


def orient(device_source: int, device_destination: int, width: int, height: int, pixel_bytes: int,
           orientation: int, stream: int = 0) -> None:
    """apply_orientation (crates/jxr/src/decoder/orientation.rs:5-211) on a
    device surface: `width` x `height` pixels of `pixel_bytes` each (0: one-bit
    luma) into a second device buffer of oriented_bytes(...) bytes."""
    _check(lib().jxrb_orient(device_source, device_destination, width, height, pixel_bytes, orientation,
                             stream or None))


class CudaDecoderSession:
    """CudaDecoderSession (crates/jxr-cuda/src/session.rs:35-268)."""

    @staticmethod
    def is_available() -> bool:
        try:
            return bool(lib().jxrb_available())
        except CudaError:
            return False

    def __init__(self, ordinal: int = 0, streams: int = 4):
        self._handle = C.c_void_p()
        # resident sets and images live in the session's device memory and
        # must be released before it
        self._dependents = weakref.WeakSet()
        self.ordinal = ordinal
        opts = SessionOptionsC(streams, 0)
        _check(lib().jxrb_session_create(ordinal, C.byref(opts), C.byref(self._handle)))

    @classmethod
    def system_default(cls) -> "CudaDecoderSession":
        """CudaDecoderSession::system_default (session.rs:42-45): device 0."""
        self = cls.__new__(cls)
        self._handle = C.c_void_p()
        self._dependents = weakref.WeakSet()
        self.ordinal = 0
        _check(lib().jxrb_session_create_default(C.byref(self._handle)))
        return self

    def allocate_destination(self, nbytes: int) -> "DeviceDestination":
        """allocate_destination (session.rs:85-92): zeroed device memory the caller owns."""
        p = C.c_void_p()
        _check(lib().jxrb_allocate_destination(self._handle, nbytes, C.byref(p)))
        return DeviceDestination(self, int(p.value), nbytes)

    def allocate_batch_destination(self, plans: Sequence[CudaDecodePlan]) -> "DeviceDestination":
        """allocate_batch_destination (session.rs:94-101): the dense batch layout's bytes."""
        arr = (C.c_void_p * len(plans))(*[p.handle.value for p in plans])
        p, n = C.c_void_p(), C.c_uint64()
        _check(lib().jxrb_allocate_batch_destination(self._handle, arr, len(plans), C.byref(p), C.byref(n)))
        return DeviceDestination(self, int(p.value), int(n.value))

    def decode_batch_to_host(self, plans: Sequence[CudaDecodePlan]) -> list:
        """decode_batch_to_host (session.rs:221-235): one batched launch, each
        image's bytes in caller order."""
        outs = [np.empty(p.output_bytes(), np.uint8) for p in plans]
        arr = (C.c_void_p * len(plans))(*[p.handle.value for p in plans])
        hosts = (C.c_void_p * len(plans))(*[o.ctypes.data for o in outs])
        sizes = (C.c_uint64 * len(plans))(*[o.size for o in outs])
        _check(lib().jxrb_decode_batch_to_host(self._handle, arr, len(plans), hosts, sizes))
        return outs

    def submit(self, plan: CudaDecodePlan) -> CudaSubmission:
        h = C.c_void_p()
        _check(lib().jxrb_submit(self._handle, plan.handle, C.byref(h)))
        return CudaSubmission(h, 1, [plan])

    def submit_into(self, plan: CudaDecodePlan, device_ptr: int, nbytes: int) -> CudaSubmission:
        h = C.c_void_p()
        _check(lib().jxrb_submit_into(self._handle, plan.handle, device_ptr, nbytes, C.byref(h)))
        return CudaSubmission(h, 1, [plan])

    def submit_batch(self, plans: Sequence[CudaDecodePlan], device_ptr: int = 0, nbytes: int = 0) -> CudaSubmission:
        arr = (C.c_void_p * len(plans))(*[p.handle.value for p in plans])
        h = C.c_void_p()
        _check(lib().jxrb_submit_batch(self._handle, arr, len(plans), device_ptr or None, nbytes, C.byref(h)))
        return CudaSubmission(h, len(plans), list(plans))

    def decode_to_host(self, plan: CudaDecodePlan) -> np.ndarray:
        out = np.empty(plan.output_bytes(), np.uint8)
        _check(lib().jxrb_decode_to_host(self._handle, plan.handle, out.ctypes.data, out.size))
        return out

    def diagnostics(self) -> dict:
        d = DiagnosticsC()
        _check(lib().jxrb_session_diagnostics(self._handle, C.byref(d)))
        return {n: int(getattr(d, n)) for n, _ in DiagnosticsC._fields_}

    def resident(self, plans: Sequence[CudaDecodePlan]) -> "ResidentSet":
        return ResidentSet(self, plans)

    def upload(self, arena: Arena, geometry: Geometry, alpha_arena: Optional[Arena] = None) -> "ResidentImage":
        return ResidentImage(self, arena, geometry, alpha_arena)

    def submit_requests(self, requests: Sequence["Request"], device_ptr: int = 0, nbytes: int = 0) -> CudaSubmission:
        arr = (C.c_void_p * len(requests))(*[r.handle.value for r in requests])
        h = C.c_void_p()
        _check(lib().jxrb_submit_requests(self._handle, arr, len(requests), device_ptr or None, nbytes,
                                          C.byref(h)))
        return CudaSubmission(h, len(requests), list(requests))

    def close(self):
        if self._handle:
            for dependent in list(self._dependents):
                dependent.close()
            lib().jxrb_session_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ResidentSet:
    """Arenas uploaded once and reconstructed many times (upload cache,
    crates/jxr-cuda/src/upload_cache.rs:65-153)."""

    def __init__(self, session: CudaDecoderSession, plans: Sequence[CudaDecodePlan]):
        self.session, self.plans = session, list(plans)
        arr = (C.c_void_p * len(plans))(*[p.handle.value for p in plans])
        self._handle = C.c_void_p()
        _check(lib().jxrb_resident_create(session._handle, arr, len(plans), C.byref(self._handle)))
        session._dependents.add(self)

    def output_bytes(self) -> int:
        return int(lib().jxrb_resident_output_bytes(self._handle))

    def launches(self, batched: bool) -> int:
        return int(lib().jxrb_resident_launches(self._handle, int(batched)))

    def run(self, device_ptr: int, nbytes: int, batched: bool = True, stream: int = 0) -> None:
        _check(lib().jxrb_resident_run(self._handle, device_ptr, nbytes, int(batched), stream or None))

    def status(self) -> int:
        w = C.c_uint32()
        _check(lib().jxrb_resident_status(self._handle, C.byref(w)))
        return w.value

    def set_tuning(self, blocks_per_sm: Sequence[int] = (0, 0, 0, 0, 0), side_stream: bool = True) -> None:
        """Launch shape of the tile kernels (see jxr_b200.autotune)."""
        t = LaunchTuningC((C.c_uint32 * 5)(*blocks_per_sm), int(side_stream))
        _check(lib().jxrb_resident_set_tuning(self._handle, C.byref(t)))

    def capture(self, device_ptr: int, nbytes: int, batched: bool = True) -> None:
        """Record one run's launch sequence as a CUDA graph bound to `device_ptr`."""
        _check(lib().jxrb_resident_capture(self._handle, device_ptr, nbytes, int(batched)))

    def replay(self, stream: int = 0) -> None:
        _check(lib().jxrb_resident_replay(self._handle, stream or None))

    def close(self):
        if self._handle:
            lib().jxrb_resident_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ResidentImage:
    """An image whose arena stays on the device (jxrb_image): requests on it
    upload only their descriptors."""

    def __init__(self, session: CudaDecoderSession, arena: Arena, geometry: Geometry,
                 alpha_arena: Optional[Arena] = None):
        self.session, self.geometry = session, geometry
        a, ap = arena.to_c()
        b, bp = alpha_arena.to_c() if alpha_arena is not None else (None, None)
        g, keep = geometry.to_c()
        self._handle = C.c_void_p()
        _check(lib().jxrb_image_create(session._handle, C.byref(a), C.byref(b) if b is not None else None,
                                       C.byref(g), C.byref(self._handle)))
        session._dependents.add(self)

    @property
    def handle(self):
        return self._handle

    def device_bytes(self) -> int:
        return int(lib().jxrb_image_device_bytes(self._handle))

    def request(self, output: OutputFormat, denominator: int = 1) -> "Request":
        return Request(self, output, denominator)

    def close(self):
        if self._handle:
            lib().jxrb_image_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Request:
    """A decode of a region (output.crop_*, image coordinates) of a resident
    image, at full resolution (denominator 1), a quarter of it (4) or a
    sixteenth (16)."""

    def __init__(self, image: ResidentImage, output: OutputFormat, denominator: int = 1):
        self.image, self.output, self.denominator = image, output, denominator
        self._handle = C.c_void_p()
        o = output.to_c()
        _check(lib().jxrb_request_create_scaled(image.handle, C.byref(o), denominator, C.byref(self._handle)))

    @property
    def handle(self):
        return self._handle

    def output_bytes(self) -> int:
        return int(lib().jxrb_request_output_bytes(self._handle))

    def traffic_bytes(self) -> int:
        return int(lib().jxrb_request_traffic_bytes(self._handle))

    def window(self):
        w = (C.c_uint32 * 4)()
        _check(lib().jxrb_request_window(self._handle, w))
        return tuple(w)

    def close(self):
        if self._handle:
            lib().jxrb_request_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# synthetic inputs
# ---------------------------------------------------------------------------
@dataclass
class SynthImage:
    arena: Arena
    alpha_arena: Optional[Arena]
    geometry: Geometry
    source: np.ndarray = field(repr=False)


def _copy(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))), shape=(n,)).copy()


def synth(width: int, height: int, *, content: int = CONTENT["PHOTO_RGB8"], color_format: int = COLOR["YUV444"],
          alpha_mode: int = 0, overlap: int = 1, alpha_overlap: int = 0, scaled: int = 1, quality: int = 75,
          qp=(0, 0, 0), alpha_qp=(0, 0, 0), tile_width: int = 0, tile_height: int = 0, hard_tiles: int = 0,
          bands: int = 3, seed: int = 1, threads: int = 8) -> SynthImage:
    """Seeded synthetic image coded by the forward analysis (csrc/synth.h)."""
    L = synth_lib()
    req = SynthRequestC(width, height, content, color_format, alpha_mode, overlap, alpha_overlap, scaled, quality,
                        (C.c_int32 * 3)(*qp), (C.c_int32 * 3)(*alpha_qp), tile_width, tile_height, hard_tiles,
                        bands, seed)
    h = C.c_void_p()
    _check_synth(L.jxrb_synth_create(C.byref(req), threads, C.byref(h)), "create")
    try:
        arenas = []
        for which in (0, 1):
            v = SynthArenaViewC()
            _check_synth(L.jxrb_synth_arena(h, which, C.byref(v)), "arena")
            if not v.coefficients:
                arenas.append(None)
                continue
            n = v.macroblock_count
            arenas.append(Arena(
                coefficients=_copy(v.coefficients, v.coefficient_count, np.int32),
                coefficient_offsets=_copy(v.coefficient_offsets, n, np.uint32),
                quantizers=_copy(v.quantizers, n * 3, np.uint32),
                bands=_copy(v.bands, n, np.uint8), hp_predictions=_copy(v.hp_predictions, n, np.uint8),
                coded_x=_copy(v.coded_x, n, np.uint32), coded_y=_copy(v.coded_y, n, np.uint32),
                planes=_copy(v.plane_words, v.plane_count * 6, np.uint64)))
        mx, my, tc, tr = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        tw, th = C.c_void_p(), C.c_void_p()
        _check_synth(L.jxrb_synth_geometry(h, C.byref(mx), C.byref(my), C.byref(tw), C.byref(tc), C.byref(th),
                                           C.byref(tr)), "geometry")
        widths = _copy(tw, tc.value, np.uint32).tolist()
        heights = _copy(th, tr.value, np.uint32).tolist()
        ch, nb = C.c_uint32(), C.c_uint32()
        sp = L.jxrb_synth_source(h, C.byref(ch), C.byref(nb))
        src = _copy(sp, width * height * ch.value, np.uint8 if nb.value == 1 else np.uint16)
        src = src.reshape(height, width, ch.value)
    finally:
        L.jxrb_synth_destroy(h)
    comps = 1 if color_format == COLOR["LUMA"] else 4 if color_format == COLOR["YUVK"] else 3
    geom = Geometry(mx.value, my.value, color_format=color_format, components=comps, overlap=overlap,
                    scaled=scaled, tile_column_widths=widths, tile_row_heights=heights, hard_tiles=hard_tiles,
                    alpha_mode=alpha_mode, alpha_overlap=alpha_overlap,
                    alpha_scaled=int(scaled and alpha_qp[0] > 0 and content != CONTENT["HDR_HALF"]))
    return SynthImage(arenas[0], arenas[1], geom, src)


# ---------------------------------------------------------------------------
# forward analysis on the GPU
# ---------------------------------------------------------------------------
@dataclass
class AnalysisPlane:
    """One sample plane to analyse (jxrb_analysis_plane); `samples` and the
    outputs are torch CUDA tensors (int32), made by analyze()."""
    samples: object
    block_columns: int = 4
    block_rows: int = 4
    scaled: int = 0
    overlap: int = 1
    steps: Sequence[int] = (1, 1, 1)
    column_boundaries: Sequence[int] = ()
    row_boundaries: Sequence[int] = ()
    hard_tiles: int = 0


def analyze(planes: Sequence[AnalysisPlane], stream: int = 0):
    """analyze_component (crates/jxr-native/src/analyze.rs:56-131) of each
    plane on the GPU: [(low_q, high_q)] as torch int32 tensors of
    (macroblocks, 16) and (macroblocks, 256).  The sample tensors are
    prefiltered in place."""
    import torch
    keep, out = [], []
    arr = (AnalysisPlaneC * len(planes))()
    for i, p in enumerate(planes):
        h, w = p.samples.shape
        mbs = (w // (p.block_columns * 4)) * (h // (p.block_rows * 4))
        low = torch.empty((h // 4) * (w // 4), dtype=torch.int32, device=p.samples.device)
        lq = torch.empty((mbs, 16), dtype=torch.int32, device=p.samples.device)
        hq = torch.empty((mbs, 256), dtype=torch.int32, device=p.samples.device)
        cb = np.ascontiguousarray(p.column_boundaries or [0, w // (p.block_columns * 4)], np.uint32)
        rb = np.ascontiguousarray(p.row_boundaries or [0, h // (p.block_rows * 4)], np.uint32)
        keep += [low, cb, rb]
        arr[i] = AnalysisPlaneC(p.samples.data_ptr(), w, h, p.block_columns, p.block_rows, p.scaled, p.overlap,
                                (C.c_uint32 * 3)(*p.steps), cb.ctypes.data, cb.size, rb.ctypes.data, rb.size,
                                p.hard_tiles, low.data_ptr(), lq.data_ptr(), hq.data_ptr())
        out.append((lq, hq))
    _check(lib().jxrb_analyze_planes(arr, len(planes), stream or None))
    return out


def analyze_plane_cpu(samples: np.ndarray, block_columns=4, block_rows=4, scaled=0, overlap=1, steps=(1, 1, 1),
                      column_boundaries=(), row_boundaries=(), hard_tiles=0):
    """The generator's CPU analysis of one plane (the checker of analyze())."""
    s = np.ascontiguousarray(samples, np.int32)
    h, w = s.shape
    mbs = (w // (block_columns * 4)) * (h // (block_rows * 4))
    lq = np.zeros((mbs, 16), np.int32)
    hq = np.zeros((mbs, 256), np.int32)
    cb = np.ascontiguousarray(column_boundaries or [0, w // (block_columns * 4)], np.uint32)
    rb = np.ascontiguousarray(row_boundaries or [0, h // (block_rows * 4)], np.uint32)
    st = np.ascontiguousarray(steps, np.uint32)
    _check_synth(synth_lib().jxrb_analyze_plane_cpu(s.ctypes.data, w, h, block_columns, block_rows, scaled, overlap,
                                                    st.ctypes.data, cb.ctypes.data, cb.size, rb.ctypes.data, rb.size,
                                                    hard_tiles, lq.ctypes.data, hq.ctypes.data), "analysis")
    return lq, hq
