"""ctypes binding of the CPU oracle (oracle/libjxr_oracle.so).

Test infrastructure: the oracle is the checker the CUDA engine is compared
with.  Only tests, the smoke check and the benchmark's CPU-baseline leg load it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
LIB_PATH = ROOT / "oracle" / "libjxr_oracle.so"

JO_OK, JO_ERR_OVERFLOW, JO_ERR_INVALID, JO_ERR_UNSUPPORTED = 0, 1, 2, 3


class JoPlane(C.Structure):
    _fields_ = [
        ("coefficients", C.POINTER(C.c_int32)),
        ("coefficient_count", C.c_size_t),
        ("offsets", C.POINTER(C.c_uint32)),
        ("quantizers", C.POINTER(C.c_uint32)),
        ("bands", C.POINTER(C.c_uint8)),
        ("hp_prediction", C.POINTER(C.c_uint8)),
        ("macroblocks_x", C.c_uint32),
        ("macroblocks_y", C.c_uint32),
        ("block_columns", C.c_uint32),
        ("block_rows", C.c_uint32),
        ("scale_after_first_transform", C.c_int),
        ("overlap", C.c_int),
        ("hard_tiles", C.c_int),
        ("column_boundaries", C.POINTER(C.c_uint32)),
        ("column_boundary_count", C.c_uint32),
        ("row_boundaries", C.POINTER(C.c_uint32)),
        ("row_boundary_count", C.c_uint32),
    ]


class JoOutput(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "internal_color", "output_color", "depth", "shift_bits", "mantissa_length",
        "exponent_bias", "storage", "layout", "ncomponents", "scaled", "alpha_depth",
        "alpha_shift_bits", "alpha_mantissa_length", "alpha_exponent_bias", "alpha_scaled",
        "red_blue_not_swapped", "premultiply")] + [
        ("crop_x", C.c_uint32), ("crop_y", C.c_uint32),
        ("crop_width", C.c_uint32), ("crop_height", C.c_uint32),
        ("nchw", C.c_int), ("widen_f16", C.c_int)]


class JoImage(C.Structure):
    _fields_ = [
        ("planes", C.POINTER(JoPlane)), ("plane_count", C.c_int),
        ("alpha", C.POINTER(JoPlane)), ("coded_color", C.c_int),
        ("centering_x", C.c_int), ("centering_y", C.c_int),
    ]


_lib = None


def lib() -> C.CDLL:
    """Load the oracle, building it with its Makefile when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        subprocess.run(["make", "-C", str(LIB_PATH.parent)], check=True,
                       stdout=subprocess.DEVNULL)
    L = C.CDLL(str(LIB_PATH))
    i32p, u32p = C.POINTER(C.c_int32), C.POINTER(C.c_uint32)
    for name, n in [("jo_inverse_core_transform", 16), ("jo_inverse_chroma_420", 4),
                    ("jo_inverse_chroma_422", 8), ("jo_inverse_overlap_4", 4),
                    ("jo_inverse_overlap_4x4", 16), ("jo_inverse_overlap_2x2", 4),
                    ("jo_inverse_overlap_2", 2)]:
        getattr(L, name).argtypes = [i32p]
        getattr(L, name).restype = C.c_int
    L.jo_dequantize.argtypes = [C.c_int32, C.c_uint32, i32p]
    L.jo_predict_high_pass.argtypes = [i32p, C.c_int, C.c_int, C.c_int]
    L.jo_upsample_pair.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int, i32p]
    L.jo_postscale_rgbe.argtypes = [i32p, C.POINTER(C.c_uint8)]
    L.jo_postscale_rgbe.restype = None
    L.jo_premultiply_unsigned.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p]
    L.jo_premultiply_signed.argtypes = [C.c_int32, C.c_int32, C.c_int32, i32p]
    L.jo_premultiply_sign_magnitude_15.argtypes = [C.c_uint16, C.c_uint16, C.POINTER(C.c_uint16)]
    L.jo_premultiply_f32.argtypes = [C.c_float, C.c_float]
    L.jo_premultiply_f32.restype = C.c_float
    L.jo_widen_f16.argtypes = [C.c_uint16]
    L.jo_widen_f16.restype = C.c_uint32
    L.jo_reconstruct_plane.argtypes = [C.POINTER(JoPlane), i32p, C.c_int]
    L.jo_upsample_chroma.argtypes = [i32p, C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.c_int, i32p, C.c_int]
    L.jo_output_bytes.argtypes = [C.POINTER(JoOutput)]
    L.jo_output_bytes.restype = C.c_size_t
    L.jo_format_output.argtypes = [C.POINTER(i32p), C.c_int, i32p, C.c_uint32, C.c_uint32,
                                   C.POINTER(JoOutput), C.c_void_p, C.c_size_t]
    L.jo_decode_image.argtypes = [C.POINTER(JoImage), C.POINTER(JoOutput), C.c_void_p, C.c_size_t, C.c_int]
    L.jo_decode_image_scaled.argtypes = [C.POINTER(JoImage), C.c_int, C.POINTER(JoOutput), C.c_void_p,
                                         C.c_size_t, C.c_int]
    L.jo_analyze_plane.argtypes = [C.POINTER(JoPlane), i32p, i32p]
    L.jo_reconstruct_plane_quarter.argtypes = [C.POINTER(JoPlane), i32p]
    for name in ("jo_apply_overlap", "jo_apply_subsampled_first_overlap"):
        getattr(L, name).argtypes = [i32p, C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p, C.c_uint32, C.c_int]
        getattr(L, name).restype = C.c_int
    L.jo_full_schedule.argtypes = [C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p, C.c_uint32, C.c_int, u32p,
                                   u32p, u32p, C.c_uint32, u32p]
    L.jo_full_schedule.restype = C.c_int
    L.jo_place_high_pass.argtypes = [i32p, C.c_uint32, C.c_int, C.c_uint32, C.c_uint32, i32p, C.c_size_t,
                                     C.c_size_t]
    L.jo_place_high_pass.restype = C.c_int
    L.jo_reconstruct_plane_sixteenth.argtypes = [C.POINTER(JoPlane), i32p]
    L.jo_reconstruct_plane_sixteenth.restype = C.c_int
    L.jo_orient.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int]
    L.jo_orient.restype = C.c_int
    _lib = L
    return L


def _arr(values, ctype):
    return (ctype * len(values))(*values)


def block_op(name: str, values):
    """Run one in-place math operator; returns (status, values)."""
    buf = _arr(list(values), C.c_int32)
    rc = getattr(lib(), name)(buf)
    return rc, list(buf)


def dequantize(coefficient: int, step: int):
    out = C.c_int32()
    rc = lib().jo_dequantize(coefficient, step, C.byref(out))
    return rc, out.value


def predict_high_pass(coefficients, direction, columns, rows):
    buf = _arr(list(coefficients), C.c_int32)
    rc = lib().jo_predict_high_pass(buf, direction, columns, rows)
    return rc, list(buf)


def upsample_pair(previous, current, nxt, centering):
    out = (C.c_int32 * 2)()
    rc = lib().jo_upsample_pair(previous, current, nxt, centering, out)
    return rc, list(out)


def postscale_rgbe(rgb):
    out = (C.c_uint8 * 4)()
    lib().jo_postscale_rgbe(_arr(list(rgb), C.c_int32), out)
    return list(out)


def premultiply_unsigned(value, alpha, maximum):
    out = C.c_uint32()
    rc = lib().jo_premultiply_unsigned(value, alpha, maximum, C.byref(out))
    return rc, out.value


def premultiply_signed(value, alpha, maximum):
    out = C.c_int32()
    rc = lib().jo_premultiply_signed(value, alpha, maximum, C.byref(out))
    return rc, out.value


def premultiply_sign_magnitude_15(value, alpha):
    out = C.c_uint16()
    rc = lib().jo_premultiply_sign_magnitude_15(value, alpha, C.byref(out))
    return rc, out.value


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class PlaneHandle:
    """A JoPlane whose numpy buffers stay alive as long as the handle."""

    def __init__(self, plane: dict):
        self.keep = []
        def keep(a, dtype):
            a = np.ascontiguousarray(a, dtype=dtype)
            self.keep.append(a)
            return a
        co = keep(plane["coefficients"], np.int32)
        off = keep(plane["offsets"], np.uint32)
        q = keep(plane["quantizers"], np.uint32)
        bands = keep(plane["bands"], np.uint8)
        hp = keep(plane["hp_prediction"], np.uint8)
        cols = keep(plane.get("column_boundaries", [0, plane["macroblocks_x"]]), np.uint32)
        rows = keep(plane.get("row_boundaries", [0, plane["macroblocks_y"]]), np.uint32)
        self.s = JoPlane(
            _ptr(co, C.c_int32), co.size, _ptr(off, C.c_uint32), _ptr(q, C.c_uint32),
            _ptr(bands, C.c_uint8), _ptr(hp, C.c_uint8), plane["macroblocks_x"], plane["macroblocks_y"],
            plane["block_columns"], plane["block_rows"], int(plane.get("scale_after_first_transform", 0)),
            int(plane["overlap"]), int(plane.get("hard_tiles", 0)), _ptr(cols, C.c_uint32), cols.size,
            _ptr(rows, C.c_uint32), rows.size)


def reconstruct_plane(plane: dict, threads: int = 1):
    h = PlaneHandle(plane)
    w = plane["macroblocks_x"] * plane["block_columns"] * 4
    hh = plane["macroblocks_y"] * plane["block_rows"] * 4
    out = np.zeros((hh, w), dtype=np.int32)
    rc = lib().jo_reconstruct_plane(C.byref(h.s), _ptr(out, C.c_int32), threads)
    return rc, out


def make_output(**kw) -> JoOutput:
    o = JoOutput()
    for k, v in kw.items():
        setattr(o, k, int(v))
    return o


def output_bytes(o: JoOutput) -> int:
    return lib().jo_output_bytes(C.byref(o))


def decode_image(planes, alpha, coded_color, centering, output: JoOutput, threads: int = 1, denominator: int = 1):
    """Reconstruct and format one image (at 1/denominator resolution);
    returns (status, bytes)."""
    handles = [PlaneHandle(p) for p in planes]
    arr = (JoPlane * len(handles))(*[h.s for h in handles])
    ah = PlaneHandle(alpha) if alpha is not None else None
    img = JoImage(arr, len(handles), C.pointer(ah.s) if ah else None, coded_color,
                  centering[0], centering[1])
    n = output_bytes(output)
    out = np.zeros(max(n, 1), dtype=np.uint8)
    rc = lib().jo_decode_image_scaled(C.byref(img), denominator, C.byref(output), out.ctypes.data, n, threads)
    return rc, out[:n]


def analyze_plane(plane: dict, samples: np.ndarray):
    """Unit-step analysis of a sample plane (geometry from `plane`); returns
    (status, coefficients in arena order)."""
    geo = dict(plane)
    geo.setdefault("coefficients", np.zeros(1, np.int32))
    mbs = plane["macroblocks_x"] * plane["macroblocks_y"]
    for k, v in (("offsets", np.zeros(mbs, np.uint32)), ("quantizers", np.ones(mbs * 3, np.uint32)),
                 ("bands", np.full(mbs, 3, np.uint8)), ("hp_prediction", np.zeros(mbs, np.uint8))):
        geo.setdefault(k, v)
    h = PlaneHandle(geo)
    count = plane["block_columns"] * plane["block_rows"]
    out = np.zeros(mbs * count * 16, np.int32)
    s = np.ascontiguousarray(samples, np.int32)
    rc = lib().jo_analyze_plane(C.byref(h.s), _ptr(s, C.c_int32), _ptr(out, C.c_int32))
    return rc, out


def unit_plane(coefficients: np.ndarray, mx: int, my: int, bc: int, br: int, **kw) -> dict:
    """A plane of unit quantizers and all bands over analysed coefficients."""
    count = bc * br
    mbs = mx * my
    return dict(coefficients=coefficients, offsets=np.arange(mbs, dtype=np.uint32) * (count * 16),
                quantizers=np.ones(mbs * 3, np.uint32), bands=np.full(mbs, 3, np.uint8),
                hp_prediction=np.zeros(mbs, np.uint8), macroblocks_x=mx, macroblocks_y=my, block_columns=bc,
                block_rows=br, **kw)


def reconstruct_plane_quarter(plane: dict):
    h = PlaneHandle(plane)
    w = plane["macroblocks_x"] * plane["block_columns"]
    hh = plane["macroblocks_y"] * plane["block_rows"]
    out = np.zeros((hh, w), dtype=np.int32)
    rc = lib().jo_reconstruct_plane_quarter(C.byref(h.s), _ptr(out, C.c_int32))
    return rc, out


def upsample_chroma(chroma: np.ndarray, sampling: int, cx: int, cy: int):
    chroma = np.ascontiguousarray(chroma, dtype=np.int32)
    h, w = chroma.shape
    out = np.zeros((h * 2 if sampling == 1 else h, w * 2), dtype=np.int32)
    rc = lib().jo_upsample_chroma(_ptr(chroma, C.c_int32), w, h, sampling, cx, cy, _ptr(out, C.c_int32), 1)
    return rc, out


def _u32s(values):
    a = np.ascontiguousarray(np.asarray(values, dtype=np.uint32))
    return a, a.ctypes.data_as(C.POINTER(C.c_uint32))


def apply_overlap(samples, width, height, columns, rows, hard, subsampled=False):
    """(status, filtered plane) of the full-resolution postfilter, or of the
    subsampled first-level one, over a bare sample plane."""
    s = np.ascontiguousarray(np.asarray(samples, dtype=np.int32).copy())
    cols, cp = _u32s(columns)
    rws, rp = _u32s(rows)
    fn = lib().jo_apply_subsampled_first_overlap if subsampled else lib().jo_apply_overlap
    rc = fn(s.ctypes.data_as(C.POINTER(C.c_int32)), width, height, cp, len(cols), rp, len(rws), int(hard))
    return rc, s


def full_schedule(width, height, columns, rows, hard, capacity=1 << 16):
    """(offsets, steps, kinds) of the full-resolution schedule's operators."""
    cols, cp = _u32s(columns)
    rws, rp = _u32s(rows)
    off, st, kd = (np.zeros(capacity, np.uint32) for _ in range(3))
    n = C.c_uint32()
    u = C.POINTER(C.c_uint32)
    rc = lib().jo_full_schedule(width, height, cp, len(cols), rp, len(rws), int(hard), off.ctypes.data_as(u),
                                st.ctypes.data_as(u), kd.ctypes.data_as(u), capacity, C.byref(n))
    assert rc == 0
    return off[:n.value], st[:n.value], kd[:n.value]


def place_high_pass(high, step, bands, block_columns, block_rows, rows, width, column):
    """(status, rows) after placing one macroblock's dequantized high-pass band."""
    h = np.ascontiguousarray(np.asarray(high, dtype=np.int32))
    r = np.ascontiguousarray(np.asarray(rows, dtype=np.int32).copy())
    rc = lib().jo_place_high_pass(h.ctypes.data_as(C.POINTER(C.c_int32)), step, bands, block_columns, block_rows,
                                  r.ctypes.data_as(C.POINTER(C.c_int32)), width, column)
    return rc, r


def reconstruct_plane_sixteenth(plane: dict):
    """(status, macroblocks_y x macroblocks_x picture) at a sixteenth."""
    h = PlaneHandle(plane)
    out = np.zeros((plane["macroblocks_y"], plane["macroblocks_x"]), np.int32)
    rc = lib().jo_reconstruct_plane_sixteenth(C.byref(h.s), out.ctypes.data_as(C.POINTER(C.c_int32)))
    return rc, out


ORIENTATIONS = ["identity", "mirror_horizontal", "rotate180", "mirror_vertical", "transpose", "rotate90",
                "transverse", "rotate270"]


def orient(src: np.ndarray, width: int, height: int, pixel_bytes: int, orientation: int):
    """(status, oriented bytes) of a packed surface (pixel_bytes 0: one-bit luma)."""
    src = np.ascontiguousarray(src, np.uint8)
    out = np.zeros(src.size, np.uint8) if pixel_bytes else np.zeros(((height if orientation >= 4 else width) + 7)
                                                                    // 8 * (width if orientation >= 4 else height),
                                                                    np.uint8)
    rc = lib().jo_orient(src.ctypes.data, out.ctypes.data, width, height, pixel_bytes, orientation)
    return rc, out
