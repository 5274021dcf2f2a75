"""Forward operators of the input generator are exact inverses of the
oracle's inverse operators -- the reference's round-trip property tests
(crates/jxr-math/src/transform.rs:417-458, overlap.rs:459-509), with its
seeded sample generator (transform.rs:402-415)."""
import ctypes as C

import numpy as np
import pytest

import jxr_b200 as J
from tests import _oracle as O

M64 = (1 << 64) - 1


def samples(seed, bits):
    state = seed

    def nxt():
        nonlocal state
        state = (state * 6364136223846793005 + 1442695040888963407) & M64
        mag = (state >> 33) % (1 << bits)
        return mag if state >> 63 == 0 else -mag
    return nxt


def fwd(name, values):
    buf = (C.c_int32 * len(values))(*values)
    getattr(J.api.synth_lib(), name)(buf)
    return list(buf)


CASES = [("jxrb_forward_core_transform", "jo_inverse_core_transform", 16, 0),
         ("jxrb_forward_chroma_420", "jo_inverse_chroma_420", 4, 200),
         ("jxrb_forward_chroma_422", "jo_inverse_chroma_422", 8, 200),
         ("jxrb_forward_overlap_4", "jo_inverse_overlap_4", 4, 100),
         ("jxrb_forward_overlap_4x4", "jo_inverse_overlap_4x4", 16, 100),
         ("jxrb_forward_overlap_2", "jo_inverse_overlap_2", 2, 300),
         ("jxrb_forward_overlap_2x2", "jo_inverse_overlap_2x2", 4, 300)]


@pytest.mark.parametrize("forward,inverse,n,seed0", CASES)
@pytest.mark.parametrize("bits", [1, 4, 9, 17, 24])
def test_forward_then_inverse_is_identity(forward, inverse, n, seed0, bits):
    nxt = samples(bits + seed0, bits)
    for _ in range(300):
        orig = [nxt() for _ in range(n)]
        rc, back = O.block_op(inverse, fwd(forward, orig))
        assert rc == 0 and back == orig


# crates/jxr-math/src/overlap.rs:511-520
def test_forward_subsampled_filters_undo_the_postfilter_results():
    assert fwd("jxrb_forward_overlap_2", [2, 3]) == [1, 2]
    assert fwd("jxrb_forward_overlap_2x2", [3, 4, 4, 5]) == [1, 2, 3, 4]


def test_quantizer_steps():
    # quant_map (crates/jxr-native/src/tile_decode/quantizer.rs:309-331)
    step = J.api.synth_lib().jxrb_quant_step
    assert step(0, 1, 0, 0) == 1
    assert step(34, 1, 0, 0) == 72 and step(50, 1, 0, 1) == 144 and step(50, 1, 0, 2) == 144
    assert step(66, 1, 1, 2) == 288 and step(50, 1, 1, 0) == 72
    assert step(4, 0, 0, 0) == 1 and step(8, 0, 0, 1) == 2 and step(16, 0, 0, 2) == 4
