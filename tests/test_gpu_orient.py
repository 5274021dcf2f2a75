"""The presentation orientation on the GPU (jxrb_orient) against the oracle's
restatement of apply_orientation (crates/jxr/src/decoder/orientation.rs:5-211),
byte for byte: every orientation, pixel sizes of 1 to 48 bytes, odd and tile-
straddling extents, one-bit luma, and an oriented decode end to end."""
import numpy as np
import pytest

import jxr_b200 as J
from jxr_b200 import api
from tests import _oracle as O
from tests._bridge import decode_synth

pytestmark = pytest.mark.gpu

C_, D, S, L = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT


@pytest.fixture(scope="module")
def torch():
    import torch as T
    if not J.CudaDecoderSession.is_available():
        pytest.fail("no B200 visible: the GPU tests need the CUDA engine")
    return T


def gpu_orient(torch, src: np.ndarray, width, height, pixel_bytes, orientation, offset=0):
    n_out = api.oriented_bytes(width, height, pixel_bytes, orientation)
    s = torch.zeros(src.size + offset, dtype=torch.uint8, device="cuda:0")
    s[offset:] = torch.from_numpy(src).to("cuda:0")
    d = torch.full((n_out + offset,), 0xA5, dtype=torch.uint8, device="cuda:0")
    api.orient(s.data_ptr() + offset, d.data_ptr() + offset, width, height, pixel_bytes, orientation)
    torch.cuda.synchronize()
    return d[offset:].cpu().numpy()


@pytest.mark.parametrize("orientation", range(8))
@pytest.mark.parametrize("pixel_bytes", [1, 2, 3, 4, 6, 8, 12, 16, 20, 48])
def test_orientation_matches_the_oracle(torch, orientation, pixel_bytes):
    rng = np.random.default_rng(pixel_bytes * 8 + orientation)
    for width, height in [(1, 1), (3, 2), (37, 29), (64, 33), (130, 97)]:
        src = rng.integers(0, 256, width * height * pixel_bytes, dtype=np.uint8)
        rc, want = O.orient(src, width, height, pixel_bytes, orientation)
        assert rc == 0
        got = gpu_orient(torch, src, width, height, pixel_bytes, orientation)
        assert np.array_equal(got, want), (width, height)


@pytest.mark.parametrize("orientation", [0, 4, 5])
def test_unaligned_surfaces_take_narrower_words(torch, orientation):
    src = np.random.default_rng(3).integers(0, 256, 45 * 31 * 8, dtype=np.uint8)
    rc, want = O.orient(src, 45, 31, 8, orientation)
    for offset in (1, 2):
        assert np.array_equal(gpu_orient(torch, src, 45, 31, 8, orientation, offset), want)


@pytest.mark.parametrize("orientation", range(8))
def test_bit_packed_orientation_matches_the_oracle(torch, orientation):
    rng = np.random.default_rng(orientation)
    for width, height in [(3, 2), (9, 17), (70, 33)]:
        src = rng.integers(0, 256, (width + 7) // 8 * height, dtype=np.uint8)
        src.reshape(height, -1)[:, -1] &= np.uint8((0xFF00 >> (width % 8 or 8)) & 0xFF)   # padding bits clear
        rc, want = O.orient(src, width, height, 0, orientation)
        assert rc == 0
        assert np.array_equal(gpu_orient(torch, src, width, height, 0, orientation), want), (width, height)


def test_oriented_decode(torch):
    """decode_oriented (crates/jxr/src/decoder.rs:327-333): the decode, then
    the orientation of its surface, all on the device."""
    img = J.synth(200, 136, quality=85, overlap=2, tile_width=6, tile_height=5, seed=77)
    out = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 200, 136)
    plan = J.CudaDecodePlan(img.arena, img.geometry, out)
    session = J.CudaDecoderSession(0)
    try:
        n = plan.output_bytes()
        dst = torch.empty(n, dtype=torch.uint8, device="cuda:0")
        rot = torch.empty(n, dtype=torch.uint8, device="cuda:0")
        sub = session.submit_into(plan, dst.data_ptr(), n)
        sub.wait()
        sub.close()
        api.orient(dst.data_ptr(), rot.data_ptr(), 200, 136, 3, api.ORIENTATION["ROTATE90"])
        torch.cuda.synchronize()
        rc, ref = decode_synth(img, out)
        assert rc == 0
        rc, want = O.orient(ref, 200, 136, 3, api.ORIENTATION["ROTATE90"])
        assert rc == 0 and np.array_equal(rot.cpu().numpy(), want)
    finally:
        session.close()


def test_orientation_rejections(torch):
    s = torch.zeros(64, dtype=torch.uint8, device="cuda:0")
    d = torch.zeros(64, dtype=torch.uint8, device="cuda:0")
    with pytest.raises(J.CudaError):
        api.orient(s.data_ptr(), d.data_ptr(), 4, 4, 1, 8)             # no such orientation
    with pytest.raises(J.CudaError):
        api.orient(s.data_ptr(), s.data_ptr(), 4, 4, 1, 5)             # in place
    with pytest.raises(J.CudaError):
        api.orient(s.data_ptr(), d.data_ptr(), 1, 1, 49, 5)            # pixel above 48 bytes
