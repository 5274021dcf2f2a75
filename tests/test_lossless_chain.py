"""Lossless coding (step 1, unscaled) through the generator's forward
analysis and the oracle's reconstruction returns the source pixels exactly:
every transform, overlap schedule (soft and hard tiles, both levels), the
colour transform and the output store are exact inverses end to end."""
import numpy as np
import pytest

import jxr_b200 as J
from tests._bridge import decode_synth

C_, D, S, L = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT


@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("tiles", [(0, 0, 0), (2, 1, 1), (3, 2, 0), (1, 1, 1)])
def test_rgb8_lossless(overlap, tiles):
    tw, th, hard = tiles
    img = J.synth(80, 48, quality=100, scaled=0, overlap=overlap, tile_width=tw, tile_height=th,
                  hard_tiles=hard, seed=overlap * 10 + tw)
    out = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 80, 48)
    rc, b = decode_synth(img, out)
    assert rc == 0
    assert np.array_equal(b.reshape(48, 80, 3), img.source)


@pytest.mark.parametrize("overlap", [0, 1, 2])
def test_gray16_lossless(overlap):
    img = J.synth(48, 64, content=J.CONTENT["GRAY16"], color_format=C_["LUMA"], quality=100, scaled=0,
                  overlap=overlap, tile_width=2, tile_height=3, hard_tiles=1, seed=7)
    out = J.OutputFormat(C_["LUMA"], D["U16"], S["U16"], L["LUMA"], 48, 64)
    rc, b = decode_synth(img, out)
    assert rc == 0
    assert np.array_equal(b.view(np.uint16).reshape(64, 48), img.source[..., 0])


def test_lossy_photo_is_close():
    img = J.synth(128, 96, quality=90, overlap=2, tile_width=4, tile_height=4, hard_tiles=1, seed=3)
    out = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 128, 96)
    rc, b = decode_synth(img, out)
    assert rc == 0
    err = np.abs(b.reshape(96, 128, 3).astype(int) - img.source.astype(int))
    assert err.mean() < 6 and np.percentile(err, 99) < 40
