"""Pins the oracle's analysis and quarter-resolution reconstruction to the
reference's own known-answer tests (each cites its source)."""
import numpy as np
import pytest

from tests import _oracle as O


def dc_plane(value, bc=4, br=4, overlap=2, bands=1, scale2=0, mx=1, my=1):
    count = bc * br
    coeff = np.zeros(mx * my * count, np.int32)
    coeff[::count] = value
    mbs = mx * my
    return dict(coefficients=coeff, offsets=np.arange(mbs, dtype=np.uint32) * count,
                quantizers=np.ones(mbs * 3, np.uint32), bands=np.full(mbs, bands, np.uint8),
                hp_prediction=np.zeros(mbs, np.uint8), macroblocks_x=mx, macroblocks_y=my, block_columns=bc,
                block_rows=br, scale_after_first_transform=scale2, overlap=overlap)


# crates/jxr-native/src/reconstruct/pipeline_tests.rs:47-83
def test_native_quarter_stops_after_the_first_inverse_transform():
    p = dc_plane(256, overlap=2, bands=1)
    rc, full = O.reconstruct_plane(p)
    assert rc == 0 and full.min() == 32 and full.max() == 36
    means = full.reshape(4, 4, 4, 4).transpose(0, 2, 1, 3).reshape(16, 16).mean(axis=1)
    assert (np.floor(means) == 33).all()
    rc, q = O.reconstruct_plane_quarter(p)
    assert rc == 0 and q.shape == (4, 4)
    assert q.ravel().tolist() == [33, 33, 33, 33, 34, 34, 34, 34, 33, 33, 33, 33, 33, 34, 34, 34]


# pipeline_tests.rs:85-122
@pytest.mark.parametrize("bc,br", [(4, 4), (2, 4), (2, 2)])
def test_reduced_subsampled_chroma_keeps_the_sample_scale(bc, br):
    p = dc_plane(256 if bc == 4 else 128, bc, br, overlap=0, bands=1)
    rc, full = O.reconstruct_plane(p)
    assert rc == 0 and (full == 16).all()
    rc, q = O.reconstruct_plane_quarter(p)
    assert rc == 0 and q.shape == (br, bc) and (q == 16).all()


LAYOUTS = [  # (macroblocks x, y, column boundaries, row boundaries, hard)
    (1, 1, [0, 1], [0, 1], False),
    (1, 4, [0, 1], [0, 4], False),
    (5, 1, [0, 5], [0, 1], False),
    (3, 3, [0, 1, 2, 3], [0, 1, 2, 3], True),
    (9, 7, [0, 9], [0, 7], False),
    (9, 7, [0, 2, 3, 9], [0, 6, 7], True),
]


def flat_case(level, bc, br, overlap, layout, scale2=0):
    mx, my, cols, rows, hard = layout
    geo = dict(macroblocks_x=mx, macroblocks_y=my, block_columns=bc, block_rows=br, overlap=overlap,
               scale_after_first_transform=scale2, hard_tiles=int(hard), column_boundaries=cols,
               row_boundaries=rows)
    samples = np.full((my * br * 4, mx * bc * 4), level, np.int32)
    rc, coeff = O.analyze_plane(geo, samples)
    assert rc == 0
    plane = O.unit_plane(coeff, mx, my, bc, br, scale_after_first_transform=scale2, overlap=overlap,
                         hard_tiles=int(hard), column_boundaries=cols, row_boundaries=rows)
    return plane, samples


# analysis is the exact inverse of full reconstruction (the analysis tests of
# crates/jxr-native/src/analyze.rs, and pipeline_tests.rs:482-484)
@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("bc,br", [(4, 4), (2, 4), (2, 2)])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_analysis_round_trips(overlap, bc, br, layout):
    mx, my = layout[0], layout[1]
    rng = np.random.default_rng(mx * 31 + my)
    samples = rng.integers(-300, 300, size=(my * br * 4, mx * bc * 4)).astype(np.int32)
    geo = dict(macroblocks_x=mx, macroblocks_y=my, block_columns=bc, block_rows=br, overlap=overlap,
               hard_tiles=int(layout[4]), column_boundaries=layout[2], row_boundaries=layout[3])
    rc, coeff = O.analyze_plane(geo, samples)
    assert rc == 0
    plane = O.unit_plane(coeff, mx, my, bc, br, overlap=overlap, hard_tiles=int(layout[4]),
                         column_boundaries=layout[2], row_boundaries=layout[3])
    rc, full = O.reconstruct_plane(plane)
    assert rc == 0 and np.array_equal(full, samples)


# pipeline_tests.rs:459-531: a flat image's reduced picture is flat at every
# position (within the reference's tolerance under overlap, exactly without)
@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("bc,br", [(4, 4), (2, 4), (2, 2)])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_quarter_of_a_flat_image_is_flat(overlap, bc, br, layout):
    for level in (-128, -78, -1, 0, 62, 127):
        plane, samples = flat_case(level, bc, br, overlap, layout)
        rc, full = O.reconstruct_plane(plane)
        assert rc == 0 and (full == level).all()
        rc, q = O.reconstruct_plane_quarter(plane)
        assert rc == 0
        tol = 0 if overlap == 0 or level == 0 else 2
        assert np.abs(q - level).max() <= tol, (level, q)


# ---- sixteenth resolution ---------------------------------------------------

# pipeline_tests.rs:85-122: the DC-only macroblock at every scale
@pytest.mark.parametrize("bc,br", [(4, 4), (2, 4), (2, 2)])
def test_reduced_subsampled_chroma_keeps_the_sample_scale_at_a_sixteenth(bc, br):
    p = dc_plane(256 if bc == 4 else 128, bc, br, overlap=0, bands=1)
    rc, s = O.reconstruct_plane_sixteenth(p)
    assert rc == 0 and s.tolist() == [[16]]


# pipeline_tests.rs:124-157
def test_native_sixteenth_applies_both_dc_gain_steps_without_expansion():
    rc, s = O.reconstruct_plane_sixteenth(dc_plane(256, overlap=2, bands=0))
    assert rc == 0 and s.tolist() == [[33]]
    rc, full = O.reconstruct_plane(dc_plane(256, overlap=2, bands=0))
    assert rc == 0 and int((2 * full.sum() + 256) // 512) == 33
    rc, s = O.reconstruct_plane_sixteenth(dc_plane(256, overlap=0, bands=0))
    assert rc == 0 and s.tolist() == [[16]]


REDUCED_LAYOUTS = [  # pipeline_tests.rs:353-368
    (1, 1, [0, 1], [0, 1], False),
    (2, 1, [0, 2], [0, 1], False),
    (1, 3, [0, 1], [0, 3], False),
    (7, 6, [0, 1, 3, 7], [0, 2, 3, 6], False),
    (9, 8, [0, 1, 2, 9], [0, 6, 8], False),
    (7, 6, [0, 1, 3, 7], [0, 2, 3, 6], True),
    (9, 8, [0, 1, 2, 9], [0, 6, 8], True),
]


def busy_dc_plane(bc, br, overlap, layout, seed):
    """busy_dc_macroblocks (pipeline_tests.rs:567-577): DC coefficients from
    the crate's LCG, (state >> 40) % 8001 - 4000, DC band only, unit steps."""
    mx, my, cols, rows, hard = layout
    state, values = seed, []
    for _ in range(mx * my):
        state = (state * 6364136223846793005 + 1442695040888963407) & (2**64 - 1)
        values.append((state >> 40) % 8001 - 4000)
    count = bc * br
    coeff = np.zeros(mx * my * count, np.int32)
    coeff[::count] = values
    return dict(coefficients=coeff, offsets=np.arange(mx * my, dtype=np.uint32) * count,
                quantizers=np.ones(mx * my * 3, np.uint32), bands=np.zeros(mx * my, np.uint8),
                hp_prediction=np.zeros(mx * my, np.uint8), macroblocks_x=mx, macroblocks_y=my, block_columns=bc,
                block_rows=br, overlap=overlap, hard_tiles=int(hard), column_boundaries=cols, row_boundaries=rows)


def unit_means(picture, across, down):
    """unit_means (pipeline_tests.rs:413-427): each unit's mean, rounded half up."""
    h, w = picture.shape
    out = []
    for y in range(0, h, down):
        for x in range(0, w, across):
            total = int(picture[y:y + down, x:x + across].astype(np.int64).sum())
            n = across * down
            out.append((2 * total + n) // (2 * n))
    return out


# pipeline_tests.rs:587-632
@pytest.mark.parametrize("bc,br", [(4, 4), (2, 4), (2, 2)])
@pytest.mark.parametrize("index", range(len(REDUCED_LAYOUTS)))
def test_sixteenth_is_the_quarter_picture_of_the_dc_band_by_macroblock(bc, br, index):
    layout = REDUCED_LAYOUTS[index]
    if bc == 2 and (layout[0] == 1 or (layout[4] and 1 in layout[2])):
        pytest.skip("chroma regions one macroblock wide are filtered unlike any other (as the reference skips)")
    plane = busy_dc_plane(bc, br, 2, layout, 50 + index)
    rc, quarter = O.reconstruct_plane_quarter(plane)
    assert rc == 0
    expected = unit_means(quarter, bc, br)
    rc, s = O.reconstruct_plane_sixteenth(plane)
    assert rc == 0 and s.size == len(expected)
    assert np.abs(s.ravel().astype(np.int64) - np.array(expected)).max() <= 1
    # without the low-pass-level filter the coefficients scaled on their own
    # are far from this picture
    rc, unfiltered = O.reconstruct_plane_sixteenth(dict(plane, overlap=1))
    assert rc == 0
    if len(expected) > 4:
        assert np.abs(unfiltered.ravel().astype(np.int64) - np.array(expected)).max() > 64


# pipeline_tests.rs:634-655: soft tile boundaries change no reduced picture
@pytest.mark.parametrize("overlap", [1, 2])
@pytest.mark.parametrize("bc,br", [(4, 4), (2, 2)])
def test_soft_tile_boundaries_do_not_change_a_reduced_picture(overlap, bc, br):
    tiled = busy_dc_plane(bc, br, overlap, (7, 6, [0, 1, 3, 7], [0, 2, 3, 6], False), 9)
    single = dict(tiled, column_boundaries=[0, 7], row_boundaries=[0, 6])
    for fn in (O.reconstruct_plane_quarter, O.reconstruct_plane_sixteenth):
        a, b = fn(tiled), fn(single)
        assert a[0] == b[0] == 0 and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("bc,br", [(4, 4), (2, 4), (2, 2)])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_sixteenth_of_a_flat_image_is_flat(overlap, bc, br, layout):
    for level in (-128, -78, -1, 0, 62, 127):
        plane, samples = flat_case(level, bc, br, overlap, layout)
        rc, s = O.reconstruct_plane_sixteenth(plane)
        assert rc == 0 and s.shape == (layout[1], layout[0])
        tol = 0 if overlap == 0 or level == 0 else 2
        assert np.abs(s - level).max() <= tol, (level, s)


# ---- orientation (crates/jxr/src/decoder/orientation.rs) -------------------

# orientation.rs:288-300
def test_orientation_maps_rectangular_pixels_without_channel_reordering():
    rc, out = O.orient(np.arange(1, 13, dtype=np.uint8), 2, 2, 3, 5)          # Rotate90
    assert rc == 0 and out.tolist() == [7, 8, 9, 1, 2, 3, 10, 11, 12, 4, 5, 6]
    rc, out = O.orient(np.arange(1, 7, dtype=np.uint8), 3, 2, 1, 7)           # Rotate270
    assert rc == 0 and out.tolist() == [3, 6, 2, 5, 1, 4]


# orientation.rs:302-330
def test_orientation_rotates_bitpacked_rows():
    rc, out = O.orient(np.array([0b1010_0000, 0b0100_0000], np.uint8), 3, 2, 0, 5)
    assert rc == 0 and out.tolist() == [0b0100_0000, 0b1000_0000, 0b0100_0000]


# orientation.rs:332-350
@pytest.mark.parametrize("orientation", range(1, 8))
def test_every_bitpacked_orientation_matches_the_pixel_mapping(orientation):
    source = np.array([1, 0, 1, 0, 1, 0], np.uint8)
    rc, want = O.orient(source, 3, 2, 1, orientation)
    assert rc == 0
    rc, packed = O.orient(np.array([0b1010_0000, 0b0100_0000], np.uint8), 3, 2, 0, orientation)
    assert rc == 0
    ow = 2 if orientation >= 4 else 3
    oh = 3 if orientation >= 4 else 2
    stride = (ow + 7) // 8
    bits = [(packed[y * stride + x // 8] >> (7 - x % 8)) & 1 for y in range(oh) for x in range(ow)]
    assert bits == want.tolist()
