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
