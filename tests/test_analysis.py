"""The forward analysis (the encoder's front half, analyze_component,
crates/jxr-native/src/analyze.rs:56-131).  On the CPU: the generator's
analysis with unit steps is the exact inverse of the oracle's reconstruction.
On the GPU (jxrb_analyze_planes): every quantized coefficient equals the CPU
analysis's, over every block shape, overlap mode, tiling and step."""
import numpy as np
import pytest

from jxr_b200 import api
from tests import _oracle as O

SHAPES = [(4, 4), (2, 4), (2, 2)]
LAYOUTS = [  # macroblocks x, y, column boundaries, row boundaries, hard
    (1, 1, [0, 1], [0, 1], 0),
    (3, 2, [0, 3], [0, 2], 0),
    (5, 4, [0, 2, 5], [0, 1, 4], 1),
    (6, 5, [0, 1, 3, 6], [0, 2, 5], 1),
    (7, 3, [0, 3, 7], [0, 3], 0),
]


def plane_samples(bc, br, layout, seed, lo=-2048, hi=2048):
    mx, my = layout[0], layout[1]
    return np.random.default_rng(seed).integers(lo, hi, (my * br * 4, mx * bc * 4)).astype(np.int32)


def arena_of(lq, hq, bc, br):
    """Analysed macroblocks as arena coefficients (all bands): block b's DC /
    low-pass value then its fifteen high-pass coefficients."""
    count = bc * br
    c = hq.reshape(-1, 16, 16)[:, :count, :].copy()
    c[:, :, 0] = lq[:, :count]
    return c.reshape(-1)


@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("bc,br", SHAPES)
@pytest.mark.parametrize("li", range(len(LAYOUTS)))
def test_unit_step_analysis_is_the_exact_inverse_of_reconstruction(overlap, bc, br, li):
    mx, my, cols, rows, hard = LAYOUTS[li]
    s = plane_samples(bc, br, LAYOUTS[li], seed=li * 9 + overlap)
    lq, hq = api.analyze_plane_cpu(s, bc, br, 0, overlap, (1, 1, 1), cols, rows, hard)
    plane = O.unit_plane(arena_of(lq, hq, bc, br), mx, my, bc, br, overlap=overlap, hard_tiles=hard,
                         column_boundaries=cols, row_boundaries=rows)
    rc, back = O.reconstruct_plane(plane)
    assert rc == 0 and np.array_equal(back, s)


@pytest.mark.gpu
@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("bc,br", SHAPES)
def test_gpu_analysis_equals_the_cpu_analysis(overlap, bc, br):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("no B200 visible: the GPU tests need the CUDA engine")
    rng = np.random.default_rng(bc * 10 + br + overlap)
    planes, wants = [], []
    for li, layout in enumerate(LAYOUTS):
        for scaled in (0, 1):
            steps = tuple(int(v) for v in rng.integers(1, 40, 3))
            s = plane_samples(bc, br, layout, seed=100 * li + scaled, lo=-40000, hi=40000)
            wants.append(api.analyze_plane_cpu(s, bc, br, scaled, overlap, steps, layout[2], layout[3], layout[4]))
            planes.append(api.AnalysisPlane(torch.from_numpy(s).to("cuda:0"), bc, br, scaled, overlap, steps,
                                            layout[2], layout[3], layout[4]))
    got = api.analyze(planes)
    torch.cuda.synchronize()
    for k, ((lq, hq), (wl, wh)) in enumerate(zip(got, wants)):
        for name, g, w in (("low", lq.cpu().numpy(), wl), ("high", hq.cpu().numpy(), wh)):
            bad = np.argwhere(g != w)
            assert bad.size == 0, (k, name, bad[:4].tolist(), [(int(g[tuple(i)]), int(w[tuple(i)])) for i in bad[:4]])


@pytest.mark.gpu
def test_gpu_analysis_of_a_large_plane_round_trips():
    """A 1024 x 768 two-level plane with unit steps: the GPU analysis then the
    oracle's reconstruction give the samples back."""
    import torch
    s = np.random.default_rng(5).integers(-3000, 3000, (768, 1024)).astype(np.int32)
    cols, rows = [0, 16, 40, 64], [0, 24, 48]
    (lq, hq), = api.analyze([api.AnalysisPlane(torch.from_numpy(s).to("cuda:0"), 4, 4, 0, 2, (1, 1, 1), cols, rows,
                                               1)])
    plane = O.unit_plane(arena_of(lq.cpu().numpy(), hq.cpu().numpy(), 4, 4), 64, 48, 4, 4, overlap=2, hard_tiles=1,
                         column_boundaries=cols, row_boundaries=rows)
    rc, back = O.reconstruct_plane(plane, threads=8)
    assert rc == 0 and np.array_equal(back, s)
