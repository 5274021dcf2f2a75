"""The benchmark configurations at full size, byte for byte against the oracle.

C2: 4096x4096 8-bit RGB, quality 90, two-level overlap, 256x256 soft tiles,
to U8 RGB.  C3: 8192x8192 half-float RGB with a separate alpha plane, to F32
RGBA NCHW (1 GiB of output).  C4: the whole 256-image mixed batch in one
batched launch and in per-image launches.  Outputs are integer bytes (float
outputs are exact bit patterns), so the tolerance is zero.  The oracle runs
on every host core."""
import os

import numpy as np
import pytest

import jxr_b200 as J
from jxr_b200 import workloads as W
from tests._bridge import decode_synth

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 8


@pytest.fixture(scope="module")
def session():
    if not J.CudaDecoderSession.is_available():
        pytest.fail("no B200 visible: the GPU tests need the CUDA engine")
    s = J.CudaDecoderSession(0)
    yield s
    s.close()


def first_difference(got, want):
    bad = np.flatnonzero(got != want)
    return None if bad.size == 0 else (int(bad[0]), int(bad.size))


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_single_image_config_full_size(session, name):
    img, out = W.single_image(name, threads=THREADS)
    plan = J.CudaDecodePlan(img.arena, img.geometry, out, img.alpha_arena)
    kinds = plan.tile_kinds()
    assert kinds["interior"] > 0            # the interior tile kernel carries the image
    got = session.decode_to_host(plan)
    rc, want = decode_synth(img, out, threads=THREADS)
    assert rc == 0
    assert got.shape == want.shape
    assert first_difference(got, want) is None


def test_mixed_batch_full_256(session):
    items = W.mixed_batch(256, seed=4, threads=THREADS)
    plans = W.plans_of(items)
    wants = []
    for it in items:
        rc, want = decode_synth(it.image, it.output, threads=THREADS)
        assert rc == 0
        wants.append(want)
    res = session.resident(plans)
    try:
        import torch
        n = res.output_bytes()
        dst = torch.empty(n, dtype=torch.uint8, device="cuda:0")
        for batched in (True, False):
            dst.fill_(0xA5)
            res.run(dst.data_ptr(), n, batched, 0)
            torch.cuda.synchronize()
            assert res.status() == 0
            got = dst.cpu().numpy()
            at = 0
            for k, (p, want) in enumerate(zip(plans, wants)):
                at = (at + 255) // 256 * 256
                m = p.output_bytes()
                assert first_difference(got[at:at + m], want) is None, (batched, k, items[k].kind)
                at += m
    finally:
        res.close()
