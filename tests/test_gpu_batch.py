"""The batched paths against the oracle: one persistent launch sequence over
a mixed batch, one launch sequence per image, CUDA-graph replay, and every
launch shape the autotuner may choose -- all bit-exact."""
import numpy as np
import pytest

import jxr_b200 as J
from jxr_b200 import autotune, workloads as W
from tests._bridge import decode_synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def session():
    if not J.CudaDecoderSession.is_available():
        pytest.fail("no B200 visible: the GPU tests need the CUDA engine")
    s = J.CudaDecoderSession(0)
    yield s
    s.close()


@pytest.fixture(scope="module")
def batch():
    items = W.mixed_batch(count=14, seed=7, lo=64, hi=720, threads=8)
    refs = []
    for it in items:
        rc, ref = decode_synth(it.image, it.output, threads=8)
        assert rc == 0
        refs.append(ref)
    return items, W.plans_of(items), refs


def split(buf, plans):
    out, at = [], 0
    for p in plans:
        at = (at + 255) // 256 * 256
        out.append(buf[at:at + p.output_bytes()])
        at += p.output_bytes()
    return out


def check_all(buf, plans, refs):
    for i, (got, ref) in enumerate(zip(split(buf, plans), refs)):
        assert np.array_equal(got, ref), f"image {i} differs"


def test_mix_covers_all_kinds(batch):
    items, _, _ = batch
    assert {it.kind for it in items} == {"rgb420", "gray16", "rgba"}


def test_batched_per_image_and_graph(session, batch):
    import torch
    items, plans, refs = batch
    res = session.resident(plans)
    n = res.output_bytes()
    stream = torch.cuda.Stream()
    for batched in (True, False):
        dst = torch.full((n,), 0x33, dtype=torch.uint8, device="cuda")
        res.run(dst.data_ptr(), n, batched, stream.cuda_stream)
        stream.synchronize()
        assert res.status() == 0
        check_all(dst.cpu().numpy(), plans, refs)
    for batched in (True, False):
        dst = torch.full((n,), 0x44, dtype=torch.uint8, device="cuda")
        res.capture(dst.data_ptr(), n, batched)
        for _ in range(2):
            res.replay(stream.cuda_stream)
        stream.synchronize()
        check_all(dst.cpu().numpy(), plans, refs)
    res.close()


@pytest.mark.parametrize("blocks,side", autotune.candidates()[::3])
def test_every_launch_shape_is_exact(session, batch, blocks, side):
    import torch
    _, plans, refs = batch
    res = session.resident(plans)
    n = res.output_bytes()
    res.set_tuning(blocks, side)
    dst = torch.zeros(n, dtype=torch.uint8, device="cuda")
    res.run(dst.data_ptr(), n, True, 0)
    torch.cuda.synchronize()
    check_all(dst.cpu().numpy(), plans, refs)
    res.close()


def test_autotuner_picks_a_candidate(session, batch, tmp_path, monkeypatch):
    import torch
    monkeypatch.setenv("JXRB_TUNING_CACHE", str(tmp_path / "tuning.json"))
    _, plans, refs = batch
    res = session.resident(plans)
    n = res.output_bytes()
    dst = torch.zeros(n, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    first = autotune.tune(res, plans, dst.data_ptr(), n, stream, reps=3)
    assert first["source"] == "measured"
    assert (tuple(first["blocks_per_sm"]), first["side_stream"]) in set(autotune.candidates())
    again = autotune.tune(res, plans, dst.data_ptr(), n, stream, reps=3)
    assert again["source"] == "cache" and again["blocks_per_sm"] == first["blocks_per_sm"]
    res.run(dst.data_ptr(), n, True, stream.cuda_stream)
    stream.synchronize()
    check_all(dst.cpu().numpy(), plans, refs)
    res.close()
