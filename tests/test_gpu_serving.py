"""The continuous-batching server: every served result equals the same
request decoded alone, under load and under a tight memory budget."""
import numpy as np
import pytest

import jxr_b200 as J
from jxr_b200 import serving, workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    if not J.CudaDecoderSession.is_available():
        pytest.fail("no B200 visible: the GPU tests need the CUDA engine")
    session = J.CudaDecoderSession(0)
    pool = W.mixed_batch(6, seed=11, lo=96, hi=640, threads=8)
    images = [session.upload(it.image.arena, it.image.geometry, it.image.alpha_arena) for it in pool]
    yield session, pool, images
    for im in images:
        im.close()
    session.close()


def alone(session, image, output, denominator=1):
    h = image.request(output, denominator)
    sub = session.submit_requests([h])
    sub.wait()
    out = sub.readback(0)
    sub.close()
    h.close()
    return out


@pytest.mark.parametrize("rate", [0.0, 4000.0])
def test_served_results_equal_alone(setup, rate):
    session, pool, images = setup
    stream = serving.request_stream(pool, 300, rate, seed=3, roi_share=0.4, quarter_share=0.3)
    server = serving.Server(session, images, budget_bytes=8 * 10**9, slots=3, max_batch=32, keep_results=True)
    stats = server.serve(stream)
    assert stats["requests"] == 300 and stats["batches"] >= 10
    assert stats["peak_device_bytes"] <= 8 * 10**9
    for r in stream:
        assert r.done >= r.admitted >= r.arrival
        assert np.array_equal(r.result, alone(session, images[r.image], r.output, r.denominator))


def test_tight_budget_still_serves_everything(setup):
    session, pool, images = setup
    stream = serving.request_stream(pool, 40, 0.0, seed=4, roi_share=0.0)
    resident = sum(im.device_bytes() for im in images)
    biggest = max(serving.Server.request_bytes(images[r.image].request(r.output)) for r in stream)
    server = serving.Server(session, images, budget_bytes=resident + biggest, slots=4, max_batch=64,
                            keep_results=True)
    stats = server.serve(stream)
    assert stats["requests"] == 40 and stats["batches"] > 4
    assert stats["peak_device_bytes"] <= resident + biggest
    for r in stream[:8]:
        assert np.array_equal(r.result, alone(session, images[r.image], r.output, r.denominator))


def test_catalog_larger_than_the_budget_uploads_on_admission(setup):
    """A catalog of twice the pool's images (each arena listed twice) under a
    budget that holds only a few of them: images are uploaded when their
    requests are admitted and the least recently used idle ones released;
    every result equals the same request decoded alone, and the server never
    holds more than the budget."""
    session, pool, images = setup
    catalog = [serving.CatalogImage(it.image.arena, it.image.geometry, it.image.alpha_arena) for it in pool] * 2
    biggest = max(c.device_bytes_estimate() for c in catalog)
    budget = biggest * 10 // 3              # 3/4 of it for uploads: room for about two and a half images
    stream = serving.request_stream(pool + pool, 240, 6000.0, seed=12, roi_share=0.3, quarter_share=0.2)
    server = serving.Server(session, catalog, budget_bytes=budget, slots=3, max_batch=16, keep_results=True,
                            output_share=0.25)
    try:
        stats = server.serve(stream)
    finally:
        server.release()
    assert stats["requests"] == 240
    assert stats["peak_device_bytes"] <= budget
    cache = stats["cache"]
    assert cache["uploads"] > len(catalog) // 2 and cache["evictions"] > 0
    assert cache["hits"] + cache["misses"] >= cache["uploads"]
    for r in stream:
        assert np.array_equal(r.result, alone(session, images[r.image % len(pool)], r.output, r.denominator))
