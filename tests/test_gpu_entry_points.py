"""Submission entry points of the C ABI that the parity tests do not reach:
bounded waits, completion queries, consumer-stream waits, output device
pointers, session diagnostics and the submission-time rejections
(crates/jxr-cuda/src/submission.rs:43-155, session.rs:103-268)."""
import ctypes as C

import numpy as np
import pytest

import jxr_b200 as J
from tests._bridge import decode_synth

pytestmark = pytest.mark.gpu

C_, D, S, L = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT
TIMEOUT, INVALID_PLAN, INVALID_DESTINATION = 13, 4, 5


@pytest.fixture(scope="module")
def session():
    if not J.CudaDecoderSession.is_available():
        pytest.fail("no B200 visible: the GPU tests need the CUDA engine")
    s = J.CudaDecoderSession(0)
    yield s
    s.close()


@pytest.fixture(scope="module")
def image():
    img = J.synth(1024, 768, quality=85, overlap=2, tile_width=16, tile_height=16, seed=61, threads=8)
    out = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 1024, 768)
    rc, want = decode_synth(img, out, threads=8)
    assert rc == 0
    return img, out, want


def pinned_plan(img, out):
    """A plan whose coefficients live in page-locked host memory, so that its
    upload is asynchronous and submit returns before it has crossed."""
    import torch
    t = torch.from_numpy(img.arena.coefficients).pin_memory()
    a = img.arena
    arena = J.Arena(t.numpy(), a.coefficient_offsets, a.quantizers, a.bands, a.hp_predictions, a.coded_x, a.coded_y,
                    a.planes)
    return J.CudaDecodePlan(arena, img.geometry, out), t


def test_bounded_wait_times_out_then_completes(session, image):
    img, out, want = image
    # 48 images from page-locked memory: about 450 MB to upload, so the
    # submission is certainly still running when the zero-length wait looks
    plan, keep = pinned_plan(img, out)
    sub = session.submit_batch([plan] * 48)
    try:
        with pytest.raises(J.CudaError) as e:
            sub.wait(timeout_ns=0)
        assert e.value.status == TIMEOUT
        assert isinstance(sub.is_complete(), bool)     # a query, never an error
        sub.wait()
        assert sub.is_complete() is True
        for k in (0, 17, 47):
            assert np.array_equal(sub.readback(k), want)
    finally:
        sub.close()


def test_consumer_stream_waits_for_the_submission(session, image):
    import torch
    img, out, want = image
    plan, keep = pinned_plan(img, out)
    n = plan.output_bytes()
    dst = torch.empty(n, dtype=torch.uint8, device="cuda:0")
    consumer = torch.cuda.Stream()
    host = torch.empty(n, dtype=torch.uint8).pin_memory()
    sub = session.submit_into(plan, dst.data_ptr(), n)
    try:
        # the consumer stream copies the output out without any host wait
        sub.enqueue_consumer_wait(consumer.cuda_stream)
        with torch.cuda.stream(consumer):
            host.copy_(dst, non_blocking=True)
        consumer.synchronize()
        assert np.array_equal(host.numpy(), want)
        assert sub.device_ptr(0) == dst.data_ptr()
    finally:
        sub.close()


def test_output_device_pointers_follow_the_layout(session, image):
    img, out, want = image
    small = J.synth(48, 32, quality=80, overlap=1, seed=62, threads=1)
    sout = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 48, 32)
    plans = [J.CudaDecodePlan(small.arena, small.geometry, sout), J.CudaDecodePlan(img.arena, img.geometry, out)]
    sub = session.submit_batch(plans)
    try:
        sub.wait()
        offs = sub.output_offsets()
        assert offs[0] == 0 and offs[1] % 256 == 0 and offs[1] >= plans[0].output_bytes()
        assert J.lib().jxrb_submission_device_ptr(sub._handle, 2) is None    # past the last image
        assert np.array_equal(sub.readback(1), want)
    finally:
        sub.close()


def test_diagnostics_count_submissions_uploads_and_launches(session, image):
    img, out, want = image
    plan = J.CudaDecodePlan(img.arena, img.geometry, out)
    before = session.diagnostics()
    got = session.decode_to_host(plan)
    after = session.diagnostics()
    assert np.array_equal(got, want)
    assert after["submissions"] == before["submissions"] + 1
    assert after["bytes_uploaded"] - before["bytes_uploaded"] >= img.arena.coefficients.nbytes
    assert after["bytes_read_back"] - before["bytes_read_back"] == plan.output_bytes()
    assert after["kernel_launches"] > before["kernel_launches"]


def test_submission_time_rejections(session, image):
    img, out, _ = image
    plan = J.CudaDecodePlan(img.arena, img.geometry, out)
    h = C.c_void_p()
    lib = J.lib()
    assert lib.jxrb_submit_batch(session._handle, None, 0, None, 0, C.byref(h)) == INVALID_PLAN
    empty = (C.c_void_p * 1)(None)
    assert lib.jxrb_submit_batch(session._handle, empty, 1, None, 0, C.byref(h)) == INVALID_PLAN
    import torch
    small = torch.empty(16, dtype=torch.uint8, device="cuda:0")
    with pytest.raises(J.CudaError) as e:
        session.submit_into(plan, small.data_ptr(), 16)
    assert e.value.status == INVALID_DESTINATION
    sub = session.submit(plan)
    try:
        buf = np.empty(plan.output_bytes() + 1, np.uint8)
        assert lib.jxrb_readback(sub._handle, 0, buf.ctypes.data, buf.size) == INVALID_DESTINATION
        assert lib.jxrb_readback(sub._handle, 1, buf.ctypes.data, 1) == INVALID_DESTINATION
        assert lib.jxrb_readback_all(sub._handle, buf.ctypes.data, buf.size + (1 << 20)) == INVALID_DESTINATION
    finally:
        sub.close()


def test_system_default_session_and_batch_decode_to_host(image):
    img, out, want = image
    small = J.synth(48, 32, quality=80, overlap=1, seed=63, threads=1)
    sout = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 48, 32)
    rc, swant = decode_synth(small, sout)
    assert rc == 0
    plans = [J.CudaDecodePlan(img.arena, img.geometry, out), J.CudaDecodePlan(small.arena, small.geometry, sout)]
    s = J.CudaDecoderSession.system_default()
    try:
        got = s.decode_batch_to_host(plans + plans[::-1])
        assert [np.array_equal(g, w) for g, w in zip(got, [want, swant, swant, want])] == [True] * 4
    finally:
        s.close()


def test_caller_owned_destinations(session, image):
    img, out, want = image
    plan = J.CudaDecodePlan(img.arena, img.geometry, out)
    dest = session.allocate_destination(plan.output_bytes())
    try:
        sub = session.submit_into(plan, dest.ptr, dest.nbytes)
        sub.wait()
        assert np.array_equal(sub.readback(0), want)
        sub.close()
    finally:
        dest.free()
    small = J.synth(48, 32, quality=80, overlap=1, seed=64, threads=1)
    sout = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 48, 32)
    plans = [J.CudaDecodePlan(small.arena, small.geometry, sout), plan]
    batch = session.allocate_batch_destination(plans)
    try:
        offs, total = api_batch_layout(plans)
        assert batch.nbytes == total
        sub = session.submit_batch(plans, batch.ptr, batch.nbytes)
        sub.wait()
        assert sub.output_offsets() == offs
        assert np.array_equal(sub.readback(1), want)
        sub.close()
    finally:
        batch.free()


def api_batch_layout(plans):
    from jxr_b200 import api
    return api.batch_layout(plans)


def test_decode_report_names_the_stages_and_times_them(session, image):
    img, out, want = image
    plan, keep = pinned_plan(img, out)
    sub = session.submit(plan)
    try:
        got = sub.readback(0)
        assert np.array_equal(got, want)
        r = sub.report()
        assert r["selected"] == "Cuda" and r["fallback"] is None
        stages = dict(r["stages"])
        assert stages["EntropyDecode"] == "CpuScalar"
        assert stages["SecondOverlap"] == "Cuda" and stages["CropClipAndPack"] == "Cuda"
        assert stages["HostReadback"] == "CpuScalar"
        assert r["upload_ms"] > 0 and r["reconstruct_ms"] > 0 and r["readback_ms"] > 0
    finally:
        sub.close()


def test_pageable_arena_is_consumed_before_submit_returns(session, image):
    """A pageable arena goes through the session's pinned staging ring and is
    read in full before submit returns: overwriting it right after submit
    cannot change the result.  A page-locked one is copied directly."""
    img, out, want = image
    coeff = img.arena.coefficients.copy()
    a = img.arena
    arena = J.Arena(coeff, a.coefficient_offsets, a.quantizers, a.bands, a.hp_predictions, a.coded_x, a.coded_y,
                    a.planes)
    plan = J.CudaDecodePlan(arena, img.geometry, out)
    before = session.diagnostics()
    sub = session.submit(plan)
    coeff[:] = 0x7FFFFFFF            # the caller reuses its buffer at once
    try:
        sub.wait()
        assert np.array_equal(sub.readback(0), want)
    finally:
        sub.close()
    after = session.diagnostics()
    assert after["bytes_staged"] - before["bytes_staged"] >= coeff.nbytes
    pinned, keep = pinned_plan(img, out)
    before = session.diagnostics()
    got = session.decode_to_host(pinned)
    after = session.diagnostics()
    assert np.array_equal(got, want)
    assert after["bytes_staged"] - before["bytes_staged"] < coeff.nbytes   # tables only
