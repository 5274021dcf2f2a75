"""Continuous-batching decode server over resident images.

Requests (full decodes and region decodes of images whose arenas are resident
on the device) arrive on a clock.  The loop admits every request that has
arrived while there is a free launch slot and room in the device memory
budget, plans it (jxrb_request_create: window, output descriptor), and sends
the admitted requests as one batched launch (jxrb_submit_requests) on the
next session stream.  Requests that arrive while earlier batches are still on
the GPU are admitted into new batches at once, so their work overlaps on the
device; a batch's memory is returned when it completes.  Latency is arrival to
observed completion of the request's batch.
"""
from __future__ import annotations

import gc
import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import api as J


@dataclass
class ServeRequest:
    image: int                       # index into the server's resident images
    output: J.OutputFormat           # crop = region in image coordinates
    arrival: float                   # seconds after the stream starts
    kind: str = "full"               # "full", "roi" or "quarter"
    pixels: int = 0                  # output pixels
    denominator: int = 1             # 4: a quarter-resolution decode
    admitted: float = math.nan
    done: float = math.nan
    result: Optional[np.ndarray] = field(default=None, repr=False)


@dataclass
class _Batch:
    submission: J.CudaSubmission
    requests: List[ServeRequest]
    handles: List[J.Request]
    bytes: int
    slot: int


class Server:
    """Serves requests on `images` (resident on the session's device) under
    `budget_bytes` of device memory, with at most `slots` batches in flight and
    `max_batch` requests a batch."""

    def __init__(self, session: J.CudaDecoderSession, images: Sequence[J.ResidentImage], budget_bytes: int,
                 slots: int = 4, max_batch: int = 256, keep_results: bool = False):
        self.session, self.images = session, list(images)
        self.budget = int(budget_bytes)
        self.resident_bytes = sum(im.device_bytes() for im in self.images)
        if self.resident_bytes > self.budget:
            raise ValueError("resident images exceed the device memory budget")
        self.slots, self.max_batch, self.keep = slots, max_batch, keep_results
        # Each batch slot keeps a device output buffer for the batches it
        # serves: allocating every batch's output from the device's memory
        # pool cost milliseconds a batch under load, more than the host's
        # other work for it.  A slot may grow to its share of the budget.
        self.slot_share = (self.budget - self.resident_bytes) // max(1, slots)
        self._slot_free = list(range(slots))
        self._slot_buf: List = [None] * slots

    def _take_slot(self, nbytes: int):
        """A free slot whose buffer holds `nbytes`, grown in 64 MiB steps
        (never beyond the slot's share of the budget)."""
        import torch
        k = self._slot_free.pop()
        buf = self._slot_buf[k]
        if buf is None or buf.numel() < nbytes:
            size = min(max(nbytes, -(-nbytes // (64 << 20)) * (64 << 20)), max(nbytes, self.slot_share))
            self._slot_buf[k] = None
            buf = self._slot_buf[k] = torch.empty(size, dtype=torch.uint8,
                                                  device=f"cuda:{self.session.ordinal}")
        return k, buf

    @staticmethod
    def request_bytes(handle: J.Request) -> int:
        # output (256-byte aligned in the batch) and its descriptors
        return (handle.output_bytes() + 255) // 256 * 256 + 4096

    def serve(self, stream: Sequence[ServeRequest], poll_s: float = 20e-6) -> Dict:
        # The loop allocates a few small objects a request; a cyclic garbage
        # collection in the middle of it would stall every request in flight,
        # so collection waits until the stream is served.
        enabled = gc.isenabled()
        gc.disable()
        try:
            return self._serve(stream, poll_s)
        finally:
            if enabled:
                gc.enable()

    def _serve(self, stream: Sequence[ServeRequest], poll_s: float) -> Dict:
        pending = deque(sorted(stream, key=lambda r: r.arrival))
        queue: deque = deque()
        inflight: List[_Batch] = []
        used = self.resident_bytes
        peak = used
        batches = 0
        t0 = time.perf_counter()
        while pending or queue or inflight:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            progressed = False
            for b in list(inflight):
                if b.submission.is_complete():
                    t = time.perf_counter() - t0
                    b.submission.wait()
                    for i, r in enumerate(b.requests):
                        r.done = t
                        if self.keep:
                            r.result = b.submission.readback(i)
                    b.submission.close()
                    for h in b.handles:
                        h.close()
                    self._slot_free.append(b.slot)
                    used -= b.bytes
                    inflight.remove(b)
                    progressed = True
            if queue and len(inflight) < self.slots:
                batch, handles, nbytes = [], [], 0
                while queue and len(batch) < self.max_batch:
                    r = queue[0]
                    h = self.images[r.image].request(r.output, r.denominator)
                    b = self.request_bytes(h)
                    if used + nbytes + b > self.budget or (batch and nbytes + b > self.slot_share):
                        h.close()
                        break
                    queue.popleft()
                    r.admitted = time.perf_counter() - t0
                    batch.append(r)
                    handles.append(h)
                    nbytes += b
                if batch:
                    slot, buf = self._take_slot(nbytes)
                    sub = self.session.submit_requests(handles, buf.data_ptr(), buf.numel())
                    inflight.append(_Batch(sub, batch, handles, nbytes, slot))
                    used += nbytes
                    peak = max(peak, used)
                    batches += 1
                    progressed = True
            if not progressed:
                wait = poll_s
                if pending and not queue and not inflight:
                    wait = max(0.0, pending[0].arrival - (time.perf_counter() - t0))
                if wait > 0:
                    time.sleep(min(wait, 1e-3) if inflight or queue else wait)
        end = time.perf_counter() - t0
        return summarize(stream, end, batches, peak)


def summarize(stream: Sequence[ServeRequest], end: float, batches: int, peak: int) -> Dict:
    lat = np.array([r.done - r.arrival for r in stream]) * 1e3
    first = min(r.arrival for r in stream)
    span = max(r.done for r in stream) - first
    mpix = sum(r.pixels for r in stream) / 1e6
    return {"requests": len(stream), "batches": batches, "mpix": round(mpix, 3), "span_s": round(span, 4),
            "p50_ms": round(float(np.percentile(lat, 50)), 3),
            "p99_ms": round(float(np.percentile(lat, 99)), 3), "mean_ms": round(float(lat.mean()), 3),
            "mpix_per_s": round(mpix / span, 2), "requests_per_s": round(len(stream) / span, 1),
            "peak_device_bytes": int(peak), "seconds": round(end, 3)}


# ---------------------------------------------------------------------------
# the request stream of the serving benchmark
# ---------------------------------------------------------------------------
def output_for(kind: str, x: int, y: int, w: int, h: int) -> J.OutputFormat:
    C_, D, S, L = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT
    if kind == "gray16":
        return J.OutputFormat(C_["LUMA"], D["U16"], S["U16"], L["LUMA"], w, h, crop_x=x, crop_y=y)
    if kind == "rgba":
        return J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGBA"], w, h, crop_x=x, crop_y=y,
                              alpha_bit_depth=D["U8"])
    return J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], w, h, crop_x=x, crop_y=y)


def request_stream(pool: Sequence, count: int, rate: float, seed: int, roi_share: float = 0.3,
                   quarter_share: float = 0.0) -> List[ServeRequest]:
    """`count` requests with Poisson arrivals at `rate` a second (rate <= 0:
    all at once) on the images of `pool` (workloads.BatchItem): a share
    `roi_share` are region decodes of 10..50 % of the image's area, a share
    `quarter_share` quarter-resolution decodes of the whole image
    (thumbnails), the rest full decodes."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(count):
        if rate > 0:
            t += float(rng.exponential(1.0 / rate))
        i = int(rng.integers(len(pool)))
        item = pool[i]
        W, H = item.output.crop_width, item.output.crop_height
        u = rng.random()
        if u >= roi_share and u < roi_share + quarter_share:
            qw, qh = -(-W // 4), -(-H // 4)
            out.append(ServeRequest(i, output_for(item.kind, 0, 0, W, H), t, "quarter", qw * qh, 4))
            continue
        if u < roi_share:
            f = float(rng.uniform(0.1, 0.5))
            aspect = float(math.exp(rng.uniform(-0.7, 0.7)))
            w = int(min(W, max(1, round(math.sqrt(f * W * H * aspect)))))
            h = int(min(H, max(1, round(f * W * H / w))))
            x, y = int(rng.integers(0, W - w + 1)), int(rng.integers(0, H - h + 1))
            kind = "roi"
        else:
            x, y, w, h, kind = 0, 0, W, H, "full"
        out.append(ServeRequest(i, output_for(item.kind, x, y, w, h), t, kind, w * h))
    return out
