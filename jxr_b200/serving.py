"""Continuous-batching decode server over a catalog of images.

Requests (full, region and reduced-resolution decodes) arrive on a clock.  The
loop admits every request that has arrived while there is a free launch slot
and room in the device memory budget, plans it (jxrb_request_create: window,
output descriptor), and sends the admitted requests as one batched launch
(jxrb_submit_requests) on the next session stream.  Requests that arrive while
earlier batches are still on the GPU are admitted into new batches at once, so
their work overlaps on the device; a batch's memory is returned when it
completes.  Latency is arrival to observed completion of the request's batch.

Images are either resident for the server's life (J.ResidentImage) or kept
on the host (CatalogImage) and uploaded when a request on them is admitted --
the reference's upload cache (crates/jxr-cuda/src/upload_cache.rs:65-153)
under a budget: when the budget binds, the least recently used uploaded
images that no batch in flight references are released to make room.
"""
from __future__ import annotations

import gc
import math
import time
from collections import OrderedDict, deque
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
class CatalogImage:
    """An image of the catalog kept on the host, uploaded on demand."""
    arena: J.Arena
    geometry: J.Geometry
    alpha_arena: Optional[J.Arena] = None

    def device_bytes_estimate(self) -> int:
        """An upper bound of jxrb_image_device_bytes: the coefficients, 16 bytes
        a macroblock a plane of tables, and slack for the tile maps and
        alignment."""
        n = self.arena.coefficients.nbytes + (self.alpha_arena.coefficients.nbytes if self.alpha_arena else 0)
        mbs = self.geometry.macroblocks_x * self.geometry.macroblocks_y
        planes = len(self.arena.planes) + (1 if self.alpha_arena is not None else 0)
        return n + planes * (16 * mbs + self.geometry.macroblocks_x + self.geometry.macroblocks_y + 1024) + 4096


@dataclass
class _Batch:
    submission: J.CudaSubmission
    requests: List[ServeRequest]
    handles: List[J.Request]
    bytes: int
    slot: int
    images: List[int] = field(default_factory=list)


class Server:
    """Serves requests on `images` (resident on the session's device) under
    `budget_bytes` of device memory, with at most `slots` batches in flight and
    `max_batch` requests a batch."""

    def __init__(self, session: J.CudaDecoderSession, images: Sequence, budget_bytes: int,
                 slots: int = 4, max_batch: int = 256, keep_results: bool = False,
                 output_share: Optional[float] = None):
        self.session, self.images = session, list(images)
        self.budget = int(budget_bytes)
        self.resident_bytes = sum(im.device_bytes() for im in self.images if isinstance(im, J.ResidentImage))
        if self.resident_bytes > self.budget:
            raise ValueError("resident images exceed the device memory budget")
        self.slots, self.max_batch, self.keep = slots, max_batch, keep_results
        # Each batch slot keeps a device output buffer for the batches it
        # serves: allocating every batch's output from the device's memory
        # pool cost milliseconds a batch under load, more than the host's
        # other work for it.  A slot may grow to its share of the budget
        # (of `output_share` of what the resident images leave, when the
        # catalog also needs room for uploads).
        on_demand = any(isinstance(im, CatalogImage) for im in self.images)
        share = output_share if output_share is not None else (0.25 if on_demand else 1.0)
        # the part of the budget outputs of batches in flight may use; the
        # rest (beside the resident images) holds uploaded catalog images
        self.output_reserve = int((self.budget - self.resident_bytes) * share)
        self.cache_room = self.budget - self.resident_bytes - self.output_reserve
        self.slot_share = self.output_reserve // max(1, slots)
        self._slot_free = list(range(slots))
        self._slot_buf: List = [None] * slots
        # uploaded catalog images: index -> (resident image, device bytes), least recently used first
        self._cache: "OrderedDict[int, tuple]" = OrderedDict()
        self._cached_bytes = 0
        self._refs: Dict[int, int] = {}
        self.cache_stats = dict(uploads=0, upload_bytes=0, evictions=0, hits=0, misses=0)

    def _take_slot(self, nbytes: int):
        """A free slot whose buffer holds `nbytes`, grown in 64 MiB steps up
        to the slot's share (a larger batch gets a buffer of its own size).
        Buffers of idle slots are released when the output reserve needs the
        room; None when the buffers of the batches in flight leave too little,
        until one of them finishes."""
        import torch
        k = self._slot_free[-1]
        buf = self._slot_buf[k]
        if buf is None or buf.numel() < nbytes:
            size = max(nbytes, min(-(-nbytes // (64 << 20)) * (64 << 20), self.slot_share))
            held = sum(b.numel() for j, b in enumerate(self._slot_buf) if b is not None and j != k)
            if held + size > self.output_reserve:
                for j in self._slot_free:
                    if j != k and self._slot_buf[j] is not None:
                        held -= self._slot_buf[j].numel()
                        self._slot_buf[j] = None
            if held + size > self.output_reserve:
                return None
            self._slot_buf[k] = None
            buf = self._slot_buf[k] = torch.empty(size, dtype=torch.uint8, device=f"cuda:{self.session.ordinal}")
        self._slot_free.pop()
        return k, buf

    def device_bytes(self) -> int:
        """What the server holds on the device: resident and uploaded images
        and the batch slots' output buffers."""
        return self.resident_bytes + self._cached_bytes + sum(b.numel() for b in self._slot_buf if b is not None)

    def _resident(self, i: int, room: int, pinned: set):
        """Image `i` on the device, uploaded if it is not; `room`: the bytes
        the budget keeps for uploaded images.  Releases the least recently
        used uploaded images no batch references (nor `pinned`, the batch
        being built) to make room.  None when it does not fit."""
        im = self.images[i]
        if isinstance(im, J.ResidentImage):
            return im
        if i in self._cache:
            self._cache.move_to_end(i)
            self.cache_stats["hits"] += 1
            return self._cache[i][0]
        need = im.device_bytes_estimate()
        if need > room:
            return None
        while self._cached_bytes + need > room:
            victim = next((k for k in self._cache if self._refs.get(k, 0) == 0 and k not in pinned), None)
            if victim is None:
                return None
            handle, nbytes = self._cache.pop(victim)
            handle.close()
            self._cached_bytes -= nbytes
            self.cache_stats["evictions"] += 1
        handle = self.session.upload(im.arena, im.geometry, im.alpha_arena)
        nbytes = handle.device_bytes()
        self._cache[i] = (handle, nbytes)
        self._cached_bytes += nbytes
        self.cache_stats["misses"] += 1
        self.cache_stats["uploads"] += 1
        self.cache_stats["upload_bytes"] += im.arena.coefficients.nbytes + (
            im.alpha_arena.coefficients.nbytes if im.alpha_arena is not None else 0)
        return handle

    def release(self):
        """Release every uploaded catalog image."""
        for handle, _ in self._cache.values():
            handle.close()
        self._cache.clear()
        self._cached_bytes = 0

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
        used = 0                            # outputs of the batches in flight
        peak = self.device_bytes()
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
                    for k in b.images:
                        self._refs[k] -= 1
                    self._slot_free.append(b.slot)
                    used -= b.bytes
                    inflight.remove(b)
                    progressed = True
            if queue and len(inflight) < self.slots:
                batch, handles, nbytes, pinned = [], [], 0, set()
                while queue and len(batch) < self.max_batch:
                    r = queue[0]
                    image = self._resident(r.image, self.cache_room, pinned)
                    if image is None:
                        break
                    pinned.add(r.image)
                    h = image.request(r.output, r.denominator)
                    b = self.request_bytes(h)
                    if used + nbytes + b > self.output_reserve or (batch and nbytes + b > self.slot_share):
                        h.close()
                        break
                    queue.popleft()
                    r.admitted = time.perf_counter() - t0
                    batch.append(r)
                    handles.append(h)
                    nbytes += b
                taken = self._take_slot(nbytes) if batch else None
                if batch and taken is None:
                    # no room for the batch's outputs yet: back to the queue
                    for h in handles:
                        h.close()
                    for r in reversed(batch):
                        r.admitted = math.nan
                        queue.appendleft(r)
                    batch = []
                if batch:
                    slot, buf = taken
                    sub = self.session.submit_requests(handles, buf.data_ptr(), buf.numel())
                    images = [r.image for r in batch]
                    for k in images:
                        self._refs[k] = self._refs.get(k, 0) + 1
                    inflight.append(_Batch(sub, batch, handles, nbytes, slot, images))
                    used += nbytes
                    peak = max(peak, self.device_bytes())
                    batches += 1
                    progressed = True
            if not progressed:
                wait = poll_s
                if pending and not queue and not inflight:
                    wait = max(0.0, pending[0].arrival - (time.perf_counter() - t0))
                if wait > 0:
                    time.sleep(min(wait, 1e-3) if inflight or queue else wait)
        end = time.perf_counter() - t0
        out = summarize(stream, end, batches, peak)
        if any(isinstance(im, CatalogImage) for im in self.images):
            out["cache"] = dict(self.cache_stats)
        return out


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


def zipf_popularity(n: int, exponent: float = 1.1, seed: int = 0) -> np.ndarray:
    """Request probabilities of `n` images ranked by a Zipf law, the ranks
    shuffled over the images."""
    p = 1.0 / np.arange(1, n + 1) ** exponent
    np.random.default_rng(seed).shuffle(p)
    return p / p.sum()


def request_stream(pool: Sequence, count: int, rate: float, seed: int, roi_share: float = 0.3,
                   quarter_share: float = 0.0, popularity: Optional[np.ndarray] = None) -> List[ServeRequest]:
    """`count` requests with Poisson arrivals at `rate` a second (rate <= 0:
    all at once) on the images of `pool` (workloads.BatchItem), uniformly or
    with the probabilities `popularity`: a share `roi_share` are region
    decodes of 10..50 % of the image's area, a share `quarter_share`
    quarter-resolution decodes of the whole image (thumbnails), the rest full
    decodes."""
    rng = np.random.default_rng(seed)
    cdf = None if popularity is None else np.cumsum(popularity)
    t = 0.0
    out = []
    for _ in range(count):
        if rate > 0:
            t += float(rng.exponential(1.0 / rate))
        i = int(rng.integers(len(pool))) if cdf is None else min(int(np.searchsorted(cdf, rng.random() * cdf[-1])),
                                                                    len(pool) - 1)
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
