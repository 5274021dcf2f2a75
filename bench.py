"""Benchmark of the B200 JPEG XR reconstruction engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c3|c4] [--impl engine|reference]

A step is one reconstruction of the workload's coefficient arena(s) into the
output surface.  `value` is reconstruction throughput in output Mpix/s with the
arena resident in HBM (device-timed with CUDA events on the launching stream,
max over ranks); `e2e` is the same metric through the public C ABI with host
buffers: every step uploads the arena from pinned host memory, reconstructs,
and reads the pixels back.  Inputs (201 MB arena for c2) exceed the 126 MB L2,
so no flush is needed between steps.

Default workload (c2): one 4096x4096 8-bit RGB image, quality 90, two-level
overlap, 256x256 soft tiles, decoded to U8 RGB in device memory.
c3: one 8192x8192 half-float RGB image with a separate alpha plane, decoded to
F32 RGBA NCHW.  c4: 256 mixed images (sizes log-uniform 64..2048; 50 % RGB8
4:2:0, 30 % 16-bit gray lossless, 20 % RGBA8), reconstructed by one persistent
batched launch sequence replayed from a CUDA graph, beside the same images
reconstructed by one plain launch sequence per image.

Before timing, the launch shape (CTAs per SM of each tile kernel, second
stream for edge tiles) is chosen by jxr_b200.autotune on the workload itself;
the timed steps replay the captured CUDA graph of one run.

--impl reference times the reference's CPU reconstruction -- the C
restatement of it under oracle/ (the Rust reference has no toolchain here) --
on the host's cores for the same workload and metric.

Multi-GPU (torchrun): replicas, one image per rank, no data-path collective;
value = all ranks' pixels / max rank time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "c2": dict(desc="4096x4096 RGB8 q90, two-level overlap, 256x256 soft tiles -> U8 RGB (device)",
               width=4096, height=4096),
    "c3": dict(desc="8192x8192 RGB half + separate alpha, QP 4/8/16, two-level overlap, 512x512 tiles, "
                    "frequency bitstream -> F32 RGBA NCHW (device)", width=8192, height=8192),
    "c3_4096": dict(desc="4096x4096 RGB half + separate alpha, QP 4/8/16, two-level overlap, 512x512 tiles "
                         "-> F32 RGBA NCHW (device): the C3 configuration at a quarter of its area, a small "
                         "case for profiling captures", width=4096, height=4096),
    "c4": dict(desc="256 mixed images, sizes log-uniform 64..2048 (x16): 50% RGB8 4:2:0 q75 overlap 1, "
                    "30% gray16 lossless overlap 0, 20% RGBA8 q85 overlap 2, tiles 128-512 -> device "
                    "(persistent batched launch from a CUDA graph vs per-image launches)"),
    "c5": dict(desc="serving: Poisson stream of 20000 requests on 32 resident images of the c4 mix with sizes "
                    "log-uniform 128..4096, 30% region decodes (10-50% of the area), 20% quarter-resolution "
                    "thumbnails, 40 GB device budget, "
                    "continuous batching; throughput saturated and p50/p99 at three offered loads; then the same "
                    "on a catalog of twice the budget (Zipf popularity), uploaded on admission"),
}


def config_of(workload, world, items=None):
    """The `config` object of the bench line: the same dict in both arms."""
    cfg = {"workload": WORKLOADS[workload]["desc"], "global_batch": world, "parallelism": f"replicas x{world}",
           "l2": "inputs (arena) larger than L2, no flush"}
    if workload == "c4":
        cfg["images"] = 256
    if workload == "c5":
        cfg.update({"step": "one request", "l2": "resident arenas larger than L2",
                    "timing": "host clock of the serving loop (arrival to observed completion)"})
    return cfg


def items_in_child(workload, threads):
    """The workload's inputs, generated by a child process (which maps the
    generator library) and read back from a file, so that this process maps
    no library of the engine package."""
    import tempfile
    from jxr_b200 import workloads as W
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "items.pkl")
        subprocess.run([sys.executable, str(ROOT / "bench.py"), "--workload", workload, "--export-items", path,
                        "--threads", str(threads)], check=True)
        return W.load(path)


def make_items(name, rank=0, threads=None):
    """The workload as a list of (synthetic image, output format)."""
    if name == "c4":
        from jxr_b200 import workloads as W
        return [(it.image, it.output) for it in W.mixed_batch(256, seed=4 + 1000 * rank, threads=threads)]
    return [make_workload(name, rank, threads)]


def make_workload(name, rank=0, threads=None):
    from jxr_b200 import workloads as W
    if name not in ("c2", "c3", "c3_4096"):
        raise SystemExit(f"unknown workload {name}")
    return W.single_image(name, 1000 * rank, threads)


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device_index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        time.sleep(0.15)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        time.sleep(0.15)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


KERNEL_SOURCES = ("recon_kernel.cu", "lifting.cuh", "engine.h")


def kernel_source_digest(read=None) -> str:
    """sha256 over the reconstruction kernel's sources in a fixed order, with
    comments and runs of whitespace removed, so that only a change of code
    makes a captured figure stale.  `read(name)` returns a source's text
    (default: the working tree's)."""
    import hashlib
    import re
    read = read or (lambda name: (ROOT / "jxr_b200" / "csrc" / name).read_text())
    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        code = re.sub(r"/\*.*?\*/", " ", read(name), flags=re.S)
        code = re.sub(r"//[^\n]*", " ", code)
        h.update(" ".join(code.split()).encode())
    return h.hexdigest()


def captured_traffic(workload: str) -> dict:
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary `profiles/traffic_<workload>.txt`, used only while the digest it
    records matches the kernel sources built now; otherwise traffic is null
    and the line says the capture is stale."""
    path = ROOT / "profiles" / f"traffic_{workload}.txt"
    if not path.exists():
        return {"traffic": None}
    fields = {}
    for entry in path.read_text().splitlines():
        key, sep, val = entry.partition("=")
        if sep and not key.lstrip().startswith("#"):
            fields[key.strip()] = val.strip()
    if fields.get("kernel_source_sha256") != kernel_source_digest():
        return {"traffic": None, "traffic_note": "ncu capture predates the current kernel sources"}
    return {"traffic": int(fields["dram_bytes_per_launch"]),
            "traffic_note": "ncu capture of this kernel source: " + fields.get("capture", "")}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class OracleImage:
    """One image prepared for the oracle (the checker; C restatement of the
    reference's CPU reconstruction)."""

    def __init__(self, img, out):
        import ctypes as C
        from tests import _bridge as B, _oracle as O
        planes, alpha = B.oracle_planes(img.arena, img.geometry, img.alpha_arena)
        self.handles = [O.PlaneHandle(p) for p in planes]
        self.arr = (O.JoPlane * len(self.handles))(*[h.s for h in self.handles])
        self.ah = O.PlaneHandle(alpha) if alpha is not None else None
        g = img.geometry
        self.im = O.JoImage(self.arr, len(self.handles), C.pointer(self.ah.s) if self.ah else None, g.color_format,
                            g.chroma_centering_x, g.chroma_centering_y)
        self.jo = B.oracle_output(g, out)
        self.n = O.output_bytes(self.jo)
        self.buf = np.empty(self.n, np.uint8)
        self.mpix = out.crop_width * out.crop_height / 1e6

    def run(self, threads):
        import ctypes as C
        from tests import _oracle as O
        rc = O.lib().jo_decode_image(C.byref(self.im), C.byref(self.jo), self.buf.ctypes.data, self.n, threads)
        if rc != 0:
            raise RuntimeError(f"oracle failed with {rc}")


def cpu_baseline(items, seconds=10.0, threads=None):
    """The oracle on the host cores over the workload's images, repeated
    until about `seconds` have passed; returns the baseline and the oracle's
    output bytes of every image."""
    threads = threads or os.cpu_count() or 1
    oracles = [OracleImage(img, out) for img, out in items]
    passes, images, mpix, t0 = 0, 0, 0.0, time.perf_counter()
    while True:
        for o in oracles:
            o.run(threads)
            images += 1
            mpix += o.mpix
            if passes and time.perf_counter() - t0 >= seconds:
                break
        passes += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    what = "full reconstructions of the workload's arena" if len(items) == 1 else "image reconstructions"
    return {"value": round(mpix / dt, 3), "unit": "Mpix/s", "cores": threads, "kind": "port",
            "sample": f"{images} {what} ({dt:.1f} s)"}, [o.buf for o in oracles]


def cpu_single_thread(items, seconds=5.0):
    """The oracle on one host thread: bands of the single image, or the
    batch's images in turn, until about `seconds` have passed."""
    if len(items) == 1:
        img, out = items[0]
        units = band_items(img, out, max(1, img.geometry.macroblocks_y // 16), 16)
        what = f"bands of {units[0][0].geometry.macroblocks_y} macroblock rows of the image"
    else:
        units, what = items, "images of the batch in turn"
    oracles = [OracleImage(i, o) for i, o in units]
    done, mpix, t0 = 0, 0.0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        o = oracles[done % len(oracles)]
        o.run(1)
        done += 1
        mpix += o.mpix
    dt = time.perf_counter() - t0
    return {"value": round(mpix / dt, 3), "unit": "Mpix/s", "cores": 1, "kind": "port",
            "sample": f"{done} {what} ({dt:.1f} s)"}


_REPLICAS = None


def dist_setup(args):
    """Join the torchrun process group (one rank per GPU, replicas)."""
    global _REPLICAS
    from jxr_b200 import replicas
    _REPLICAS = replicas.init()
    return _REPLICAS.world, _REPLICAS.rank, _REPLICAS.local


def max_over_ranks(value, world):
    return value if world == 1 else _REPLICAS.max(value)


def sum_over_ranks(value, world):
    return value if world == 1 else _REPLICAS.sum(value)


def barrier(world):
    if world > 1:
        _REPLICAS.barrier()


def band_items(img, out, rows, count):
    """`count` horizontal bands of `rows` macroblock rows of one image (at
    least one, at most the image's), each a region decode (the window treated
    as a plane, cropped to the band)."""
    import dataclasses
    g = img.geometry
    rows = max(1, min(rows, g.macroblocks_y))
    starts = np.linspace(0, g.macroblocks_y - rows, num=max(1, count)).astype(int)
    bands = []
    for y0 in dict.fromkeys(int(v) for v in starts):
        wg = dataclasses.replace(g, macroblock_origin_y=g.macroblock_origin_y + y0, macroblocks_y=rows)
        wo = dataclasses.replace(out, crop_y=0, crop_height=min(16 * rows, out.crop_height - 16 * y0))
        bands.append((dataclasses.replace(img, geometry=wg), wo))
    return bands


def run_reference(args, world, rank):
    """The reference arm: the reference's CPU reconstruction path (its C
    restatement under oracle/; the Rust reference has no toolchain here) on all
    host cores, same workload and metric.  A step is a bounded sample of the
    workload sized so that warm-up plus timed steps take about two minutes:
    a band of macroblock rows of the single-image workloads, the next image
    of the mixed batch.  The inputs come from a child process: this process
    maps the oracle and no library of the engine package."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    items = items_in_child(args.workload, threads)
    per_step_s = max(0.005, 120.0 / (args.steps + args.warmup))
    if len(items) == 1:
        img, out = items[0]
        whole = OracleImage(img, out)
        t = time.perf_counter()
        whole.run(threads)
        full_s = max(1e-4, time.perf_counter() - t)
        bands = band_items(img, out, int(img.geometry.macroblocks_y * per_step_s / full_s), 8)
        oracles = [OracleImage(i, o) for i, o in bands]
        rows = bands[0][0].geometry.macroblocks_y
        sample = (f"bands of {rows} of the image's {img.geometry.macroblocks_y} macroblock rows "
                  f"({oracles[0].mpix:.3f} Mpix each)")
    else:
        oracles = [OracleImage(i, o) for i, o in items]
        sample = "one image of the batch per step, cycling"
    for k in range(args.warmup):
        oracles[k % len(oracles)].run(threads)
    mpix = 0.0
    t0 = time.perf_counter()
    for k in range(args.steps):
        o = oracles[k % len(oracles)]
        o.run(threads)
        mpix += o.mpix
    dt = time.perf_counter() - t0
    value = mpix / dt
    line = {"metric": "recon Mpix/s", "value": round(value, 3), "unit": "Mpix/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dt * 1e3 / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded forward analysis of generated images; reference corpus unavailable)",
            "config": config_of(args.workload, args.gpus),
            "cpu_baseline": {"value": round(value, 3), "unit": "Mpix/s", "cores": threads, "kind": "port",
                             "sample": f"{args.steps} timed steps, each {sample}, {threads} threads"},
            "e2e": {"value": round(value, 3), "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def pinned_plans(items):
    """Plans whose coefficient arrays live in pinned host memory (the e2e leg)."""
    import torch
    import jxr_b200 as J
    keep, plans, h2d = [], [], 0

    def pinned(a):
        if a is None:
            return None
        t = torch.from_numpy(a.coefficients).pin_memory()
        keep.append(t)
        return J.Arena(t.numpy(), a.coefficient_offsets, a.quantizers, a.bands, a.hp_predictions, a.coded_x,
                       a.coded_y, a.planes)

    for img, out in items:
        plans.append(J.CudaDecodePlan(pinned(img.arena), img.geometry, out, pinned(img.alpha_arena)))
        h2d += img.arena.coefficients.nbytes + (img.alpha_arena.coefficients.nbytes if img.alpha_arena else 0)
    return plans, keep, int(h2d)


def timed_runs(fn, steps, stream, dev):
    """Device time of `steps` calls of fn(): (total ms between two events
    around the calls, mean ms between the events bracketing each call).  The
    two come from separate passes: events between the calls cost about 5 us a
    step on the stream, so the total is taken without them."""
    import torch
    first = torch.cuda.Event(enable_timing=True)
    last = torch.cuda.Event(enable_timing=True)
    first.record(stream)
    for _ in range(steps):
        fn()
    last.record(stream)
    torch.cuda.synchronize(dev)
    total = first.elapsed_time(last)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for k in range(steps):
        starts[k].record(stream)
        fn()
        ends[k].record(stream)
    torch.cuda.synchronize(dev)
    return total, sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / steps


def run_serving(args, world, rank, local):
    """c5: the continuous-batching server (jxr_b200.serving) on resident
    images.  Latency and throughput are host-clock figures of the serving loop
    (arrival to observed completion); each rank serves its own request stream
    (replicas)."""
    import torch
    import jxr_b200 as J
    from jxr_b200 import serving, workloads as W
    from jxr_b200 import build as jbuild
    jbuild.build()
    torch.cuda.set_device(local)
    pool = W.mixed_batch(32, seed=5 + 1000 * rank, lo=128, hi=4096)
    session = J.CudaDecoderSession(local)
    images = [session.upload(it.image.arena, it.image.geometry, it.image.alpha_arena) for it in pool]
    server = serving.Server(session, images, budget_bytes=40 * 10**9, slots=4, max_batch=256)
    count = 20000
    roi, quarter = 0.3, 0.2
    # warm-up: a saturated stream long enough that the device memory pool
    # reaches the peak of four batches in flight (its growth, mapping fresh
    # memory, would otherwise land in the timed stream)
    warm = 2000
    server.serve(serving.request_stream(pool, warm, 0.0, seed=99, roi_share=roi, quarter_share=quarter))
    before = session.diagnostics()
    barrier(world)
    with ClockSampler(local) as clocks:
        sat = server.serve(serving.request_stream(pool, count, 0.0, seed=1 + rank, roi_share=roi,
                                                  quarter_share=quarter))
    launches = session.diagnostics()["kernel_launches"] - before["kernel_launches"]
    loads = []
    for frac in (0.25, 0.5, 0.8):
        rate = frac * sat["requests_per_s"]
        st = server.serve(serving.request_stream(pool, count, rate, seed=10 + rank, roi_share=roi,
                                                 quarter_share=quarter))
        loads.append(dict(offered_requests_per_s=round(rate, 1), offered_fraction=frac, **st))
    # a catalog larger than the budget: every image listed many times (the
    # copies share the generated host arenas, each its own upload), requests
    # spread over them by a Zipf law; images are uploaded on admission and
    # the least recently used idle ones released when the budget binds
    budget = 40 * 10**9
    per_copy = sum(serving.CatalogImage(it.image.arena, it.image.geometry, it.image.alpha_arena)
                   .device_bytes_estimate() for it in pool)
    copies = max(2, -(-2 * budget // per_copy))
    catalog = [serving.CatalogImage(it.image.arena, it.image.geometry, it.image.alpha_arena) for it in pool] * copies
    cpool = list(pool) * copies
    popularity = serving.zipf_popularity(len(catalog), 1.1, seed=21)
    cserver = serving.Server(session, catalog, budget_bytes=budget, slots=4, max_batch=256)
    cserver.serve(serving.request_stream(cpool, warm, 0.0, seed=97, roi_share=roi, quarter_share=quarter,
                                         popularity=popularity))
    csat = cserver.serve(serving.request_stream(cpool, count, 0.0, seed=31 + rank, roi_share=roi,
                                                quarter_share=quarter, popularity=popularity))
    cloads = []
    for frac in (0.25, 0.5, 0.8):
        rate = frac * csat["requests_per_s"]
        st = cserver.serve(serving.request_stream(cpool, count, rate, seed=40 + rank, roi_share=roi,
                                                  quarter_share=quarter, popularity=popularity))
        cloads.append(dict(offered_requests_per_s=round(rate, 1), offered_fraction=frac, **st))
    catalog_stats = {"images": len(catalog), "catalog_bytes": int(per_copy * copies), "budget_bytes": budget,
                     "cache_room_bytes": cserver.cache_room, "output_reserve_bytes": cserver.output_reserve,
                     "popularity": "Zipf 1.1 over the catalog", "saturated": csat, "loads": cloads}
    cserver.release()
    # end to end: every output read back to host memory
    e2e_stream = serving.request_stream(pool, 2000, 0.0, seed=7 + rank, roi_share=roi, quarter_share=quarter)
    keep = serving.Server(session, images, budget_bytes=40 * 10**9, slots=4, max_batch=256, keep_results=True)
    # warm-up: the server's output and pinned readback buffers grow to size
    keep.serve(serving.request_stream(pool, warm, 0.0, seed=98, roi_share=roi, quarter_share=quarter))
    e2e = keep.serve(e2e_stream)
    d2h = sum(r.result.nbytes for r in e2e_stream)
    span = max_over_ranks(sat["span_s"], world)
    total_mpix = sum_over_ranks(sat["mpix"], world)
    value = total_mpix / span
    result = None
    if rank == 0:
        line = {"metric": "recon Mpix/s", "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world,
                "steps": count, "warmup": warm, "ms_per_step": round(1e3 / sat["requests_per_s"], 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
                "data": "synthetic (seeded forward analysis of generated images; reference corpus unavailable)",
                "config": config_of("c5", world),
                "serving": {"saturated": sat, "loads": loads, "resident_bytes": server.resident_bytes,
                            "budget_bytes": server.budget, "catalog": catalog_stats},
                "e2e": {"value": e2e["mpix_per_s"], "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": int(d2h // len(e2e_stream)),
                        "note": "arenas resident (upload cache); every output read back"},
                "gpu_launches": int(launches), "clocks": clocks.summary()}
        # parity: a sample of served requests against the oracle
        if not args.no_cpu_baseline:
            from tests._bridge import oracle_decode
            import dataclasses
            ok = True
            for r in e2e_stream[:64]:
                img = pool[r.image].image
                h = images[r.image].request(r.output, r.denominator)
                ox, oy, wx, wy = h.window()
                g = dataclasses.replace(img.geometry, macroblock_origin_x=ox, macroblock_origin_y=oy,
                                        macroblocks_x=wx, macroblocks_y=wy)
                d, c = r.denominator, r.output
                x0, y0 = c.crop_x // d, c.crop_y // d
                x1, y1 = -(-(c.crop_x + c.crop_width) // d), -(-(c.crop_y + c.crop_height) // d)
                o = dataclasses.replace(c, crop_x=x0 - 16 // d * ox, crop_y=y0 - 16 // d * oy, crop_width=x1 - x0,
                                        crop_height=y1 - y0)
                rc, ref = oracle_decode(img.arena, g, o, img.alpha_arena, threads=os.cpu_count() or 8,
                                        denominator=d)
                ok &= rc == 0 and bool(np.array_equal(ref, r.result))
            line["parity_vs_oracle"] = ok
        result = line
    for im in images:
        im.close()
    session.close()
    return result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="default launch shape instead of the autotuner's")
    ap.add_argument("--no-sub", action="store_true", help="the headline workload only (no c3/c4/c5 sub-objects)")
    ap.add_argument("--export-items", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--threads", type=int, default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.export_items:
        # the reference arm's input generation, in a process of its own
        from jxr_b200 import build as jbuild, workloads as W
        jbuild.build_synth()
        W.export(make_items(args.workload, threads=args.threads), args.export_items)
        return
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    if args.workload == "c5":
        line = run_serving(args, world, rank, local)
    else:
        line = run_images(args, args.workload, args.steps, world, rank, local)
        # the default run also carries the other configurations' figures
        # (single GPU only: the scaling runs time the headline workload)
        if world == 1 and args.workload == "c2" and not args.no_sub:
            sub = {}
            for w in ("c3", "c4"):
                sub[w] = summarize(run_images(args, w, min(args.steps, 20 if w == "c3" else 50), world, rank,
                                              local))
            sub["c5"] = summarize(run_serving(args, world, rank, local))
            line["workloads"] = sub
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


SUMMARY_KEYS = ("value", "unit", "ms_per_step", "steps", "config", "roofline", "e2e", "per_image", "serving",
                "cpu_baseline", "cpu_baseline_single_thread", "parity_vs_oracle", "gpu_launches", "clocks",
                "launch_shape")


def summarize(line):
    """The parts of a workload's line kept as a sub-object of the default line."""
    return None if line is None else {k: line[k] for k in SUMMARY_KEYS if k in line}


def run_images(args, workload, steps, world, rank, local):
    """The engine arm for the image workloads (c2, c3, c4): device-resident
    throughput, per-image launches (c4), end to end through the C ABI, the
    roofline, the CPU baselines and parity against the oracle.  Returns rank
    0's line (None elsewhere)."""
    import torch
    import jxr_b200 as J
    from jxr_b200 import autotune
    from jxr_b200 import build as jbuild
    jbuild.build()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    items = make_items(workload, rank)
    plans = [J.CudaDecodePlan(img.arena, img.geometry, out, img.alpha_arena) for img, out in items]
    session = J.CudaDecoderSession(local)
    mpix = sum(out.crop_width * out.crop_height for _, out in items) / 1e6
    traffic = sum(p.traffic_bytes() for p in plans)
    batch = len(items) > 1

    # ---- device-resident throughput ------------------------------------
    res = session.resident(plans)
    nbytes = res.output_bytes()
    dst = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    # a dedicated stream: its handle is what the kernels launch on and what
    # the CUDA events below are recorded on
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    res.run(dst.data_ptr(), nbytes, True, stream.cuda_stream)
    torch.cuda.synchronize(dev)
    tuning = None
    if not args.no_tune:
        tuning = autotune.tune(res, plans, dst.data_ptr(), nbytes, stream, batched=True)
    # the timed launch sequence: one run captured as a CUDA graph, replayed
    res.capture(dst.data_ptr(), nbytes, True)
    for _ in range(args.warmup):
        res.replay(stream.cuda_stream)
    torch.cuda.synchronize(dev)
    if res.status() != 0:
        raise SystemExit("reconstruction reported an arithmetic error")
    barrier(world)
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clocks:
        # nvidia-smi samples every 100 ms and a timed region of a few steps is
        # shorter than that: the sampler also covers about a second of the
        # same replays run untimed right before it
        soak_until = time.perf_counter() + 1.0
        while time.perf_counter() < soak_until:
            for _ in range(10):
                res.replay(stream.cuda_stream)
            torch.cuda.synchronize(dev)
        total_ms, per_launch_ms = timed_runs(lambda: res.replay(stream.cuda_stream), steps, stream, dev)
    barrier(world)
    total_ms = max_over_ranks(total_ms, world)
    ms_per_step = total_ms / steps
    value = world * mpix * steps / (total_ms / 1e3)
    launches = steps * res.launches(True)

    # ---- the same images, one plain launch sequence per image -------------
    per_image = None
    if batch:
        pi_steps = max(3, steps // 20)
        for _ in range(args.warmup):
            res.run(dst.data_ptr(), nbytes, False, stream.cuda_stream)
        torch.cuda.synchronize(dev)
        barrier(world)
        pi_ms, _ = timed_runs(lambda: res.run(dst.data_ptr(), nbytes, False, stream.cuda_stream), pi_steps,
                              stream, dev)
        pi_ms = max_over_ranks(pi_ms, world)
        pi_value = world * mpix * pi_steps / (pi_ms / 1e3)
        per_image = {"value": round(pi_value, 2), "unit": "Mpix/s", "ms_per_step": round(pi_ms / pi_steps, 4),
                     "steps": pi_steps, "launches_per_step": res.launches(False),
                     "batched_over_per_image": round(value / pi_value, 3)}
        # leave the batched output in dst for the parity check below
        res.replay(stream.cuda_stream)
        torch.cuda.synchronize(dev)

    # ---- end to end through the C ABI with host buffers ------------------
    e2e_plans, _pins, h2d = pinned_plans(items)
    host_out = torch.empty(nbytes + 256 * len(plans), dtype=torch.uint8).pin_memory()
    offsets = np.cumsum([0] + [p.output_bytes() for p in plans])
    # two device outputs, so that step k+1 (upload, reconstruction) runs on
    # its own stream while step k's result is read back: the copy engines
    # move both directions at once, as a streaming caller would have them
    e2e_dst = [torch.empty(nbytes, dtype=torch.uint8, device=dev) for _ in range(2)]
    e2e_steps = max(3, min(steps, 20 if not batch else 5))

    use_plans = [e2e_plans]

    def e2e_submit(k):
        dst = e2e_dst[k % 2].data_ptr()
        return session.submit_batch(use_plans[0], dst, nbytes) if batch else \
            session.submit_into(use_plans[0][0], dst, nbytes)

    region = []   # bytes of the output region to read back (the outputs with their alignment gaps)

    def e2e_finish(sub):
        sub.wait()
        if not region:
            region.append(sub.output_offsets()[-1] + int(offsets[-1] - offsets[-2]))
        sub.readback_all(host_out.data_ptr(), region[0])
        sub.close()

    def e2e_run(steps):
        prev = None
        for k in range(steps):
            sub = e2e_submit(k)
            if prev is not None:
                e2e_finish(prev)
            prev = sub
        e2e_finish(prev)

    e2e_run(2)
    barrier(world)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e2e_run(e2e_steps)
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world)
    e2e_value = world * mpix * e2e_steps / e2e_s
    d2h = int(region[0])
    # the same from the generator's pageable arenas: the library stages them
    # through its pinned ring
    use_plans[0] = plans
    e2e_run(2)
    barrier(world)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e2e_run(e2e_steps)
    pageable_s = max_over_ranks(time.perf_counter() - t0, world)
    pageable_value = world * mpix * e2e_steps / pageable_s

    result = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        achieved = traffic / (per_launch_ms / 1e3) / 1e9
        line = {
            "metric": "recon Mpix/s", "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded forward analysis of generated images; reference corpus unavailable)",
            "config": config_of(workload, world),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": traffic},
            "e2e": {"value": round(e2e_value, 2), "unit": "Mpix/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "note": "pinned host arena -> device -> pinned host every step; two steps in flight",
                    "pageable_arena": {"value": round(pageable_value, 2), "unit": "Mpix/s",
                                       "note": "same, arenas in pageable memory (staged by the library's pinned ring)"}},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        if batch:
            line["per_image"] = per_image
        if tuning is not None:
            line["launch_shape"] = {k: tuning[k] for k in ("blocks_per_sm", "side_stream", "source")}
        line["roofline"].update(captured_traffic(workload))
        if world == 1 and not args.no_cpu_baseline:
            base, ref_bytes = cpu_baseline(items, seconds=args.cpu_seconds)
            line["cpu_baseline"] = base
            line["cpu_baseline_single_thread"] = cpu_single_thread(items, seconds=min(args.cpu_seconds, 5.0))
            got = dst.cpu().numpy()
            ok, at = True, 0
            for p, ref in zip(plans, ref_bytes):
                at = (at + 255) // 256 * 256        # resident outputs: plan order, 256-byte aligned
                n = p.output_bytes()
                ok &= bool(np.array_equal(got[at:at + n], ref))
                at += n
            line["parity_vs_oracle"] = ok
        result = line
    res.close()
    session.close()
    return result


if __name__ == "__main__":
    main()
