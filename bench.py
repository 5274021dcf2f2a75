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
}


def make_workload(name, rank=0, threads=None):
    import jxr_b200 as J
    threads = threads or os.cpu_count() or 8
    C_, D, S, L, A = J.COLOR, J.DEPTH, J.STORE, J.LAYOUT, J.ALPHA
    if name == "c2":
        img = J.synth(4096, 4096, quality=90, overlap=2, tile_width=16, tile_height=16, hard_tiles=0,
                      seed=2 + 1000 * rank, threads=threads)
        out = J.OutputFormat(C_["RGB"], D["U8"], S["U8"], L["RGB"], 4096, 4096)
        return img, out
    if name == "c3":
        img = J.synth(8192, 8192, content=J.CONTENT["HDR_HALF"], alpha_mode=A["SEPARATE"], scaled=0, quality=0,
                      qp=(4, 8, 16), overlap=2, alpha_overlap=0, tile_width=32, tile_height=32, hard_tiles=0,
                      seed=3 + 1000 * rank, threads=threads)
        out = J.OutputFormat(C_["RGB"], D["F16"], S["F16"], L["RGBA"], 8192, 8192, alpha_bit_depth=D["F16"],
                             nchw=1, widen_f16=1)
        return img, out
    raise SystemExit(f"unknown workload {name}")


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


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(img, out, seconds=10.0, threads=None):
    """The oracle (C restatement of the reference CPU reconstruction) on the
    host cores, on the same arena: full-image reconstructions repeated until
    about `seconds` have passed."""
    import ctypes as C
    from tests import _bridge as B, _oracle as O
    threads = threads or os.cpu_count() or 1
    planes, alpha = B.oracle_planes(img.arena, img.geometry, img.alpha_arena)
    handles = [O.PlaneHandle(p) for p in planes]
    arr = (O.JoPlane * len(handles))(*[h.s for h in handles])
    ah = O.PlaneHandle(alpha) if alpha is not None else None
    g = img.geometry
    im = O.JoImage(arr, len(handles), C.pointer(ah.s) if ah else None, g.color_format, g.chroma_centering_x,
                   g.chroma_centering_y)
    jo = B.oracle_output(g, out)
    n = O.output_bytes(jo)
    buf = np.empty(n, np.uint8)
    L = O.lib()
    runs, t0 = 0, time.perf_counter()
    while True:
        rc = L.jo_decode_image(C.byref(im), C.byref(jo), buf.ctypes.data, n, threads)
        if rc != 0:
            raise RuntimeError(f"oracle failed with {rc}")
        runs += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    mpix = out.crop_width * out.crop_height / 1e6
    return {"value": round(mpix * runs / dt, 3), "unit": "Mpix/s", "cores": threads, "kind": "port",
            "sample": f"{runs} full reconstructions of the workload's arena ({dt:.1f} s)"}, buf


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args, world, rank):
    if rank != 0:
        return
    img, out = make_workload(args.workload)
    base, _ = cpu_baseline(img, out, seconds=max(5.0, 3.0 * args.steps / max(1, args.steps)))
    # timed steps of the reference CPU path: full reconstructions of the workload
    import ctypes as C
    from tests import _bridge as B, _oracle as O
    threads = os.cpu_count() or 1
    planes, alpha = B.oracle_planes(img.arena, img.geometry, img.alpha_arena)
    handles = [O.PlaneHandle(p) for p in planes]
    arr = (O.JoPlane * len(handles))(*[h.s for h in handles])
    ah = O.PlaneHandle(alpha) if alpha is not None else None
    g = img.geometry
    im = O.JoImage(arr, len(handles), C.pointer(ah.s) if ah else None, g.color_format, g.chroma_centering_x,
                   g.chroma_centering_y)
    jo = B.oracle_output(g, out)
    n = O.output_bytes(jo)
    buf = np.empty(n, np.uint8)
    L = O.lib()
    for _ in range(args.warmup):
        L.jo_decode_image(C.byref(im), C.byref(jo), buf.ctypes.data, n, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        L.jo_decode_image(C.byref(im), C.byref(jo), buf.ctypes.data, n, threads)
    dt = time.perf_counter() - t0
    mpix = out.crop_width * out.crop_height / 1e6
    value = mpix * args.steps / dt
    line = {"metric": "recon Mpix/s", "value": round(value, 3), "unit": "Mpix/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dt * 1e3 / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded forward analysis of generated images)",
            "config": {"workload": WORKLOADS[args.workload]["desc"], "l2": "inputs larger than L2"},
            "cpu_baseline": dict(base, value=round(value, 3),
                                 sample=f"{args.steps} timed full reconstructions on {threads} threads"),
            "e2e": {"value": round(value, 3), "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    import jxr_b200 as J
    from jxr_b200 import build as jbuild
    jbuild.build()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    img, out = make_workload(args.workload, rank)
    plan = J.CudaDecodePlan(img.arena, img.geometry, out, img.alpha_arena)
    session = J.CudaDecoderSession(local)
    nbytes = plan.output_bytes()
    mpix = out.crop_width * out.crop_height / 1e6
    traffic = plan.traffic_bytes()

    # ---- device-resident throughput ------------------------------------
    res = session.resident([plan])
    dst = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    # a dedicated stream: its handle is what the kernels launch on and what
    # the CUDA events below are recorded on
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    for _ in range(args.warmup):
        res.run(dst.data_ptr(), nbytes, True, stream.cuda_stream)
    torch.cuda.synchronize(dev)
    if res.status() != 0:
        raise SystemExit("reconstruction reported an arithmetic error")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clocks:
        t_first = torch.cuda.Event(enable_timing=True)
        t_last = torch.cuda.Event(enable_timing=True)
        t_first.record(stream)
        for k in range(args.steps):
            starts[k].record(stream)
            res.run(dst.data_ptr(), nbytes, True, stream.cuda_stream)
            ends[k].record(stream)
        t_last.record(stream)
        torch.cuda.synchronize(dev)
    barrier(world)
    total_ms = t_first.elapsed_time(t_last)
    per_launch_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / args.steps
    total_ms = max_over_ranks(total_ms, world)
    ms_per_step = total_ms / args.steps
    value = world * mpix * args.steps / (total_ms / 1e3)
    launches = args.steps * res.launches(True)

    # ---- end to end through the C ABI with host buffers ------------------
    arena_pinned = torch.from_numpy(img.arena.coefficients).pin_memory()
    alpha_pinned = torch.from_numpy(img.alpha_arena.coefficients).pin_memory() if img.alpha_arena else None
    host_out = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    a_np = arena_pinned.numpy()
    e2e_plan = J.CudaDecodePlan(J.Arena(a_np, img.arena.coefficient_offsets, img.arena.quantizers, img.arena.bands,
                                        img.arena.hp_predictions, img.arena.coded_x, img.arena.coded_y,
                                        img.arena.planes),
                                img.geometry, out,
                                None if alpha_pinned is None else J.Arena(
                                    alpha_pinned.numpy(), img.alpha_arena.coefficient_offsets,
                                    img.alpha_arena.quantizers, img.alpha_arena.bands,
                                    img.alpha_arena.hp_predictions, img.alpha_arena.coded_x,
                                    img.alpha_arena.coded_y, img.alpha_arena.planes))
    e2e_steps = max(3, min(args.steps, 20))
    h2d = int(img.arena.coefficients.nbytes + (img.alpha_arena.coefficients.nbytes if img.alpha_arena else 0))
    for _ in range(2):
        sub = session.submit_into(e2e_plan, dst.data_ptr(), nbytes)
        sub.wait()
        sub.close()
    barrier(world)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sub = session.submit_into(e2e_plan, dst.data_ptr(), nbytes)
        sub.wait()
        import ctypes as C
        J.lib().jxrb_readback(sub._handle, 0, host_out.data_ptr(), nbytes)
        sub.close()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world)
    e2e_value = world * mpix * e2e_steps / e2e_s

    result = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        achieved = traffic / (per_launch_ms / 1e3) / 1e9
        line = {
            "metric": "recon Mpix/s", "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded forward analysis of generated images; reference corpus unavailable)",
            "config": {"workload": WORKLOADS[args.workload]["desc"], "global_batch": world,
                       "parallelism": f"replicas x{world}", "l2": "inputs (arena) larger than L2, no flush"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": traffic},
            "e2e": {"value": round(e2e_value, 2), "unit": "Mpix/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": int(nbytes)},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        traffic_file = ROOT / "profiles" / f"traffic_{args.workload}.txt"
        if traffic_file.exists():
            for entry in traffic_file.read_text().splitlines():
                key, _, val = entry.partition("=")
                if key.strip() == "dram_bytes_per_launch":
                    line["roofline"]["traffic"] = int(val.strip())
        if world == 1 and not args.no_cpu_baseline:
            base, ref_bytes = cpu_baseline(img, out, seconds=args.cpu_seconds)
            line["cpu_baseline"] = base
            got = dst.cpu().numpy()
            line["parity_vs_oracle"] = bool(np.array_equal(got, ref_bytes))
        result = line
        print(json.dumps(line), flush=True)
    res.close()
    session.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return result


if __name__ == "__main__":
    main()
