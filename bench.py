#!/usr/bin/env python
"""bench.py -- 1M-Gaussian fwd+bwd views/s on B200: batched vs plain per view.

Workload (default): 1,048,576 Gaussians, SH degree 3, 16 cameras on a
radius-3 sphere with resolutions drawn from {320x240, 640x480, 1280x720,
1920x1080}, tile size and pixels per lane autotuned, L2 loss against a
seeded U[0,1] target, forward + hand-written backward to all parameters.  One step = the whole batch of
views through forward + backward; `value` is whole-job views/s of the
batched path with inputs resident in HBM.  The plain per-view path (the same
kernels, one view per call) is timed beside it.

Launch: python bench.py [--gpus N --steps K --warmup W]; for N > 1 under
torchrun, every rank renders its own 16 cameras of the same scene (weak
scaling, no data-path collective); time = max over ranks.
`--impl reference` times the CPU restatement of the reference algorithm
(oracle, all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "del-splat_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "1M-Gaussian 1080p fwd+bwd views/s: batched vs plain per-view (1 B200)"
UNIT = "views/s"


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region.  NVML is polled every `period_s` from a thread of this process,
    so even a region of ~100 ms gets tens of samples; without NVML,
    `nvidia-smi -lms 200` runs beside the region instead.  Only reads the
    GPU's state."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits (nvml.h nvmlClocksEventReason*)
    REASON_BITS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
                   0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device: int, period_s: float = 0.005):
        self.dev = device
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm MHz, max sm MHz, reason bits)
        self.stop = threading.Event()
        self.source = None

    def _bus_id(self):
        pr = torch.cuda.get_device_properties(self.dev)
        return f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"

    def _start_nvml(self):
        import pynvml
        pynvml.nvmlInit()
        h = pynvml.nvmlDeviceGetHandleByPciBusId(self._bus_id())
        mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons

        def poll():
            while True:
                self.samples.append((pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM), mx, int(get_reasons(h))))
                if self.stop.wait(self.period):
                    return

        self.nvml = pynvml
        self.t = threading.Thread(target=poll, daemon=True)
        self.t.start()
        self.source = "nvml"

    def __enter__(self):
        try:
            self._start_nvml()
            return self
        except Exception:  # no NVML on this host: fall back to nvidia-smi
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self._bus_id(), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.source = "nvidia-smi"
        except (OSError, RuntimeError, AssertionError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nvml is not None:
            self.stop.set()
            self.t.join(timeout=2)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        for clk, cmax, bits in self.samples:
            sm.append(float(clk))
            mx = float(cmax)
            reasons.update(name for bit, name in self.REASON_BITS.items() if bits & bit)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": self.source}


# --------------------------------------------------------------------------- helpers
def source_hash() -> str:
    """SHA-256 over the CUDA sources and the C header: the build an ncu
    capture in profiles/ belongs to."""
    import hashlib
    h = hashlib.sha256()
    csrc = os.path.join(PKG, "csrc")
    files = sorted(f for f in os.listdir(csrc) if f.endswith((".cu", ".cuh")))
    for f in files:
        with open(os.path.join(csrc, f), "rb") as fh:
            h.update(f.encode() + b"\0" + fh.read())
    with open(os.path.join(ROOT, "include", "dsplat.h"), "rb") as fh:
        h.update(fh.read())
    return h.hexdigest()[:16]


KERNEL_OF_STAGE = {"raster_fwd": "k_raster_fwd", "raster_bwd": "k_raster_bwd", "sb_lists": "k_sb_scatter_staged",
                   "project_bwd": "k_project_bwd_colour", "project_fwd": "k_fused_project"}


def captured_figures(stage: str, workload: str):
    """Per-launch figures of a stage's kernel from the committed ncu summary
    of this very build: lines `capture_build <hash>`, `workload <workload>:
    <description>` and `per_launch <workload> <kernel> inst
    <warp-instructions> dram_bytes <bytes>` in a profiles/*.md.  None when
    no capture of the current sources exists (the line then says so instead
    of reporting a stale figure)."""
    import glob
    import re
    kernel = KERNEL_OF_STAGE.get(stage)
    if kernel is None:
        return None
    want = source_hash()
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            txt = f.read()
        m_build = re.search(r"capture_build\s+([0-9a-f]+)", txt)
        m = re.search(r"per_launch\s+" + workload + r"\s+" + kernel + r"\s+inst\s+(\d+)\s+dram_bytes\s+(\d+)", txt)
        if m and m_build and m_build.group(1) == want:
            wl = re.search(r"^\s*workload\s+" + workload + r":\s*(.+)$", txt, re.M)
            return {"inst": int(m.group(1)), "dram_bytes": int(m.group(2)),
                    "capture": os.path.relpath(path, ROOT), "workload": wl.group(1).strip() if wl else None}
    return None


def num_sms(dev) -> int:
    return int(torch.cuda.get_device_properties(dev).multi_processor_count)


def issue_roofline(stage: str, launch_ms: float, clocks: dict, dev, hbm_peak: float, peak_kind: str,
                   workload: str = "gauss-batch") -> dict:
    """Instruction-issue roofline of one launch of `stage`'s kernel: warp-
    instructions per launch (ncu capture of this build) / this run's CUDA-
    event launch time, against 4 warp-instructions per clock per SM at this
    run's median sampled SM clock; the capture's DRAM bytes per launch give
    the HBM fraction beside it."""
    fig = captured_figures(stage, workload)
    clk = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    ceiling = num_sms(dev) * 4 * clk * 1e6 / 1e9  # G warp-instructions/s
    out = {"kernel": KERNEL_OF_STAGE.get(stage, stage), "stage": stage, "bound": "issue",
           "unit": "G warp-instructions/s", "peak": ceiling, "launch_ms": launch_ms,
           "peak_note": f"{num_sms(dev)} SMs x 4 schedulers x {clk:.0f} MHz (median SM clock sampled in the run)"}
    if fig is None:
        out.update({"achieved": None, "frac": None, "traffic": None,
                    "note": "no ncu capture of this build in profiles/ (source hash " + source_hash() + ")"})
        return out
    achieved = fig["inst"] / (launch_ms / 1e3) / 1e9
    gbs = fig["dram_bytes"] / (launch_ms / 1e3) / 1e9
    out.update({"achieved": achieved, "frac": achieved / ceiling, "traffic": fig["dram_bytes"],
                "inst_per_launch": fig["inst"], "capture": fig["capture"], "capture_workload": fig["workload"],
                "hbm": {"achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                        "peak_kind": peak_kind}})
    return out


def cpu_model() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo), for the CPU baseline."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def single_thread_sample(scene, nthreads: int, tile_size: int):
    """1-thread vs all-thread time of the workload's smallest view (the
    reference's CPU path is single-threaded); returns (s 1 thread, s all
    threads, view description)."""
    i = min(range(len(scene.cameras)), key=lambda k: scene.cameras[k].width * scene.cameras[k].height)
    t1, cam = cpu_sample(scene, i, 1, tile_size)
    tn, _ = cpu_sample(scene, i, nthreads, tile_size)
    return t1, tn, f"{cam.width}x{cam.height}"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def rank_cameras(base, rank: int, views: int):
    """Weak scaling: every rank renders its own `views` cameras of the same
    scene (rank 0 the workload's own; rank r > 0 seeded from 1000 + r)."""
    from dsplat import scenes
    if rank == 0:
        return base.cameras
    return scenes.sphere_cameras(np.random.default_rng(1000 + rank), views, 3.0, scenes.CONFIG3_RESOLUTIONS)


def max_over_ranks(x: float, world: int, dev) -> float:
    if world == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------- CPU arm
def cpu_sample(scene, cam_index: int, nthreads: int, tile_size: int, steps: int = 1):
    """Oracle fwd+bwd (FP32, OpenMP) of one view of the workload; returns s/view."""
    import oracle
    cam = scene.cameras[cam_index]
    tgt = np.random.default_rng(99).uniform(0, 1, (cam.height, cam.width, 3)).astype(np.float32)
    dummy_lists = np.zeros(1, np.uint32)
    S = oracle.Scene(scene.means, scene.log_scales, scene.quats, scene.opacity, scene.colors.reshape(scene.n, -1),
                     scene.sh_degree, cam.mvp, cam.campos, cam.width, cam.height, tile_size, dummy_lists,
                     dummy_lists, np.zeros(1, np.int32), np.zeros((1, 4), np.float32), tgt)
    t0 = time.perf_counter()
    for _ in range(steps):
        S.cpu_fwd_bwd(nthreads)
    return (time.perf_counter() - t0) / steps, cam


def cpu_workload_rate(scene, nthreads: int, tile_size: int, reps: int = 1):
    """CPU views/s of the whole workload, estimated from one timed fwd+bwd of
    one view per distinct resolution, weighted by how many of the workload's
    views have that resolution.  Returns (views/s, sample description)."""
    by_res = {}
    for i, c in enumerate(scene.cameras):
        by_res.setdefault((c.width, c.height), []).append(i)
    total = 0.0
    for res, idx in sorted(by_res.items()):
        t, _ = cpu_sample(scene, idx[0], nthreads, tile_size, steps=reps)
        total += t * len(idx)
    desc = ("one fwd+bwd of one view per resolution (" + ", ".join(f"{w}x{h} x{len(v)}" for (w, h), v in
                                                                  sorted(by_res.items())) +
            f") of the {scene.n}-Gaussian SH{scene.sh_degree} workload, weighted to its {len(scene.cameras)} "
            f"views; oracle C++ restatement, OpenMP {nthreads} threads")
    return len(scene.cameras) / total, desc


def run_reference(args, rank, world):
    if rank != 0:
        return
    from dsplat import scenes
    nthreads = os.cpu_count() or 1
    scene = scenes.config3(seed=3, n=args.n, views=args.views, tile_size=args.tile)
    ts = 16  # the reference's tile size; the CPU blend's results do not depend on it
    # a step is one view's fwd+bwd; steps cycle through the workload's views
    # in order, so a multiple of the view count weights resolutions exactly
    nv = len(scene.cameras)
    for i in range(args.warmup):
        cpu_sample(scene, i % nv, nthreads, ts)
    total = 0.0
    for i in range(args.steps):
        t, _ = cpu_sample(scene, i % nv, nthreads, ts)
        total += t
    per_view = total / max(args.steps, 1)
    v = 1.0 / per_view
    desc = (f"{args.steps} timed steps after {args.warmup} untimed, each one fwd+bwd of one view of the "
            f"{scene.n}-Gaussian SH{scene.sh_degree} workload, cycling through its {nv} views "
            f"(320x240..1920x1080); oracle C++ restatement, OpenMP {nthreads} threads")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_view * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": "1M Gaussians SH3, 16 views mixed 320x240..1920x1080, fwd+bwd, L2 loss",
                       "num_gaussians": args.n, "views_per_gpu": args.views, "tile_size": ts,
                       "step": "one view (steps cycle through the views)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- other workloads
def covered_pixel_tests(xyd: np.ndarray, rad: np.ndarray, w: int, h: int) -> int:
    """Number of (circle, pixel) pairs with the pixel centre within the radius
    and inside the image: the atomicMin operations one frame issues."""
    x, y, r = xyd[:, 0].astype(np.float64), xyd[:, 1].astype(np.float64), rad.astype(np.float64)
    rmax = int(np.ceil(r.max())) + 1
    total = 0
    bx, by = np.floor(x), np.floor(y)
    for oy in range(-rmax, rmax + 1):
        py = by + oy
        for ox in range(-rmax, rmax + 1):
            px = bx + ox
            d2 = (x - (px + 0.5)) ** 2 + (y - (py + 0.5)) ** 2
            total += int(np.count_nonzero((d2 <= r * r) & (px >= 0) & (px < w) & (py >= 0) & (py < h)))
    return total


def run_zbuffer(args, rank, world, local):
    """1,048,576 points in [-1,1]^3 seen from (0,0,-3), 1024x1024, pixel radius
    1..4, RGBA u32: one frame = circle projection + packed depth|index
    atomicMin z-buffer + colour resolve (dsplat_circle_splat_zbuffer)."""
    from dsplat import _native, scenes
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L = _native.lib()
    sc = scenes.config1(seed=1 + rank)
    W, H = sc.camera.width, sc.camera.height
    n = sc.xyz.shape[0]
    st = torch.cuda.current_stream(dev).cuda_stream
    xyz = torch.from_numpy(sc.xyz).to(dev)
    rad = torch.from_numpy(sc.radius_px).to(dev)
    rgba = torch.from_numpy(sc.rgba.view(np.int32)).to(dev)
    mvp = torch.from_numpy(np.ascontiguousarray(sc.camera.mvp, np.float32).reshape(-1)).to(dev)
    xyd = torch.empty((n, 3), device=dev)
    rad_world = torch.empty(n, device=dev)
    pix = torch.empty((H, W), dtype=torch.int32, device=dev)
    zbuf = torch.empty(W * H, dtype=torch.int64, device=dev)
    ts = 16

    def frame(xyz=xyz, rad=rad, rgba=rgba, pix=pix):
        _native.check(L.dsplat_circle_pnt2splat3_to_pnt2splat2(st, n, xyz.data_ptr(), xyd.data_ptr(),
                                                               rad_world.data_ptr(), mvp.data_ptr(), W, H, 0.0),
                      "project")
        _native.check(L.dsplat_circle_splat_zbuffer(st, n, xyd.data_ptr(), rad.data_ptr(), rgba.data_ptr(), 1,
                                                    pix.data_ptr(), None, W, H, ts, zbuf.data_ptr()), "zbuffer")

    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize()
    tests = covered_pixel_tests(xyd.cpu().numpy(), sc.radius_px, W, H)
    # splat kernels alone (fill + atomicMin + resolve), for the roofline line
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record()
    for _ in range(args.steps):
        _native.check(L.dsplat_circle_splat_zbuffer(st, n, xyd.data_ptr(), rad.data_ptr(), rgba.data_ptr(), 1,
                                                    pix.data_ptr(), None, W, H, ts, zbuf.data_ptr()), "zbuffer")
    a1.record()
    torch.cuda.synchronize()
    splat_ms = a0.elapsed_time(a1) / args.steps
    c0 = L.dsplat_launch_count()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record()
        for _ in range(args.steps):
            frame()
        e1.record()
        torch.cuda.synchronize()
    launches = L.dsplat_launch_count() - c0
    t_ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    fps = world * args.steps / (t_ms / 1e3)
    # end to end: points from pinned host memory in, the image out, every
    # frame; the copies run on side streams (dsplat.feed), so frame k+1's
    # points arrive and frame k-1's image leaves while frame k is splatted
    from dsplat.feed import DeviceToHostDrain, HostToDeviceFeed
    host = {"xyz": torch.from_numpy(sc.xyz).pin_memory(), "rad": torch.from_numpy(sc.radius_px).pin_memory(),
            "rgba": torch.from_numpy(sc.rgba.view(np.int32)).pin_memory()}
    feed = HostToDeviceFeed(host, dev)
    outs = [torch.empty_like(pix) for _ in feed.slots]
    drain = DeviceToHostDrain({"pix": outs[0]}, dev, slots=len(feed.slots))

    def run_e2e(frames):
        feed.put(host)
        for k in range(frames):
            d = feed.get()
            i = next(j for j, sl in enumerate(feed.slots) if sl is d)
            if k + 1 < frames:
                feed.put(host)
            drain.reclaim(i)
            frame(d["xyz"], d["rad"], d["rgba"], outs[i])
            drain.push(i, {"pix": outs[i]})
            feed.release()
        for i in range(len(feed.slots)):  # every readback has landed
            drain.wait(i)

    run_e2e(args.warmup)
    torch.cuda.synchronize()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record()
    run_e2e(args.steps)
    q1.record()
    torch.cuda.synchronize()
    e2e = world * args.steps / (max_over_ranks(q0.elapsed_time(q1), world, dev) / 1e3)
    e2e_equal = bool(torch.equal(drain.host[(args.steps - 1) % len(feed.slots)]["pix"], pix.cpu()))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:  # the CPU baseline: rank 0 at N=1 only
        import oracle
        xyd_h = xyd.cpu().numpy()
        t0 = time.perf_counter()
        aabb = oracle.circle_aabb(xyd_h, sc.radius_px)
        t2i, i2p, _ = oracle.tile2pnt(xyd_h, aabb, W, H, ts)
        oracle.circle_splat_tiled(W, H, ts, t2i, i2p, xyd_h, sc.radius_px)
        cpu_s = time.perf_counter() - t0
        cpu = {"value": 1.0 / cpu_s, "unit": "frames/s", "cores": 1, "kind": "port", "cpu_model": cpu_model(),
               "sample": "one full frame: tile lists + tiled circle painter (oracle C++ restatement of "
                         "del-splat-cpu's sorted painter), 1 thread; projection excluded"}
    peak, peak_kind = peaks()
    alg = n * (12 + 4 + 4) + W * H * (8 + 4)
    if rank == 0:
        print(json.dumps({
            "metric": "1M-point 1024x1024 circle z-buffer frames/s (1 B200)", "value": fps, "unit": "frames/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 keys / f32",
            "data": "synthetic (seeded PCG64)",
            "config": {"workload": "1M points U[-1,1]^3, camera (0,0,-3), 1024x1024, pixel radius 1..4, RGBA u32, "
                                   "tile span 16", "num_points": n, "covered_pixel_tests": tests,
                       "splat_ms": splat_ms, "atomic_min_per_s": tests / (splat_ms / 1e3),
                       "l2": "z-buffer (8 MB) is L2-resident by design; inputs 20 MB"},
            "roofline": {"kernel": "circle z-buffer splat (fill + atomicMin + resolve)", "bound": "hbm",
                         "achieved": alg / (splat_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (splat_ms / 1e3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                         "note": "algorithmic bytes N*(12+4+4) + W*H*(8+4); the limiter is L2 atomic throughput "
                                 "(atomic_min_per_s)"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "frames/s", "h2d_bytes_per_step": n * 20, "d2h_bytes_per_step": W * H * 4,
                    "result": "the RGBA image to pinned host memory every frame, copies on side streams",
                    "image_equal_resident_run": e2e_equal},
            "gpu_launches": int(launches), "clocks": clk.summary()}), flush=True)


STAGE_NAMES = ["project_fwd", "depth_sort", "sb_lists", "task_order", "raster_fwd", "(host gap)", "grad_clear",
               "raster_bwd", "project_bwd"]


def time_dropin(base, cams, dev, steps: int, warmup: int, world: int) -> dict:
    """Forward only, one view per call, through the reference-shaped chain a
    del-splat-cudarc caller runs (splat_gauss.rs:6-195): the drop-in
    projection, tile2idx_idx2pnt (the count with its device-to-host read of
    the pair total, then the fill into buffers allocated per call, as the
    reference allocates them) and rasterize_pnt2splat2 at the reference's
    16x16 tiles.  That chain takes per-point RGB (the reference has no SH), so
    the SH DC colours stand in.  Beside it, the batched forward of the same
    views (SH 3) with the same event timing."""
    from dsplat import cudarc
    n = base.n
    means = torch.from_numpy(np.ascontiguousarray(base.means)).to(dev)
    scales = torch.from_numpy(np.ascontiguousarray(base.scales)).to(dev)
    quats = torch.from_numpy(np.ascontiguousarray(base.quats)).to(dev)
    opacity = torch.from_numpy(np.ascontiguousarray(base.opacity)).to(dev)
    rgb = torch.from_numpy(np.ascontiguousarray(base.colors.reshape(n, -1, 3)[:, 0, :])).to(dev)
    xyd, conic, aabb = (torch.empty((n, k), device=dev) for k in (3, 3, 4))
    mvps = [torch.from_numpy(np.ascontiguousarray(c.mvp)).to(dev) for c in cams]
    imgs = [torch.zeros((c.height, c.width, 3), device=dev) for c in cams]

    def step():
        for c, mvp, img in zip(cams, mvps, imgs):
            size = (c.width, c.height)
            cudarc.splat_gauss_pnt2splat3_to_pnt2splat2(None, means, scales, quats, xyd, conic, aabb, mvp, size)
            t2i, i2p = cudarc.splat_gauss_tile2idx_idx2pnt(None, size, 16, xyd, aabb)
            img.zero_()
            cudarc.splat_gauss_rasterize_pnt2splat2(None, size, img, xyd, conic, aabb, opacity, rgb, 16, t2i, i2p)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    t = max_over_ranks(e0.elapsed_time(e1), world, dev)
    return {"views_per_s": world * len(cams) * steps / (t / 1e3), "ms_per_16_views": t / steps,
            "chain": "pnt2splat3_to_pnt2splat2 -> tile2idx_idx2pnt (count: D2H sync; fill: per-call buffers) "
                     "-> rasterize_pnt2splat2, 16x16 tiles, one view per call, forward only, SH DC as RGB"}


def measure_stages(L, step, steps: int) -> np.ndarray:
    """Mean per-stage times (ms, CUDA events recorded on the launch stream by
    the library's stage hook) of `steps` eager runs of step()."""
    from dsplat import _native
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(10)]
    for e in evs:
        e.record()
    torch.cuda.synchronize()
    handles = (_native.c_void_p * 10)(*[e.cuda_event for e in evs])
    stage_ms = np.zeros(9)
    for _ in range(steps):
        L.dsplat_set_stage_events(handles, 10)
        step()
        L.dsplat_set_stage_events(None, 0)
        torch.cuda.synchronize()
        stage_ms += [evs[i].elapsed_time(evs[i + 1]) for i in range(9)]
    return stage_ms / max(steps, 1)


def _train_state(params, adam):
    """The tensors that define a training step's starting point: parameters,
    Adam moments and the device-side step count."""
    names = sorted(params)
    return ([params[k] for k in names] + [adam.exp_avg[k] for k in names] + [adam.exp_avg_sq[k] for k in names] +
            [adam.step_count])


def run_train4m(args, rank, world, local):
    """4,194,304 Gaussians (SH 3), 8 views at 1920x1080, one training step =
    forward with L2 loss + backward + fused Adam (lr 1e-3, betas 0.9/0.999)
    on all parameters, captured in one CUDA graph with the Adam step count
    on the device.  e2e: each step's target images come from pinned host
    memory and its loss goes back (the parameters live on the device, as in
    training)."""
    from dsplat import _native, scenes
    from dsplat.feed import DeviceToHostDrain, HostToDeviceFeed
    from dsplat.gauss import Adam, CapturedStep, GaussBatch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L = _native.lib()
    sc = scenes.config4(seed=4 + rank)
    host = {"means": sc.means, "log_scales": sc.log_scales, "quats": sc.quats, "opacity": sc.opacity,
            "colors": sc.colors.reshape(sc.n, -1)}
    params = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in host.items()}
    grads = {k: torch.zeros_like(v) for k, v in params.items()}
    tgt = np.concatenate([t.reshape(-1) for t in scenes.targets_for(sc, seed=99 + rank)])
    target = torch.from_numpy(tgt).to(dev)
    ts, ppl = (args.tile, args.ppl) if args.tile else (8, 2)
    batch = GaussBatch(sc.n, sc.cameras, ts, 3, pair_capacity=1 << 26, device=dev, pixels_per_lane=ppl,
                       check_overflow=False)
    batch.ensure_capacity(params)
    V = len(sc.cameras)

    # untimed parity check before any update: the batched images against the
    # plain per-view path (each view rendered alone), max-abs
    batch.forward(params)
    imgs = batch.images()
    worst = 0.0
    for v, cam in enumerate(sc.cameras):
        one = GaussBatch(sc.n, [cam], ts, 3, pair_capacity=1 << 25, device=dev, pixels_per_lane=ppl)
        one.ensure_capacity(params)
        one.forward(params)
        worst = max(worst, float((one.images()[0] - imgs[v]).abs().max()))
        del one
    torch.cuda.empty_cache()

    def eager_step(opt):
        for g in grads.values():
            g.zero_()
        batch.forward(params, target=target)
        batch.backward(params, grads)
        opt.step(grads)

    # stage times (one eager pass per timed step, on a throw-away optimizer
    # state; the parameters are reset afterwards)
    snapshot = {k: v.clone() for k, v in params.items()}
    scratch = Adam(params, 3, lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    stage_ms = measure_stages(L, lambda: eager_step(scratch), max(1, min(args.steps, 5)))
    for k in params:
        params[k].copy_(snapshot[k])
    del scratch, snapshot

    adam = Adam(params, 3, lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    graph = CapturedStep(batch, params, grads, target, warmup=args.warmup, optimizer=adam)
    flags, _, _ = batch.status()
    if flags:
        raise RuntimeError("pair capacity overflow in the warm-up")
    c0 = L.dsplat_launch_count()
    eager_step(adam)  # one more real step, to count this library's launches per step
    torch.cuda.synchronize()
    per_step_launches = L.dsplat_launch_count() - c0
    # the training state the timed steps start from; the e2e run below starts
    # from it again, so that both time the same stretch of the training
    # trajectory (the work per step changes as the scene trains)
    start = [t.clone() for t in _train_state(params, adam)]
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record()
        for _ in range(args.steps):
            graph.replay()
        e1.record()
        torch.cuda.synchronize()
    flags, _, pairs = batch.status()
    if flags:
        raise RuntimeError("pair capacity overflow inside the timed region")
    t_ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    clocks = clk.summary()

    # end to end: targets in, loss out, every step (graphs per feed slot)
    tgt_pinned = target.cpu().pin_memory()
    feed = HostToDeviceFeed({"target": tgt_pinned}, dev)
    loss_dev = [torch.zeros(1, device=dev) for _ in feed.slots]
    drain = DeviceToHostDrain({"loss": loss_dev[0]}, dev, slots=len(feed.slots))
    for sl in feed.slots:
        sl["target"].copy_(target)
    slot_graphs = [CapturedStep(batch, params, grads, sl["target"], warmup=1, optimizer=adam) for sl in feed.slots]

    def run_e2e(steps):
        feed.put({"target": tgt_pinned})
        for k in range(steps):
            d = feed.get()
            i = next(j for j, sl in enumerate(feed.slots) if sl is d)
            if k + 1 < steps:
                feed.put({"target": tgt_pinned})
            drain.reclaim(i)
            slot_graphs[i].replay()
            torch.sum(batch.slab_loss(), dim=0, keepdim=True, out=loss_dev[i])
            drain.push(i, {"loss": loss_dev[i]})
            feed.release()
        for i in range(len(feed.slots)):
            drain.wait(i)

    run_e2e(max(1, args.warmup))
    torch.cuda.synchronize()
    for t, t0 in zip(_train_state(params, adam), start):  # in place: the graphs hold these buffers
        t.copy_(t0)
    del start
    torch.cuda.synchronize()
    barrier(world)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record()
    run_e2e(args.steps)
    q1.record()
    torch.cuda.synchronize()
    et = max_over_ranks(q0.elapsed_time(q1), world, dev)

    peak, peak_kind = peaks()
    dom = max((n for n in STAGE_NAMES if not n.startswith("(") and n != "task_order"),
              key=lambda n: stage_ms[STAGE_NAMES.index(n)])
    roofline = issue_roofline(dom, float(stage_ms[STAGE_NAMES.index(dom)]), clocks, dev, peak, peak_kind,
                              workload="train4m")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:  # the CPU baseline: rank 0 at N=1 only
        try:
            nth = os.cpu_count() or 1
            t1, cam = cpu_sample(sc, 0, nth, 16)
            cpu = {"value": 1.0 / (t1 * V), "unit": "steps/s", "cores": nth, "kind": "port",
                   "sample": f"one fwd+bwd of one {cam.width}x{cam.height} view of the {sc.n}-Gaussian SH3 "
                             f"scene (oracle C++ restatement, OpenMP {nth} threads), x{V} views per step; "
                             "Adam not included", "cpu_model": cpu_model()}
        except Exception as ex:
            cpu = {"value": None, "unit": "steps/s", "cores": 0, "kind": "port", "sample": f"failed: {ex}"}

    if rank == 0:
        value = world * args.steps / (t_ms / 1e3)
        print(json.dumps({
            "metric": "4M-Gaussian 8x1080p fwd+bwd+Adam steps/s (1 B200)", "value": value,
            "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded PCG64)",
            "config": {"workload": "4M Gaussians SH3, 8 views 1920x1080, fwd+bwd+fused Adam, CUDA graph",
                       "num_gaussians": sc.n, "views": V, "views_per_s": world * V * args.steps / (t_ms / 1e3),
                       "tile_size": ts, "pixels_per_lane": ppl, "pairs_per_step": int(pairs), "cuda_graph": True,
                       "l2": "inputs larger than L2 (params 944 MB)",
                       "stage_ms": {n: round(float(stage_ms[i]), 4) for i, n in enumerate(STAGE_NAMES)}},
            "parity": {"batched_vs_plain_max_abs": worst, "tolerance": 1e-4,
                       "note": "the 8 views before any update, batched vs each view rendered alone"},
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": world * args.steps / (et / 1e3), "unit": "steps/s",
                    "h2d_bytes_per_step": int(tgt_pinned.numel() * 4), "d2h_bytes_per_step": 4,
                    "result": "targets in, loss out every step; parameters stay on the device",
                    "start": "the same training state as the timed steps (parameters, moments, step count)"},
            "gpu_launches": int(per_step_launches * args.steps), "clocks": clocks}), flush=True)


# --------------------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--views", type=int, default=16)
    ap.add_argument("--tile", type=int, default=0, help="tile size 8/16/32; 0: autotune (with --ppl)")
    ap.add_argument("--ppl", type=int, default=0, help="rasteriser pixels per lane (0: default / autotune)")
    ap.add_argument("--no-graph", action="store_true", help="time the batched step without CUDA-graph replay")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-dropin", action="store_true", help="skip the forward-only drop-in chain leg")
    ap.add_argument("--workload", default="gauss-batch", choices=["gauss-batch", "zbuffer", "train4m"],
                    help="gauss-batch: the headline (default); zbuffer: 1M-point circle z-buffer at 1024x1024; "
                         "train4m: 4M Gaussians, 8 views at 1080p, fwd+bwd+Adam")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    if args.impl == "reference":  # CPU only: no process group, no GPU
        run_reference(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")))
        return
    rank, world, local = dist_setup()
    if args.workload in ("zbuffer", "train4m"):
        (run_zbuffer if args.workload == "zbuffer" else run_train4m)(args, rank, world, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    from dsplat import _native, scenes
    from dsplat.gauss import GaussBatch

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L = _native.lib()
    base = scenes.config3(seed=3, n=args.n, views=args.views, tile_size=args.tile)
    # weak scaling: every rank gets its own cameras of the same scene
    cams = rank_cameras(base, rank, args.views)
    host = {"means": base.means, "log_scales": base.log_scales, "quats": base.quats, "opacity": base.opacity,
            "colors": base.colors.reshape(base.n, -1)}
    params = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in host.items()}
    rng = np.random.default_rng(99 + rank)
    tgt_np = [rng.uniform(0, 1, (c.height, c.width, 3)).astype(np.float32) for c in cams]
    target = torch.from_numpy(np.concatenate([t.reshape(-1) for t in tgt_np])).to(dev)
    grads = {k: torch.zeros_like(v) for k, v in params.items()}

    tune_report = {}
    if args.tile == 0:
        from dsplat import autotune
        args.tile, args.ppl = autotune.tune(params, cams, 3, target, use_cache=False, report=tune_report)
    batch = GaussBatch(base.n, cams, args.tile, 3, pair_capacity=1 << 24, device=dev, pixels_per_lane=args.ppl)
    pairs = batch.ensure_capacity(params)
    V = len(cams)
    pix_off = batch.pix_offsets

    def zero_grads():
        for g in grads.values():
            g.zero_()

    def step_batched():
        zero_grads()
        batch.forward(params, target=target)
        batch.backward(params, grads)

    # plain per-view path: the same kernels one view per call, at the batch's
    # (tile, pixels per lane) and at 16x16 tiles (the reference's tile size);
    # the faster one is reported
    plain_cfgs = []
    if not args.no_plain:
        for ts_p, ppl_p in dict.fromkeys([(args.tile, args.ppl), (16, 4)]):
            lst = []
            for v, c in enumerate(cams):
                b = GaussBatch(base.n, [c], ts_p, 3, pair_capacity=1 << 22, device=dev, pixels_per_lane=ppl_p)
                b.ensure_capacity(params)
                lst.append((b, target[3 * pix_off[v]: 3 * pix_off[v + 1]]))
            plain_cfgs.append(((ts_p, ppl_p), lst))

    def step_plain(plain):
        zero_grads()
        for b, t in plain:
            b.forward(params, target=t)
            b.backward(params, grads)

    for _ in range(args.warmup):
        step_batched()
    torch.cuda.synchronize()
    stage_ms = measure_stages(L, step_batched, args.steps)

    graph = None
    if not args.no_graph:
        from dsplat.gauss import CapturedStep
        graph = CapturedStep(batch, params, grads, target)
        for _ in range(args.warmup):
            graph.replay()
        torch.cuda.synchronize()
    run_batched = graph.replay if graph is not None else step_batched

    c0 = L.dsplat_launch_count()
    step_batched()
    torch.cuda.synchronize()
    per_step_launches = L.dsplat_launch_count() - c0
    n_launch0 = L.dsplat_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record()
        for _ in range(args.steps):
            run_batched()
        e1.record()
        torch.cuda.synchronize()
    barrier(world)
    launches = L.dsplat_launch_count() - n_launch0
    if graph is not None:  # a replay re-issues the captured launches without calling the library
        launches = per_step_launches * args.steps
    t_ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    value = world * V * args.steps / (t_ms / 1e3)
    clocks = clk.summary()

    # untimed check: no capacity overflow happened
    flags, needed_now, pairs_now = batch.status()
    if flags:
        raise RuntimeError("pair capacity overflow inside the timed region")

    # plain per-view path, same kernels one view per call
    plain_vps = None
    parity = {}
    plain_by_cfg = {}
    plain_cfg = None
    plain = None
    for cfg, plain in plain_cfgs:
        for _ in range(args.warmup):
            step_plain(plain)
        torch.cuda.synchronize()
        barrier(world)
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record()
        for _ in range(args.steps):
            step_plain(plain)
        p1.record()
        torch.cuda.synchronize()
        pt = max_over_ranks(p0.elapsed_time(p1), world, dev)
        vps = world * V * args.steps / (pt / 1e3)
        plain_by_cfg[f"ts{cfg[0]}_ppl{cfg[1]}"] = vps
        if plain_vps is None or vps > plain_vps:
            plain_vps, plain_cfg = vps, cfg
        # untimed parity check: every view of the batched step against the
        # same view rendered alone (same kernels, one view per call)
        worst = 0.0
        for v, (b, _) in enumerate(plain):
            worst = max(worst, float((b.images()[0] - batch.images()[v]).abs().max()))
        parity[f"batched_vs_plain_max_abs_ts{cfg[0]}_ppl{cfg[1]}"] = worst
    plain_cfgs = plain = None  # release the per-view workspaces

    # forward only: the reference-shaped drop-in chain one view per call,
    # beside the batched forward of the same views
    fwd_only = None
    if not args.no_dropin:
        fwd_only = {"dropin": time_dropin(base, cams, dev, args.steps, args.warmup, world)}
        for _ in range(args.warmup):
            batch.forward(params)
        torch.cuda.synchronize()
        barrier(world)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(args.steps):
            batch.forward(params)
        f1.record()
        torch.cuda.synchronize()
        ft = max_over_ranks(f0.elapsed_time(f1), world, dev)
        fwd_only["batched"] = {"views_per_s": world * V * args.steps / (ft / 1e3), "ms_per_16_views": ft / args.steps,
                               "chain": "dsplat_gauss_batch_forward, eager, SH 3"}
        fwd_only["batched_over_dropin"] = fwd_only["batched"]["views_per_s"] / fwd_only["dropin"]["views_per_s"]

    # end to end through the public API: every step's inputs (parameters and
    # targets) come from pinned host memory and every step's result -- the
    # rendered images of all views and the loss -- goes back to pinned host
    # memory.  Copies in (dsplat.feed.HostToDeviceFeed) and out
    # (DeviceToHostDrain) run on side streams: step k+1's inputs and step
    # k-1's images move while step k computes.
    host_pinned = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in host.items()}
    tgt_pinned = target.cpu().pin_memory()
    h2d = sum(t.numel() * 4 for t in host_pinned.values()) + tgt_pinned.numel() * 4

    from dsplat.feed import DeviceToHostDrain, HostToDeviceFeed
    host_step = dict(host_pinned, target=tgt_pinned)
    feed = HostToDeviceFeed(host_step, dev)
    outs = [torch.empty_like(batch.out_rgb) for _ in feed.slots]
    loss_dev = [torch.zeros(1, device=dev) for _ in feed.slots]
    drain = DeviceToHostDrain({"images": outs[0], "loss": loss_dev[0]}, dev, slots=len(feed.slots))
    d2h = drain.bytes_per_push()

    # one captured step per feed slot (the graph bakes in its slot's buffers)
    slot_graphs = None
    if graph is not None:
        from dsplat.gauss import CapturedStep
        for sl in feed.slots:  # valid inputs for the capture's warm-up runs
            for name in params:
                sl[name].copy_(params[name])
            sl["target"].copy_(target)
        slot_graphs = [CapturedStep(batch, {name: sl[name] for name in params}, grads, sl["target"], out_rgb=outs[i])
                       for i, sl in enumerate(feed.slots)]

    def run_e2e(steps):
        feed.put(host_step)
        last = 0
        for k in range(steps):
            d = feed.get()
            i = next(j for j, sl in enumerate(feed.slots) if sl is d)
            if k + 1 < steps:
                feed.put(host_step)
            drain.reclaim(i)
            if slot_graphs is not None:
                slot_graphs[i].replay()
            else:
                p = {name: d[name] for name in params}
                zero_grads()
                batch.forward(p, target=d["target"], out_rgb=outs[i])
                batch.backward(p, grads)
            torch.sum(batch.slab_loss(), dim=0, keepdim=True, out=loss_dev[i])
            drain.push(i, {"images": outs[i], "loss": loss_dev[i]})
            feed.release()
            last = i
        return drain.wait(last)

    run_e2e(args.warmup)
    torch.cuda.synchronize()
    barrier(world)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record()
    result = run_e2e(args.steps)
    for i in range(len(feed.slots)):  # every readback has landed
        drain.wait(i)
    q1.record()
    torch.cuda.synchronize()
    et = max_over_ranks(q0.elapsed_time(q1), world, dev)
    e2e_vps = world * V * args.steps / (et / 1e3)
    e2e_images_equal = bool(torch.equal(result["images"], batch.out_rgb.cpu()))

    # roofline of the dominant kernel: instruction issue (the rasterisers are
    # issue-bound with DRAM nearly idle); see issue_roofline
    peak, peak_kind = peaks()
    npix = int(batch.layout.num_pix)
    names = STAGE_NAMES
    dom = max((n for n in names if not n.startswith("(") and n != "task_order"),
              key=lambda n: stage_ms[names.index(n)])
    roofline = issue_roofline(dom, float(stage_ms[names.index(dom)]), clocks, dev, peak, peak_kind)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:  # the CPU baseline: rank 0 at N=1 only
        try:
            nth = os.cpu_count() or 1
            rate, desc = cpu_workload_rate(base, nth, 16)  # the reference's tile size; results do not depend on it
            t1, tn, res = single_thread_sample(base, nth, 16)
            cpu = {"value": rate, "unit": UNIT, "cores": nth, "kind": "port", "sample": desc,
                   "cpu_model": cpu_model(),
                   "single_thread": {"view": res, "s_per_view_1_thread": t1, "s_per_view_all_threads": tn,
                                     "estimated_value_1_thread": rate * tn / t1,
                                     "note": "workload rate scaled by this view's all-thread / 1-thread time"}}
        except Exception as ex:  # the CPU baseline must not hide the GPU result
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "port", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG64; no public dataset)",
            "config": {"workload": "1M Gaussians SH3, 16 views mixed 320x240..1920x1080, fwd+bwd, L2 loss",
                       "num_gaussians": base.n, "views_per_gpu": V, "tile_size": args.tile,
                       "pixels_per_lane": batch.ppl or None, "cuda_graph": graph is not None,
                       "autotune": tune_report or None,
                       "pairs_per_step": int(pairs_now), "pixels_per_step": npix,
                       "plain_views_per_s": plain_vps,
                       "plain_config": {"tile_size": plain_cfg[0], "pixels_per_lane": plain_cfg[1]}
                       if plain_cfg else None,
                       "plain_views_per_s_by_config": plain_by_cfg or None,
                       "batched_over_plain": (value / world) / (plain_vps / world) if plain_vps else None,
                       "forward_only": fwd_only,
                       "l2": "inputs larger than L2 (params 236 MB, pair lists > 1 GB)",
                       "parallelism": f"replicas x{world} (views sharded, no collective)",
                       "stage_ms": {n: round(float(stage_ms[i]), 4) for i, n in enumerate(names)}},
            "parity": dict(parity, batched_vs_plain_max_abs=max(parity.values()) if parity else None,
                           tolerance=1e-4, note="every view's image, batched step vs the view rendered alone"),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_vps, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "result": "rendered images of all views + loss, to pinned host memory every step",
                    "images_equal_resident_run": e2e_images_equal},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
