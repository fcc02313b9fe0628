#!/usr/bin/env python3
"""Benchmark of the GR-ray-tracer hot path on B200.

Workload (default, the configuration the headline metric is quoted on):
  C2 -- 256x256 image-mode rays, adaptive RK45 (rtol = atol = 1e-8), Kerr
  a = 0.94, Fishbone-Moncrief torus on a 128x64x64 (r, theta, phi) grid,
  camera at 1000 M, inclination 17 deg, absorption and emission on.
  Synthetic inputs (the torus generator), one ray per pixel centre.

Forms, each timed over the same steps:
  fp64           the plain FP64 parity kernel, one 256x256 image per step
                 (initialise the 65,536 pixel rays on the device, trace them
                 to termination, build the image products), run as the
                 context's CUDA graph like the batched forms;
  fp64_batched   the same kernel on the C2 image at four frequency channels
                 (230/345/86/43 GHz: custom generator frequency and emission
                 coefficient scaled by f/230 GHz) traced by ONE persistent
                 launch, 262,144 rays per step, run as the context's CUDA
                 graph (init + trace + every image's products);
  mixed_batched  the mixed FP32/FP64 kernel on that batch (autotuned launch
                 shape) -- the headline when every channel's Stokes-I image is
                 within 1e-5 (L2 relative) of the FP64 image of that channel.
`value` is rays/s of the headline form with the grid resident in HBM.
`e2e` repeats the headline step through the C ABI with host buffers: the
photon SoA is uploaded from pinned host memory and every image's products are
copied back every step.  For the batched forms it streams: two contexts on one
stream, used in turn through grt_render_async / grt_render_wait, so one
context's copies overlap the other's trace while the traces stay in order
(`e2e_serial` is the same step with upload, trace and copy-back one after
another on one context).  L2 is flushed (a 256 MB device write) before every
timed step: outside the events for the forms and the serial e2e, on the
stream inside the timed region for the streamed e2e.

On one GPU the default run then measures the other configurations, each by
this script in a child process of its own after the headline's timed region
(C1 64x64 RK4; C3 the 64-image batch; C4 the adjoint; C5 disk mode), and
reports a summary of each under `other_workloads` in the same line
(--no-other-workloads skips them; --workload c1/c3/c4/c5 runs one alone).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank renders one frame of a camera orbit (camera_phi =
2 pi k / N) and the image products are all-gathered over NCCL every step
(weak scaling); times are CUDA-event times, max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "gr-ray-tracer_b200"))

METRIC = "rays/s & RK steps/s on 1 B200: mixed+batched vs FP64 at ≤1e-5 Stokes-I rel err"

# Algorithmic FP64 operations per unit (add/sub, mul, div, sqrt, pow each 1),
# pinned by the oracle's op-counting instantiation of the reference source
# (tests/test_opcount.py): one right-hand side, one RK4 step, one RKF45 attempt.
OPS_RHS = 243
OPS_RK4_STEP = 1100
OPS_RK45_ATTEMPT = 1691
PHOTON_BYTES = 8 * 18 + 2  # id + 17 float64 fields + terminate + phase


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def algorithmic_flops(stats, integrator):
    if integrator == 0:
        return stats["accepted_steps"] * OPS_RK4_STEP
    attempts = stats["accepted_steps"] + stats["rejected_attempts"]
    return stats["accepted_steps"] * OPS_RHS + attempts * OPS_RK45_ATTEMPT


class ClockSampler:
    """SM clock, power and clock-event (throttle) reasons of this rank's GPU,
    sampled through NVML every 10 ms by a background thread while the timed
    regions run (nvidia-smi's 200 ms loop would see only a sample or two of a
    sub-second region)."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, device_index, period_s=0.010):
        self.dev = device_index
        self.period = period_s
        self.rows = []
        self.handle = None
        self.max_mhz = None
        self._stop = None
        self._thread = None
        self._active = None

    def _open(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.dev)
        try:
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.dev)
        self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)

    def _loop(self):
        import pynvml
        while not self._stop.is_set():
            if not self._active.is_set():
                self._active.wait(0.05)
                continue
            try:
                sm = pynvml.nvmlDeviceGetClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
                reasons = pynvml.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                power = pynvml.nvmlDeviceGetPowerUsage(self.handle) / 1000.0
                self.rows.append((sm, reasons, power))
            except Exception:
                pass
            self._stop.wait(self.period)

    def __enter__(self):
        import threading
        try:
            self._open()
        except Exception as e:  # no NVML: report the clocks as unsampled
            log(f"clock sampler unavailable: {e}")
            return self
        self._stop = threading.Event()
        self._active = threading.Event()
        self._thread = threading.Thread(target=self._loop, daemon=True)
        self._thread.start()
        return self

    def timed(self, on):
        """Sample only while a timed region runs."""
        if self._active is not None:
            (self._active.set if on else self._active.clear)()

    def __exit__(self, *exc):
        if self._thread:
            self._stop.set()
            self._thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "samples": 0}
        sm = [r[0] for r in self.rows]
        reasons = sorted({name for _, bits, _ in self.rows for name, bit in self.REASONS if bits & bit})
        return {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm), "sm_max_mhz": self.max_mhz,
                "power_w_max": max(r[2] for r in self.rows), "reasons": reasons, "samples": len(self.rows),
                "source": f"NVML every {self.period * 1e3:.0f} ms during the timed regions"}


def dist_setup(n_gpus, collectives=True):
    """(world, rank, local rank) from torchrun's environment; joins the NCCL
    process group when several ranks run and `collectives` is set."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if world > 1 and not collectives:
        torch.cuda.set_device(local)
    elif world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_rel_diff(a, b):
    """Largest |a - b| / max(|a|, |b|) over the entries (0 where equal)."""
    import numpy as np
    scale = np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-300)
    d = np.where(a == b, 0.0, np.abs(a - b) / scale)
    return float(d.max()) if d.size else 0.0


def pinned_photons(n):
    """Photon SoA in one pinned (page-locked) host block laid out like the
    library's device block (grt_host_photon_layout), so it moves in one copy."""
    import torch
    from grt.abi import PhotonArrays
    t = torch.empty(146 * n, dtype=torch.uint8, pin_memory=True)
    pa = PhotonArrays.block(n, t.numpy())
    pa._keep = t
    return pa


def pinned_products(p, nx, ny):
    import numpy as np
    import torch
    from grt.abi import ProductArrays
    out = ProductArrays(0, 0, 0)
    out.nx, out.ny, out.bins = nx, ny, p.spectrum_bins
    keep = []

    def mk(shape, dtype=torch.float64):
        t = torch.zeros(shape, dtype=dtype, pin_memory=True)
        keep.append(t)
        return t.numpy()
    for f in ("image_I", "image_Q", "image_U", "image_V"):
        setattr(out, f, mk((ny, nx)))
    out.spectrum_frequency_hz = mk((p.spectrum_bins,))
    out.spectrum_I = mk((p.spectrum_bins,))
    out.arrived_count = mk((1,), torch.int64).view(np.uint64)
    out._keep = keep
    return out


def load_traffic():
    """DRAM bytes per trace launch from the committed ncu summary, if any."""
    path = ROOT / "profiles" / "trace_kernel_traffic.json"
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def run_ours(args):
    import numpy as np
    import torch
    from grt import abi, autotune, lib, workloads

    world, rank, local = dist_setup(args.gpus)
    w = workloads.WORKLOADS[args.workload]
    bw = workloads.BATCHES[args.workload]
    # N GPUs: a camera orbit of N frames (camera_phi = 2 pi k / N; the torus
    # and the metric are axisymmetric, so every frame costs the same), whole
    # frames assigned to ranks by shard_images -- the per-image partition of
    # the multi-GPU design -- and every step ends with an all-gather of the
    # frames' image products over NCCL.  One GPU renders frame 0, the workload.
    from grt import parallel
    frame_phis = [2.0 * math.pi * k / world for k in range(world)]
    my_frames = parallel.shard_images([1.0] * world, world)[rank]
    assert len(my_frames) == 1
    frame_phi = frame_phis[my_frames[0]]

    def frame_params(wl):
        q = wl.params()
        q.camera_phi = q.camera_phi + frame_phi
        return q

    if args.images:
        # a slice of the batch (its first N images), for profiling runs
        bw = workloads.BatchWorkload(f"{bw.name}_first{args.images}", bw.base, bw.images[:args.images])
    grid = w.torus()
    stream = torch.cuda.Stream()
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # Forms (all on the same torus, all through the C ABI, each step one
    # render through the context's CUDA graph: init the rays, trace them,
    # build every image's products on the device):
    #   fp64           -- the plain FP64 parity kernel on one image (one
    #                     frequency channel), the library's default launch shape;
    #   fp64_batched   -- the FP64 kernel on the batch (every frequency channel
    #                     of the image in one persistent launch);
    #   mixed_batched  -- the mixed FP32/FP64 kernel on the batch;
    #   mixed_grid_batched -- the same with the FP32 right-hand side inside the
    #                     fluid grid too after emission (GRT_PREC_MIXED_GRID).
    # The batched forms pick their launch shape with the autotuner.
    FORMS = {"fp64": (abi.PREC_FP64, False), "fp64_batched": (abi.PREC_FP64, True),
             "mixed_batched": (abi.PREC_MIXED, True), "mixed_grid_batched": (abi.PREC_MIXED_GRID, True)}
    wanted = [f for f in args.forms.split(",") if f]
    forms = {}
    for name in wanted:
        prec, batched = FORMS[name]
        p = frame_params(bw if batched else w)
        p.precision = prec
        ctx = lib.Context(p)
        ctx.set_stream(stream.cuda_stream)
        ctx.upload_grid(grid)
        forms[name] = (ctx, batched)
    specs = bw.specs(frame_params(bw))

    def prepare(ctx, batched):
        if batched:
            ctx.init_image_batch(specs)
        else:
            ctx.init_image_photons(w.pixels, w.pixels)

    # the batched forms pick their launch shape with the autotuner; the plain
    # FP64 form keeps the library's default shape
    cfg = {}
    for name, (ctx, batched) in forms.items():
        if batched and args.launch:
            b, r, g, sp = (int(v) for v in args.launch.split(","))
            ctx.set_launch_config(threads_per_block=128, blocks_per_sm=b, refill_threshold=r,
                                  photons_per_grab=g, split_legs=sp)
            cfg[name] = ctx.launch_config()
        elif batched and not args.no_autotune:
            cfg[name], _, table = autotune.tune(ctx, lambda c: prepare(c, True), bw.name, log=None)
            for c, ms in sorted(table, key=lambda x: x[1])[:4]:
                log(f"autotune {name} {c} {ms:.3f} ms")
        else:
            cfg[name] = ctx.launch_config()
    peak64, peak32 = lib.measure_fma_peaks()

    results = {}
    images = {}
    gathered_ok = {}
    sampler = ClockSampler(local).__enter__()
    for name, (ctx, batched) in forms.items():
        prepare(ctx, batched)
        gather = None
        if world > 1:
            import torch.distributed as dist
            nbytes = ctx.products_block_bytes
            mine = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
            every = torch.empty(world * nbytes, dtype=torch.uint8, device="cuda")

            def gather():
                # this rank's frame products, device to device, then every
                # rank's frames on every rank (NCCL), ordered on `stream`
                ctx.copy_products_block(mine.data_ptr(), nbytes)
                with torch.cuda.stream(stream):
                    dist.all_gather_into_tensor(every, mine)
        for _ in range(args.warmup):
            ctx.render_graph()  # graph: init rays, trace, every image's products
            if gather:
                gather()
        torch.cuda.synchronize()
        barrier(world)
        total_ms = 0.0
        trace_ms = 0.0
        launches = 0
        stats_acc = None
        sampler.timed(True)
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush_buf.zero_()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            st = ctx.render_graph()
            if gather:
                gather()
            ev1.record(stream)
            ev1.synchronize()
            total_ms += ev0.elapsed_time(ev1)
            trace_ms += st["trace_ms"]
            # our kernels per step: one init per image, the trace launches and
            # the products launches (up to 32 images each)
            launches += (len(specs) + -(-len(specs) // 32) if batched else 2) + st["launches"]
            stats_acc = st
        sampler.timed(False)
        torch.cuda.synchronize()
        if gather:
            # the gathered block of this rank equals its own products
            gathered_ok[name] = bool(torch.equal(every[rank * nbytes:(rank + 1) * nbytes], mine))
        barrier(world)
        total_ms = max_over_ranks(total_ms, world)
        n_rays = bw.rays if batched else w.pixels * w.pixels
        if batched:
            images[name] = [ctx.batch_image_products(k).image_I.copy() for k in range(len(specs))]
        else:
            images[name] = [ctx.image_products().image_I.copy()]
        results[name] = dict(ms_per_step=total_ms / args.steps, trace_ms_per_launch=trace_ms / args.steps,
                             stats=stats_acc, launches=launches, rays=n_rays, geodesics=ctx.geodesics,
                             geodesics_per_s=world * ctx.geodesics * args.steps / (total_ms * 1e-3),
                             rays_per_s=world * n_rays * args.steps / (total_ms * 1e-3),
                             rk_steps_per_s=world * stats_acc["accepted_steps"] * args.steps / (total_ms * 1e-3))

    # Stokes-I error of every frequency channel of each mixed batch against the
    # FP64 image of the same channel (the FP64 batch is bitwise the FP64 form
    # per image; without it, the channels are rendered once by the FP64 form).
    mixed_forms = [k for k in images if k.startswith("mixed")]
    errors = {}
    if mixed_forms:
        if "fp64_batched" in images:
            ref_imgs = images["fp64_batched"]
        else:
            q = frame_params(bw)
            ctx = lib.Context(q)
            ctx.upload_grid(grid)
            ctx.init_image_batch(specs)
            ctx.run()
            ref_imgs = [ctx.batch_image_products(k).image_I.copy() for k in range(len(specs))]
            ctx.close()
        for name in mixed_forms:
            errs, pix = [], []
            for got, ref_img in zip(images[name], ref_imgs):
                diff = got - ref_img
                nref = float(np.linalg.norm(ref_img))
                errs.append(float(np.linalg.norm(diff) / nref) if nref > 0 else float(np.linalg.norm(diff)))
                mask = np.abs(ref_img) > 1e-3 * np.abs(ref_img).max()
                pix.append(float(np.max(np.abs(diff[mask]) / np.abs(ref_img[mask]))) if mask.any() else 0.0)
            errors[name] = (max(errs), max(pix))
    # headline form: the fastest mixed batch whose images meet the 1e-5
    # Stokes-I bar, else the FP64 batch
    passing = [k for k in mixed_forms if errors[k][0] <= 1e-5]
    if passing:
        head = max(passing, key=lambda k: results[k]["rays_per_s"])
    elif "fp64_batched" in results:
        head = "fp64_batched"
    else:
        head = next(iter(results))
    stokes_err, per_pixel = errors.get(head, (None, None))
    H = results[head]
    ctx, batched = forms[head]

    # ---- e2e: the C ABI with host buffers (pinned), copies inside the timed region ----
    # serial: upload, trace and products back, one after another on one context
    prepare(ctx, batched)
    n_rays = ctx.n
    host_in = pinned_photons(n_rays)
    ctx.download_photons(host_in)
    if batched:
        host_out = [pinned_products(ctx.params, sp.nx, sp.ny) for sp in specs]
    else:
        host_out = [pinned_products(ctx.params, w.pixels, w.pixels)]

    def e2e_step():
        ctx.upload_photons(host_in)
        ctx.run()
        if batched:
            ctx.all_batch_image_products(host_out)
        else:
            ctx.image_products(host_out[0])

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    serial_ms = 0.0
    sampler.timed(True)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush_buf.zero_()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        e2e_step()
        ev1.record(stream)
        ev1.synchronize()
        serial_ms += ev0.elapsed_time(ev1)
    sampler.timed(False)
    serial_ms = max_over_ranks(serial_ms, world)
    p = ctx.params
    d2h = sum(8 * (4 * o.nx * o.ny + p.spectrum_bins + 1) for o in host_out)
    e2e_serial = {"value": world * n_rays * args.steps / (serial_ms * 1e-3), "unit": "rays/s",
                  "ms_per_step": serial_ms / args.steps}

    # streamed (batched forms): two contexts on the one stream, used in turn
    # through grt_render_async / grt_render_wait, each with its own pinned
    # input block and product buffers.  One context's upload and copy-back
    # overlap the other's trace; the traces stay in order on the shared stream.
    # The L2 flush before every render is on that stream, inside the timed
    # region.
    e2e_ms = None
    host_wall_ms = None
    if batched:
        ctx2 = lib.Context(ctx.params)
        ctx2.set_stream(stream.cuda_stream)
        ctx2.upload_grid(grid)
        ctx2.set_launch_config(**cfg[head])
        prepare(ctx2, True)
        host_in2 = pinned_photons(n_rays)
        host_in2._buffer[:] = host_in._buffer
        ctxs = [ctx, ctx2]
        ins = [host_in, host_in2]
        outs = [host_out, [pinned_products(ctx.params, sp.nx, sp.ny) for sp in specs]]

        def streamed(nsteps):
            pending = [False, False]
            for k in range(nsteps):
                c = k % 2
                if pending[c]:
                    ctxs[c].render_wait()
                with torch.cuda.stream(stream):
                    flush_buf.zero_()
                ctxs[c].render_async(ins[c], outs[c])
                pending[c] = True
            for c in (0, 1):
                if pending[c]:
                    ctxs[c].render_wait()

        streamed(max(args.warmup, 2))
        torch.cuda.synchronize()
        barrier(world)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler.timed(True)
        t0 = time.perf_counter()
        ev0.record(stream)
        streamed(args.steps)
        ev1.record(stream)
        ev1.synchronize()
        host_wall_ms = (time.perf_counter() - t0) * 1e3
        sampler.timed(False)
        e2e_ms = max_over_ranks(ev0.elapsed_time(ev1), world)
        # per-pixel sums of several arrivals are in atomic order: equal up to rounding
        diff_images = max(max_rel_diff(outs[c][k].image_I, images[head][k])
                          for c in (0, 1) for k in range(len(specs)))
        ctx2.close()
    sampler.__exit__(None, None, None)
    clocks = sampler.summary()
    if e2e_ms is None:
        e2e = dict(e2e_serial, mode="serial: upload, trace, products back on one context")
    else:
        e2e = {"value": world * n_rays * args.steps / (e2e_ms * 1e-3), "unit": "rays/s",
               "ms_per_step": e2e_ms / args.steps, "host_wall_ms_per_step": host_wall_ms / args.steps,
               "mode": "streamed: two contexts in turn on one stream (grt_render_async)",
               "image_I_max_rel_diff_vs_value_form": diff_images}
    e2e.update(h2d_bytes_per_step=PHOTON_BYTES * n_rays, d2h_bytes_per_step=d2h)

    # ---- roofline of the dominant kernel (the headline form's trace kernel) ----
    integrator = w.integrator
    flops = algorithmic_flops(H["stats"], integrator)
    achieved = flops / (H["trace_ms_per_launch"] * 1e-3) / 1e12
    traffic = load_traffic().get(f"{bw.name if batched else w.name}:{head}")
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                "frac": achieved / peak64, "traffic": traffic,
                "peak_source": "measured this run: FP64 FMA microbenchmark (grt_measure_fma_peaks)",
                "fp32_peak_tflops": peak32,
                "flops_per_launch": flops,
                "ops_per_unit": {"rhs": OPS_RHS, "rk4_step": OPS_RK4_STEP, "rk45_attempt": OPS_RK45_ATTEMPT}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w)
    for c, _ in forms.values():
        c.close()
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": H["rays_per_s"],
            "unit": "rays/s",
            "rk_steps_per_s": H["rk_steps_per_s"],
            # one traced geodesic carries every frequency channel of its pixel
            # (channel sharing), so rays/s counts channel images and
            # geodesics_per_s counts traced geodesics
            "geodesics_per_s": H["geodesics_per_s"],
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": H["ms_per_step"],
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64" if head.startswith("mixed") else "f64",
            "data": "synthetic (Fishbone-Moncrief torus generator, deterministic pixel-centre rays)",
            "config": {"workload": bw.name if batched else w.name,
                       "images": [{"inclination_deg": i, "pixels": f"{px}x{px}", "frequency_ghz": f}
                                  for i, px, f in bw.images] if batched else None,
                       "pixels": f"{w.pixels}x{w.pixels}",
                       "grid": "x".join(map(str, w.grid)), "spin": w.spin, "inclination_deg": w.inclination_deg,
                       "integrator": "rk45" if w.integrator else "rk4", "rtol": w.rtol,
                       "headline_form": head, "launch": cfg.get(head),
                       "rays_per_step": H["rays"], "geodesics_per_step": H["geodesics"],
                       "channel_sharing": bool(batched and H["geodesics"] < H["rays"]),
                       "l2": "flushed by a 256 MB device write before every timed step (outside the events)",
                       "parallelism": (f"frames x{world}: a camera orbit (camera_phi = 2 pi k / {world}), one "
                                       "frame per GPU (shard_images), image products all-gathered over NCCL every "
                                       "step inside the timed region" if world > 1 else "one GPU"),
                       "frames": world},
            "forms": {k: {"rays_per_step": v["rays"], "rays_per_s": v["rays_per_s"],
                          "geodesics_per_step": v["geodesics"], "geodesics_per_s": v["geodesics_per_s"],
                          "rk_steps_per_s": v["rk_steps_per_s"],
                          "ms_per_step": v["ms_per_step"], "trace_ms_per_launch": v["trace_ms_per_launch"],
                          "accepted_steps": v["stats"]["accepted_steps"],
                          "rejected_attempts": v["stats"]["rejected_attempts"],
                          "launch": cfg.get(k)} for k, v in results.items()},
            # where the speed-up comes from: batching with channel sharing
            # (rays per traced geodesic) and the precision form at equal
            # geodesics (mixed batch against the FP64 batch, trace only)
            "speedup_mixed_batched_vs_fp64": (results[head]["rays_per_s"] / results["fp64"]["rays_per_s"]
                                              if head.startswith("mixed") and "fp64" in results else None),
            "speedup_mixed_vs_fp64_same_batch": (
                results["fp64_batched"]["trace_ms_per_launch"] / results[head]["trace_ms_per_launch"]
                if head.startswith("mixed") and "fp64_batched" in results else None),
            "speedup_fp64_batched_vs_fp64_per_geodesic": (
                results["fp64_batched"]["geodesics_per_s"] / results["fp64"]["geodesics_per_s"]
                if "fp64_batched" in results and "fp64" in results else None),
            "stokes_I_rel_err": stokes_err,
            "stokes_I_max_pixel_rel_err": per_pixel,
            "stokes_I_rel_err_by_form": {k: {"l2": v[0], "max_pixel": v[1]} for k, v in errors.items()},
            "e2e": e2e,
            "e2e_serial": e2e_serial,
            "gpu_launches": H["launches"],
            "products_gather_check": gathered_ok or None,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        if world == 1 and args.workload == "c2" and not args.no_other_workloads:
            line["other_workloads"] = other_workloads()
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# The other configurations: workload and timed steps of each.
OTHER_WORKLOADS = (("c1", 10), ("c3", 3), ("c4", 10), ("c5", 2))


def other_workloads():
    """C1, C3, C4 and C5, each run by this script in a child process of its own
    (its own timing rules: warm-up, L2 flush, CUDA events) after the headline's
    timed region has ended, so that one default run reports every
    configuration.  Each entry is a summary of that run's JSON line, or the
    reason it failed."""
    out = {}
    for wl, steps in OTHER_WORKLOADS:
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", wl, "--steps", str(steps), "--warmup", "3",
               "--no-cpu-baseline"]
        env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE")}
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, env=env)
            lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
            if r.returncode != 0 or not lines:
                out[wl] = {"error": f"exit {r.returncode}: {r.stderr.strip()[-300:]}"}
                continue
            d = json.loads(lines[-1])
        except Exception as e:  # a failed configuration must not cost the headline line
            out[wl] = {"error": repr(e)[:300]}
            continue
        keys = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "dtype", "gpu_launches", "forward_ms",
                "adjoint_ms", "emission_ms", "transport_ms", "rk_steps_per_s", "geodesics_per_s", "packets")
        summary = {k: d[k] for k in keys if k in d}
        summary["workload"] = (d.get("config") or {}).get("workload")
        if d.get("roofline"):
            summary["roofline_frac"] = d["roofline"].get("frac")
        if isinstance(d.get("e2e"), dict):
            summary["e2e"] = d["e2e"].get("value")
        if d.get("forms"):
            summary["forms"] = {k: {"rays_per_s": v.get("rays_per_s"), "trace_ms_per_launch": v.get("trace_ms_per_launch")}
                                for k, v in d["forms"].items()}
        if d.get("clocks"):
            summary["clocks"] = {k: d["clocks"].get(k) for k in ("sm_mhz", "reasons")}
        out[wl] = summary
    return out


def cpu_baseline(w, reps=2, params=None, label=None):
    """The reference's own integrate_geodesics (shim-compiled, oracle/_ref) on
    the host cores, on one full image of workload w (params: that image's
    parameters, default w's); falls back to the oracle port."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    from grt import config, torus
    p = params if params is not None else w.params()
    n = w.pixels * w.pixels
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        torus.write_numpy_dir(w.torus(), d / "np")
        toml = config.write_toml(p, d / "c.toml", d / "np", d / "out")
        best = None
        if pyoracle.Reference.available():
            ref = pyoracle.Reference()
            kind = "reference"
            for _ in range(reps):
                ph = ref.init_image_photons(toml, w.pixels, w.pixels)
                _, st = ref.run(toml, ph, None)
                if best is None or st["elapsed_s"] < best[0]:
                    best = (st["elapsed_s"], st["stepped"])
        else:
            o = pyoracle.Oracle()
            kind = "port"
            for _ in range(reps):
                ph = o.init_image_photons(p, w.pixels, w.pixels)
                t0 = time.perf_counter()
                st = o.run(p, w.torus(), ph)
                dt = time.perf_counter() - t0
                if best is None or dt < best[0]:
                    best = (dt, st["accepted_steps"])
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return {"value": n / best[0], "unit": "rays/s", "rk_steps_per_s": best[1] / best[0], "cores": cores,
            "kind": kind,
            "sample": f"{label or 'full ' + w.name + ' workload'} ({n} rays), best of {reps}; reference Kokkos "
                      "functor via the project OpenMP shim (real Kokkos is not installable offline), "
                      "OMP threads = all cores"}


def run_reference(args):
    """The reference arm: the reference's own CPU code (oracle/_ref) on the
    workload of our arm -- for the default, the C2 image at its four frequency
    channels.  The reference traces one camera per run, so each step is one
    channel's full 256x256 image (a bounded sample of the batch), cycling
    through the channels; rays/s is the batch's metric."""
    import math
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from grt import workloads
    w = workloads.WORKLOADS[args.workload]
    bw = workloads.BATCHES.get(args.workload)
    # one parameter set per channel image of the batch with w's resolution
    chans = []
    if bw is not None:
        for incl, px, f_ghz in bw.images:
            if px != w.pixels:
                continue
            q = w.params()
            q.update(camera_theta=math.radians(incl), custom_frequency_hz=f_ghz * 1e9,
                     emission_coefficient=q.emission_coefficient * f_ghz / 230.0)
            chans.append((q, f"{incl:g} deg, {f_ghz:g} GHz"))
    if not chans:
        chans = [(w.params(), w.name)]
    vals = []
    for i in range(args.warmup):
        cpu_baseline(w, reps=1, params=chans[i % len(chans)][0])
    t_total = 0.0
    steps_total = 0.0
    for i in range(args.steps):
        q, lab = chans[i % len(chans)]
        c = cpu_baseline(w, reps=1, params=q, label=f"one {w.pixels}x{w.pixels} channel image per step ({lab})")
        vals.append(c)
        t_total += (w.pixels * w.pixels) / c["value"]
        steps_total += c["rk_steps_per_s"] * (w.pixels * w.pixels) / c["value"]
    n = w.pixels * w.pixels * args.steps
    value = n / t_total
    c = vals[-1]
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rays/s",
        "rk_steps_per_s": steps_total / t_total, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": bw.name if bw is not None else w.name, "pixels": f"{w.pixels}x{w.pixels}",
                   "grid": "x".join(map(str, w.grid)),
                   "sample": f"one channel image per step, cycling through {len(chans)} channel(s)"},
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": c["cores"], "kind": c["kind"],
                         "sample": c["sample"]},
        "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def timed_call(stream, fn):
    """(result, ms) of fn() bracketed by CUDA events on `stream`."""
    import torch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    out = fn()
    ev1.record(stream)
    ev1.synchronize()
    return out, ev0.elapsed_time(ev1)


def run_adjoint(args):
    """C4: the adjoint of the radiative-transfer sweep -- checkpointed forward
    trace of the 128x128 line-of-sight image over the 96x48x48 torus, then the
    reverse sweep for an L2 loss to a target rendered from perturbed
    multipliers.  One step = forward + adjoint; reports rays/s of the pair."""
    import numpy as np
    import torch
    from grt import lib, workloads
    world, rank, _ = dist_setup(args.gpus, collectives=False)
    if rank != 0:  # a one-GPU measurement: rank 0 runs it, the other ranks exit
        return
    w = workloads.C4
    p = w.params()
    grid = w.torus()
    shape = grid["r.npy"].shape
    stream = torch.cuda.Stream()
    ta, te = workloads.c4_target_multipliers(shape)
    ctx = lib.Context(p)
    ctx.set_stream(stream.cuda_stream)
    ctx.upload_grid(grid)
    ctx.set_cell_multipliers(ta, te)
    ctx.init_image_forward_photons(p.image_nx, p.image_ny, workloads.C4_BACK_DISTANCE)
    ctx.run()
    target = ctx.image_products().image_I.copy()
    ctx.set_cell_multipliers(None, None)
    fwd_ms = adj_ms = 0.0
    st = None
    for it in range(args.warmup + args.steps):
        ctx.init_image_forward_photons(p.image_nx, p.image_ny, workloads.C4_BACK_DISTANCE)
        st, f_ms = timed_call(stream, lambda: ctx.forward_checkpointed(workloads.C4_CHECKPOINT_INTERVAL))
        img = ctx.image_products().image_I
        dL = 2.0 * (img - target)
        (ga, ge), a_ms = timed_call(stream, lambda: ctx.adjoint_image_I(dL, shape))
        if it >= args.warmup:
            fwd_ms += f_ms
            adj_ms += a_ms
    ctx.close()
    n = p.image_nx * p.image_ny
    total = fwd_ms + adj_ms
    print(json.dumps({
        "metric": "adjoint (checkpointed forward + reverse sweep) rays/s on 1 B200", "value": n * args.steps / (total * 1e-3),
        "unit": "rays/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps, "forward_ms": fwd_ms / args.steps, "adjoint_ms": adj_ms / args.steps,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic (Fishbone-Moncrief torus, seeded lognormal target)",
        "photon_calls": st["photon_calls"], "nonzero_gradient_cells": int(np.count_nonzero(ga) + np.count_nonzero(ge)),
        "config": {"workload": w.name, "pixels": f"{p.image_nx}x{p.image_ny}", "grid": "x".join(map(str, w.grid)),
                   "checkpoint_interval": workloads.C4_CHECKPOINT_INTERVAL}}), flush=True)


def run_disk(args):
    """C5: disk-mode scattering Monte Carlo -- about 1e7 packets emitted on the
    device from the 128x64x64 torus, traced with isotropic fluid-frame
    scattering to escape or capture.  One step = emission + transport."""
    import torch
    from grt import lib, workloads
    world, rank, _ = dist_setup(args.gpus, collectives=False)
    if rank != 0:  # a one-GPU measurement: rank 0 runs it, the other ranks exit
        return
    w = workloads.C5
    if args.disk_normalization:
        # fewer packets (a smaller case of the same run, for profiling)
        w = workloads.DiskWorkload(f"{w.name}_norm{args.disk_normalization:g}", w.grid, w.spin,
                                   args.disk_normalization)
    p = w.params()
    stream = torch.cuda.Stream()
    ctx = lib.Context(p)
    ctx.set_stream(stream.cuda_stream)
    ctx.upload_grid(w.torus())
    n = ctx.init_disk_photons()
    q = p.copy()
    q.nphotons = n
    ctx.set_params(q)
    if args.launch:
        b, r, g, sp = (int(v) for v in args.launch.split(","))
        ctx.set_launch_config(threads_per_block=128, blocks_per_sm=b, refill_threshold=r, photons_per_grab=g,
                              split_legs=sp)
    elif not args.no_autotune:
        from grt import autotune
        autotune.tune(ctx, lambda c: c.init_disk_photons(), w.name, reps=1)
    cfg = ctx.launch_config()
    init_ms = run_ms = 0.0
    st = None
    for it in range(args.warmup + args.steps):
        n, i_ms = timed_call(stream, ctx.init_disk_photons)
        st, r_ms = timed_call(stream, ctx.run)
        if it >= args.warmup:
            init_ms += i_ms
            run_ms += r_ms
    ctx.close()
    total = init_ms + run_ms
    print(json.dumps({
        "metric": "disk-mode packets/s on 1 B200 (emission + scattering transport)", "value": n * args.steps / (total * 1e-3),
        "unit": "packets/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps,
        "emission_ms": init_ms / args.steps, "transport_ms": run_ms / args.steps,
        "rk_steps_per_s": st["accepted_steps"] * args.steps / (total * 1e-3), "packets": n,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic (Fishbone-Moncrief torus)",
        "config": {"workload": w.name, "grid": "x".join(map(str, w.grid)), "spin": w.spin, "launch": cfg}}),
          flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="c2", choices=("c1", "c2", "c3", "c4", "c5"),
                    help="c2 (the headline), c1, c3 (the 64-image batch), c4 (adjoint), c5 (disk mode)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other-workloads", action="store_true",
                    help="c2 on one GPU: skip the runs of c1, c3, c4 and c5 that follow the headline")
    ap.add_argument("--no-autotune", action="store_true", help="use the library's default launch shape")
    ap.add_argument("--forms", default="fp64,fp64_batched,mixed_batched",
                    help="comma list of fp64, fp64_batched, mixed_batched, mixed_grid_batched")
    ap.add_argument("--images", type=int, default=0,
                    help="only the first N images of the workload's batch (a slice for profiling)")
    ap.add_argument("--launch", default="",
                    help="fixed launch shape of the batched forms (and of c5): blocks_per_sm,refill_threshold,"
                         "photons_per_grab,split_legs (instead of the autotuner)")
    ap.add_argument("--disk-normalization", type=float, default=0.0,
                    help="c5 only: superphoton normalisation (packets per unit density) instead of the "
                         "workload's 210, e.g. 21 for about 1e6 packets (a smaller case for profiling)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)  # at least three untimed warm-up steps
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c4":
        run_adjoint(args)
    elif args.workload == "c5":
        run_disk(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
