#!/usr/bin/env python
"""Benchmark of the FDTD step: Gvoxel-updates/s and the HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl virs|reference]

One step = one time step of the simulation over the whole grid.  The default
workload is the large hall, 1024x768x512 FP32 voxels (402.7 M) with two
3-section absorbing materials, one Gaussian-pulse source and 8 receivers;
all fields (1.6 GB each) are far larger than the 126 MB L2, so no flush is
needed between steps.  With --gpus N under torchrun every rank runs its own
hall (independent replicas, no collective on the data path; weak scaling);
the time is the maximum over ranks.

The JSON line carries:
  value       Gvoxel-updates/s of the device-resident run (virs_run, CUDA
              graph), inputs already in HBM
  e2e         the same through virs_run_host with pinned host buffers: the
              step's source samples in and the receiver samples out are
              copied inside the timed region
  roofline    algorithmic bytes of the stencil kernel (13 B per voxel
              update in FP32: p 4 + p^{n-1} 4 + p^{n+1} 4 + cell code 1) over
              its CUDA-event duration, against the measured HBM copy
              bandwidth of MEASURED_PEAKS.json
  cpu_baseline  the CPU oracle's FP32 step (OpenMP, all host threads) on a
              crop of the hall
  variants    the BF16-storage form of the same hall, and the batched
              workload (64 source positions in a 256^3 room + 16 rooms of
              96^3..320^3, 1.29 G voxels per step) in FP32 and BF16 storage

--impl reference times the reference's CPU implementation of this path.
The reference's own CPU build cannot be compiled here (oneTBB, Embree,
tinyobjloader, kfr, AudioFile are absent), so this arm runs the CPU
restatement of its step (oracle/), on all host threads, on a crop of the
same hall sized so that the run ends within a few minutes.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

GRAPH_WARMUP = 64  # warm-up steps at least: both step graphs (32 steps per parity) built and launched once
BYTES_F32 = 13.0   # per voxel update: p 4 + p^{n-1} 4 + p^{n+1} 4 + code 1
BYTES_16 = 7.0     # 16-bit storage: 2 + 2 + 2 + 1
# two steps per pass (time blocking), per voxel and launch: p^n, p^{n-1} in,
# the code, p^{n+1}, p^{n+2} out
PAIR_F32 = 17.0    # 4 + 4 + 1 + 4 + 4
PAIR_16 = 9.0      # 2 + 2 + 1 + 2 + 2
METRIC = "Gvoxel-updates/s"
STORAGE_NAMES = {"f32": "FP32", "bf16": "BF16 storage (FP32 update)", "f16": "FP16 storage (FP32 update)"}
KERNEL_TYPES = {"f32": "float", "bf16": "__nv_bfloat16", "f16": "__half"}


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_traffic(path: Path, storage: str, nvox: int):
    """DRAM bytes (read + write) per launch of the stencil kernel, from the ncu
    summary: lines `storage=<s> voxels=<n> bytes_per_launch=<b> ...`, scaled by
    the voxel count when the capture ran a smaller grid."""
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        f = dict(kv.split("=", 1) for kv in line.split() if "=" in kv)
        if f.get("storage") == storage and "voxels" in f and "bytes_per_launch" in f:
            n, b = int(f["voxels"]), float(f["bytes_per_launch"])
            src = f"ncu dram__bytes_read.sum + dram__bytes_write.sum, {path.name}"
            if n != nvox:
                src += f", captured on {n} voxels and scaled by {nvox / n:.3f}"
            return {"bytes": round(b * nvox / n), "source": src}
    return None


def stencil_roofline(r, storage: str):
    """(algorithmic bytes per voxel and launch, steps per launch, kernel name,
    traffic file) of the run's dominant kernel: the two-step kernel when the
    autotuner chose time blocking, else the single-step stencil."""
    f32 = storage == "f32"
    if r.get("time_blocking", {}).get("active"):
        return (PAIR_F32 if f32 else PAIR_16, 2, "k_pair_tma<%s> (two steps per pass; then the boundary passes, "
                "post kernels and the fix-up of the voxels next to boundary voxels and sources)" % KERNEL_TYPES[storage],
                ROOT / "profiles" / "k_pair_tma_dram_traffic.txt")
    return (BYTES_F32 if f32 else BYTES_16, 1,
            "k_step_tma<%s> (stencil; boundary voxels in a separate list pass)" % KERNEL_TYPES[storage],
            ROOT / "profiles" / "k_step_tma_dram_traffic.txt")


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---- clocks -------------------------------------------------------------------

class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.path:
            return {"unavailable": "nvidia-smi not runnable"}
        rows = []
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), float(f[3]), f[4:]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"unavailable": "no samples"}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[3][1:5]) if v.lower() == "active"})
        loaded = [r for r in rows if r[2] > 200.0] or rows
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(rows), "reasons": reasons}


# ---- the CUDA path ----------------------------------------------------------------

def gpu_uuid(dev):
    import torch
    u = str(torch.cuda.get_device_properties(dev).uuid)
    return u if u.startswith("GPU-") else "GPU-" + u


def max_over_ranks(ms: float, dist, device: str) -> float:
    """The slowest rank's time: every rank takes part, and every rank gets
    the maximum (a no-op without a process group)."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def time_run(sim, steps, stream):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    sim.run(steps, stream.cuda_stream)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def bench_storage(sc, storage, args, stream, dev, world, dist, want_e2e, rounding=0):
    """Warm up, then time K steps: device-resident graph run, a per-kernel
    CUDA-event pass, and (optionally) the end-to-end host run.  rounding:
    the 16-bit stores' rounding (virs_set_rounding)."""
    import torch
    from virs_b200 import scenes
    warm = max(args.warmup, GRAPH_WARMUP)
    total = warm + args.steps + (args.kernel_steps if args.kernel_steps else 0) + (args.steps if want_e2e else 0)
    total += args.sustained_steps if want_e2e else 0
    sim, meta = scenes.build_simulation(sc, storage=storage, device=dev, steps=total)
    if rounding:
        sim.set_rounding(rounding)
    t_pre = time.perf_counter()
    tiling = sim.autotune(args.tune_steps) if args.tune_steps else sim.tiling()
    tune_s = time.perf_counter() - t_pre
    if args.steps_per_pass:
        # forced: single steps, or two steps per pass with the autotuner's
        # two-step tiling when it chose one, else --pair-tiling
        tb = sim.time_blocking()
        rows, planes = (tb["rows"], tb["planes"]) if tb["active"] and not args.pair_tiling else \
            tuple(args.pair_tiling or (14, 42))
        sim.set_time_blocking(args.steps_per_pass, rows, planes)
    sim.run(warm, stream.cuda_stream)
    torch.cuda.synchronize()
    pre_s = time.perf_counter() - t_pre
    if dist:
        dist.barrier()
    with Clocks(gpu_uuid(dev)) as clk:
        ms = time_run(sim, args.steps, stream)
    ms = max_over_ranks(ms, dist, f"cuda:{dev}")
    out = {"ms": ms, "clocks": clk.summary(), "meta": meta,
           "warmup": {"steps": warm, "autotune_s": round(tune_s, 2), "seconds": round(pre_s, 2),
                      "autotune_trial_steps": args.tune_steps},
           "tiling": {"tile_rows": tiling.tile_rows, "planes_per_block": tiling.planes_per_block,
                      "pipeline_depth": tiling.pipeline_depth},
           "time_blocking": sim.time_blocking()}
    # per-kernel events over K' steps (no graph; events around each stencil launch)
    if args.kernel_steps:
        sim.set_timing(True)
        sim.run(args.kernel_steps, stream.cuda_stream)
        sim.synchronize()
        t = sim.timing()
        sim.set_timing(False)
        # per launch of the dominant kernel (two steps with time blocking);
        # the boundary pass per step
        out["kernel_ms"] = t.step_kernel_ms / max(t.step_launches, 1)
        per = 2 if out["time_blocking"]["active"] else 1
        out["boundary_ms"] = t.boundary_kernel_ms / max(t.step_launches * per, 1)
        # the library's count of its kernel launches (5 per two steps with
        # time blocking, 3 per step otherwise)
        out["launches_per_step"] = t.kernel_launches / args.kernel_steps
    if want_e2e:
        nsrc, nrcv = len(sc.src_pos), len(sc.rcv_pos)
        first = int(sim.info().steps_done)
        sig = torch.empty((nsrc, args.steps), dtype=torch.float32, pin_memory=True)
        sig.copy_(torch.from_numpy(np.ascontiguousarray(sc.src_sig[:, first:first + args.steps])))
        ir = torch.empty((nrcv, args.steps), dtype=torch.float32, pin_memory=True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        e0.record(stream)
        sim.run_host_ptr(args.steps, sig.data_ptr(), ir.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        ems = e0.elapsed_time(e1)
        ems = max_over_ranks(ems, dist, f"cuda:{dev}")
        out["e2e_ms"] = ems
        out["e2e_wall_ms"] = wall
        out["h2d"] = 4 * nsrc
        out["d2h"] = 4 * nrcv
        out["ir_finite"] = bool(torch.isfinite(ir).all())
    if want_e2e and args.sustained_steps:
        # the configuration's whole run at once: within about a second the
        # GPU reaches its power cap, so this rate sits below the short
        # timed region's; reported beside it with its own clock record
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        with Clocks(gpu_uuid(dev)) as clk:
            sms = time_run(sim, args.sustained_steps, stream)
        out["sustained"] = {"ms": max_over_ranks(sms, dist, f"cuda:{dev}"), "clocks": clk.summary()}
    sim.close()
    return out


def bench_batch(storage, args, stream, dev, dist=None):
    """The batched workload: 64 source positions in a 256^3 room plus 16 rooms
    of 96^3..320^3, advanced by three launches per step (virs_batch)."""
    import torch
    from virs_b200 import capi, scenes
    steps, warm = args.batch_steps, GRAPH_WARMUP
    scs = scenes.batched(steps=steps + warm + 2 * 3 + 4)
    sims = [scenes.build_simulation(sc, storage=storage, device=dev)[0] for sc in scs]
    nvox = sum(int(np.prod(s.shape)) for s in sims)
    b = capi.Batch(sims)
    t = b.autotune(2)
    b.run(warm, stream.cuda_stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0.record(stream)
    b.run(steps, stream.cuda_stream)
    e1.record(stream)
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{dev}")
    b.synchronize()
    ok = all(bool(np.isfinite(s.ir()).all()) for s in sims)
    b.close()
    for s in sims:
        s.close()
    return {"value": nvox * steps / (ms * 1e-3) / 1e9, "ms_per_step": ms / steps, "members": len(scs),
            "voxels_per_step": nvox, "steps": steps, "tiling": [t.tile_rows, t.planes_per_block, t.pipeline_depth],
            "ir_finite": ok, "launches_per_step": 3}


CPU_CROP_PLANES = 16   # planes of the hall crop both CPU figures time


def bench_ir_postprocess(dev, steps=4000, reps=5):
    """The end of a simulation on the GPU: the 8 receiver traces of a
    4000-step run of the 128^3 hall crop resampled to 48 kHz, by the
    reference's Chebyshev-I cascade plus linear interpolation
    (virs_postprocess_ir) and by the Kaiser-windowed sinc
    (virs_postprocess_ir_sinc), each peak-normalised.  Host clock around a
    whole call (size query, kernels, copy of the result to the host), best
    of `reps` after one untimed call.  The hall's simulation rate (38 kHz)
    is below 48 kHz: the step upsamples, and the anti-alias design for that
    rate, with its stop band at the simulation's Nyquist frequency, is one
    section."""
    from virs_b200 import capi, scenes
    sc = scenes.large_hall(steps=steps, size=(128, 128, 128))
    sim, _ = scenes.build_simulation(sc, device=dev)
    sim.run(steps)
    sim.synchronize()
    dt = float(sim.info().dt)
    fs = float(np.float32(1.0) / np.float32(dt))
    band = min(fs, 48000.0)
    sos = capi.design_chebyshev_lowpass(fs, 0.45 * band, 0.5 * band)
    out = {"receivers": int(sim.ir().shape[0]), "samples_in": steps, "rate_in_hz": round(fs, 1),
           "sections": int(sos.shape[0])}
    for name, call in (("chebyshev_linear", lambda: sim.postprocess_ir(48000.0, sos, True)),
                       ("kaiser_sinc", lambda: sim.postprocess_ir_sinc(48000.0))):
        y = call()
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            call()
            best = min(best, time.perf_counter() - t0)
        out[name + "_ms"] = round(best * 1e3, 3)
        out["samples_out"] = int(y.shape[1])
    sim.close()
    return out


def bench_adjoint(args, stream, dev):
    """The inverse-design configuration: 128x128x96, 6 materials x 2
    sections, 4 receivers, 4000 steps, checkpoints every 64.  The forward
    pass (virs_forward_checkpointed) is timed with CUDA events; the reverse
    pass (virs_adjoint: recomputation of every segment, the adjoint steps,
    the FP64 gradient sums, gradients copied to the host) by the host clock
    around the synchronous call."""
    import torch
    from virs_b200 import scenes
    sc, guess = scenes.inverse_design(steps=args.adjoint_steps)
    every = 64
    sim, _ = scenes.build_simulation(sc)
    nvox = int(np.prod(sim.shape))
    # warm-up: both passes once at the full length, so that the checkpoint
    # and segment buffers exist before the timed passes
    sim.forward_checkpointed(sc.steps, every)
    sim.adjoint(np.zeros((len(sc.rcv_pos), sc.steps), np.float32), sc.n_materials, sc.n_sections)
    sim.start(sc.steps)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    sim.forward_checkpointed(sc.steps, every, stream.cuda_stream)
    e1.record(stream)
    e1.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    ir = sim.ir(0, sc.steps)
    dl = (2.0 * ir / ir.size).astype(np.float32)
    t0 = time.perf_counter()
    gc, gs = sim.adjoint(dl, sc.n_materials, sc.n_sections)
    adj_ms = (time.perf_counter() - t0) * 1e3
    sim.close()
    return {"workload": "inverse design 128x128x96, 6 materials x 2 sections, 4 receivers, %d steps, "
                        "checkpoint every %d" % (sc.steps, every),
            "forward_ms": round(fwd_ms, 2), "adjoint_ms": round(adj_ms, 2),
            "forward_value": round(nvox * sc.steps / (fwd_ms * 1e-3) / 1e9, 3),
            "gradient_value": round(nvox * sc.steps / ((fwd_ms + adj_ms) * 1e-3) / 1e9, 3),
            "unit": "Gvoxel-updates/s (forward; forward + reverse for the gradient)",
            "grad_finite": bool(np.isfinite(gc).all() and np.isfinite(gs).all())}


def bench_slabs(sc, args, dev, parts=2, steps=100):
    """The hall split into `parts` z-slabs on this GPU, advanced by
    virs_slab_run (ghost planes pulled by device copies every step beside
    the interior stencil, single steps, the 16-step slab graph): the cost of
    the slab machinery against the whole grid.  The warm-up captures the
    graph.  Timed by the host clock around the queued run and a
    synchronisation of every slab."""
    from virs_b200 import capi, scenes
    parts_, meta = scenes.build_slabs(sc, parts, device=dev)
    sims = [p[0] for p in parts_]
    nvox = int(np.prod(meta["shape"]))
    capi.slab_run(sims, 32)                             # warm-up: captures the graph
    for s in sims:
        s.synchronize()
    t0 = time.perf_counter()
    capi.slab_run(sims, steps)
    for s in sims:
        s.synchronize()
    secs = time.perf_counter() - t0
    for s in sims:
        s.close()
    return {"parts": parts, "steps": steps, "value": round(nvox * steps / secs / 1e9, 3),
            "ms_per_step": secs * 1e3 / steps, "timing": "host clock around virs_slab_run and the synchronisations"}


def cpu_sample(shape, steps_budget_s, threads):
    """The oracle's FP32 step on a crop of the hall (same x, y extent,
    CPU_CROP_PLANES planes), timed on the host in chunks of about a second
    until the budget is spent; returns (Gvox/s, description, seconds).  The
    main arm's cpu_baseline and the reference arm both report this figure.
    The scene's absorbers are designed with the oracle's FP64 designs, so
    this leg runs no part of the library."""
    import oracle
    from virs_b200 import scenes
    sys.path.insert(0, str(ROOT / "tests"))
    from helpers import oracle_grid, oracle_scene
    oracle.set_threads(threads)
    nx, ny, nz = shape
    nzc = CPU_CROP_PLANES
    with scenes.designs(oracle.design_first_order, oracle.design_octave_cascade):
        sc = scenes.large_hall(steps=64, size=(nx, ny, nzc))
    g = oracle_grid(sc)
    osc = oracle_scene(sc, g)
    n = nx * ny * nzc
    st = (np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(g["bidx"].size * 12 + 1, np.float32))
    osc.run(4, state=st)                               # touch the pages, start the threads
    t0 = time.perf_counter()
    osc.run(4, state=st, step0=4)
    per_step = (time.perf_counter() - t0) / 4
    # chunks of about a second until the budget is spent
    chunk = max(1, min(20000, int(1.0 / max(per_step, 1e-6))))
    k, dt, step = 0, 0.0, 8
    while dt < steps_budget_s and k < 200000:
        t0 = time.perf_counter()
        osc.run(chunk, state=st, step0=step)
        dt += time.perf_counter() - t0
        k += chunk
        step += chunk
    return n * k / dt / 1e9, f"{k} steps of a {nx}x{ny}x{nzc} crop of the hall ({n * k / 1e9:.2f} G voxel updates)", dt


def run_virs(args):
    import torch
    rank, world, local = env_rank()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    dev = local
    torch.cuda.set_device(dev)
    from virs_b200 import capi, scenes
    total_steps = max(args.warmup, GRAPH_WARMUP) + 3 * args.steps + args.kernel_steps + args.sustained_steps + 16
    sc = scenes.large_hall(steps=total_steps, size=tuple(args.size))
    nvox = int(np.prod(args.size))
    stream = torch.cuda.Stream(device=dev)
    storage = {"f32": capi.STORAGE_F32, "bf16": capi.STORAGE_BF16, "f16": capi.STORAGE_F16}[args.storage]
    fbytes = 4 if storage == capi.STORAGE_F32 else 2   # bytes of one field value
    r32 = bench_storage(sc, storage, args, stream, dev, world, dist, want_e2e=True)
    variants = {}
    if args.variants and storage == capi.STORAGE_F32:
        rb = bench_storage(sc, capi.STORAGE_BF16, args, stream, dev, world, dist, want_e2e=False)
        gv = nvox * args.steps / (rb["ms"] * 1e-3) / 1e9 * world
        peak, _ = peaks()
        _, bsteps, bkern, _ = stencil_roofline(rb, "bf16")
        variants["bf16_storage"] = {
            "value": gv, "ms_per_step": rb["ms"] / args.steps,
            "speedup_vs_f32": (r32["ms"] / rb["ms"]),
            "roofline_frac": (nvox * BYTES_16 * bsteps / (rb["kernel_ms"] * 1e-3) / 1e9) / peak
            if rb.get("kernel_ms") else None,
            "bytes_per_voxel": BYTES_16,
            "kernel": bkern.split(" ")[0],
            "kernel_ms": rb.get("kernel_ms"),
            "boundary_ms": rb.get("boundary_ms"),
            "time_blocking": rb["time_blocking"],
        }
        # the same with stochastic rounding of the 16-bit stores: the cost of
        # the per-voxel hash (two steps per pass do not apply it)
        rs = bench_storage(sc, capi.STORAGE_BF16, args, stream, dev, world, dist, want_e2e=False,
                           rounding=capi.ROUND_STOCHASTIC)
        variants["bf16_storage_stochastic_rounding"] = {
            "value": nvox * args.steps / (rs["ms"] * 1e-3) / 1e9 * world, "ms_per_step": rs["ms"] / args.steps,
            "vs_bf16_nearest": rb["ms"] / rs["ms"],
            "kernel_ms": rs.get("kernel_ms"), "kernel_ms_nearest": rb.get("kernel_ms"),
            "boundary_ms": rs.get("boundary_ms"),
        }
    if args.adjoint:
        variants["adjoint_inverse_design"] = bench_adjoint(args, stream, dev)
    if args.variants:
        variants["ir_postprocess"] = bench_ir_postprocess(dev)
    if args.slabs and world == 1:
        variants["slabs_2_one_gpu"] = bench_slabs(sc, args, dev)
    if args.batch_steps:
        for name, st in (("batched_f32", capi.STORAGE_F32), ("batched_bf16", capi.STORAGE_BF16)):
            rb = bench_batch(st, args, stream, dev, dist)
            rb["value"] *= world
            variants[name] = rb
        variants["bf16_batched_vs_f32_plain"] = None   # filled below
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peak, peak_kind = peaks()
    value = nvox * args.steps / (r32["ms"] * 1e-3) / 1e9 * world
    interior = int(np.prod([d - 2 for d in args.size]))
    kernel_ms = r32.get("kernel_ms")
    bpv, steps_per_launch, kernel_name, traffic_file = stencil_roofline(r32, args.storage)
    # achieved: the launch's own algorithmic bytes (13 / 7 B per voxel for a
    # single step; 17 / 9 B per voxel for a two-step launch, which reads p^n,
    # p^{n-1} and the code once and writes p^{n+1} and p^{n+2}) over its
    # CUDA-event duration.  The per-update basis (13 / 7 B per voxel update
    # times the updates a launch makes) is reported beside it as an
    # effective bandwidth: with time blocking it exceeds the bytes moved.
    upd = BYTES_F32 if args.storage == "f32" else BYTES_16
    effective = nvox * upd * steps_per_launch / (kernel_ms * 1e-3) / 1e9 if kernel_ms else None
    achieved = nvox * bpv / (kernel_ms * 1e-3) / 1e9 if kernel_ms else None
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "Gvoxel-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        # untimed steps run right before the timed region (at least the 64
        # that build and launch both step graphs); before them the autotuner
        # timed its candidates
        "warmup": r32["warmup"]["steps"],
        "warmup_detail": dict(r32["warmup"], requested=args.warmup,
                              note="autotuner: every candidate tiling timed twice for autotune_trial_steps steps "
                                   "(at least 8 for two-step candidates), then the simulation restarted from rest; "
                                   "seconds = autotuner + warm-up steps"),
        "ms_per_step": r32["ms"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": args.storage,
        "data": "synthetic (seeded hall geometry, Gaussian-pulse source)",
        "config": {
            "workload": "large_hall %dx%dx%d %s, 2 materials x 3-section cascades, sponge 1, 1 source, "
                        "8 receivers, Courant 1/sqrt(3), centered boundary form"
                        % (*args.size, STORAGE_NAMES[args.storage]),
            "voxels": nvox,
            # the count above is every cell the stencil streams; the interior
            # (border planes excluded) alongside, with its own rate
            "interior_voxels": interior,
            "interior_value": round(interior * args.steps / (r32["ms"] * 1e-3) / 1e9 * world, 3),
            "boundary_voxels": int(r32["meta"]["info"].boundary_count),
            "l2": "inputs larger than L2 (%d x %.2f GB fields), no flush"
                  % (4 if steps_per_launch == 2 else 2, nvox * fbytes / 1e9),
            "parallelism": "replicas" if world > 1 else "single GPU",
            "timing": "CUDA events on the launching stream around virs_run (CUDA graph), max over ranks",
            "tiling": r32["tiling"],
            "time_blocking": r32["time_blocking"],
        },
        "roofline": {
            "bound": "hbm",
            "achieved": round(achieved, 1) if achieved else None,
            "peak": peak,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4) if achieved else None,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s",
            "traffic": None,
            "kernel": kernel_name,
            "kernel_ms": kernel_ms,
            "steps_per_launch": steps_per_launch,
            "basis": "%g B per voxel per launch (the launch's own algorithmic bytes)" % bpv,
            "bytes_per_voxel": bpv,
            "updates_per_launch": steps_per_launch,
            "effective_achieved": round(effective, 1) if effective else None,
            "effective_frac": round(effective / peak, 4) if effective else None,
            "effective_basis": "%g B per voxel update x %d update(s) per voxel per launch: with time blocking an "
                               "effective bandwidth above the bytes moved" % (upd, steps_per_launch),
            "boundary_pass_ms": r32.get("boundary_ms"),
            "boundary_pass_note": ("per step: a two-step pass's two boundary launches (the second also recomputes "
                                   "the voxels next to boundary voxels and sources), halved" if steps_per_launch == 2
                                   else "per step"),
        },
        "e2e": {
            "value": round(nvox * args.steps / (r32["e2e_ms"] * 1e-3) / 1e9 * world, 3),
            "unit": "Gvoxel-updates/s",
            "h2d_bytes_per_step": r32["h2d"],
            "d2h_bytes_per_step": r32["d2h"],
            "api": "virs_run_host (pinned host buffers)",
            "wall_ms": r32["e2e_wall_ms"],
        },
        "gpu_launches": round(r32.get("launches_per_step", 3) * args.steps),
        "clocks": r32["clocks"],
        "variants": variants,
    }
    if r32.get("sustained"):
        su = r32["sustained"]
        variants["sustained"] = {
            "steps": args.sustained_steps,
            "value": round(nvox * args.sustained_steps / (su["ms"] * 1e-3) / 1e9 * world, 3),
            "ms_per_step": su["ms"] / args.sustained_steps,
            "clocks": su["clocks"],
            "note": "the configuration's whole run in one timed region, after the headline's; the power cap "
                    "(sw_power_cap) engages within about a second",
        }
    if "batched_bf16" in variants:
        # against the headline FP32 hall, and against FP32 storage on the same
        # batched workload
        variants["bf16_batched_vs_f32_plain"] = round(variants["batched_bf16"]["value"] / value, 3)
        variants["bf16_batched_vs_f32_batched"] = round(variants["batched_bf16"]["value"] /
                                                        variants["batched_f32"]["value"], 3)
    tr = measured_traffic(Path(args.traffic) if args.traffic else traffic_file, args.storage, nvox)
    if tr:
        line["roofline"]["traffic"] = tr["bytes"]
        line["roofline"]["traffic_source"] = tr["source"]
        if kernel_ms:
            line["roofline"]["dram_frac"] = round(tr["bytes"] / (kernel_ms * 1e-3) / 1e9 / peak, 4)
    if world == 1 and not args.no_cpu:
        th = host_threads()
        gv, desc, secs = cpu_sample(tuple(args.size), args.cpu_seconds, th)
        line["cpu_baseline"] = {"value": round(gv, 4), "unit": "Gvoxel-updates/s", "cores": th, "kind": "port",
                                "sample": desc + f", {secs:.1f} s"}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's step (the
    reference's own CPU build cannot be compiled: oneTBB, Embree,
    tinyobjloader, kfr and AudioFile are absent) on all host threads, timed
    exactly as the main arm's cpu_baseline: the same crop of the hall, the
    same chunks, the same budget.  Nothing of the library is loaded."""
    rank, world, _ = env_rank()
    if rank != 0:
        return
    th = host_threads()
    nx, ny, nz = args.size
    gv, desc, secs = cpu_sample(tuple(args.size), max(10.0, args.cpu_seconds), th)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(gv, 4),
        "unit": "Gvoxel-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": nx * ny * CPU_CROP_PLANES / (gv * 1e9) * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded hall geometry)",
        "config": {"workload": "large_hall %dx%dx%d FP32 (the CPU arm runs a %d-plane crop; one step = one time step "
                               "of the crop)" % (nx, ny, nz, CPU_CROP_PLANES)},
        "cpu_baseline": {"value": round(gv, 4), "unit": "Gvoxel-updates/s", "cores": th, "kind": "port",
                         "sample": f"{desc}, {secs:.1f} s; the reference CPU build (oneTBB, Embree, tinyobjloader, "
                                   "kfr, AudioFile) cannot be compiled here, so this is the CPU restatement of its step"},
        "e2e": {"value": round(gv, 4), "unit": "Gvoxel-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        maps = Path("/proc/self/maps").read_text()
        line["config"]["libvirs_b200_mapped"] = "libvirs_b200" in maps
    except OSError:
        pass
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["virs", "reference"], default="virs")
    ap.add_argument("--size", type=int, nargs=3, default=[1024, 768, 512])
    ap.add_argument("--kernel-steps", type=int, default=100, help="steps of the per-kernel CUDA-event pass")
    ap.add_argument("--sustained-steps", type=int, default=4000,
                    help="steps of the sustained variant: the configuration's whole run in one timed region (0 = skip)")
    ap.add_argument("--tune-steps", type=int, default=4, help="steps per candidate of virs_autotune (0 = no tuning)")
    ap.add_argument("--no-variants", dest="variants", action="store_false")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-slabs", dest="slabs", action="store_false",
                    help="skip the variant that runs the hall as two z-slabs on one GPU")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false",
                    help="skip the inverse-design (adjoint) variant")
    ap.add_argument("--adjoint-steps", type=int, default=4000,
                    help="steps of the inverse-design leg (4000: the configuration; fewer for profiling)")
    ap.add_argument("--batch-steps", type=int, default=60, help="timed steps of the batched workload (0 = skip)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--storage", choices=list(STORAGE_NAMES), default="f32",
                    help="field storage of the timed hall (f32 is the headline; bf16/f16 store 16-bit fields)")
    ap.add_argument("--steps-per-pass", type=int, choices=[0, 1, 2], default=0,
                    help="0: the autotuner's choice; 1: single steps; 2: two steps per pass (time blocking)")
    ap.add_argument("--pair-tiling", type=int, nargs=2, default=None, metavar=("ROWS", "PLANES"),
                    help="tile rows (12/14/16/32) and planes per block of the two-step kernel with --steps-per-pass 2")
    ap.add_argument("--traffic", default=None,
                    help="ncu DRAM-traffic summary of the stencil kernel")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_virs(args)


if __name__ == "__main__":
    main()
