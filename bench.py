"""Benchmark: photoelectric system-matrix entries per second on B200.

Workload (``pe_large``): 64x64x32 voxels of 0.5 mm, two tungsten plates with
400 seeded holes each, 4 layers of 40x40 crystals (6400 rows x 131072
columns, 3.4 GB float32), 4x4x4 voxel sub-samples x 2x4x2 crystal sub-cells
= 1024 rays per entry.  A step is one z-slab of 4 planes for every crystal
(6400 x 16384 entries, the reference CLI's slab size); 8 steps cover the
whole matrix.  Inputs are seeded synthetic tables (no public dataset exists
for this path).

``--impl ours`` (default) times the sm_100a kernel through the C ABI with the
geometry resident on the device (``value``), then end to end through the
public API with host tables in and the slab copied back to pinned host memory
(``e2e``).  It also times the reference's own CUDA kernel on the same GPU on a
bounded sample (``ref_cuda``) and the reference's code on the host cores
(``cpu_baseline``).  ``--impl reference`` times the reference's CPU
implementation (the reference kernel code compiled for the host, OpenMP over
entries) on a bounded sample per step.

Multi-GPU (torchrun): ranks take different slabs (weak scaling, no
collective on the data path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-spect-pet-sysmat_b200"))

SLAB_Z = 4
L2_FLUSH_BYTES = 256 << 20
# DRAM traffic of one full pe_large slab launch (6400 x 16384 entries):
# dram__bytes_read.sum 126.68 MB + dram__bytes_write.sum 579.35 MB from one
# single-pass ncu capture of pe_trace_kernel on B200.  Algorithmic bytes of the
# same launch: 4 B per entry of output, 419.4 MB, plus 0.64 MB of tables.
PE_LARGE_SLAB_DRAM_BYTES = 706.03e6
PE_LARGE_SLAB_ALGORITHMIC_BYTES = 4 * 6400 * 16384 + 2 * 4 * 80000

# FP32 operations per unit of work, counted from the tracer's source
# (gpu-spect-pet-sysmat_b200/csrc/tracer.cuh, pe_kernel.cu): add/sub/mul/fma
# and each div/sqrt/exp as 1.  Used for the roofline numerator.
F_RAY = 64          # sub-cell point, distance, solid angle, self path, absorption, two exp
F_BOX = 31          # chord_through, general case
F_XF = 18           # crystal-frame transform of both ray ends
F_CYL = 60          # chord_hole
F_CONE = 26         # one candidate cone test
F_IN = 31           # chord_to_end


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "of measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "of fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def pe_workload(name: str):
    from sysmat_b200 import configs
    return configs.NAMED[name]()


def workload_config(name: str, p, rows: int):
    """The workload description both arms print (the same dict)."""
    nx, ny, _ = p.grid
    return {"workload": name, "crystals": rows, "voxels": p.n_voxels, "holes": p.n_holes, "plates": p.n_plates,
            "sv": list(p.sv), "sc": list(p.sc), "rays_per_entry": p.rays_per_entry,
            "step": "one %d-plane z-slab x all crystals (%d entries); the host arm times a seeded sample of "
                    "entries of the same matrix per step" % (SLAB_Z, rows * nx * ny * SLAB_Z),
            "l2": "GPU arm: L2 flushed between steps (%d MiB memset)" % (L2_FLUSH_BYTES >> 20),
            "parallelism": "slabs sharded across ranks, no data-path collective"}


# ---------------------------------------------------------------------------
# CPU side: the reference's own code on the host cores
# ---------------------------------------------------------------------------

def cpu_reference_rate(p, target_s: float, seed: int = 0, max_entries: int = 1 << 16):
    """Entries/s of the reference kernel code on all host cores, on a seeded
    random sample of entries grown until it takes >= target_s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    kind = "f32"
    if not oracle_py.ref_available("pe_f32"):
        return None
    rng = np.random.default_rng(seed)
    n, spent, done = 64, 0.0, 0
    while spent < target_s and done < max_entries:
        rows = rng.integers(0, p.n_crystals, n)
        vox = rng.integers(0, p.n_voxels, n)
        t0 = time.perf_counter()
        oracle_py.ref_pe_entries(p, rows, vox, kind)
        spent += time.perf_counter() - t0
        done += n
        n = min(n * 2, max_entries - done) if done < max_entries else 0
        if n <= 0:
            break
    return {"value": done / spent, "unit": "entries/s", "cores": os.cpu_count(), "kind": "reference",
            "sample": "%d seeded random entries (%d rays each), reference kernel code built for the host, "
                      "OpenMP over entries, %.1f s" % (done, p.rays_per_entry, spent)}


def error_vs_reference_fp64(p, slab_host, row0, n_rows=96, seed=3):
    """Max and median relative error, on nonzero entries, of GPU-computed
    entries of slab 0 against the reference's own code built with double
    (the CPU-baseline leg's library).  Per sampled row: its 4 largest entries
    (voxels seen through holes) and 4 random nonzero ones."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    if not oracle_py.ref_available("pe_f64"):
        return None
    rng = np.random.default_rng(seed)
    rows_local = rng.choice(slab_host.shape[0], min(n_rows, slab_host.shape[0]), replace=False)
    rows, cols = [], []
    for r in rows_local:
        row = slab_host[r]
        top = np.argsort(-row)[:4]
        nz = np.flatnonzero(row)
        extra = rng.choice(nz, min(4, nz.size), replace=False) if nz.size else top[:0]
        c = np.unique(np.concatenate([top, extra]))
        rows.append(np.full(c.size, r))
        cols.append(c)
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    got = slab_host[rows, cols].astype(np.float64)
    t0 = time.perf_counter()
    ref = oracle_py.ref_pe_entries(p, rows + row0, cols, "f64")   # slab 0: column index = voxel index
    dt = time.perf_counter() - t0
    nz = ref != 0
    e = np.abs(got[nz] - ref[nz]) / np.abs(ref[nz])
    return {"median": float(np.median(e)) if e.size else None, "max": float(e.max()) if e.size else None,
            "n_entries": int(rows.size), "n_nonzero": int(nz.sum()),
            "zero_pattern_equal": bool(np.array_equal(got == 0, ref == 0)),
            "vs": "fp64: the reference's kernel code built for the host with double",
            "sample": "%d rows of slab 0, per row the 4 largest and 4 random nonzero entries; %.1f s on %d cores"
                      % (len(rows_local), dt, os.cpu_count())}


def run_reference_impl(args, world, rank):
    if rank != 0:
        return
    p = pe_workload(args.workload)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    if not oracle_py.ref_available("pe_f32"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_pe_f32.so not built (no reference tree at build time)"}))
        return
    rng = np.random.default_rng(1)
    per_step = args.ref_entries
    for _ in range(args.warmup):
        oracle_py.ref_pe_entries(p, rng.integers(0, p.n_crystals, per_step), rng.integers(0, p.n_voxels, per_step))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle_py.ref_pe_entries(p, rng.integers(0, p.n_crystals, per_step), rng.integers(0, p.n_voxels, per_step))
    dt = time.perf_counter() - t0
    value = args.steps * per_step / dt
    sample = ("%d seeded random entries per step of %s (%d rays each), reference kernel code built for the host, "
              "OpenMP over entries" % (per_step, args.workload, p.rays_per_entry))
    line = {"metric": "pe sysmat entries/s", "value": value, "unit": "entries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded %s geometry)" % args.workload, "impl": "reference",
            "config": workload_config(args.workload, p, p.n_crystals),
            "cpu_baseline": {"value": value, "unit": "entries/s", "cores": os.cpu_count(), "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# GPU: the reference's CUDA kernel on this GPU (bounded sample)
# ---------------------------------------------------------------------------

def ref_cuda_rate(p, device: int, n_rows: int = 64):
    """The reference's photodetectorCudaMe (built for sm_100a with this
    workload's crystal sub-cells) on a seeded random set of n_rows crystals
    (moved to the front of the detector table) and one fine slab of 4 planes
    of the k-times finer voxel grid that emulates voxel sub-sampling."""
    import torch
    path = os.path.join(ROOT, "oracle", "_ref", "libref_pe_cuda_%dx%dx%d.so" % tuple(p.sc))
    if not os.path.exists(path):
        return {"unavailable": "%s not built" % os.path.basename(path)}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    lib = ctypes.CDLL(path)
    lib.ref_cuda_pe_kernel.restype = ctypes.c_int
    rng = np.random.default_rng(5)
    N = p.n_crystals
    pick = rng.choice(N, n_rows, replace=False)
    order = np.concatenate([pick, np.setdiff1d(np.arange(N), pick)])
    det = np.zeros(max(80000, p.detector.size), np.float32)
    det[0] = N
    body = p.detector[1:1 + 12 * N].reshape(N, 12)[order]
    det[1:1 + 12 * N] = body.ravel()
    col = np.zeros(max(80000, p.collimator.size), np.float32)
    col[:p.collimator.size] = p.collimator
    img = oracle_py.fine_image(p)
    fnz = int(img[2])
    z0 = fnz // 2 - SLAB_Z // 2
    img[30] = fnz
    img[31] = z0
    img[2] = SLAB_Z
    img[20] = 0
    cells = int(img[0]) * int(img[1]) * SLAB_Z
    dev = torch.device("cuda", device)
    d_col = torch.from_numpy(col).to(dev)
    d_det = torch.from_numpy(det).to(dev)
    d_img = torch.from_numpy(img).to(dev)
    d_dst = torch.zeros(n_rows * cells, dtype=torch.float32, device=dev)
    ms = ctypes.c_float(0)
    fp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = lib.ref_cuda_pe_kernel(fp(d_col), fp(d_det), fp(d_img), fp(d_dst), n_rows, cells, 1, ctypes.byref(ms))
    if rc != 0:
        return {"unavailable": "reference kernel returned CUDA error %d" % rc}
    rc = lib.ref_cuda_pe_kernel(fp(d_col), fp(d_det), fp(d_img), fp(d_dst), n_rows, cells, 1, ctypes.byref(ms))
    n_sv = int(np.prod(p.sv))
    entries = n_rows * cells / n_sv
    return {"value": entries / (ms.value / 1e3), "unit": "entries/s", "kernel_ms": ms.value,
            "sample": "%d random crystals x one %d-plane slab of the %dx finer grid (%d fine cells = %d entries of "
                      "%d rays); reference launch shape 16x32" % (n_rows, SLAB_Z, p.sv[0], n_rows * cells,
                                                                   int(entries), p.rays_per_entry)}


# ---------------------------------------------------------------------------
# Our kernel
# ---------------------------------------------------------------------------

def run_ours(args, world, rank, local):
    import torch
    import sysmat_b200
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    p = pe_workload(args.workload)
    ctx = sysmat_b200.Context(local)
    geo = sysmat_b200.Geometry(ctx, p)
    nx, ny, nz = p.grid
    n_slabs = nz // SLAB_Z
    slab_vox = nx * ny * SLAB_Z
    rows = p.n_crystals if args.rows <= 0 else min(args.rows, p.n_crystals - args.row0)
    row_range = (0, rows) if args.rows <= 0 else (args.row0, args.row0 + rows)
    out = torch.empty((rows, slab_vox), dtype=torch.float32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    opts = geo.options()

    from sysmat_b200.shard import max_over_ranks, slab_of

    def step(i):
        s = slab_of(i, rank, world, n_slabs)
        flush.zero_()
        geo.pe(z=(s * SLAB_Z, SLAB_Z), rows=row_range, opts=opts, out=out.data_ptr(), stream=stream.cuda_stream)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(i)
    ctx.sync(stream.cuda_stream)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            t_start.record(stream)
            for i in range(args.steps):
                s = slab_of(i, rank, world, n_slabs)
                flush.zero_()
                starts[i].record(stream)
                geo.pe(z=(s * SLAB_Z, SLAB_Z), rows=row_range, opts=opts, out=out.data_ptr(), stream=stream.cuda_stream)
                ends[i].record(stream)
            t_end.record(stream)
        torch.cuda.synchronize()
    barrier()
    ctx.sync(stream.cuda_stream)
    total_ms = t_start.elapsed_time(t_end)
    kernel_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_ms, kernel_sum = max_over_ranks([total_ms, sum(kernel_ms)], device=dev)
    entries_per_step = rows * slab_vox
    value = world * args.steps * entries_per_step / (total_ms / 1e3)

    # Work counters of one slab (separate, counted run).
    ctx.set_counters(True)
    geo.pe(z=(0, SLAB_Z), rows=row_range, opts=opts, out=out.data_ptr(), stream=stream.cuda_stream)
    n_rays, n_cry, n_hole, n_cone = ctx.last_counters()
    ctx.set_counters(False)
    flops = (n_rays * (F_RAY + p.n_plates * F_BOX + 2 * F_IN + F_BOX) + n_cry * (F_BOX + F_XF) + n_hole * F_CYL
             + n_cone * F_CONE)
    kernel_s = kernel_sum / args.steps / 1e3
    peaks, peak_src = load_peaks()
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12
    achieved = flops / kernel_s / 1e12
    # DRAM bytes (read + write) of one pe_trace_kernel launch of this step,
    # from one ncu capture of a full pe_large slab (dram__bytes_read.sum +
    # dram__bytes_write.sum); None for other workloads or row subsets.
    traffic = PE_LARGE_SLAB_DRAM_BYTES if (args.workload == "pe_large" and rows == p.n_crystals) else None

    # End to end through the public API: tables in from host memory, slab out to pinned host memory.
    e2e = None
    if args.e2e_steps < 0:
        args.e2e_steps = args.steps
    if args.e2e_steps > 0:
        host = torch.empty((rows, slab_vox), dtype=torch.float32, pin_memory=True).numpy()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(args.e2e_steps):
            s = (i * world + rank) % n_slabs
            g2 = sysmat_b200.Geometry(ctx, p)
            g2.pe(z=(s * SLAB_Z, SLAB_Z), rows=row_range, opts=opts, out=host)
            g2.close()
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t[0])
        e2e = {"value": world * args.e2e_steps * entries_per_step / e2e_s, "unit": "entries/s",
               "h2d_bytes_per_step": 4 * (p.collimator.size + p.detector.size + p.image.size + p.physics.size),
               "d2h_bytes_per_step": 4 * rows * slab_vox, "steps": args.e2e_steps,
               "path": "sysmat_b200.Geometry(tables) + Geometry.pe(host out) per step"}

    if rank == 0:
        line = {
            "metric": "pe sysmat entries/s", "value": value, "unit": "entries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded %s geometry)" % args.workload,
            "config": workload_config(args.workload, p, rows),
            "rays_per_s": value * p.rays_per_entry,
            "kernel_ms_per_step": kernel_sum / args.steps,
            "gpu_launches": args.steps,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak, "traffic": traffic,
                         "traffic_algorithmic_bytes": PE_LARGE_SLAB_ALGORITHMIC_BYTES if traffic else None,
                         "peak_source": "FP32 issue peak 148 SMs x 128 lanes x 2 FLOP x sm_max %.0f MHz (%s clock)" % (sm_max, peak_src.split()[1]),
                         "work": {"rays": n_rays, "exact_crystal_tests": n_cry, "exact_hole_tests": n_hole,
                                  "cone_tests": n_cone, "flops_per_step": flops},
                         "hbm_write_gbs": 4 * entries_per_step / kernel_s / 1e9,
                         "hbm_frac": 4 * entries_per_step / kernel_s / 1e9 / float(peaks.get("hbm_gbs", 6650.0))},
            "clocks": clocks.summary(),
        }
        if e2e:
            line["e2e"] = e2e
        if not args.no_ref_cuda:
            try:
                line["ref_cuda"] = ref_cuda_rate(p, local)
            except Exception as exc:  # the reference kernel is a baseline, not the product
                line["ref_cuda"] = {"unavailable": "%s" % exc}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_reference_rate(p, args.cpu_seconds)
            slab0 = out.cpu().numpy()   # slab 0 of the timed rows (the counted run computed it last)
            line["error"] = error_vs_reference_fp64(p, slab0, row_range[0])
        if world == 1:
            line["beam_metrics"] = run_beam_metrics(out, stream)
        if world == 1 and args.scatter_steps > 0:
            line["scatter"] = run_scatter(args, ctx, dev)
        if world == 1 and args.sweep_steps > 0:
            line["sweep"] = run_sweep(args, ctx, dev)
            line["sweep_small"] = run_sweep(args, ctx, dev, small=True)
            line["rotations"] = run_rotations(args, ctx, dev)
        if world == 1 and args.surrogate_steps > 0:
            line["surrogate"] = run_surrogate(args, ctx, dev)
        print(json.dumps(line))
    geo.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Beam masks and MPXI of the resident slab (sysmat_b200.beams)
# ---------------------------------------------------------------------------

def run_beam_metrics(block, stream, reps: int = 5):
    """sm_beam_metrics on a resident sysmat block (masks kept): HBM-bound;
    algorithmic bytes per entry = 4 (sysmat read) + 1 (mask written) + 1
    (mask read for MPXI).  The block (419 MB for pe_large) exceeds L2."""
    import torch
    from sysmat_b200 import beams
    peaks, src = load_peaks()
    with torch.cuda.stream(stream):
        beams.beam_metrics(block, stream=stream)          # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # Keep the GPU busy (~20 ms) while the host enqueues the timed calls, so
        # that host-side delays (e.g. the CPU baseline's worker threads still
        # spinning) leave no gaps between the timed kernels.
        torch.cuda._sleep(40_000_000)
        e0.record(stream)
        for _ in range(reps):
            m = beams.beam_metrics(block, stream=stream)
        e1.record(stream)
    stream.synchronize()
    ms = e0.elapsed_time(e1) / reps
    entries = block.shape[0] * block.shape[1]
    gbs = 6.0 * entries / (ms / 1e3) / 1e9
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    return {"entries": entries, "ms": ms, "bytes_per_entry": 6, "achieved_gbs": gbs, "peak_gbs": hbm,
            "frac": gbs / hbm, "peak_source": src, "active_rows": int((m["row_count"] > 0).sum()),
            "mpxi_max": int(m["mpxi"].max()),
            "timed": "row stats + int8 masks + MPXI of the resident slab 0, CUDA events, mean of %d" % reps}


# ---------------------------------------------------------------------------
# Exact primary-Compton scatter (scatter_small: 2048 x 16384)
# ---------------------------------------------------------------------------

def ref_cuda_scatter_rate(p, d_pe, bitmaps, n_rows: int = 16):
    """The reference's crystalScatterSysMatCuda / collimatorScatterSysMatCuda
    (built for sm_100a) on the first n_rows detector rows, with the reference's
    own launch shape; seconds per full matrix extrapolated by rows."""
    import torch
    path = os.path.join(ROOT, "oracle", "_ref", "libref_scatter_cuda.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libref_scatter_cuda.so not built"}
    lib = ctypes.CDLL(path)
    N, V = p.n_crystals, p.n_voxels
    pad = lambda a, n: np.pad(a.astype(np.float32), (0, max(0, n - a.size)))  # noqa: E731
    dev = d_pe.device
    det = torch.from_numpy(pad(p.detector, 80000)).to(dev)
    col = torch.from_numpy(pad(p.collimator, 80000)).to(dev)
    img = torch.from_numpy(p.image.astype(np.float32).copy()).to(dev)
    phy = torch.from_numpy(p.physics.astype(np.float32).copy()).to(dev)
    bc = torch.from_numpy(bitmaps[0].view(np.int32)).to(dev)
    bh = torch.from_numpy(bitmaps[1].view(np.int32)).to(dev)
    rows16 = (n_rows + 15) // 16 * 16
    dst = torch.zeros((rows16, V), dtype=torch.float32, device=dev)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    ms_c, ms_h = ctypes.c_float(0), ctypes.c_float(0)
    h0 = int(np.floor(np.float32(p.collimator[10]) + np.float32(0.01)))
    rc = lib.ref_cuda_crystal_scatter(vp(dst), vp(det), vp(img), vp(phy), vp(d_pe), vp(bc), N, V, n_rows, ctypes.byref(ms_c))
    rc |= lib.ref_cuda_collimator_scatter(vp(dst), vp(col), vp(det), vp(img), vp(phy), vp(bh), N, V, h0, n_rows,
                                          ctypes.byref(ms_h))
    if rc != 0:
        return {"unavailable": "reference scatter kernel returned CUDA error %d" % rc}
    full_s = (ms_c.value + ms_h.value) / 1e3 * N / n_rows
    return {"seconds_full_matrix": full_s, "entries_per_s": N * V / full_s, "sample_rows": n_rows,
            "crystal_ms": ms_c.value, "collimator_ms": ms_h.value, "scatter_points": [1, 1, 1],
            "note": "reference kernels scatter from crystal centres only (1 point per crystal)"}


def run_scatter(args, ctx, dev):
    """Exact crystal + collimator scatter of the scatter workload on the device
    (PE sysmat resident in HBM), timed with CUDA events on the launch stream."""
    import torch
    import sysmat_b200
    p = pe_workload("scatter_small")
    g = sysmat_b200.Geometry(ctx, p)
    N, V = p.n_crystals, p.n_voxels
    stream = torch.cuda.Stream(device=dev)
    d_pe = torch.zeros((N, V), dtype=torch.float32, device=dev)
    d_out = torch.zeros((N, V), dtype=torch.float32, device=dev)
    sp = tuple(args.scatter_points)
    with torch.cuda.stream(stream):
        g.pe(opts=g.options(sv=(1, 1, 1), sc=(2, 4, 2)), out=d_pe.data_ptr(), stream=stream.cuda_stream)
    stream.synchronize()
    res = {}
    for parts in ("crystal", "collimator"):
        times = []
        for i in range(1 + args.scatter_steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                g.scatter(pe=d_pe.data_ptr(), sp=sp, parts=parts, out=d_out.data_ptr(), stream=stream.cuda_stream)
                e1.record(stream)
            stream.synchronize()
            if i > 0:
                times.append(e0.elapsed_time(e1) / 1e3)
        res[parts] = min(times)
    total = res["crystal"] + res["collimator"]
    bitmaps = g.scatter_bitmaps()
    out = {"workload": "scatter_small: 32x32x16 voxels of 1 mm, pe_small collimator (49 holes), 2 layers of 32x32 "
                       "crystals [2048 x 16384]; PE input from the tracer (voxel centres, 2x4x2 sub-cells)",
           "scatter_points": list(sp), "crystal_s": res["crystal"], "collimator_s": res["collimator"],
           "seconds": total, "entries_per_s": N * V / total,
           "terms_per_s": N * (N - 1) * V * int(np.prod(sp)) / res["crystal"],
           "timed": "bitmaps + pair sums + main kernel per call, device-resident PE, CUDA events, best of %d"
                    % args.scatter_steps}
    if not args.no_ref_cuda:
        try:
            out["ref_cuda"] = ref_cuda_scatter_rate(p, d_pe, bitmaps)
        except Exception as exc:  # the reference kernel is a baseline, not the product
            out["ref_cuda"] = {"unavailable": str(exc)}
    g.close()
    return out


# ---------------------------------------------------------------------------
# Scatter surrogate (scatter_large: 2048 x 131072) against the all-exact matrix
# ---------------------------------------------------------------------------

def run_surrogate(args, ctx, dev):
    """Crystal + collimator scatter of scatter_large: all exact, then through
    the surrogate with the learned correction (the configured MLP) and without
    it (baseline only); wall time of each on the device (CUDA events around the
    whole call, PE resident in HBM) and each output row's true relative L2
    error against the all-exact matrix."""
    import torch
    import sysmat_b200
    p = pe_workload(args.surrogate_workload)
    g = sysmat_b200.Geometry(ctx, p)
    N, V = p.n_crystals, p.n_voxels
    sp = tuple(args.scatter_points)
    stream = torch.cuda.Stream(device=dev)
    d_pe = torch.zeros((N, V), dtype=torch.float32, device=dev)
    exact = torch.zeros((N, V), dtype=torch.float32, device=dev)
    out = torch.zeros((N, V), dtype=torch.float32, device=dev)
    with torch.cuda.stream(stream):
        g.pe(opts=g.options(sv=(1, 1, 1), sc=(2, 4, 2)), out=d_pe.data_ptr(), stream=stream.cuda_stream)
    stream.synchronize()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            r = fn()
            e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1) / 1e3, r

    t_exact, _ = timed(lambda: g.scatter(pe=d_pe.data_ptr(), sp=sp, parts="both", out=exact.data_ptr(),
                                         stream=stream.cuda_stream))
    den = exact.double().pow(2).sum(1).sqrt().clamp_min(1e-300)
    res = {"workload": "%s [%d x %d]: scatter_small's collimator and 2 x 32 x 32 crystals, image %dx%dx%d voxels of "
                       "1 mm; crystal + collimator scatter, %dx%dx%d scatter points"
                       % ((args.surrogate_workload, N, V) + tuple(p.grid) + sp),
           "exact_s": t_exact, "exact_entries_per_s": N * V / t_exact, "variants": {}}
    # one untimed run first: the context's memory pool then holds the workspaces
    # (transfer matrices, pair table), as in any application that calls it again
    g.scatter_surrogate(d_pe.data_ptr(), out.data_ptr(),
                        options=sysmat_b200.SurrogateOptions.make(sp=sp, parts=3, network=0))
    torch.cuda.synchronize()
    res["warmup"] = "one untimed baseline-only run before the timed ones (workspaces mapped in the context's pool)"
    for name, kw in (("network", dict(network=1)), ("baseline_only", dict(network=0))):
        opts = sysmat_b200.SurrogateOptions.make(sp=sp, parts=3, **kw)
        for i in range(args.surrogate_steps):
            t, st = timed(lambda: g.scatter_surrogate(d_pe.data_ptr(), out.data_ptr(), options=opts,
                                                      stream=stream.cuda_stream))
        err = ((out.double() - exact.double()).pow(2).sum(1).sqrt() / den).cpu().numpy()
        kept = st["row_state"] != 2
        stats = {k: v for k, v in st.items() if k not in ("row_error", "row_state")}
        res["variants"][name] = {
            "seconds": t, "speedup_vs_exact": t_exact / t, "entries_per_s": N * V / t,
            "rows_recomputed": int(st["rows_recomputed"]), "rows_corrected": int(st["rows_corrected"]),
            "true_row_error": {"median": float(np.median(err)), "p90": float(np.quantile(err, 0.9)),
                               "p99": float(np.quantile(err, 0.99)), "max": float(err.max()),
                               "frac_above_tol": float((err > opts.tol).mean()),
                               "verified_rows_median": float(np.median(err[kept])) if kept.any() else 0.0},
            "options": {"train_frac": opts.train_frac, "holdout_frac": opts.holdout_frac, "tol": opts.tol,
                        "anchors": list(opts.anchors), "network": opts.network,
                        "mlp": [opts.layers, opts.width, opts.freqs, opts.emb], "steps": opts.steps},
            "stats": stats}
    g.close()
    return res


# ---------------------------------------------------------------------------
# Batched design sweep: 64 seeded geometries in one persistent graph launch
# ---------------------------------------------------------------------------

def run_sweep(args, ctx, dev, small: bool = False):
    import torch
    import sysmat_b200
    from sysmat_b200 import configs
    params = configs.sweep_small() if small else configs.sweep()
    geos = [sysmat_b200.Geometry(ctx, p) for p in params]
    t0 = time.perf_counter()
    opts = []
    for g in geos:
        tuned, _ = sysmat_b200.autotune(g)
        opts.append(tuned)
    tune_s = time.perf_counter() - t0
    outs = [torch.empty((g.n_crystals, g.nx * g.ny * g.nz), dtype=torch.float32, device=dev) for g in geos]
    entries = sum(o.numel() for o in outs)
    rays = sum(o.numel() * int(np.prod(p.sv)) * int(np.prod(p.sc)) for o, p in zip(outs, params))
    stream = torch.cuda.Stream(device=dev)
    batch = sysmat_b200.PeBatch(ctx, geos, opts, [o.data_ptr() for o in outs], [o.shape[1] for o in outs])

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            fn()
            e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1) / 1e3

    batch.run(stream.cuda_stream)          # captures the graph
    stream.synchronize()
    t_batch = min(timed(lambda: batch.run(stream.cuda_stream)) for _ in range(args.sweep_steps))

    def sequential():
        for g, o, op in zip(geos, outs, opts):
            g.pe(opts=op, out=o.data_ptr(), stream=stream.cuda_stream)
    t_seq = min(timed(sequential) for _ in range(args.sweep_steps))

    def sequential_default():
        for g, o in zip(geos, outs):
            g.pe(opts=g.options(), out=o.data_ptr(), stream=stream.cuda_stream)
    t_default = min(timed(sequential_default) for _ in range(args.sweep_steps))
    ctx.sync(stream.cuda_stream)
    info = batch.info()
    batch.close()
    for g in geos:
        g.close()
    workload = ("64 small seeded geometries (grids 8^3..20^3, 1-2 plates of 16-100 holes, 8^2..24^2 crystals x 1-2 "
                "layers)" if small else "64 seeded geometries (grids 16^3..48^3, 1-3 plates, 16-400 holes per plate, "
                                        "16^2..48^2 crystals x 1-4 layers)")
    return {"workload": workload + ", whole PE sysmat of each, voxel centres x 2x4x2 sub-cells",
            "entries": entries, "rays": rays, "output_gb": entries * 4 / 1e9,
            "batched_s": t_batch, "batched_entries_per_s": entries / t_batch, "batched_rays_per_s": rays / t_batch,
            "sequential_s": t_seq, "sequential_entries_per_s": entries / t_seq, "speedup": t_seq / t_batch,
            "sequential_default_brick_s": t_default, "autotune_gain": t_default / t_seq,
            "work_items": info["items"], "persistent_ctas": info["ctas"], "autotune_s": tune_s,
            "bricks": sorted(set(tuple(o.tile_voxels) + (o.group,) for o in opts)),
            "timed": "one CUDA-graph launch of the persistent kernel vs 64 sm_pe_compute launches on one stream, "
                     "same autotuned bricks, CUDA events, best of %d" % args.sweep_steps}


# ---------------------------------------------------------------------------
# Rotations as work items of one persistent launch (the CLI's multi-rotation path)
# ---------------------------------------------------------------------------

def run_rotations(args, ctx, dev, n_rot: int = 16):
    """pe_small's geometry turned through n_rot image rotations (2 pi / n_rot
    apart), voxel centres x 2x4x2 sub-cells: every rotation's whole matrix in
    one persistent launch (sm_pe_batch with per-item rotations, CUDA graph) vs
    one sm_pe_compute launch per rotation, outputs resident in HBM."""
    import torch
    import sysmat_b200
    from sysmat_b200 import configs
    p = configs.pe_small()
    p.image = p.image.copy()
    p.image[6] = n_rot
    p.image[7] = np.float32(2 * np.pi / n_rot)
    p.sv = (1, 1, 1)
    g = sysmat_b200.Geometry(ctx, p)
    opts = g.options()
    N, V = p.n_crystals, p.n_voxels
    outs = torch.empty((n_rot, N, V), dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    batch = sysmat_b200.PeBatch(ctx, [g] * n_rot, [opts] * n_rot, [outs[r].data_ptr() for r in range(n_rot)],
                                [V] * n_rot, rotations=list(range(n_rot)))

    def timed(fn, reps=3):
        best = 1e30
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                fn()
                e1.record(stream)
            stream.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        return best

    batch.run(stream.cuda_stream)
    stream.synchronize()
    t_batch = timed(lambda: batch.run(stream.cuda_stream))
    ref = outs.clone()

    def per_rotation():
        for r in range(n_rot):
            g.pe(rotation=r, opts=opts, out=outs[r].data_ptr(), stream=stream.cuda_stream)
    t_seq = timed(per_rotation)
    ctx.sync(stream.cuda_stream)
    same = bool(torch.equal(ref, outs))
    batch.close()
    g.close()
    entries = n_rot * N * V
    return {"workload": "pe_small geometry, %d image rotations, voxel centres x 2x4x2 sub-cells [%d x %d] per rotation"
                        % (n_rot, N, V),
            "batched_s": t_batch, "per_rotation_s": t_seq, "speedup": t_seq / t_batch,
            "batched_entries_per_s": entries / t_batch, "identical_outputs": same,
            "timed": "one CUDA-graph launch of the persistent kernel over %d rotations vs %d sm_pe_compute launches, "
                     "CUDA events, best of 3" % (n_rot, n_rot)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="pe_large")
    ap.add_argument("--e2e-steps", type=int, default=-1, help="end-to-end steps (default: as many as --steps)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-entries", type=int, default=4096)
    ap.add_argument("--rows", type=int, default=0, help="limit the crystal rows per step (profiling runs)")
    ap.add_argument("--row0", type=int, default=0, help="first crystal row when --rows limits them")
    ap.add_argument("--no-ref-cuda", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scatter-steps", type=int, default=1, help="timed runs of the exact scatter (0 skips it)")
    ap.add_argument("--scatter-points", type=int, nargs=3, default=[2, 4, 2])
    ap.add_argument("--sweep-steps", type=int, default=1, help="timed runs of the batched sweep (0 skips it)")
    ap.add_argument("--surrogate-steps", type=int, default=1,
                    help="timed runs of the scatter surrogate (0 skips it)")
    ap.add_argument("--surrogate-workload", default="scatter_large")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_impl(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
