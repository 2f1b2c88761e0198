"""Benchmark of the FDTD time-step path.

Workload (the configuration the headline metric is quoted on): 256^3 FP32 dispersive
plasmonics -- Drude+Lorentz gold-like sphere, 12-cell CPML, TFSF broadband plane wave and
DFT monitors on six box faces at 64 frequencies with FP64 sums.  One step = one full time
step of the whole grid (H update with the deferred Sa/E2 sums, E update with CPML/ADE,
TFSF injection, monitor gather; the DFT accumulation runs every 64 staged steps).

  value   : Gcell-updates/s with all inputs resident in HBM, CUDA events on the library's
            stream around the K timed steps (one mfd_run call), max over ranks.  The model is
            the configuration's 4000-step run; the timed steps follow W warm-up steps, and a
            second window (value_late) times K steps after step 1500, when the pulse fills
            the TFSF box.  --mode selects the arithmetic of the field updates (fast: the
            tolerance mode, the default; exact: the reference's operation order bit for bit);
            other_mode times the same window in the other one.
  e2e     : the same metric through the public API with host buffers: model upload
            (mfd_create), K steps, and the read-back of what the reference's solve! writes
            for this run with its default outputs (no field frames requested): Sa, E2 and
            the DFT spectra; wall-clock with the device synchronised.
  roofline: the dominant kernel pair (the E update: core rows + CPML slabs; the H update
            alongside), algorithmic bytes per update / its mean time from CUDA events around
            each update, measured over the K steps after the timed ones (the timed steps
            themselves carry no per-launch events), against the measured HBM copy bandwidth.
  dft_fold: the same for the DFT fold of one spectral face monitor (the tensor-core fold in
            the tolerance mode): its spectra read and written once, its 64 staged steps read.

Multi-GPU: replicas (the path does not shard); each rank runs the same workload on its own
GPU, scaling "weak".  ``--impl reference`` times the CPU oracle (the restatement of the
reference's CPU path) on the host cores instead.

Other workloads (``--workload``): ``dielectric100`` (100^3 FP64), ``nonlinear`` (192x192x1024
FP32 glass with Kerr and plasma), ``batch2d`` (256 uneven 2-D models in one batch),
``batch3d`` (small uneven 3-D models in one batch), ``serve`` (a Poisson stream of 2-D and
3-D solves through the serving loop); each prints one JSON line with the same keys.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM traffic of one E and one H update (every launch of the update) of the 256^3 workload,
# per arithmetic mode, from ncu captures of the launches of whole steps (dram__bytes_read.sum
# + dram__bytes_write.sum; the tolerance mode's without cache flushes between launches, the
# mean of two steps); the captures and their commands are in NCU_TRAFFIC_SOURCE.
NCU_TRAFFIC_256 = {("exact", "E"): 760_243_968, ("exact", "H"): 857_313_280,
                   ("fast", "E"): 898_029_056, ("fast", "H"): 923_752_448}
NCU_TRAFFIC_SOURCE = "profiles/update_traffic_256.md"

WORKLOAD = "plasmonics_256: 256^3 FP32, Drude+Lorentz sphere r=60nm, 12-cell CPML, TFSF 600nm/3fs, 6x DFT faces x 64 freq FP64"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(model, meta, dtype):
    """Algorithmic HBM bytes of one H launch and one E launch: every array read once and
    written once, neighbours from on-chip reuse."""
    T = np.dtype(dtype).itemsize
    g = model.grid
    N = g.Nx * g.Ny * g.Nz
    geo = np.count_nonzero(model.geometry)
    math_h = any(m.Mh != model.Mh for m in model.materials)
    h = N * (3 * T + 6 * T + (1 if math_h else 0) + 2 * T + (2 * T if geo else 0))
    e = N * (3 * T + 6 * T + 3 * T + (1 if geo else 0))
    # CPML slabs: two psi per face cell, read + write, in each kernel
    for f, L in enumerate(model.pml):
        if L.nb:
            axis = f // 2
            n_axis = (g.Nx, g.Ny, g.Nz)[axis]
            slab = N // n_axis * L.nb
            h += slab * 2 * 2 * T
            e += slab * 2 * 2 * T
    # material state: E^n read + per pole P^n, P^{n-1} read and P^{n+1} write (3 components)
    for imat, m in enumerate(model.materials, start=1):
        cells = int(np.count_nonzero(model.geometry == imat))
        if m.nq or m.isplasma:
            e += cells * 3 * T
        e += cells * m.nq * 3 * 3 * T
        if m.isplasma:
            e += cells * (3 * 3 * T + 3 * 2 * T + 2 * 2 * 8 + 2 * T)
    return int(h), int(e)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 20 ms from before the warm-up;
    summary() keeps the samples taken inside the marked (timed) window, or the nearest ones
    when the window is shorter than the sampling interval."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.window = None
        self.path = os.path.join("/tmp", f"mfd_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)   # let the sampler start before the measured work
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def stop(self):
        if self.proc is not None:
            time.sleep(0.05)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if hasattr(self, "fh"):
            self.fh.close()

    @staticmethod
    def _t(stamp):
        import datetime
        try:
            return datetime.datetime.strptime(stamp.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def summary(self, window=None):
        window = window or self.window
        if self.proc is None or not os.path.exists(self.path):
            return None
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 10 and p[2].replace(".", "").isdigit():
                    rows.append(p)
        if not rows:
            return None
        inside = rows
        if window is not None:
            t0, t1 = window
            stamped = [(self._t(r[0]), r) for r in rows]
            stamped = [(t, r) for t, r in stamped if t is not None]
            inside = [r for t, r in stamped if t0 <= t <= t1]
            if not inside and stamped:    # window shorter than the interval: the nearest samples
                mid = 0.5 * (t0 + t1)
                inside = [r for _, r in sorted(stamped, key=lambda tr: abs(tr[0] - mid))[:2]]
        sm = [float(r[2]) for r in inside]
        mx = [float(r[3]) for r in inside if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in inside for i in range(4) if r[6 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside)}


def max_over_ranks(value, ws):
    """The largest of `value` over the ranks (the job's time is its slowest rank's)."""
    if ws <= 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _timed_window(st, a, b):
    """Steps a..b in one mfd_run call: (device ms from CUDA events, kernel launches)."""
    k0 = st.kernel_times()
    st.run(a, b)
    k1 = st.kernel_times()
    return st.last_run_ms(), int(sum(k1[k][1] - k0[k][1] for k in k1))


def run_gpu(args):
    import maxwellfdtd_b200 as M
    from maxwellfdtd_b200 import _abi, workloads
    ws, rank, local = dist_setup()
    torch = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    W, K = args.warmup, args.steps
    late = max(args.late_start, W + 2 * K + 64) if args.late_start > 0 else 0
    nt = max(4000, late + K + 1, W + 2 * K + 65)   # the configuration runs 4000 steps; the TFSF data cover them all
    model, mons = workloads.plasmonics_256(nt=nt, n=args.size)
    dtype = np.float32
    lib = M.load_library()
    b, meta = model.build_desc(dtype, mons, device=local, mode=args.mode)
    st = _abi.Stepper(lib, b, dtype)
    N = model.grid.Nx * model.grid.Ny * model.grid.Nz
    clk = ClockSampler(local).start()
    st.run(1, W)                # warm-up
    if ws > 1:
        dist.barrier()
        torch.cuda.synchronize()
    t_w0 = time.time()
    ms, launches = _timed_window(st, W + 1, W + K)   # timed: K steps, CUDA events on the library's stream
    win_early = (t_w0, time.time())
    # the next K steps again with an event pair around every launch: per-kernel device times
    kt0 = st.kernel_times()
    st.set_profiling(True)
    st.run(W + K + 1, W + 2 * K)
    st.set_profiling(False)
    kt1 = st.kernel_times()
    # one whole cycle of the monitors' staging ring (64 steps, one DFT fold in it): the
    # per-step cost with the fold amortised as in a long run
    cyc0 = W + 2 * K
    ms_cyc, _ = _timed_window(st, cyc0 + 1, cyc0 + 64)
    ms_late = None
    win_late = None
    if late:
        # a second timed window once the pulse fills the TFSF box (steps after `late`)
        st.run(cyc0 + 65, late)
        if ws > 1:
            dist.barrier()
            torch.cuda.synchronize()
        t_l0 = time.time()
        ms_late, _ = _timed_window(st, late + 1, late + K)
        win_late = (t_l0, time.time())
    clk.stop()
    dev_bytes = st.device_bytes()
    st.close()
    ms_max = max_over_ranks(ms, ws)
    ms_cyc = max_over_ranks(ms_cyc, ws)
    value = N * K * ws / (ms_max * 1e-3) / 1e9
    late_out = None
    if late:
        ms_late = max_over_ranks(ms_late, ws)
        late_out = {"value": round(N * K * ws / (ms_late * 1e-3) / 1e9, 3), "ms_per_step": round(ms_late / K, 4),
                    "steps": [late + 1, late + K], "clocks": clk.summary(win_late)}
    h_bytes, e_bytes = algorithmic_bytes(model, meta, dtype)
    # one E update and one H update per step, each a core-rows kernel plus a CPML-slab kernel
    e_ms = (kt1["E"][0] - kt0["E"][0]) / K
    h_ms = (kt1["H"][0] - kt0["H"][0]) / K
    peak, peak_kind = peaks()
    e_gbs = e_bytes / (e_ms * 1e-3) / 1e9
    h_gbs = h_bytes / (h_ms * 1e-3) / 1e9
    per_kernel = {k: {"ms": round(kt1[k][0] - kt0[k][0], 4), "launches": int(kt1[k][1] - kt0[k][1])} for k in kt1}
    # the DFT fold of one spectral face monitor per launch (every 64 steps): its spectra read
    # and written once (complex128) and its staged samples (6 components x 64 steps) read once
    spec = [m for m in meta["monitors"] if m["kind"] == 1 and not m["sum"]]
    fold = None
    if spec and per_kernel["dft"]["launches"]:
        fold_ms = (kt1["dft"][0] - kt0["dft"][0]) / (kt1["dft"][1] - kt0["dft"][1])
        fold_bytes = int(np.mean([len(m["cells"]) * 6 * (m["dft"].Nw * 32 + 64 * 4) for m in spec]))
        fold_gbs = fold_bytes / (fold_ms * 1e-3) / 1e9
        fold = {"kernel": ("monitor_dft_tc_kernel (tcgen05.mma kind::tf32, TMEM accumulators)" if args.mode == "fast"
                           else "monitor_dft_kernel (FP64)"),
                "mean_launch_ms": round(fold_ms, 5), "algorithmic_bytes_per_launch": fold_bytes,
                "achieved": round(fold_gbs, 1), "unit": "GB/s", "frac": round(fold_gbs / peaks()[0], 4)}

    # the other arithmetic mode on the same workload: the same window on its own handle
    other = "exact" if args.mode == "fast" else "fast"
    b3, _ = model.build_desc(dtype, mons, device=local, mode=other)
    st3 = _abi.Stepper(lib, b3, dtype)
    st3.run(1, W)
    ms3, _ = _timed_window(st3, W + 1, W + K)
    st3.close()
    ms3 = max_over_ranks(ms3, ws)
    other_out = {"mode": other, "value": round(N * K * ws / (ms3 * 1e-3) / 1e9, 3), "ms_per_step": round(ms3 / K, 4)}

    plain = plain_stepper(lib, args, local) if rank == 0 and not args.no_plain else None

    # end to end through the public API with host buffers: results land in page-locked
    # buffers the caller owns (allocated once, before the timed region)
    pinned = _pinned_outputs(model, meta, dtype)
    t0 = time.perf_counter()
    b2, meta2 = model.build_desc(dtype, mons, device=local, host_alloc=_pinned_array, mode=args.mode)
    t_desc = time.perf_counter() - t0
    h2d = sum(a.nbytes for a in b2.keep if isinstance(a, np.ndarray))
    t0 = time.perf_counter()
    st2 = _abi.Stepper(lib, b2, dtype)
    t_create = time.perf_counter() - t0
    st2.run(1, K)
    t_run = time.perf_counter() - t0 - t_create
    d2h = 0
    d2h += st2.read_integral(_abi.MFD_INT_SA, out=pinned["Sa"]).nbytes
    d2h += st2.read_integral(_abi.MFD_INT_E2, out=pinned["E2"]).nbytes
    for m, ms_ in enumerate(meta2["monitors"]):
        for c in (0, 1, 2, 6, 7, 8):
            d2h += st2.read_monitor(m, c, (ms_["dft"].Nw, len(ms_["cells"])), True, out=pinned[("m", m, c)]).nbytes
    t_e2e = time.perf_counter() - t0
    t_read = t_e2e - t_create - t_run
    st2.close()
    t_e2e = max_over_ranks(t_e2e, ws)
    e2e = N * K * ws / t_e2e / 1e9

    out = None
    if rank == 0:
        cpu = None if (args.no_cpu or ws > 1) else cpu_baseline(args, model, mons)
        err = None if (args.no_cpu or ws > 1) else headline_error(lib, local, mode=args.mode)
        out = {
            "metric": "Gcell-updates/s",
            "value": round(value, 3),
            "unit": "Gcell-updates/s",
            "n_gpus": ws,
            "steps": K,
            "warmup": W,
            "ms_per_step": round(ms_max / K, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [args.size] * 3, "cells": N, "steps_per_sim": nt,
                       "timed_steps": [W + 1, W + K], "mode": args.mode,
                       "parallelism": f"replicas{ws}", "l2": "inputs larger than L2 (fields 604 MB)"},
            "value_late": late_out,
            "value_ring_cycle": {"value": round(N * 64 * ws / (ms_cyc * 1e-3) / 1e9, 3),
                                 "ms_per_step": round(ms_cyc / 64, 4), "steps": [cyc0 + 1, cyc0 + 64],
                                 "note": "64 steps: one fold of the DFT monitors' staging ring"},
            "other_mode": other_out,
            "e2e": {"value": round(e2e, 3), "unit": "Gcell-updates/s", "h2d_bytes_per_step": int(h2d / K),
                    "d2h_bytes_per_step": int(d2h / K),
                "includes": "mfd_create upload from page-locked inputs + K steps + read-back of the reference's default outputs (Sa, E2, spectra) into caller-owned page-locked buffers",
                    "host_setup_s_excluded": round(t_desc, 3),
                    "split_s": {"create": round(t_create, 4), "run": round(t_run, 4), "read_back": round(t_read, 4)}},
            "roofline": {"bound": "hbm", "kernel": ("E update (e3d_core_async_kernel on the core rows and, one launch per side, "
                                                    "the y-layer rows and z-layer planes + e3d_core_kernel on the material rows)"
                                                    if args.mode == "fast" else
                                                    "E update (e3d_core_async_kernel + e3d_core_kernel on the material rows + e3d_slab_kernel)"),
                         "achieved": round(e_gbs, 1),
                         "peak": peak, "unit": "GB/s", "frac": round(e_gbs / peak, 4),
                         "traffic": NCU_TRAFFIC_256.get((args.mode, "E")) if args.size == 256 else None,
                         "traffic_source": NCU_TRAFFIC_SOURCE,
                         "algorithmic_bytes_per_launch": e_bytes, "mean_launch_ms": round(e_ms, 5),
                         "peak_kind": peak_kind,
                         "h_kernel": {"achieved": round(h_gbs, 1), "frac": round(h_gbs / peak, 4),
                                      "traffic": NCU_TRAFFIC_256.get((args.mode, "H")) if args.size == 256 else None,
                                      "algorithmic_bytes_per_launch": h_bytes, "mean_launch_ms": round(h_ms, 5)}},
            "kernels": per_kernel,
            "dft_fold": fold,
            "plain_stepper": plain,
            "gpu_launches": launches,
            "device_bytes": dev_bytes,
            "cpu_baseline": cpu,
            "error_vs_fp64_oracle": err,
            "clocks": clk.summary(win_early),
        }
        print(json.dumps(out), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out


def bytes_2d(model):
    """Algorithmic HBM bytes of one 2-D cell-update (FP32): H reads Ex, Ez, Hy and writes Hy,
    with the Sa (and E2 with materials) running sums read and written; E reads Hy, Dx, Dz and
    writes Dx, Dz, Ex, Ez; the material map once per half-step; CPML psi pairs on layer cells;
    Debye/Drude/Lorentz poles on material cells (P^n, P^{n-1} read, P^{n+1} written, E^n read)."""
    g = model.grid
    N = g.Nx * g.Nz
    geo = np.count_nonzero(model.geometry)
    h = N * (4 * 4 + 8 + (8 if geo else 0) + (1 if geo else 0))
    e = N * (4 + 8 + 8 + 8 + (1 if geo else 0))
    for f, L in enumerate(model.pml):
        if L.nb and f // 2 != 1:
            n_axis = g.Nx if f // 2 == 0 else g.Nz
            h += N // n_axis * L.nb * 8
            e += N // n_axis * L.nb * 8
    for imat, m in enumerate(model.materials, start=1):
        if m.nq:
            cells = int(np.count_nonzero(model.geometry == imat))
            e += cells * (2 * 4 + m.nq * 2 * 3 * 4)
    return h + e


def run_batch2d(args, three=False):
    """Batched configuration (2-D models, or with three=True small 3-D ones): all models in one
    batch (persistent launches, CUDA graph, autotuned tiles) against the same models run as
    sequential plain solves."""
    import maxwellfdtd_b200 as M
    from maxwellfdtd_b200 import _abi, workloads
    ws, rank, local = dist_setup()
    lib = M.load_library()
    if three:
        models = workloads.batch3d(n=args.sims, seed=args.seed, steps_scale=args.steps_scale)
        comps = (0, 1, 2, 6, 7, 8)
        bytes_of = lambda m: sum(algorithmic_bytes(m, None, np.float32))
    else:
        models = workloads.batch2d(n=args.sims, seed=args.seed, steps_scale=args.steps_scale)
        comps = (1, 6, 8)
        bytes_of = bytes_2d
    ncell = lambda m: m.grid.Nx * m.grid.Ny * m.grid.Nz
    cu_total = sum(ncell(m) * m.Nt for m, _ in models)
    bytes_total = sum(bytes_of(m) * m.Nt for m, _ in models)
    clk = ClockSampler(local).start()
    # warm-up: a small batch of the first members for a few steps (loads the kernels)
    wb = _abi.Batch(lib, local)
    warm = []
    for m, mo in models[:8]:
        b, meta = m.build_desc(np.float32, mo, device=local, mode=args.mode)
        st = _abi.Stepper(lib, b, np.float32)
        wb.add(st, min(m.Nt, 3 * 16))
        warm.append(st)
    wb.run_all()
    wb.close()
    for st in warm:
        st.close()
    # batched, end to end: upload every member, run all, read every member's fields and monitors
    t0 = time.time()
    batch = _abi.Batch(lib, local)
    held = []
    h2d = 0
    for m, mo in models:
        b, meta = m.build_desc(np.float32, mo, device=local, mode=args.mode)
        h2d += sum(a.nbytes for a in b.keep if isinstance(a, np.ndarray))
        st = _abi.Stepper(lib, b, np.float32)
        batch.add(st, m.Nt)
        held.append((st, meta, m))
    t_up = time.time()
    batch.run_all()
    t_run = time.time()
    clk.mark(t_up, t_run)
    clk.stop()
    d2h = 0
    for st, meta, m in held:
        for c in comps:
            d2h += st.read_field(c).nbytes
        for k, mm in enumerate(meta["monitors"]):
            for c in comps:
                d2h += st.read_monitor(k, c, (m.Nt, len(mm["cells"])), False).nbytes
    t_end = time.time()
    info = batch.info()
    batch.close()
    for st, _, _ in held:
        st.close()
    dev_ms = info["device_ms"]
    value = cu_total / (dev_ms * 1e-3) / 1e9
    # sequential plain solves of a seeded subset (device time of each mfd_run call)
    seq = [models[i] for i in np.random.default_rng(args.seed + 1).choice(len(models), min(args.seq_sims, len(models)), replace=False)]
    seq_ms, seq_cu = 0.0, 0
    for m, mo in seq:
        b, meta = m.build_desc(np.float32, mo, device=local, mode=args.mode)
        st = _abi.Stepper(lib, b, np.float32)
        st.run(1, m.Nt)
        seq_ms += st.last_run_ms()
        seq_cu += ncell(m) * m.Nt
        st.close()
    seq_value = seq_cu / (seq_ms * 1e-3) / 1e9
    peak, kind = peaks()
    achieved = bytes_total / (dev_ms * 1e-3) / 1e9
    out = {
        "metric": "Gcell-updates/s", "value": round(value, 3), "unit": "Gcell-updates/s", "n_gpus": 1,
        "steps": int(sum(m.Nt for m, _ in models)), "warmup": 3, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": (f"batch3d: {len(models)} 3-D models, Nx,Ny,Nz in [48,128], dx=20nm, 8-cell CPML, "
                                f"1-5 spheres eps in [1,12] (half Debye), Ricker point source, 4 point monitors, "
                                f"steps 500-2000 x {args.steps_scale}") if three else
                               (f"batch2d: {len(models)} 2-D models, Nx,Nz in [128,1024], dx=20nm, 10-cell CPML, "
                                f"1-20 ellipses eps in [1,12] (half Debye), Ricker point source, 4 point monitors, "
                                f"steps 2000-6000 x {args.steps_scale}"),
                   "cells": int(sum(ncell(m) for m, _ in models)), "cell_updates": int(cu_total),
                   "seed": args.seed, "mode": args.mode, "parallelism": "one batch, persistent launches, CUDA graph",
                   "l2": "inputs larger than L2", "tile": list(info["tile"])},
        "e2e": {"value": round(cu_total / (t_end - t0) / 1e9, 3), "unit": "Gcell-updates/s",
                "h2d_bytes_per_step": int(h2d / max(1, max(m.Nt for m, _ in models))),
                "d2h_bytes_per_step": int(d2h / max(1, max(m.Nt for m, _ in models))),
                "includes": "descriptor upload of every member + batched run + read-back of fields and monitors",
                "wall_s": round(t_end - t0, 3)},
        "roofline": {"bound": "hbm", "kernel": ("batched 3-D step (batch_h3d + batch_e3d + material/sources/monitors)" if three
                                                else "batched 2-D step (batch_h2d + batch_e2d + material/sources/monitors)"),
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": None, "algorithmic_bytes": int(bytes_total), "peak_kind": kind},
        "sequential": {"value": round(seq_value, 3), "unit": "Gcell-updates/s", "sims": len(seq),
                       "note": "the same kind of models run one at a time with mfd_run (device time per run)"},
        "batched_vs_sequential": round(value / seq_value, 2),
        "gpu_launches": int(info["launches"]),
        "clocks": clk.summary(),
    }
    print(json.dumps(out), flush=True)
    return out


def run_serve(args):
    """Served mixed stream: Poisson arrivals of 2-D and 3-D solves through the serving loop
    (admission by device memory, continuous batching of 2-D and small 3-D requests, solo
    lanes for the rest),
    against the same requests solved one at a time."""
    import maxwellfdtd_b200 as M
    from maxwellfdtd_b200 import serve, workloads
    ws, rank, local = dist_setup()
    lib = M.load_library()
    stream = workloads.served(n=args.requests, rate=args.rate, seed=args.seed, steps_scale=args.steps_scale)
    reqs = [serve.Request(i, m, mo, a, mode=args.mode) for i, (a, m, mo) in enumerate(stream)]   # client-side descriptors
    # warm-up: two small requests alone (loads the kernels)
    for _, m, mo in workloads.served(n=2, seed=args.seed + 7, steps_scale=0.01, n2=(64, 96), n3=(24, 32)):
        serve.solve_alone(lib, serve.Request(-1, m, mo, 0.0))
    clk = ClockSampler(local).start()
    srv = serve.Server(lib, device=local, budget_bytes=args.budget_gb * 1e9, max_active=args.slots,
                       max_solo=args.solo_lanes, chunk=64)
    t0 = time.time()
    stats = srv.run(reqs)
    clk.mark(t0, time.time())
    clk.stop()
    h2d = sum(sum(a.nbytes for a in r.builder.keep if isinstance(a, np.ndarray)) for r in reqs)
    d2h = sum(sum(v.nbytes for v in r.out.values()) for r in reqs if r.out)
    # the same kind of requests as sequential plain solves (a seeded subset, end to end each)
    pick = np.random.default_rng(args.seed + 1).choice(len(reqs), min(args.seq_sims, len(reqs)), replace=False)
    seq_t, seq_cu = 0.0, 0
    for i in pick:
        _, _, wall = serve.solve_alone(lib, reqs[i], fields=False)
        seq_t += wall
        seq_cu += reqs[i].cell_updates
    seq_value = seq_cu / seq_t / 1e9
    value = stats["gcell_updates_per_s"]
    out = {
        "metric": "Gcell-updates/s", "value": round(value, 3), "unit": "Gcell-updates/s", "n_gpus": 1,
        "steps": int(sum(r.model.Nt for r in reqs)), "warmup": 2, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"served: {len(reqs)} requests, Poisson {args.rate}/s, 2-D sides 256-2048 / 3-D sides "
                               f"64-256 (dx=10nm), 500-5000 steps x {args.steps_scale}, dielectric/Drude/Lorentz, "
                               f"TFSF or soft plane source, spectral monitor 8-32 freq FP64",
                   "budget_gb": args.budget_gb, "slots": args.slots, "solo_lanes": args.solo_lanes, "seed": args.seed,
                   "mode": args.mode,
                   "parallelism": "one GPU: continuous batch of 2-D requests + concurrent solo lanes"},
        "latency": {"p50_s": round(stats["latency_p50_s"], 4), "p99_s": round(stats["latency_p99_s"], 4),
                    "queue_wait_p50_s": round(stats["queue_wait_p50_s"], 4),
                    "queue_wait_p99_s": round(stats["queue_wait_p99_s"], 4)},
        "e2e": {"value": round(value, 3), "unit": "Gcell-updates/s",
                "h2d_bytes_per_step": int(h2d / max(1, sum(r.model.Nt for r in reqs))),
                "d2h_bytes_per_step": int(d2h / max(1, sum(r.model.Nt for r in reqs))),
                "includes": "every request from arrival: admission, upload, steps, read-back of its monitors (spectra)"},
        "requests": {"batched": stats["batched"], "solo": stats["solo"], "errors": stats["errors"],
                     "phase_sum_s": {k: round(v, 3) for k, v in stats["phase_sum_s"].items()},
                     "makespan_s": round(stats["makespan_s"], 3), "cell_updates": stats["cell_updates"],
                     "peak_device_gb": round(srv.peak_used / 1e9, 2), "peak_active": srv.peak_active},
        "sequential": {"value": round(seq_value, 3), "unit": "Gcell-updates/s", "requests": len(pick),
                       "note": "the same kind of requests solved one at a time, end to end (create, run, read-back of monitors)"},
        "served_vs_sequential": round(value / seq_value, 2),
        "clocks": clk.summary(),
    }
    print(json.dumps(out), flush=True)
    return out


def _rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = max(np.linalg.norm(a), np.linalg.norm(b))
    return 0.0 if den == 0 else float(np.linalg.norm(a - b) / den)


def _fields(st, ndim):
    from maxwellfdtd_b200.sources import comp_index, field_components
    return {c: st.read_field(comp_index(c)) for c in field_components(ndim) if not c.startswith("D")}


def _timed_solve(lib, model, mons, dtype, W, K, local, profile_steps=0, mode="exact"):
    """Warm-up W steps, then steps W+1..W+K in one timed call, then profile_steps more with
    per-launch events; returns (stepper, ms, meta, per-kernel ms per step)."""
    from maxwellfdtd_b200 import _abi
    b, meta = model.build_desc(dtype, mons, device=local, mode=mode)
    st = _abi.Stepper(lib, b, dtype)
    st.run(1, W)
    st.run(W + 1, W + K)
    ms = st.last_run_ms()
    per = None
    if profile_steps:
        k0 = st.kernel_times()
        st.set_profiling(True)
        st.run(W + K + 1, W + K + profile_steps)
        st.set_profiling(False)
        k1 = st.kernel_times()
        per = {k: round((k1[k][0] - k0[k][0]) / profile_steps * 1e3, 2) for k in k1 if k1[k][1] > k0[k][1]}
    return st, ms, meta, per


def run_config(args):
    """The reference-style configurations other than the headline: `dielectric100` (100^3
    FP64 dielectric sphere, TFSF data from a vacuum record run, 1000 steps) and `nonlinear`
    (192 x 192 x 1024 FP32 glass with 3 Lorentz poles, Kerr and FP64 plasma).  Device
    throughput and the error against the FP64 CPU oracle (the full configuration for
    dielectric100; a 48 x 48 x 256 grid of the same medium, spacing and source for nonlinear)."""
    import tempfile
    import maxwellfdtd_b200 as M
    from maxwellfdtd_b200 import _abi, workloads
    ws, rank, local = dist_setup()
    lib = M.load_library()
    peak, kind = peaks()
    oracle = _oracle_lib()
    threads = oracle.lib.oracle_set_threads(0)
    if args.workload == "dielectric100":
        dtype = np.float64
        rec_model, box, scatter = workloads.dielectric_100_record(nt=1000)
        with tempfile.TemporaryDirectory() as tmp:
            sol = M.solve(rec_model, backend=M.B200(dtype), tfsf_record=True, tfsf_box=box,
                          tfsf_fname=os.path.join(tmp, "rec.npz"))
        model, mons = scatter(sol.out["tfsf_record"])
        W = args.warmup
        K = model.Nt - W - 20
        clk = ClockSampler(local).start()
        t0 = time.time()
        st, ms, meta, per = _timed_solve(lib, model, mons, dtype, W, K, local, profile_steps=20, mode=args.mode)
        clk.mark(t0, time.time())
        clk.stop()
        gpu = _fields(st, 3)
        gpu_mon = st.read_monitor(0, 6, (model.Nt, 1), False)
        st.close()
        # the FP64 oracle on the same descriptor, all steps
        b, meta = model.build_desc(dtype, mons)
        so = _abi.Stepper(oracle, b, dtype)
        t = time.perf_counter()
        so.run(1, model.Nt)
        cpu_s = time.perf_counter() - t
        ref = _fields(so, 3)
        ref_mon = so.read_monitor(0, 6, (model.Nt, 1), False)
        so.close()
        err = {c: _rel_l2(gpu[c], ref[c]) for c in gpu}
        err["monitor_Ex"] = _rel_l2(gpu_mon, ref_mon)
        err_note = f"full configuration, all 1000 steps, FP64 GPU ({args.mode} mode) vs FP64 oracle"
        wl = "dielectric100: 100^3 FP64, dx=20nm, 10-cell CPML, sphere r=500nm eps=2.25, TFSF 800nm/10fs from a vacuum record run, 1000 steps"
        cpu = {"value": round(model.grid.Nx * model.grid.Ny * model.grid.Nz * model.Nt / cpu_s / 1e9, 5),
               "unit": "Gcell-updates/s", "cores": int(threads), "kind": "port", "sample": f"all {model.Nt} steps ({cpu_s:.1f} s)"}
    else:
        dtype = np.float32
        W, K = args.warmup, args.steps
        model, mons = workloads.nonlinear_192(nt=W + K + 22)
        clk = ClockSampler(local).start()
        t0 = time.time()
        st, ms, meta, per = _timed_solve(lib, model, mons, dtype, W, K, local, profile_steps=20, mode=args.mode)
        clk.mark(t0, time.time())
        clk.stop()
        st.close()
        # error: the same medium, spacing and source on a 48 x 48 x 256 grid, GPU FP32 vs oracle FP64
        n_small, steps_small = (48, 48, 256), args.err_steps
        small, _ = workloads.nonlinear_192(nt=steps_small, n=n_small)
        out = {}
        cpu_s = None
        for tag, lib_, dt_ in (("gpu", lib, np.float32), ("fp64", oracle, np.float64), ("fp32", oracle, np.float32)):
            b, meta = small.build_desc(dt_, None, mode=args.mode if tag == "gpu" else "exact")
            sx = _abi.Stepper(lib_, b, dt_)
            t = time.perf_counter()
            sx.run(1, small.Nt)
            if tag == "fp64":
                cpu_s = time.perf_counter() - t
            out[tag] = {**_fields(sx, 3), "rho_end": sx.read_integral(_abi.MFD_INT_RHO)}
            sx.close()
        vec = lambda o, cs: np.concatenate([np.asarray(o[c], np.float64).ravel() for c in cs])
        groups = {"E": ("Ex", "Ey", "Ez"), "H": ("Hx", "Hy", "Hz"), "rho_end": ("rho_end",)}
        err = {g: _rel_l2(vec(out["gpu"], cs), vec(out["fp64"], cs)) for g, cs in groups.items()}
        err["oracle_fp32_vs_fp64"] = {g: _rel_l2(vec(out["fp32"], cs), vec(out["fp64"], cs)) for g, cs in groups.items()}
        err["gpu_vs_fp32_oracle"] = {g: _rel_l2(vec(out["gpu"], cs), vec(out["fp32"], cs)) for g, cs in groups.items()}
        err_note = (f"{n_small[0]}x{n_small[1]}x{n_small[2]} grid of the same configuration, {steps_small} steps, "
                    f"FP32 GPU ({args.mode} mode, rho FP64) vs FP64 oracle")
        wl = ("nonlinear: 192x192x1024 FP32, dx=dy=100nm dz=20nm, 16-cell CPML, glass: 3 Sellmeier Lorentz poles + Kerr "
              "n2=2.5e-20 + 8-photon plasma (rho FP64), Gaussian beam w0=3um 800nm 30fs 5e17 W/m^2")
        Ns = n_small[0] * n_small[1] * n_small[2]
        cpu = {"value": round(Ns * steps_small / cpu_s / 1e9, 5), "unit": "Gcell-updates/s", "cores": int(threads),
               "kind": "port", "sample": f"FP64 oracle, {steps_small} steps of the {n_small} grid ({cpu_s:.1f} s)"}
    N = model.grid.Nx * model.grid.Ny * model.grid.Nz
    value = N * K / (ms * 1e-3) / 1e9
    h_bytes, e_bytes = algorithmic_bytes(model, meta, dtype)
    achieved = (h_bytes + e_bytes) / (ms * 1e-3 / K) / 1e9
    out = {"metric": "Gcell-updates/s", "value": round(value, 3), "unit": "Gcell-updates/s", "n_gpus": 1, "steps": K,
           "warmup": W, "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if dtype == np.float64 else "f32", "data": "synthetic",
           "config": {"workload": wl, "grid": [model.grid.Nx, model.grid.Ny, model.grid.Nz], "cells": N, "mode": args.mode},
           "roofline": {"bound": "hbm", "kernel": "whole step (H + E updates, material response, sources, monitors)",
                        "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                        "traffic": None, "algorithmic_bytes_per_step": int(h_bytes + e_bytes), "peak_kind": kind},
           "kernels_us_per_step": per,
           "error_vs_fp64_oracle": {"rel_l2": err, "how": err_note},
           "cpu_baseline": cpu, "clocks": clk.summary()}
    print(json.dumps(out), flush=True)
    return out


def plain_stepper(lib, args, device, steps=20):
    """The plain FP32 stepper at 256^3 (vacuum, 12-cell CPML, Sa sum): H and E update times
    and their HBM roofline fractions, CUDA events per update."""
    from maxwellfdtd_b200 import _abi, workloads
    model, _ = workloads.plain_256(nt=steps + 5, n=args.size)
    b, meta = model.build_desc(np.float32, None, device=device, mode=args.mode)
    st = _abi.Stepper(lib, b, np.float32)
    st.run(1, 3)
    k0 = st.kernel_times()
    st.set_profiling(True)
    st.run(4, 3 + steps)
    st.set_profiling(False)
    k1 = st.kernel_times()
    ms = st.last_run_ms()
    st.close()
    h_bytes, e_bytes = algorithmic_bytes(model, meta, np.float32)
    peak, kind = peaks()
    h_ms = (k1["H"][0] - k0["H"][0]) / steps
    e_ms = (k1["E"][0] - k0["E"][0]) / steps
    N = model.grid.Nx * model.grid.Ny * model.grid.Nz
    return {"workload": f"plain_256: {args.size}^3 FP32 vacuum, 12-cell CPML, soft point source, Sa sum, {args.mode} mode",
            "value": round(N * steps / (ms * 1e-3) / 1e9, 3), "unit": "Gcell-updates/s", "steps": steps,
            "h_update": {"ms": round(h_ms, 5), "bytes": h_bytes, "frac": round(h_bytes / (h_ms * 1e-3) / 1e9 / peak, 4)},
            "e_update": {"ms": round(e_ms, 5), "bytes": e_bytes, "frac": round(e_bytes / (e_ms * 1e-3) / 1e9 / peak, 4)},
            "peak_gbs": peak, "peak_kind": kind}


def _pinned_array(n, dtype):
    """A page-locked 1-D host array (torch's pinned allocator), or an ordinary one without CUDA."""
    import torch
    tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64, np.dtype(np.uint8): torch.uint8,
           np.dtype(np.int64): torch.int64, np.dtype(np.complex128): torch.complex128}[np.dtype(dtype)]
    return torch.empty(int(n), dtype=tdt, pin_memory=torch.cuda.is_available()).numpy()


def _pinned_outputs(model, meta, dtype):
    """Page-locked host arrays for the read-back of the e2e measurement (torch's pinned
    allocator), or ordinary arrays when no CUDA is present."""
    import torch
    g = model.grid
    N = g.Nx * g.Ny * g.Nz

    def arr(n, dt):
        return _pinned_array(n, dt)
    out = {"Sa": arr(N, dtype)}
    out["E2"] = arr(N, dtype)
    for m, ms_ in enumerate(meta["monitors"]):
        for c in (0, 1, 2, 6, 7, 8):
            out[("m", m, c)] = arr(ms_["dft"].Nw * len(ms_["cells"]), np.complex128).reshape(ms_["dft"].Nw, len(ms_["cells"]))
    return out


def headline_error(lib, device, n=96, steps=60, mode="exact"):
    """Relative L2 error of the single-precision GPU result against the FP64 oracle on an
    n^3 version of the headline configuration (same spacing, sphere, TFSF and monitors
    scaled with the grid): the E and H vectors, Sa, and the DFT spectra; and the distance to
    the oracle run in single precision (the parity measure, 0 when bit-identical)."""
    from maxwellfdtd_b200 import _abi, workloads
    from maxwellfdtd_b200.sources import comp_index
    oracle = _oracle_lib()
    oracle.lib.oracle_set_threads(0)
    model, mons = workloads.plasmonics_256(nt=steps, n=n)
    res = {}
    for tag, lb, dt in (("gpu", lib, np.float32), ("fp64", oracle, np.float64), ("fp32", oracle, np.float32)):
        b, meta = model.build_desc(dt, mons, device=device if lb is lib else 0, mode=mode if lb is lib else "exact")
        st = _abi.Stepper(lb, b, dt)
        st.run(1, model.Nt)
        o = {c: st.read_field(comp_index(c)) for c in ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez")}
        o["Sa"] = st.read_integral(_abi.MFD_INT_SA)
        o["dft"] = np.concatenate([st.read_monitor(k, comp_index(c), (mm["dft"].Nw, len(mm["cells"])), True).ravel()
                                   for k, mm in enumerate(meta["monitors"]) for c in ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez")])
        st.close()
        res[tag] = o
    vec = lambda o, cs: np.concatenate([np.asarray(o[c]).ravel() for c in cs])
    groups = {"E": ("Ex", "Ey", "Ez"), "H": ("Hx", "Hy", "Hz"), "Sa": ("Sa",), "dft": ("dft",)}

    def rel(a, b):
        a = np.concatenate([a.real.ravel(), a.imag.ravel()]) if np.iscomplexobj(a) else a.astype(np.float64)
        b = np.concatenate([b.real.ravel(), b.imag.ravel()]) if np.iscomplexobj(b) else b.astype(np.float64)
        den = max(np.linalg.norm(a), np.linalg.norm(b))
        return 0.0 if den == 0 else float(np.linalg.norm(a - b) / den)
    return {"rel_l2": {g: rel(vec(res["gpu"], cs), vec(res["fp64"], cs)) for g, cs in groups.items()},
            "gpu_vs_fp32_oracle": {g: rel(vec(res["gpu"], cs), vec(res["fp32"], cs)) for g, cs in groups.items()},
            "how": f"{n}^3 version of the workload (dx=2nm, same sphere, TFSF and DFT faces scaled), {steps} steps, "
                   f"GPU in the {mode} mode"}


def _oracle_lib():
    from maxwellfdtd_b200 import _abi
    so = os.path.join(ROOT, "oracle", "libmfd_oracle.so")
    if not os.path.exists(so):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return _abi.Library(so, "oracle_")


def cpu_baseline(args, model, mons, steps=None):
    """The oracle (the reference's CPU path restated in C++, OpenMP) on the same workload,
    a bounded number of steps on all host cores."""
    from maxwellfdtd_b200 import _abi
    lib = _oracle_lib()
    threads = lib.lib.oracle_set_threads(0)
    steps = steps or args.cpu_steps
    b, meta = model.build_desc(np.float32, mons)
    st = _abi.Stepper(lib, b, np.float32)
    st.run(1, 1)
    t0 = time.perf_counter()
    st.run(2, 1 + steps)
    dt = time.perf_counter() - t0
    st.close()
    N = model.grid.Nx * model.grid.Ny * model.grid.Nz
    return {"value": round(N * steps / dt / 1e9, 5), "unit": "Gcell-updates/s", "cores": int(threads),
            "kind": "port", "sample": f"{steps} full steps of the {args.size}^3 workload ({dt:.1f} s)"}


def run_reference(args):
    ws, rank, local = dist_setup()
    if rank != 0:
        return None
    from maxwellfdtd_b200 import _abi, workloads
    W, K = args.warmup, args.steps
    # each step a bounded sample: full 256^3 steps on the host cores
    nt = W + K + 2
    model, mons = workloads.plasmonics_256(nt=nt, n=args.size)
    lib = _oracle_lib()
    threads = lib.lib.oracle_set_threads(0)
    b, meta = model.build_desc(np.float32, mons)
    st = _abi.Stepper(lib, b, np.float32)
    st.run(1, W)
    t0 = time.perf_counter()
    st.run(W + 1, W + K)
    dt = time.perf_counter() - t0
    st.close()
    N = model.grid.Nx * model.grid.Ny * model.grid.Nz
    v = N * K / dt / 1e9
    out = {"impl": "reference", "metric": "Gcell-updates/s", "value": round(v, 5), "unit": "Gcell-updates/s",
           "n_gpus": ws, "steps": K, "warmup": W, "ms_per_step": round(dt * 1e3 / K, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "grid": [args.size] * 3, "cells": N, "parallelism": "host cores"},
           "cpu_baseline": {"value": round(v, 5), "unit": "Gcell-updates/s", "cores": int(threads), "kind": "port",
                            "sample": f"{K} full steps of the {args.size}^3 workload after {W} warm-up steps"},
           "e2e": {"value": round(v, 5), "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=256, help="grid side of the headline workload")
    ap.add_argument("--cpu-steps", type=int, default=40, help="steps of the CPU-baseline sample (about 10 s on 16 cores)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-stepper roofline measurement")
    ap.add_argument("--mode", default="fast", choices=["fast", "exact"],
                    help="arithmetic of the field updates (fast: the tolerance mode; exact: bit-identical order)")
    ap.add_argument("--late-start", type=int, default=1500,
                    help="plasmonics: steps run before the second timed window (0: no late window)")
    ap.add_argument("--workload", default="plasmonics", choices=["plasmonics", "batch2d", "batch3d", "serve", "dielectric100", "nonlinear"])
    ap.add_argument("--err-steps", type=int, default=300, help="nonlinear: steps of the oracle comparison")
    ap.add_argument("--requests", type=int, default=48, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: Poisson arrival rate (1/s)")
    ap.add_argument("--budget-gb", type=float, default=160.0, help="serve: device-memory admission budget")
    ap.add_argument("--slots", type=int, default=64, help="serve: requests resident at once")
    ap.add_argument("--solo-lanes", type=int, default=16, help="serve: concurrent solo lanes")
    ap.add_argument("--sims", type=int, default=256, help="batch2d: number of models")
    ap.add_argument("--steps-scale", type=float, default=None,
                    help="batch2d / serve: scale of the step counts (default 0.25 / 0.25)")
    ap.add_argument("--seq-sims", type=int, default=16, help="batch2d / serve: models timed as sequential solves")
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if args.steps > 20:
            args.steps = 20   # each reference step is a full 256^3 step on the CPU
        run_reference(args)
    elif args.workload in ("batch2d", "batch3d"):
        args.steps_scale = 0.25 if args.steps_scale is None else args.steps_scale
        run_batch2d(args, three=args.workload == "batch3d")
    elif args.workload in ("dielectric100", "nonlinear"):
        run_config(args)
    elif args.workload == "serve":
        args.steps_scale = 0.25 if args.steps_scale is None else args.steps_scale
        run_serve(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
