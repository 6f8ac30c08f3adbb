#!/usr/bin/env python3
"""Benchmark: Mobile V2 cell-substeps/s on the config-1 plain path (701^2).

One step = one 1/60 s physics step of the plain terrain path on a 701 x 701
grid (dx 0.05 m): bucket-cut entrainment -> Mobile V2 finite-volume step (all
CFL substeps) -> large-avalanche labelling (38 deg start, 8-connected) ->
gated residual frontier relaxation, through the public Python API over the C
ABI.  Inputs: the seeded 6-octave value-noise pile (seed 1) and the straight
bucket cut of the config; synthetic data, no dataset.

  value   cell-substeps/s = 701^2 * sum(substeps) / sum(device step time), with
          the terrain resident in HBM; device time from CUDA events on the
          library's stream; L2 flushed (256 MiB write) between timed steps.
  e2e     the same cell-substeps over host wall-clock time, including per step
          the pinned-host -> device copy of the cut command (indices + target
          surfaces) and the device -> host read of the step records.
  roofline  dominant kernel = the fused FV substep kernel; achieved =
          28 B/cell * cells per launch / mean launch time from CUDA events
          recorded around the device-side substep loop.

``--impl reference`` times the CPU restatement of the reference path (NumPy,
oracle/) on the same workload, one rank only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mobile V2 cell-substeps/s at 701^2 (config-1 plain path)"
UNIT = "cell-substeps/s"
N = 701
DX = 0.05
DT = 1.0 / 60.0
BYTES_PER_CELL_SUBSTEP = 28  # FX32: read b,h,qx,qy (16 B) + write h,qx,qy (12 B)


def material():
    import soilb200
    return soilb200.MaterialScenario("config1_soil", 1600.0, 35.0, 0.0, 0.5, 38.0, 30.0, 0.55)


def cut_schedule(cut, steps: int, pinned: bool):
    """Per-step cut commands (flat indices, target surfaces), optionally pinned."""
    out = []
    for k in range(steps):
        idx, tgt = cut.footprint((k + 1) * DT)
        if pinned:
            import torch
            ti = torch.empty(idx.size, dtype=torch.int32, pin_memory=True)
            tt = torch.empty(tgt.size, dtype=torch.float64, pin_memory=True)
            ti.numpy()[:] = idx
            tt.numpy()[:] = tgt
            out.append((ti.numpy(), tt.numpy()))
        else:
            out.append((idx, tgt))
    return out


class ClockSampler:
    """SM clock / throttle-reason sampling during the timed region.

    NVML is read from a thread every 2 ms (a timed region of a few tens of
    milliseconds still gets a median); nvidia-smi polling is the fallback when
    NVML cannot be opened.  Only reads: no clock or power setting is touched.
    """

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, period_s: float = 0.002):
        self.device = device
        self.period = period_s
        self.samples = []            # (sm_mhz, sm_max_mhz, reasons bitmask)
        self.source = None
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None
        self._handle = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            self._nvml = pynvml
            try:
                uuid = str(torch.cuda.get_device_properties(device).uuid)
                self._handle = pynvml.nvmlDeviceGetHandleByUUID(
                    uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                self._handle = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.source = "nvml"
        except Exception:
            self._nvml = None
            self.source = "nvidia-smi"

    def _sample_nvml(self):
        n = self._nvml
        sm = n.nvmlDeviceGetClockInfo(self._handle, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(self._handle, n.NVML_CLOCK_SM)
        get = getattr(n, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            n.nvmlDeviceGetCurrentClocksThrottleReasons
        self.samples.append((float(sm), float(mx), int(get(self._handle))))

    def _sample_smi(self):
        out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                              "--format=csv,noheader,nounits"],
                             capture_output=True, text=True, timeout=5).stdout.strip()
        if not out:
            return
        f = [x.strip() for x in out.split(",")]
        mask = 0
        for (name, bit), val in zip(self.REASONS, f[5:9]):
            if val.lower().startswith("active"):
                mask |= bit
        try:
            self.samples.append((float(f[1]), float(f[2]), mask))
        except ValueError:
            pass

    def _run(self):
        while not self._stop.is_set():
            try:
                if self._nvml is not None:
                    self._sample_nvml()
                else:
                    self._sample_smi()
            except Exception:
                pass
            self._stop.wait(self.period if self._nvml is not None else 0.2)

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = sorted({name for _, _, m in self.samples for name, bit in self.REASONS
                          if m & bit})
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples), "reasons": reasons,
                "samples": len(self.samples), "source": self.source}


# DRAM bytes (read + write) per FV substep, from one ncu capture of the
# persistent substep-loop kernel on the same workload (dram__bytes_read.sum +
# dram__bytes_write.sum of the launch, divided by the substeps it ran).
NCU_TRAFFIC_BYTES = {
    # fv_loop_kernel at 701^2, 3 substeps in the captured launch: 8.028672 MB
    # read + 1.536 KB written (cold L2 under ncu; the state then stays in L2)
    "config1_plain_path_701": (8_028_672 + 1_536) // 3,
    # fv_loop_kernel at 4096^2, 4 substeps in the captured launch: 1.130031 GB
    # read + 805.078784 MB written
    "mobile_v2_4096": (1_130_031_000 + 805_078_784) // 4,
    # fv_loop_kernel on the config-4 site (4096^2, 64 cuts), the first timed
    # step's launch, 3 substeps: 841.548288 MB read + 592.439552 MB written
    "site_c4_4096": (841_548_288 + 592_439_552) // 3,
}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def combine_over_ranks(dev_s: float, wall_s: float, work: float, device: str):
    """Replicas: the job's time is the slowest rank's (device and wall clock),
    its work the sum over ranks.  Every rank calls this with the same
    collectives in the same order."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([dev_s, wall_s], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(work)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), float(c[0])


def run_gpu(args, rank: int, world: int, local_rank: int):
    import torch
    import soilb200
    from soilb200 import workloads
    from soilb200.pipeline import PlainPath

    torch.cuda.set_device(local_rank)
    site = args.workload == "site_c4_4096"
    if site:
        n = 4096
        cfg = workloads.config4(n, seed=4, dx=DX)

        class _Cuts:  # the 64 cuts' union as one per-step command
            @staticmethod
            def footprint(t):
                return workloads.merged_footprint(cfg["cuts"], t)
        cut = _Cuts()
    else:
        n = N
        cfg = workloads.config1(N, seed=1, dx=DX)
        cut = cfg["cut"]
    # one CUDA graph per step; with SOILB200_NO_GRAPH=1 (profilers) the same
    # kernels are launched operator by operator instead
    fused = os.environ.get("SOILB200_NO_GRAPH") != "1"
    path = PlainPath(cfg["b_eff"], cfg["z_base"], dx=DX, material=material(),
                     device=local_rank, residual="gated", fused=fused)
    grid = path.grid
    total_steps = args.warmup + args.steps
    sched = cut_schedule(cut, total_steps, pinned=True)
    stream = torch.cuda.ExternalStream(grid.stream_handle(), device=local_rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local_rank}")

    for k in range(args.warmup):
        idx, tgt = sched[k]
        path.step(DT, idx, tgt)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()

    launches0 = grid.kernel_launches()
    step_ms, substeps, loop_ms = [], [], []
    stage_sum = {}
    h2d = d2h = 0
    stats_bytes = 2 * 400  # MobileStats + LabelOut records read back per step (approx, fixed)
    wall = 0.0
    with ClockSampler(local_rank) as clocks:
        for k in range(args.warmup, total_steps):
            flush.zero_()
            torch.cuda.synchronize()
            idx, tgt = sched[k]
            if fused:
                # the step call is synchronous (its records are read back before
                # it returns): the wall clock around it is the end-to-end time,
                # and its device time comes from the step graph's own first and
                # last event nodes
                t0 = time.perf_counter()
                st = path.step(DT, idx, tgt)
                wall += time.perf_counter() - t0
                step_ms.append(path.last_stats.device_ms)
            else:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                t0 = time.perf_counter()
                e0.record(stream)
                st = path.step(DT, idx, tgt)
                e1.record(stream)
                e1.synchronize()
                wall += time.perf_counter() - t0
                step_ms.append(e0.elapsed_time(e1))
            substeps.append(st.substeps)
            if args.stages:
                for name, ms in path.stage_times().items():
                    stage_sum[name] = stage_sum.get(name, 0.0) + ms
            ls = path.mobile.last_stats
            if ls is not None and ls.substeps:
                loop_ms.append((ls.substep_loop_ms, ls.substeps))
            h2d += idx.nbytes + tgt.nbytes
            d2h += stats_bytes
    launches = grid.kernel_launches() - launches0
    # precision report (untimed): wet cells of the final state, and the FX32
    # fields against the same step sequence run in FP64 from the same inputs
    h_fx = grid.download("mobile")
    b_fx = grid.download("b_eff")
    wet_cells = int(np.count_nonzero(h_fx > 0.0))
    site_extra = site_report(path, st, h_fx, local_rank) if site else None
    if site_extra is not None and not args.no_repose:
        site_extra["settle"] = site_settle(path, local_rank)
    ref64 = PlainPath(cfg["b_eff"], cfg["z_base"], dx=DX, material=material(),
                      device=local_rank, residual="gated", precision="fp64", fused=fused)
    for k in range(total_steps):
        idx, tgt = sched[k]
        ref64.step(DT, idx, tgt)
    dh_max = float(np.abs(h_fx - ref64.grid.download("mobile")).max())
    db_max = float(np.abs(b_fx - ref64.grid.download("b_eff")).max())
    ref64.close()
    dev_s = sum(step_ms) / 1000.0
    cells = n * n
    cell_substeps = cells * sum(substeps)
    if world > 1:
        dev_s, wall, cell_substeps = combine_over_ranks(dev_s, wall, cell_substeps,
                                                        f"cuda:{local_rank}")
    peak, peak_kind = measured_peak()
    tot_loop = sum(m for m, _ in loop_ms)
    tot_launch = sum(n for _, n in loop_ms)
    per_launch_ms = tot_loop / tot_launch if tot_launch else None
    alg_bytes = BYTES_PER_CELL_SUBSTEP * cells
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms else None
    result = None
    if rank == 0:
        result = {
            "metric": ("Mobile V2 cell-substeps/s at 4096^2 (config-4 site, 64 cuts)" if site
                       else METRIC),
            "value": cell_substeps / dev_s if dev_s > 0 else 0.0, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_s * 1000.0 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32-quanta+f32 (f64/i64 ledger)",
            "data": ("synthetic (seeded config-4 value-noise site + 64 bucket cuts)" if site
                     else "synthetic (seeded config-1 value-noise pile + bucket cut)"),
            "config": {"workload": args.workload, "grid": [n, n], "dx_m": DX,
                       "dt_s": DT, "steps_simulated_before_timing": args.warmup,
                       "step": "cut entrain -> Mobile V2 (all substeps) -> labelling -> "
                               "gated residual frontier",
                       "precision": "FX32: int32 height quanta + float32 momentum",
                       "l2": "flushed (256 MiB write) between timed steps",
                       "parallelism": f"replicas x{world}",
                       "launch": "one CUDA graph per step" if fused else "operator by operator",
                       "device_time": ("event nodes at the step graph's first and last node"
                                       if fused else "CUDA events around each step"),
                       "substeps_total": int(sum(substeps))},
            "e2e": {"value": cell_substeps / wall if wall > 0 else 0.0, "unit": UNIT,
                    "h2d_bytes_per_step": h2d // max(args.steps, 1),
                    "d2h_bytes_per_step": d2h // max(args.steps, 1)},
            "roofline": {"bound": "hbm",
                         "kernel": "fv_loop_kernel (FX32 persistent substep loop; per substep)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "mean_launch_ms": per_launch_ms,
                         "traffic": NCU_TRAFFIC_BYTES.get(args.workload),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                           "of one loop launch / its substeps"},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "wet_cells": wet_cells,
            "wet_fraction": wet_cells / cells,
            "max_abs_dh_vs_fp64_m": dh_max,
            **({"site": site_extra} if site_extra else {}),
            **({"stage_ms_per_step": {k: v / args.steps for k, v in stage_sum.items()},
                "stage_note": "event nodes between the step graph's stages (they add a "
                              "little time of their own)"} if stage_sum else {}),
            "precision_vs_fp64": {
                "max_abs_dh_m": dh_max, "max_abs_db_m": db_max, "bound_m": 1.0e-5,
                "steps_compared": total_steps,
                "how": "same inputs and cut schedule stepped by the FP64 path (the "
                       "reference's arithmetic) on the GPU, fields compared after the "
                       "last step"},
        }
    return result


def site_report(path, last, h, device: int, reps: int = 10, tile: int = 64):
    """Config-4 extras for the site line: the labelling (yield + union-find +
    component reductions, sb_label) timed alone on the final state with CUDA
    events, the component count of the last step, and the fraction of 64^2
    tiles that hold mobile material or unstable cells."""
    import torch
    grid = path.grid
    stream = torch.cuda.ExternalStream(grid.stream_handle(), device=device)
    path.avalanche.label(release_settled_latches=False)  # warm
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        st = path.avalanche.label(release_settled_latches=False)
    e1.record(stream)
    e1.synchronize()
    labels = grid.download("labels")
    ny, nx = h.shape
    ty, tx = (ny + tile - 1) // tile, (nx + tile - 1) // tile
    busy = (h > 0.0) | (labels >= 0)
    pad = np.zeros((ty * tile, tx * tile), dtype=bool)
    pad[:ny, :nx] = busy
    tiles = pad.reshape(ty, tile, tx, tile).any(axis=(1, 3))
    return {"labelling_ms": e0.elapsed_time(e1) / reps,
            "labelling_what": "sb_label on the final state: cohesive yield, block-local "
                              "union-find, border merge, compression, component reductions",
            "components": int(last.regions), "unstable_cells": int(last.unstable_cells),
            "largest_component_cells": int(last.largest),
            "active_tile_fraction": float(tiles.mean()),
            "active_tile_rule": f"{tile}x{tile} tiles holding mobile material or unstable cells",
            "label_regions_check": int(st.connected_region_count)}


def site_settle(path, device: int, trials: int = 3, eps_slope: float = 1e-4,
                angle_deg: float = 35.0):
    """Config-4 settle stage, on the site's own resident state after the timed
    steps: PlainPath.settle relaxes the resting surface to 35 deg with the
    learned proposal schedule + plain sweeps, and with the plain sweeps alone,
    from the same start (restored untimed before every trial); device time
    with CUDA events on the grid's stream, median of ``trials``."""
    import torch
    from soilb200 import learned
    from soilb200.train_repose import DEFAULT_WEIGHTS
    grid = path.grid
    lr = learned.LearnedRelaxation(grid, learned.ReposeNet.load(DEFAULT_WEIGHTS), angle_deg)
    stream = torch.cuda.ExternalStream(grid.stream_handle(), device=device)
    start = grid.download("b_eff")
    q = 2.0 ** grid.height_exponent

    def quanta():
        return int(np.rint((grid.download("b_eff") - grid.datum) * q).astype(np.int64).sum())

    def one(schedule):
        grid.upload("b_eff", start)
        s0 = quanta()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        st = path.settle(lr, eps_slope * DX, schedule)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), int(st.iterations), bool(st.converged), quanta() == s0

    one(learned.PLAIN)  # warm: relaxation graphs, the network's workspace
    one(learned.SCHEDULE)
    plain = [one(learned.PLAIN) for _ in range(trials)]
    learn = [one(learned.SCHEDULE) for _ in range(trials)]
    grid.upload("b_eff", start)
    pm = statistics.median(p[0] for p in plain)
    lm = statistics.median(p[0] for p in learn)
    return {"what": "PlainPath.settle on the site's resident state after the timed steps: "
                    f"resting surface to {angle_deg:g} deg, eps {eps_slope:g}",
            "learned_ms": lm, "plain_ms": pm, "speedup_vs_plain": pm / lm,
            "learned_sweeps": learn[0][1], "plain_sweeps": plain[0][1],
            "converged": all(p[2] for p in plain + learn),
            "mass_ledger_exact": all(p[3] for p in plain + learn), "trials": trials}


def run_mobile_large(args, n: int = 4096):
    """Mobile V2 steps alone on an n^2 grid that is wet everywhere (HBM-bound:
    the 28 B/cell working set of n = 4096 is 470 MB, well above the 126 MB L2)."""
    import torch
    import soilb200
    from soilb200.bulk_state import B200BulkState, B200ProductionMobileV2Solver

    ys, xs = np.indices((n, n), dtype=np.float64)
    b = np.tan(np.deg2rad(10.0)) * xs * DX + 0.2 * np.sin(xs / 37.0) * np.cos(ys / 29.0)
    h = 0.15 + 0.1 * np.cos(xs / 53.0) * np.sin(ys / 41.0)
    state = B200BulkState((n, n), DX, DX, b, mobile_headroom_m=1.0)
    state.grid.upload("mobile", h)
    state.grid.upload("momentum_x", 0.8 * h)   # 0.8 m/s downslope: never static
    state.grid.upload("momentum_y", 0.3 * h)
    cfg = soilb200.MobileV2Config(dx_m=DX, dy_m=DX)
    solver = B200ProductionMobileV2Solver(state=state, config=cfg)
    solver.bind_device_state(state, material())
    stream = torch.cuda.ExternalStream(state.grid.stream_handle())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    warm_subs = [int(solver.step_resident(DT).substeps) for _ in range(args.warmup)]
    torch.cuda.synchronize()
    dev_ms, subs, loop = 0.0, 0, []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rec = solver.step_resident(DT)
            e1.record(stream)
            e1.synchronize()
            dev_ms += e0.elapsed_time(e1)
            subs += rec.substeps
            ls = solver.last_stats
            loop.append((ls.substep_loop_ms, ls.substeps))
    peak, kind = measured_peak()
    per = sum(m for m, _ in loop) / max(sum(k for _, k in loop), 1)
    alg = BYTES_PER_CELL_SUBSTEP * n * n
    ach = alg / (per * 1e-3) / 1e9
    return {"metric": f"Mobile V2 cell-substeps/s at {n}^2 (FV step only, wet everywhere)",
            "value": n * n * subs / (dev_ms * 1e-3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "substeps": subs, "warmup_substeps": warm_subs, "higher_is_better": True,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_source": kind, "mean_launch_ms": per,
                         "algorithmic_bytes_per_launch": alg,
                         "traffic": NCU_TRAFFIC_BYTES["mobile_v2_4096"],
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                           "of one loop launch / its substeps"},
            "clocks": clocks.summary()}


def _c2_cpu_patch(args):
    """Oracle (NumPy FP64 restatement) step of one config-2 patch; run in a
    spawned worker process."""
    i, dt = args
    import time as _t
    from oracle import mobile_v2 as M
    from soilb200 import workloads
    b, h, q = workloads.config2_patch(i, DX)
    t0 = _t.perf_counter()
    st = M.step(M.OracleConfig(), b, h, q, dt)
    return h.size * st.substeps, _t.perf_counter() - t0


def c2_cpu_baseline(budget_s: float = 20.0):
    """Config-2 patches stepped by the CPU oracle on a process pool over all
    host cores (bounded sample: the first patches in seed order until the
    budget is used)."""
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    done_cells, n = 0, 0
    with ctx.Pool(cores) as pool:
        for work, _ in pool.imap(_c2_cpu_patch, [(i, DT) for i in range(512)]):
            done_cells += work
            n += 1
            if time.perf_counter() - t0 > budget_s:
                pool.terminate()
                break
    wall = time.perf_counter() - t0
    return {"value": done_cells / wall, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} config-2 patches (seeds 1000+i), one 1/60 s Mobile V2 step each, "
                      f"NumPy FP64 oracle, process pool of {cores}; {wall:.1f} s wall"}


def run_batched_c2(args, n_patches: int = 512):
    """Config 2: 512 uneven patches stepped together by the batched runtime
    (one graph per physics step, per-patch CFL substeps, autotuned tiles)."""
    import torch
    import soilb200
    from soilb200 import workloads

    states = [soilb200.MobileV2State(b, h, q) for b, h, q in workloads.config2(n_patches, DX)]
    cells = [s.h_m.size for s in states]
    cfg = soilb200.MobileV2Config.unchecked(
        dx_m=DX, dy_m=DX, basal_friction_coefficient=float(np.tan(np.deg2rad(35.0))), cfl=0.4)
    batch = soilb200.B200PatchBatch(states, cfg)
    tuned_ms = batch.autotune(DT, trials=1)
    stream = torch.cuda.ExternalStream(batch.stream_handle())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        batch.step_stats(DT)
    torch.cuda.synchronize()
    launches0 = batch.kernel_launches()
    dev_ms, work, loop_ms, rounds = 0.0, 0, 0.0, 0
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            stats = batch.step_stats(DT)
            e1.record(stream)
            e1.synchronize()
            dev_ms += e0.elapsed_time(e1)
            work += sum(c * int(s.substeps) for c, s in zip(cells, stats))
            loop_ms += stats[0].substep_loop_ms
            rounds += max(int(s.substeps) for s in stats)
    peak, kind = measured_peak()
    ach = BYTES_PER_CELL_SUBSTEP * work / (loop_ms * 1e-3) / 1e9
    out = {"metric": "Mobile V2 cell-substeps/s, 512 batched patches (config 2)",
           "value": work / (dev_ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
           "dtype": "int32-quanta+f32 (f64/i64 ledger)", "data": "synthetic (seeded config-2 patches)",
           "config": {"workload": "batched_c2_512", "patches": n_patches, "cells": sum(cells),
                      "rows_per_warp": sorted(set(batch.rows)), "autotuned_loop_ms": tuned_ms,
                      "substep_rounds": rounds, "l2": "flushed (256 MiB write) between timed steps"},
           "roofline": {"bound": "hbm", "kernel": "batch_fv_kernel + batch_round_kernel",
                        "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                        "peak_source": kind, "algorithmic_bytes": "28 B per cell-substep",
                        "traffic": None},
           "gpu_launches": batch.kernel_launches() - launches0, "clocks": clocks.summary()}
    batch.close()
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = c2_cpu_baseline()
    return out


def c1_after_cut(n: int = N, seed: int = 1):
    """b_eff of config 1 after the whole 12 s straight cut (every footprint
    lowered to its target surface)."""
    from soilb200 import workloads
    cfg = workloads.config1(n, seed=seed, dx=DX)
    b = cfg["b_eff"].copy()
    cut = cfg["cut"]
    for k in range(1, 721):
        idx, tgt = cut.footprint(k * DT)
        b.flat[idx] = np.minimum(b.flat[idx], tgt)
    return b


def run_repose(args, eps_slope: float = 1e-4, seed: int = 1, surface=None, label=None):
    """Second headline metric: ms to repose at 701^2 after the cut, the learned
    proposal (tensor-core conv net, flux form, exact quanta) + plain sweeps
    against plain sweeps alone, same tolerance (eps * dx m), same start.  The
    proposal runs len(scales) rounds, round i moving scales[i] of the
    network's transfer (full-size rounds first, then damped ones)."""
    import torch
    import soilb200
    from soilb200 import learned
    from soilb200.train_repose import DEFAULT_WEIGHTS

    if not DEFAULT_WEIGHTS.exists():
        raise SystemExit(f"trained weights missing: {DEFAULT_WEIGHTS} (python -m soilb200.train_repose)")
    net = learned.ReposeNet.load(DEFAULT_WEIGHTS)
    fused_net = getattr(args, "net", "fused") == "fused"
    sched = learned.SCHEDULE
    scales, plain_between = sched["scales"], sched["plain_between"]
    b = c1_after_cut(seed=seed) if surface is None else surface
    k, datum = soilb200.choose_quantization(b)
    tol = eps_slope * DX
    q = 2.0 ** k

    # one resident grid per arm (buffers, graphs and the network's workspace are
    # reused across trials); each trial re-uploads the post-cut surface untimed
    rounds = len(scales)
    grids = {}
    for r in (0, rounds):
        g = soilb200.DeviceGrid(b.shape, DX, DX, precision="fx32", height_exponent=k, datum_m=datum)
        g.upload("z_base", np.zeros_like(b))
        grids[r] = (g, learned.LearnedRelaxation(g, net, 35.0, fused=fused_net))

    def one(r):
        g, lr = grids[r]
        g.upload("b_eff", b)
        s0 = int(np.rint((g.download("b_eff") - datum) * q).astype(np.int64).sum())
        stream = torch.cuda.ExternalStream(g.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        launches0 = g.kernel_launches()
        e0.record(stream)
        st = lr.relax_scheduled(tol, sched if r else learned.PLAIN, max_iterations=400000)
        e1.record(stream)
        e1.synchronize()
        s1 = int(np.rint((g.download("b_eff") - datum) * q).astype(np.int64).sum())
        return (e0.elapsed_time(e1), int(st.iterations), bool(st.converged), s0 == s1,
                g.kernel_launches() - launches0)

    for _ in range(args.warmup):
        one(0)
        one(rounds)
    plain, learn = [], []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            plain.append(one(0))
            learn.append(one(rounds))
    for g, _ in grids.values():
        g.close()
    pm = statistics.median(p[0] for p in plain)
    lm = statistics.median(p[0] for p in learn)
    n = b.shape[0]
    return {"metric": f"ms to repose at {n}^2 after the cut, learned proposal + plain sweeps (35 deg, eps 1e-4)",
            "value": lm, "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": lm, "higher_is_better": False, "dtype": "int32-quanta (bf16 net, f32 accumulate)",
            "data": label or f"synthetic (config-1 pile, seed {seed}, after the full straight cut)",
            "config": {"workload": "repose_701" if surface is None else "repose_site_4096",
                       "seed": seed, "proposal_rounds": rounds,
                       "network": ("one kernel for the four layers" if fused_net
                                   else "one launch per layer"),
                       "proposal_scales": list(scales),
                       "plain_sweeps_between_proposals": plain_between,
                       "check_sweeps": sched["check_sweeps"],
                       "extra_proposal_scales": list(sched["extra_scales"]),
                       "plain_sweeps_between_extra_proposals": sched["extra_between"],
                       "tolerance_m": tol,
                       "plain_ms": pm, "speedup_vs_plain": pm / lm,
                       "plain_iterations": plain[0][1], "learned_iterations": learn[0][1],
                       "converged": all(p[2] for p in plain + learn),
                       "mass_ledger_exact": all(p[3] for p in plain + learn)},
            "gpu_launches": learn[0][4], "clocks": clocks.summary()}


def repose_summary(seeds=(1, 2, 3, 4, 5, 6, 7, 8, 9), trials: int = 3):
    """The second metric for the default line: ms to repose, learned + plain
    sweeps against plain sweeps, on the bench surface (seed 1), on four
    held-out surfaces (seeds 2-5, never used to train the network or to tune
    the adaptive part of its schedule) and on the four surfaces that tuned it
    (seeds 6-9; 6 and 7 have long run-outs), median of ``trials`` runs each."""
    import math
    sub = argparse.Namespace(steps=trials, warmup=1)
    per = []
    for seed in seeds:
        r = run_repose(sub, seed=seed)["config"]
        per.append({"seed": seed, "plain_ms": r["plain_ms"],
                    "learned_ms": r["plain_ms"] / r["speedup_vs_plain"],
                    "speedup": r["speedup_vs_plain"], "plain_sweeps": r["plain_iterations"],
                    "learned_sweeps": r["learned_iterations"], "converged": r["converged"],
                    "mass_ledger_exact": r["mass_ledger_exact"]})
    held = [p["speedup"] for p in per if 2 <= p["seed"] <= 5]
    return {"metric": "ms to repose at 701^2 after the cut, learned proposal + plain sweeps vs "
                      "plain sweeps (35 deg, eps 1e-4)",
            "bench_surface": per[0], "held_out": [p for p in per if 2 <= p["seed"] <= 5],
            "tuning_surfaces": [p for p in per if p["seed"] >= 6],
            "held_out_geomean_speedup": math.exp(sum(math.log(x) for x in held) / len(held))
            if held else None,
            "all_geomean_speedup": math.exp(sum(math.log(p["speedup"]) for p in per) / len(per))}


# ---------------------------------------------------------------------------
# CPU baseline (oracle port, NumPy, 1 core)
# ---------------------------------------------------------------------------
def path_oracle(cfg, mat):
    """The CPU oracle of the whole plain step (FP64, NumPy): entrainment,
    Mobile V2, yield + labelling + classification, gated residual frontier."""
    from oracle.path import PathOracle, PathOracleConfig
    return PathOracle(cfg["b_eff"], cfg["z_base"], PathOracleConfig(
        dx=DX, density=mat.assumed_bulk_density_kg_m3, cohesion=mat.cohesion_proxy_pa,
        start_angle_deg=mat.start_angle_deg, stop_angle_deg=mat.stop_angle_deg,
        mobile_friction=mat.mobile_friction_coefficient))


def cpu_baseline(sample_steps: int = 6, warm_steps: int = 30, budget_s: float = 25.0):
    from oracle.path import entrain
    from soilb200 import workloads
    cfg = workloads.config1(N, seed=1, dx=DX)
    mat = material()
    sched = cut_schedule(cfg["cut"], warm_steps + sample_steps, pinned=False)
    oracle = path_oracle(cfg, mat)
    # warm-up cut with no flow (entrainment only) keeps the sample bounded
    for k in range(warm_steps):
        idx, tgt = sched[k]
        entrain(oracle.b, oracle.z, oracle.h, idx, tgt, oracle.w)
    t0 = time.perf_counter()
    subs = 0
    done = 0
    for k in range(warm_steps, warm_steps + sample_steps):
        subs += oracle.step(DT, *sched[k]).substeps
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return {"value": N * N * subs / el if el > 0 else 0.0, "unit": UNIT, "cores": 1,
            "kind": "port",
            "sample": f"{done} physics steps ({subs} substeps) of the config-1 plain path on "
                      f"the CPU oracle (NumPy FP64 restatement of the whole step: entrainment, "
                      f"MobileV2ReferenceSolver, yield/labelling/classification, gated residual "
                      f"frontier), after {warm_steps} cut steps; {el:.1f} s"}


def run_reference(args):
    """--impl reference: the CPU restatement of the path (the same step as the
    GPU arm: entrainment, Mobile V2, labelling + classification, gated
    residual frontier), on this host."""
    from soilb200 import workloads
    cfg = workloads.config1(N, seed=1, dx=DX)
    mat = material()
    total = args.warmup + args.steps
    sched = cut_schedule(cfg["cut"], total, pinned=False)
    oracle = path_oracle(cfg, mat)
    for k in range(args.warmup):
        oracle.step(DT, *sched[k])
    t0 = time.perf_counter()
    subs = 0
    for k in range(args.warmup, total):
        subs += oracle.step(DT, *sched[k]).substeps
    el = time.perf_counter() - t0
    value = N * N * subs / el if el > 0 else 0.0
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el * 1000.0 / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded config-1 value-noise pile + bucket cut)",
            "config": {"workload": "config1_plain_path_701", "grid": [N, N], "dx_m": DX,
                       "dt_s": DT, "steps_simulated_before_timing": args.warmup,
                       "step": "cut entrain -> Mobile V2 (all substeps) -> labelling -> "
                               "gated residual frontier"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"{args.steps} physics steps ({subs} substeps) after "
                                       f"{args.warmup} warm-up steps, NumPy oracle of the "
                                       f"whole step, 1 core"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--stages", action="store_true",
                    help="per-stage device times of the step graph (event nodes between stages)")
    ap.add_argument("--no-repose", action="store_true",
                    help="leave the learned-repose sub-object out of the default line")
    ap.add_argument("--net", default="fused", choices=["fused", "layers"],
                    help="repose workloads: the network's inference in one kernel or one "
                         "launch per layer")
    ap.add_argument("--workload", default="config1_plain_path_701",
                    choices=["config1_plain_path_701", "mobile_v2_4096", "batched_c2_512",
                             "repose_701", "site_c4_4096", "repose_site_4096"])
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.stages:
        os.environ["SOILB200_STAGE_EVENTS"] = "1"
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return
    if args.workload == "mobile_v2_4096":
        print(json.dumps(run_mobile_large(args)))
        return
    if args.workload == "batched_c2_512":
        print(json.dumps(run_batched_c2(args)))
        return
    if args.workload == "repose_701":
        print(json.dumps(run_repose(args)))
        return
    if args.workload == "repose_site_4096":
        from soilb200 import workloads
        site = workloads.site_after_cuts(workloads.config4(4096, seed=4, dx=DX))
        print(json.dumps(run_repose(args, surface=site, seed=4, label=(
            "synthetic (config-4 site, seed 4, after all 64 cuts ran their full travel)"))))
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    result = run_gpu(args, rank, world, local_rank)
    if rank == 0:
        if args.workload == "config1_plain_path_701" and not args.no_repose:
            result["repose"] = repose_summary()
        if not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline()
        print(json.dumps(result))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
