#!/usr/bin/env python
"""SIMPLE outer-iteration throughput (cell-iterations/s) of the B200 library.

Workload (one "step" = one steady SIMPLE outer iteration of the reference's generic_simple_v1):
  obstacle channel, 2.5 x 0.41 x 0.41 box at 200 x 70 x 70 hexes with interior nodes jittered
  by +-15 % of the local spacing (seed 0), the 0.1 x 0.1 x 0.41 obstacle block removed
  (970,480 cells, 2,876,926 internal faces), parabolic inlet Umax 0.45, fixed-p outlet, no-slip
  walls and obstacle, rho 1, mu 1e-3, relaxation U 0.7 / p 0.3, 2 non-orthogonal correctors,
  FP64 plain method, inner tolerances 1e-10 absolute (the reference defaults).
  The mesh and fields are synthetic (generated here); device working set ~1.5 GB > 126 MB L2.

Usage:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Prints one JSON line (rank 0).  N > 1 runs independent replicas (weak scaling) launched by
torchrun, one process per GPU; the timed region is bracketed by a barrier and device
synchronisation and reported as the maximum over ranks.
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

WORKLOAD = dict(nx=200, ny=70, nz=70, jitter=0.15, seed=0, obstacle=True)
PARAMS = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, n_nonorth_corr=2)
KERNEL_FAMILY = 7  # ANB_KF_PCG_SPMV: the dominant kernel of the step (see profiles/)
# DRAM bytes (read + write) per k_pcg_pq launch on this workload: mean of 3 launches of
#   ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum --clock-control none
#       -k k_pcg_pq -s 30 -c 3 python bench.py --steps 2 --warmup 3 --no-cpu
# (93.10 MB read + 3.44 MB write; profiles/k_pcg_pq_obstacle1m.md)
PCG_SPMV_TRAFFIC_BYTES = 96.53e6
FAMILY_NAMES = {1: "k_lsq_grad", 2: "k_momentum", 3: "k_pressure_rc", 4: "k_nonorth_rhs", 5: "k_flux_final",
                6: "k_bicg_v/k_bicg_t", 7: "k_pcg_pq"}


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock / throttle-reason samples during the timed region: NVML reads every 20 ms (read-only
    queries), else nvidia-smi every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows: list[list[str]] = []
        self._stop = threading.Event()
        self._nvml = self._nvml_handle()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _nvml_handle(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            bus = None
            try:
                import torch

                if torch.cuda.is_available():
                    p = torch.cuda.get_device_properties(self.device)
                    bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            except Exception:
                bus = None
            h = (pynvml.nvmlDeviceGetHandleByPciBusId(bus) if bus else pynvml.nvmlDeviceGetHandleByIndex(self.device))
            return pynvml, h
        except Exception:
            return None

    def _sample_nvml(self):
        nv, h = self._nvml
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        self.rows.append([str(self.device), str(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                          str(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)),
                          str(nv.nvmlDeviceGetPowerUsage(h) / 1000.0), hex(r)]
                         + ["Active" if r & b else "Not Active" for b in bits])

    def _run(self):
        while not self._stop.is_set():
            try:
                if self._nvml is not None:
                    self._sample_nvml()
                else:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5)
                    for line in out.stdout.strip().splitlines():
                        self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.02 if self._nvml is not None else 0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self) -> dict:
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4)
                          if r[5 + k].strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def max_over_ranks(values: list[float], dist=None, device: str = "cpu") -> list[float]:
    """Element-wise maximum over all ranks (the timed region is the slowest rank's)."""
    if dist is None:
        return list(values)
    import torch

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def replica_throughput(world: int, cells: int, steps: int, t_max: float) -> float:
    """Whole-job cell-iterations/s of `world` independent replicas (weak scaling)."""
    return world * cells * steps / t_max


def make_case():
    from tests.cases import channel, initial_state

    m, bc, _ = channel(**WORKLOAD)
    return m, bc, initial_state(m, bc)


def run_ours(args, rank: int, world: int, local_rank: int) -> dict | None:
    import anabasis_b200 as anb

    anb.lib()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as td

        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
        dist = td
    m, bc, (u0, v0, w0, p0) = make_case()
    C = m.n_cells
    s = anb.Solver(m, anb.default_params(device=local_rank, **PARAMS))
    s.set_bc(bc)
    s.set_state(u0, v0, w0, p0)
    lib = anb.lib()
    # warm-up (includes the one-time AMG structure set-up)
    s.iterate(args.warmup)
    lib.anb_profile_select(s._h, KERNEL_FAMILY)
    if dist:
        dist.barrier()
    launches0 = lib.anb_launch_count()
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        rc, st = s.iterate(args.steps)
        wall = time.perf_counter() - t0
    launches = lib.anb_launch_count() - launches0
    dev_seconds = float(sum(x["iter_seconds"] for x in st))
    n_l = ct_ll()
    secs = np.zeros(1)
    byts = np.zeros(1)
    lib.anb_profile_read(s._h, n_l, anb._d(secs), anb._d(byts))
    # end-to-end through the public API: host arrays in, one SIMPLE step, host arrays out
    g = s.get_state()
    e2e_steps = max(1, min(args.steps, 5))
    te = time.perf_counter()
    for _ in range(e2e_steps):
        s.set_state(g["u"], g["v"], g["w"], g["p"])
        s.iterate(1)
        g = s.get_state(with_phi=False)
    e2e_wall = time.perf_counter() - te
    t_max, e2e_wall = max_over_ranks([dev_seconds, e2e_wall], dist, f"cuda:{local_rank}")
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    achieved = (byts[0] / secs[0] / 1e9) if secs[0] > 0 else None
    value = replica_throughput(world, C, args.steps, t_max)
    cpu = cpu_baseline(m, bc, (u0, v0, w0, p0)) if world == 1 and not args.no_cpu else None
    out = {
        "metric": "SIMPLE cell-iters/s",
        "value": value,
        "unit": "cell-iters/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "obstacle channel 200x70x70 jittered hex (970480 cells), FP64 SIMPLE, "
                               "2 non-orthogonal correctors, inner tol 1e-10",
                   "cells": C, "internal_faces": m.n_internal, "parallelism": f"replicas{world}",
                   "l2": "working set > L2 (no flush needed)", "wall_seconds_timed": wall},
        "e2e": {"value": replica_throughput(world, C, e2e_steps, e2e_wall), "unit": "cell-iters/s",
                "h2d_bytes_per_step": 4 * 8 * C, "d2h_bytes_per_step": 4 * 8 * C},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": FAMILY_NAMES[KERNEL_FAMILY], "achieved": achieved,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "launches": int(n_l.value), "algorithmic_bytes": byts[0] / max(int(n_l.value), 1),
                     "traffic": PCG_SPMV_TRAFFIC_BYTES if KERNEL_FAMILY == 7 else None},
        "inner": {"bicgstab_last": [st[-1]["its_u"], st[-1]["its_v"], st[-1]["its_w"]],
                  "pcg_total_last": st[-1]["its_p_total"], "mass_res_last": st[-1]["mass_res"]},
        "clocks": clk.summary(),
    }
    if cpu:
        out["cpu_baseline"] = cpu
    return out


def ct_ll():
    import ctypes

    return ctypes.c_longlong(0)


def cpu_baseline(m, bc, state, steps: int = 1) -> dict:
    """Oracle port (C++/OpenMP, Jacobi-PCG) on the same mesh: one SIMPLE step, all host threads."""
    import oracle

    nthreads = os.cpu_count() or 1
    o = oracle.Oracle(m.topology())
    o.set_bc(bc)
    prm = oracle.params(n_threads=nthreads, **PARAMS)
    t0 = time.perf_counter()
    o.run(prm, steps, *state)
    dt = time.perf_counter() - t0
    return {"value": m.n_cells * steps / dt, "unit": "cell-iters/s", "cores": nthreads, "kind": "port",
            "sample": f"{steps} SIMPLE step(s) of the same 970480-cell workload from the initial state "
                      f"({dt:.1f} s)"}


def run_reference(args, rank: int) -> dict | None:
    if rank != 0:
        return None
    m, bc, state = make_case()
    steps = max(1, min(args.steps, 3))
    warm = 1 if args.warmup > 0 else 0
    import oracle

    nthreads = os.cpu_count() or 1
    o = oracle.Oracle(m.topology())
    o.set_bc(bc)
    prm = oracle.params(n_threads=nthreads, **PARAMS)
    s, _ = o.run(prm, warm, *state) if warm else ({"u": state[0], "v": state[1], "w": state[2], "p": state[3]}, None)
    t0 = time.perf_counter()
    o.run(prm, steps, s["u"], s["v"], s["w"], s["p"])
    dt = time.perf_counter() - t0
    v = m.n_cells * steps / dt
    return {
        "impl": "reference", "metric": "SIMPLE cell-iters/s", "value": v, "unit": "cell-iters/s", "n_gpus": 0,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "obstacle channel 200x70x70 jittered hex (970480 cells), FP64 SIMPLE, "
                               "2 non-orthogonal correctors, inner tol 1e-10", "cells": m.n_cells},
        "cpu_baseline": {"value": v, "unit": "cell-iters/s", "cores": nthreads, "kind": "port",
                         "sample": f"{steps} SIMPLE step(s) after {warm} warm-up step(s); the reference's HYPRE "
                                   f"path cannot be built (no HYPRE/MPI), the oracle port stands in"},
        "e2e": {"value": v, "unit": "cell-iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
    else:
        out = run_ours(args, rank, world, local_rank)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
