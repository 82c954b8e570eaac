#!/usr/bin/env python
"""SIMPLE outer-iteration throughput (cell-iterations/s) of the B200 library.

Workload (one "step" = one steady SIMPLE outer iteration of the reference's generic_simple_v1):
  obstacle channel, 2.5 x 0.41 x 0.41 box at 200 x 70 x 70 hexes with interior nodes jittered
  by +-15 % of the local spacing (seed 0), the 0.1 x 0.1 x 0.41 obstacle block removed
  (970,480 cells, 2,876,926 internal faces), parabolic inlet Umax 0.45, fixed-p outlet, no-slip
  walls and obstacle, rho 1, mu 1e-3, relaxation U 0.7 / p 0.3, 2 non-orthogonal correctors,
  FP64 plain method, inner tolerances 1e-10 absolute (the reference defaults).
  The mesh and fields are synthetic (generated here); device working set ~1.9 GB > 126 MB L2.

Reference arm (--impl reference): the CPU oracle (oracle/, a C++/OpenMP restatement of the
reference's SIMPLE iteration with an aggregation-AMG PCG for the pressure in place of HYPRE's
BoomerAMG-PCG; the reference's own HYPRE path cannot be built without HYPRE and MPI)
on the box's host cores, same case built by the oracle alone (no product library in the process),
same warm-up and timed step indices as the library arm.

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
KERNEL_FAMILY = 7  # ANB_KF_PCG_SPMV: the PCG SpMV, a level-0 SELL kernel launched outside the V-cycle graph
# DRAM bytes (read + write) per k_pcg_pq launch on this workload, from one launch of
#   ANB_NO_LOOP_GRAPH=1 ncu --set full --clock-control none -k regex:"^k_pcg_pq$" -s 30 -c 1
#       python bench.py --steps 2 --warmup 3 --no-cpu
# (93.07 MB read + 6.14 MB write)
PCG_SPMV_TRAFFIC_BYTES = 99.21e6
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


def bench_config(world: int) -> dict:
    """The `config` of both arms' JSON lines (the same workload, so the same dict)."""
    return {"workload": "obstacle channel 200x70x70 jittered hex (970480 cells), FP64 SIMPLE, "
                        "2 non-orthogonal correctors, inner tol 1e-10",
            "cells": 970480, "internal_faces": 2876926, "parallelism": f"replicas{world}",
            "l2": "working set > L2 (no flush needed)"}


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
    # the state the timed steps start from, kept on the host for the end-to-end replay below
    g0 = s.get_state(with_phi=False)
    if dist:
        dist.barrier()
    launches0 = lib.anb_launch_count()
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        rc, st = s.iterate(args.steps)
        wall = time.perf_counter() - t0
    launches = lib.anb_launch_count() - launches0
    dev_seconds = float(sum(x["iter_seconds"] for x in st))
    # The roofline kernel is timed with a CUDA event pair around each of its launches over the K
    # steps that follow the timed region (same workload, same launches).  Inside the timed region
    # the events would keep the pressure solves on the host loop (a graph's while body cannot
    # record events) and add ~0.4 ms per step at this size.
    lib.anb_profile_select(s._h, KERNEL_FAMILY)
    s.iterate(args.steps)
    n_l = ct_ll()
    secs = np.zeros(1)
    byts = np.zeros(1)
    lib.anb_profile_read(s._h, n_l, anb._d(secs), anb._d(byts))
    lib.anb_profile_select(s._h, 0)
    # End to end through the public API: the same K steps (W+1 .. W+K) replayed from the state
    # saved after the warm-up, every step with host arrays in (anb_set_state), one SIMPLE step and
    # host arrays out (anb_get_state).  A step depends only on u, v, w, p (the AMG values are
    # refreshed every step), so the replay repeats the timed steps bit for bit; the per-step
    # continuity residuals are compared to show it.
    g = {k: (a.copy() if a is not None else None) for k, a in g0.items()}
    e2e_steps = args.steps
    e2e_st = []
    te = time.perf_counter()
    for _ in range(e2e_steps):
        s.set_state(g["u"], g["v"], g["w"], g["p"])
        e2e_st += s.iterate(1)[1]
        g = s.get_state(with_phi=False, out=g)  # the caller's arrays, refilled every step
    e2e_wall = time.perf_counter() - te
    replay_same = [x["mass_res"] for x in e2e_st] == [x["mass_res"] for x in st]
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
        "config": bench_config(world),
        "wall_seconds_timed": wall,
        "e2e": {"value": replica_throughput(world, C, e2e_steps, e2e_wall), "unit": "cell-iters/s",
                "h2d_bytes_per_step": 4 * 8 * C, "d2h_bytes_per_step": 4 * 8 * C,
                "steps": f"the timed steps {args.warmup + 1}-{args.warmup + args.steps} replayed from the "
                         "state after warm-up", "replay_identical": replay_same},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": FAMILY_NAMES[KERNEL_FAMILY], "achieved": achieved,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "launches": int(n_l.value), "algorithmic_bytes": byts[0] / max(int(n_l.value), 1),
                     "window": f"CUDA events around each launch, the {args.steps} steps after the timed region",
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
    """Oracle port (C++/OpenMP, aggregation-AMG PCG for the pressure as the reference's BoomerAMG-PCG,
    Jacobi-BiCGSTAB for the momentum) on the same mesh: one SIMPLE step, all host threads."""
    import oracle

    nthreads = os.cpu_count() or 1
    o = oracle.Oracle(m.topology())
    o.set_bc(bc)
    prm = oracle.params(n_threads=nthreads, p_use_amg=1, **PARAMS)
    t0 = time.perf_counter()
    o.run(prm, steps, *state)
    dt = time.perf_counter() - t0
    return {"value": m.n_cells * steps / dt, "unit": "cell-iters/s", "cores": nthreads, "kind": "port",
            "sample": f"{steps} SIMPLE step(s) of the same 970480-cell workload from the initial state "
                      f"({dt:.1f} s)"}


def run_reference(args, rank: int, world: int) -> dict | None:
    """The oracle port on the host cores: the case is built by the oracle alone (its own channel
    generator and boundary evaluation, pinned bit for bit to the library's and the reference's),
    then the same warm-up steps and the same timed steps as the library arm, all host threads."""
    if rank != 0:
        return None
    import oracle

    o, bc, state = oracle.channel_case(**WORKLOAD)
    nthreads = os.cpu_count() or 1
    prm = oracle.params(n_threads=nthreads, tol_mass=0.0, tol_vel=0.0, p_use_amg=1, **PARAMS)  # no early stop
    s = {"u": state[0], "v": state[1], "w": state[2], "p": state[3]}
    if args.warmup > 0:
        s, _ = o.run(prm, args.warmup, *state)
    t0 = time.perf_counter()
    _, st = o.run(prm, args.steps, s["u"], s["v"], s["w"], s["p"])
    dt = time.perf_counter() - t0
    assert len(st) == args.steps
    v = o.n_cells * args.steps / dt
    return {
        "impl": "reference", "metric": "SIMPLE cell-iters/s", "value": v, "unit": "cell-iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(world),
        "cpu_baseline": {"value": v, "unit": "cell-iters/s", "cores": nthreads, "kind": "port",
                         "sample": f"steps {args.warmup + 1}-{args.warmup + args.steps} of the workload (the "
                                   f"library arm's timed steps) after {args.warmup} warm-up steps; the "
                                   f"reference's HYPRE path cannot be built (no HYPRE/MPI), the oracle port "
                                   f"(AMG-PCG / Jacobi-BiCGSTAB) stands in"},
        "e2e": {"value": v, "unit": "cell-iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_variants(args) -> dict:
    """Design switches on the benchmark workload (FP64, steps 5-14 after 4 warm-up steps, CUDA
    events): the flux correction's row form against its face-parallel form (ANB_FLUX_FORM), and
    the momentum BiCGSTAB's Jacobi preconditioner against the momentum AMG (mom_amg)."""
    import ctypes

    import anabasis_b200 as anb

    m, bc, state = make_case()
    lib = anb.lib()

    def timed(family, env, **prm):
        old = {k: os.environ.get(k) for k in env}
        os.environ.update(env)
        try:
            s = anb.Solver(m, anb.default_params(**PARAMS, **prm))
            s.set_bc(bc)
            s.set_state(*state)
            s.iterate(4)
            lib.anb_profile_select(s._h, family)
            _, st = s.iterate(10)
            n = ctypes.c_longlong(0)
            sec, by = np.zeros(1), np.zeros(1)
            lib.anb_profile_read(s._h, ctypes.byref(n), sec.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 by.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            s.close()
        finally:
            for k, v in old.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        return dict(step_ms=1e3 * sum(x["iter_seconds"] for x in st) / len(st), family_seconds=float(sec[0]),
                    family_launches=int(n.value), algo_gbs=float(by[0] / sec[0] / 1e9) if sec[0] > 0 else None,
                    bicg_its=[st[-1]["its_u"], st[-1]["its_v"], st[-1]["its_w"]])

    out = {"metric": "design switches, FP64 SIMPLE on the benchmark workload", "unit": "ms per step",
           "config": bench_config(1)}
    for form in ("row", "face"):
        r = timed(5, {"ANB_FLUX_FORM": form})
        r["us_per_flux_call"] = 1e6 * r["family_seconds"] / max(r["family_launches"], 1)
        out[f"flux_{form}"] = r
    for amg in (0, 1):
        r = timed(13, {}, mom_amg=amg)
        r["momentum_ms_per_step"] = 1e3 * r["family_seconds"] / 10
        out[f"momentum_{'amg' if amg else 'jacobi'}"] = r
    return out


def run_cpu_baselines(args) -> dict:
    """The oracle port (C++/OpenMP, all host threads, AMG-PCG / Jacobi-BiCGSTAB at the reference's
    1e-10 tolerances) on configurations 1-3, each case built by the oracle alone: config 1 (16,000
    hexes) for 300 steps from the initial state, config 2 (970,480 cells) and config 3 (3,977,792
    cells) on bounded samples of steps 1..k.  No product library is loaded."""
    import oracle

    nthreads = os.cpu_count() or 1
    rows = []
    for name, kw, steps in (("config 1: channel 40x20x20 (16000 hex)", dict(nx=40, ny=20, nz=20), 300),
                            ("config 2: obstacle channel 200x70x70 jittered (seed 0)", WORKLOAD, 3),
                            ("config 3: obstacle channel 320x112x112 jittered (seed 1)",
                             dict(nx=320, ny=112, nz=112, jitter=0.15, seed=1, obstacle=True), 2)):
        t0 = time.perf_counter()
        o, bc, state = oracle.channel_case(**kw)
        setup = time.perf_counter() - t0
        prm = oracle.params(n_threads=nthreads, tol_mass=0.0, tol_vel=0.0, p_use_amg=1, **PARAMS)
        t0 = time.perf_counter()
        _, st = o.run(prm, steps, *state)
        dt = time.perf_counter() - t0
        rows.append({"case": name, "cells": o.n_cells, "steps": len(st), "seconds": dt,
                     "cell_iters_per_s": o.n_cells * len(st) / dt, "ms_per_step": 1e3 * dt / len(st),
                     "setup_s": setup, "mass_res_last": st[-1]["mass_res"],
                     "pcg_its_last_step": st[-1]["its_p_total"]})
        del o
    return {"metric": "SIMPLE cell-iters/s, CPU oracle port", "unit": "cell-iters/s", "cores": nthreads,
            "kind": "port", "data": "synthetic", "rows": rows}


def _peak_device_bytes(device: int = 0) -> int | None:
    """Device memory in use (NVML, read-only query).  The library allocates every buffer of a
    phase up front and keeps it until the context is destroyed, so the figure taken at the end of
    a phase is that phase's high-water mark."""
    try:
        import pynvml

        pynvml.nvmlInit()
        return int(pynvml.nvmlDeviceGetMemoryInfo(pynvml.nvmlDeviceGetHandleByIndex(device)).used)
    except Exception:
        return None


def _converge(m, bc, precision, max_steps, tol_mass, tol_vel, init=None, **extra):
    """SIMPLE from the initial state until massRes < tol_mass and max du < tol_vel."""
    import anabasis_b200 as anb
    from tests.cases import initial_state

    s = anb.Solver(m, anb.default_params(precision=precision, **PARAMS, **extra))
    s.set_bc(bc)
    s.set_state(*(init if init is not None else initial_state(m, bc)))
    _, st = s.iterate(max_steps, tol_mass, tol_vel)
    names = m.topology()["patch_names"]
    f = s.patch_force(names.index("patch_3_0"), -1)
    return s, st, f


def _field_errors(a: dict, b: dict) -> dict:
    us = max(float(np.abs(a[k]).max()) for k in "uvw")
    e = {k: float(np.abs(a[k] - b[k]).max()) / us for k in "uvw"}
    e["p"] = float(np.abs(a["p"] - b["p"]).max()) / max(float(np.abs(a["p"]).max()), 1e-300)
    return e


MIXED_VARIANTS = {
    # the reference's plain method: every solve to 1e-10 absolute (velTol, pTol; relTol 0)
    "fp64": dict(precision=0),
    # FP32 inner solves, each linear solve refined in FP64 to the plain method's tolerance
    "mixed_strict": dict(precision=1),
    # one FP32 inner solve per system and outer step; the SIMPLE iteration is the refinement loop
    "mixed_outer_1e-2": dict(precision=1, mixed_refine=1, mixed_inner_rtol=1e-2),
    "mixed_outer_1e-3": dict(precision=1, mixed_refine=1, mixed_inner_rtol=1e-3),
    # FP64 with the reference's own relative-tolerance options (velRelTol, pRelTol) at 1e-3: the
    # last pressure pass of a step stays absolute (main.cu's final-pass rule); separates the effect
    # of inexact inner solves from that of the precision
    "fp64_reltol_1e-3": dict(precision=0, vel_rel_tol=1e-3, p_rel_tol=1e-3),
}


def run_mixed4m(args) -> dict:
    """Config 3: 320x112x112 jittered obstacle channel (seed 1).  Each variant runs from the
    initial state to massRes < 1e-6 and max relative velocity change < tol_vel; time ratio to the
    plain FP64 run and the field and force errors against it."""
    from tests.cases import channel

    m, bc, _ = channel(nx=320, ny=112, nz=112, jitter=0.15, seed=1, obstacle=True)
    runs = {}
    for name, kw in MIXED_VARIANTS.items():
        kw = dict(kw)
        prec = kw.pop("precision")
        t0 = time.perf_counter()
        s, st, f = _converge(m, bc, prec, args.max_steps, 1e-6, args.tol_vel, **kw)
        wall = time.perf_counter() - t0
        runs[name] = dict(steps=len(st), device_s=float(sum(x["iter_seconds"] for x in st)), wall_s=wall,
                          mass_res=st[-1]["mass_res"], du=max(st[-1]["du_rel"], st[-1]["dv_rel"], st[-1]["dw_rel"]),
                          pcg_its_per_step=float(np.mean([x["its_p_total"] for x in st])),
                          bicg_its_per_step=float(np.mean([max(x["its_u"], x["its_v"], x["its_w"]) for x in st])),
                          F=f["F"], state=s.get_state(with_phi=False), peak_bytes=_peak_device_bytes())
        s.close()
    a = runs["fp64"]
    F = np.array(a["F"])
    for name, r in runs.items():
        r["time_ratio_vs_fp64"] = a["device_s"] / r["device_s"]
        r["force_rel_error"] = float(np.abs(np.array(r["F"]) - F).max() / np.abs(F).max())
        r["field_rel_error"] = _field_errors(a["state"], r["state"])
    for r in runs.values():
        r.pop("state")
    b = runs["mixed_strict"]
    return {"metric": "time to converged solution (massRes<1e-6), FP64 / mixed precision",
            "value": b["time_ratio_vs_fp64"], "unit": "x", "higher_is_better": True, "n_gpus": 1,
            "dtype": "f64 vs f32-inner/f64-outer", "data": "synthetic",
            "config": {"workload": "obstacle channel 320x112x112 jittered hex (seed 1), 2 non-orthogonal correctors",
                       "cells": m.n_cells, "tol_mass": 1e-6, "tol_vel": args.tol_vel},
            "runs": runs}


def run_adjoint1m(args) -> dict:
    """Config 4: 1M-cell obstacle channel; converged FP64 forward (SIMPLE, then Newton to a residual
    two-norm of 1e-13), adjoint gradient of the x-force on the obstacle w.r.t. every inlet-face
    velocity and mu, checked against the tangent-linear model and central differences (h = 1e-6
    along unit random directions, seed 42, each perturbed state Newton-converged)."""
    from tests.cases import channel

    m, bc, _ = channel(**WORKLOAD)
    t0 = time.perf_counter()
    s, st, _ = _converge(m, bc, 0, args.max_steps, 1e-10, 1e-8)
    fwd_dev = float(sum(x["iter_seconds"] for x in st))
    fwd_wall = time.perf_counter() - t0
    newton = s.newton_solve(max_newton=10, tol=1e-13)
    names = m.topology()["patch_names"]
    k_in, k_obs = names.index("patch_1_0"), names.index("patch_3_0")
    direction = (1.0, 0.0, 0.0)
    g, gmu, J, ainfo = s.adjoint_force_grad(k_obs, direction)
    t = m.topology()
    F = m.n_faces
    mask = np.zeros(F, bool)
    s0, n = int(t["patch_start"][k_in]), int(t["patch_size"][k_in])
    mask[s0:s0 + n] = True
    mask = np.tile(mask, 3)
    base = s.get_state(with_phi=False)
    rng = np.random.default_rng(42)
    checks = []
    h = 1e-6
    for i in range(args.dirs):
        d = np.where(mask, rng.standard_normal(3 * F), 0.0)
        dmu = rng.standard_normal()
        nrm = np.sqrt(d @ d + dmu * dmu)
        d, dmu = d / nrm, dmu / nrm
        adj = float(g @ d + gmu * dmu)
        rec = {"adjoint": adj}
        if i < args.tl_dirs:
            tl, tinfo = s.tangent_linear(k_obs, direction, d, dmu)
            rec.update(tangent_linear=tl, tl_rel_err=abs(tl - adj) / abs(adj), tl_seconds=tinfo["seconds"])
        Jpm = []
        for sg in (1.0, -1.0):
            s.set_state(base["u"], base["v"], base["w"], base["p"])
            b = dict(bc)
            for q, k in enumerate("uvw"):
                b[k] = bc[k] + sg * h * d[q * F:(q + 1) * F]
            s.set_bc(b)
            s.set_viscosity(PARAMS["mu"] + sg * h * dmu)
            s.newton_solve(max_newton=10, tol=1e-13)
            Jpm.append(s.force_objective(k_obs, direction)[0])
        fd = (Jpm[0] - Jpm[1]) / (2 * h)
        rec.update(fd=fd, fd_rel_err=abs(fd - adj) / abs(adj))
        checks.append(rec)
        s.set_state(base["u"], base["v"], base["w"], base["p"])
        s.set_bc(bc)
        s.set_viscosity(PARAMS["mu"])
    return {"metric": "adjoint cost / forward cost", "value": ainfo["seconds"] / fwd_dev, "unit": "x",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "obstacle channel 200x70x70 jittered hex (970480 cells), J = x-force on the "
                                   "obstacle, parameters 3 x inlet-face velocities + mu", "cells": m.n_cells,
                       "inlet_faces": int(n), "fd_step": h, "directions": args.dirs},
            "forward": {"simple_steps": len(st), "device_s": fwd_dev, "wall_s": fwd_wall, "newton": newton},
            "adjoint": ainfo, "J": J, "dJ_dmu": gmu,
            "max_fd_rel_err": max(c["fd_rel_err"] for c in checks) if checks else None,
            "max_tl_rel_err": max((c["tl_rel_err"] for c in checks if "tl_rel_err" in c), default=None),
            "checks": checks}


def run_tets16m(args) -> dict:
    """Config 5: 463x76x76 jittered hexes (seed 2) split into 6 tets, obstacle removed before the
    split (~16M cells).  Mixed-precision forward for --steps SIMPLE steps from the initial state,
    the same steps in FP64 as the accuracy reference, then the adjoint gradient of the obstacle force at
    the FP64 state restored from a host checkpoint of (U, p) in a fresh FP64 context; peak device
    memory of each phase."""
    import anabasis_b200 as anb
    from tests.cases import channel

    import ctypes
    import tempfile

    t0 = time.perf_counter()
    m, bc, case_dir = channel(nx=463, ny=76, nz=76, jitter=0.15, seed=2, obstacle=True, tets=True)
    mesh_s = time.perf_counter() - t0
    out = {"metric": "mixed-precision SIMPLE cell-iters/s at 16M tets", "unit": "cell-iters/s", "n_gpus": 1,
           "higher_is_better": True, "data": "synthetic",
           "config": {"workload": "463x76x76 jittered hexes split into 6 tets, obstacle channel", "cells": m.n_cells,
                      "steps": args.steps}, "mesh_build_s": mesh_s}
    # set-up as the drop-in program does it: the ASCII polyMesh read back (parallel parse, host
    # geometry for the boundary evaluation), then the library context (device geometry, LSQ
    # moments, layout, upload)
    with tempfile.TemporaryDirectory(prefix="anb_pm_") as d:
        t0 = time.perf_counter()
        m.write(d)
        write_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        m_read = anb.HostMesh.read(d)
        read_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        s = anb.Solver(m_read, anb.default_params(**PARAMS))
        create_s = time.perf_counter() - t0
        t = np.zeros(10)
        anb.lib().anb_setup_times(s._h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        s.close()
        del m_read
    out["setup"] = {"polymesh_bytes_write_s": write_s, "read_polymesh_s": read_s, "anb_create_s": create_s,
                    "anb_create_phases_s": dict(zip(["copy_in_topology", "geometry_device", "layout", "upload"],
                                                    t[:4].tolist())),
                    "layout_parts_s": dict(zip(["adjacency", "lsq_moments_device", "rcm", "face_order_coeffs", "sell",
                                                "boundary_cells"], t[4:].tolist())),
                    "host_threads": os.cpu_count()}
    runs = {}
    for prec in (1, 0):
        t0 = time.perf_counter()
        s, st, f = _converge(m, bc, prec, args.steps, -1.0, -1.0)
        runs[prec] = dict(device_s=float(sum(x["iter_seconds"] for x in st[1:])), steps=len(st), F=f["F"],
                          setup_and_run_wall_s=time.perf_counter() - t0, peak_bytes=_peak_device_bytes(),
                          state=s.get_state(with_phi=False))
        s.close()
    out["value"] = m.n_cells * (runs[1]["steps"] - 1) / runs[1]["device_s"]
    out["fp64_cell_iters_per_s"] = m.n_cells * (runs[0]["steps"] - 1) / runs[0]["device_s"]
    F = np.array(runs[0]["F"])
    out["mixed_vs_fp64"] = {"force_rel_error": float(np.abs(np.array(runs[1]["F"]) - F).max() / np.abs(F).max()),
                            "field_rel_error": _field_errors(runs[0]["state"], runs[1]["state"])}
    ck = runs[0]["state"]
    os.environ.setdefault("ANB_ADJ_RTOL", "1e-8")  # 1e-10 stagnates on this tet mesh; 1e-8 is ample for 1e-5
    s = anb.Solver(m, anb.default_params(**PARAMS))
    s.set_bc(bc)
    s.set_state(ck["u"], ck["v"], ck["w"], ck["p"])
    names = m.topology()["patch_names"]
    _, res = s.steady_residual()
    g, gmu, J, ainfo = s.adjoint_force_grad(names.index("patch_3_0"), (1.0, 0.0, 0.0))
    out["adjoint"] = dict(ainfo, dJ_dmu=gmu, J=J, residual_norms=list(map(float, res)),
                          rtol=float(os.environ["ANB_ADJ_RTOL"]), peak_bytes=_peak_device_bytes())
    for k in (0, 1):
        runs[k].pop("state")
    out["mixed"], out["fp64"] = runs[1], runs[0]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--config", default="obstacle1m",
                    choices=["obstacle1m", "mixed4m", "adjoint1m", "tets16m", "cpu3", "variants"],
                    help="obstacle1m: the headline SIMPLE throughput line; the others are single-GPU studies "
                         "of the mixed-precision, adjoint and 16M-tet configurations")
    ap.add_argument("--max-steps", type=int, default=4000)
    ap.add_argument("--tol-vel", type=float, default=1e-6)
    ap.add_argument("--dirs", type=int, default=8, help="adjoint1m: finite-difference directions")
    ap.add_argument("--tl-dirs", type=int, default=4, help="adjoint1m: tangent-linear directions")
    args = ap.parse_args()
    if args.warmup < 3:  # both arms: at least 3 warm-up steps, the same steps timed
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    studies = {"mixed4m": run_mixed4m, "adjoint1m": run_adjoint1m, "tets16m": run_tets16m,
               "cpu3": run_cpu_baselines, "variants": run_variants}
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.config in studies:
        out = studies[args.config](args) if rank == 0 else None
    else:
        out = run_ours(args, rank, world, local_rank)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
