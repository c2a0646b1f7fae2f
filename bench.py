"""Benchmark of the D2Q9 solver step on B200.

Workload (one bench "step" = S lattice time steps of one case):
  free-surface culvert dam break scaled to 8192x2048 (the precision-sweep case),
  FP32 populations + FP64 mass/fill level, half-way walls, conservative free
  surface.  Working set ~1.2 GB, far above the 126 MB L2, so no L2 flush is
  needed between steps.

  value  MLUPS (million cell updates / s) over all ranks, inputs resident in
         HBM, device time from CUDA events on the engine's stream, max over ranks.
  e2e    the same metric through the C ABI with host buffers: per step
         flb_reset from pinned host geometry flags (H2D), S steps, and a read of
         density, velocity, fill level and flags into pinned host memory (D2H).

Multi-GPU: the path does not shard (one GPU per case), so --gpus N runs N
independent replicas, one per rank (weak scaling).

--impl reference times the CPU restatement of the reference step (the oracle,
OpenMP on the host cores) on a bounded sample of the same workload.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS, %HBM peak: FP32 vs FP16-store @L2<1e-3; batch cases/s; adjoint/fwd"
WORKLOAD = ("free-surface culvert dam break 8192x2048 (precision-sweep geometry), tau 0.55, g_y -5e-5, FP32 "
            "populations + FP64 mass, half-way walls, conservative free surface, velocity limiter 0.25")
U_MAX = 0.25  # keeps the surge front stable (plain BGK at tau 0.55 diverges near Mach 0.6)


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fp:
            d = json.load(fp)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.lines: list[str] = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes_sc(counts: dict, N: int) -> float:
    """Stream-collide pass, free-surface FP32 build, over the super-tiles it
    visits: every visited cell reads its flag (1 B); every fluid/interface
    cell loads and stores its 9 populations (72 B), writes density and
    velocity (12 B) and reads its wall-neighbour mask (1 B); interface cells
    also read their FP64 mass (8 B) and rewrite their flag (1 B).  Gas cells
    outside the visited super-tiles are not counted (they are not touched)."""
    active = counts["fluid"] + counts["interface"]
    return active * 86.0 + counts["interface"] * 9.0


def run_ours(args, rank, local_rank, world):
    import torch

    from flowlb_b200 import cases
    from flowlb_b200 import engine as E

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    case = cases.dam_break(4)
    N = case.cells
    S = args.lattice_steps
    solver = E.Solver(case.flags, free_surface=True, precision=32, mass_precision=64, tau=case.tau, fy=case.fy,
                      bounce_back=E.BB_HALFWAY, fs_mode=E.FS_CONSERVATIVE, device=local_rank, u_max=U_MAX)
    stream = torch.cuda.ExternalStream(solver.stream, device=local_rank)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing -------------------------------------------
    for _ in range(args.warmup):
        solver.step(S)
    solver.sync()
    counts0 = solver.cell_counts()
    launches0 = solver.launches
    barrier()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            solver.step(S)
        stop.record(stream)
        stop.synchronize()
    barrier()
    elapsed_ms = start.elapsed_time(stop)
    launches = solver.launches - launches0
    counts1 = solver.cell_counts()
    t_max = elapsed_ms
    if dist is not None:
        tt = torch.tensor([elapsed_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    value = world * N * S * args.steps / (t_max * 1e-3) / 1e6

    # ---- dominant-kernel roofline: per-pass CUDA-event timing -------------
    prof_steps = max(20, S // 4)
    ca = solver.cell_counts()
    passes = solver.profile_steps(prof_steps)
    cb = solver.cell_counts()
    counts_avg = {k: 0.5 * (ca[k] + cb[k]) for k in ca}
    sc_ms = passes["stream_collide"] / prof_steps
    sc_bytes = algorithmic_bytes_sc(counts_avg, N)
    peak, peak_kind = measured_peaks()
    achieved = sc_bytes / (sc_ms * 1e-3) / 1e9
    shares = {k: v / max(1e-12, sum(passes.values())) for k, v in passes.items()}

    # ---- end to end through the C ABI with host buffers -------------------
    host_flags = torch.from_numpy(np.ascontiguousarray(case.flags.ravel())).pin_memory()
    out_rho = torch.empty(N, dtype=torch.float32).pin_memory()
    out_u = torch.empty(2 * N, dtype=torch.float32).pin_memory()
    out_phi = torch.empty(N, dtype=torch.float64).pin_memory()
    out_flags = torch.empty(N, dtype=torch.uint8).pin_memory()
    L = E.load_library()

    def e2e_step():
        solver._check(L.flb_reset(solver.handle, host_flags.data_ptr()))
        solver.step(S)
        for fid, buf in ((E.FIELD_RHO, out_rho), (E.FIELD_U, out_u), (E.FIELD_PHI, out_phi),
                         (E.FIELD_FLAGS, out_flags)):
            solver._check(L.flb_read_field(solver.handle, fid, buf.data_ptr(), 0))

    e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    barrier()
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        tt = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e_value = world * N * S * args.steps / e2e_s / 1e6

    # ---- side measurements on rank 0 (FP16 storage, single-phase probe) ---
    extra = {}
    if rank == 0 and not args.no_extra:
        extra = side_measurements(args, local_rank, E, cases, peak)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(case, args)

    if dist is not None:
        dist.barrier()
    solver.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nx": case.nx, "ny": case.ny, "cells": N,
                       "lattice_steps_per_step": S, "parallelism": f"replicas x{world}",
                       "l2": "working set ~1.2 GB > 126 MB L2; no flush needed",
                       "cells_by_type_at_start": counts0, "cells_by_type_at_end": counts1},
            "e2e": {"value": round(e2e_value, 1), "unit": "MLUPS", "h2d_bytes_per_step": int(N),
                    "d2h_bytes_per_step": int(N * (4 + 8 + 8 + 1))},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "k_stream_collide (free-surface FP32 build)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": None, "algorithmic_bytes_per_launch": int(sc_bytes),
                         "avg_launch_ms": round(sc_ms, 5), "pass_share": {k: round(v, 3) for k, v in shares.items()}},
            "clocks": clocks.summary(),
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        line.update(extra)
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def side_measurements(args, device, E, cases, peak):
    """FP16 scaled-deviation storage on the same workload, and the plain FP32
    single-phase step on an 8192x2048 grid (the >=80% HBM target)."""
    import torch

    out = {}
    c = cases.dam_break(4)
    S = args.lattice_steps
    s16 = E.Solver(c.flags, free_surface=True, precision=16, mass_precision=64, tau=c.tau, fy=c.fy,
                   bounce_back=E.BB_HALFWAY, fs_mode=E.FS_CONSERVATIVE, device=device, u_max=U_MAX)
    st = torch.cuda.ExternalStream(s16.stream, device=device)
    s16.step(S)
    s16.sync()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(max(2, args.steps // 2)):
        s16.step(S)
    b.record(st)
    b.synchronize()
    ms = a.elapsed_time(b)
    out["fp16s_same_workload"] = {"value": round(c.cells * S * max(2, args.steps // 2) / (ms * 1e-3) / 1e6, 1),
                                  "unit": "MLUPS"}
    s16.close()
    p = cases.hbm_probe(8192, 2048)
    for prec, key, bytes_per in ((32, "single_phase_fp32_8192x2048", 74.0), (16, "single_phase_fp16s_8192x2048",
                                                                               38.0)):
        s = E.Solver(p.flags, free_surface=False, precision=prec, tau=p.tau, fx=p.fx, bounce_back=E.BB_HALFWAY,
                     device=device)
        st = torch.cuda.ExternalStream(s.stream, device=device)
        s.step(50)
        s.sync()
        n = 400
        a.record(st)
        s.step(n)
        b.record(st)
        b.synchronize()
        ms = a.elapsed_time(b)
        cnt = s.cell_counts()
        fluid = cnt["fluid"]
        mlups = p.cells * n / (ms * 1e-3) / 1e6
        # bytes: flag of every cell + populations and wall mask of fluid cells
        gbs = (p.cells * 1.0 + fluid * (bytes_per - 1.0)) * n / (ms * 1e-3) / 1e9
        out[key] = {"value": round(mlups, 1), "unit": "MLUPS", "achieved_gbs": round(gbs, 1),
                    "frac_of_measured_hbm": round(gbs / peak, 4)}
        s.close()
    out["fp16s_speedup_single_phase"] = round(out["single_phase_fp16s_8192x2048"]["value"] /
                                              out["single_phase_fp32_8192x2048"]["value"], 3)
    return out


def cpu_baseline(case, args):
    """The oracle (C, OpenMP) on the host cores, same mode, bounded sample."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    o = O.Oracle(case.flags, O.OracleConfig(variant=O.F32, free_surface=True, bb=O.BB_HALFWAY,
                                            fs_mode=O.FS_CONSERVATIVE, tau=case.tau, fy=case.fy, threads=threads,
                                            u_max=U_MAX, arithmetic=O.ARITH_FUSED))
    o.step(1)
    n = args.cpu_steps
    t0 = time.perf_counter()
    o.step(n)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": round(case.cells * n / dt / 1e6, 2), "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{case.nx}x{case.ny} dam break, {n} time steps after the first, same storage and modes"}


def run_reference(args, rank, world):
    """CPU restatement of the reference step timed on the host cores."""
    if rank != 0:
        return
    from flowlb_b200 import cases
    from oracle import oracle as O

    case = cases.dam_break(4)
    threads = os.cpu_count() or 1
    o = O.Oracle(case.flags, O.OracleConfig(variant=O.F32, free_surface=True, bb=O.BB_HALFWAY,
                                            fs_mode=O.FS_CONSERVATIVE, tau=case.tau, fy=case.fy, threads=threads,
                                            u_max=U_MAX))
    S = args.ref_lattice_steps
    for _ in range(args.warmup):
        o.step(S)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(S)
    dt = time.perf_counter() - t0
    value = case.cells * S * args.steps / dt / 1e6
    sample = f"{case.nx}x{case.ny} dam break, {S} time steps per bench step"
    line = {"metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "nx": case.nx, "ny": case.ny, "cells": case.cells,
                       "lattice_steps_per_step": S, "parallelism": "host cores"},
            "cpu_baseline": {"value": round(value, 2), "unit": "MLUPS", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--lattice-steps", type=int, default=200, help="lattice time steps per bench step")
    ap.add_argument("--ref-lattice-steps", type=int, default=2)
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, local_rank, world = env_rank()
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, local_rank, world)


if __name__ == "__main__":
    main()
