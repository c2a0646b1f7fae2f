"""Benchmark of the D2Q9 solver step on B200.

Workload (one bench "step" = S lattice time steps of one case): the
free-surface culvert dam break, 2048x512, FP32 populations + FP64 mass,
tau 0.55, g_y -5e-5, half-way walls, conservative free surface, velocity
limiter 0.25.  Its working set (~70 MB) fits in the 126 MB L2, so the L2 is
flushed (a 256 MB buffer is zeroed) before every timed step, outside the
timed events.

  value  MLUPS over all ranks, inputs resident in HBM, device time from CUDA
         events on the engine's stream (per step, summed), max over ranks.
  e2e    the same metric through the C ABI with host buffers: per step
         flb_reset from pinned host geometry flags (H2D), S steps, and a read
         of density, velocity, fill level and flags into pinned host memory.

Side measurements on rank 0 (--no-extra skips them): the plain FP32 and FP16
scaled-deviation single-phase step on 8192x2048 (HBM fraction, FP16/FP32
ratio) with the FP16 velocity error against FP64 on the 256x64 channel after
10,000 steps; the dam break at 8192x2048; the 512-case batched ensemble
against a per-case loop; the adjoint's backward/forward cost.

Multi-GPU: the path does not shard (one GPU per case), so --gpus N runs N
independent replicas, one per rank (weak scaling).

--impl reference times the CPU restatement of the reference step (the oracle,
OpenMP on all host cores, the reference's per-cell arithmetic) over the same
window of lattice steps and in the same modes as the GPU arm.
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
WORKLOAD = ("free-surface culvert dam break 2048x512, tau 0.55, g_y -5e-5, FP32 populations + FP64 mass, "
            "half-way walls, conservative free surface, velocity limiter 0.25")
U_MAX = 0.25  # keeps the surge front stable (plain BGK at tau 0.55 diverges near Mach 0.6)
KERNEL_OF_PASS = {"stream_collide": "k_sc_list (free-surface stream-collide)", "fs1": "k_fs1 (mass exchange)",
                  "fs234": "k_fs234 (flag stencil, mass/fill update, next step's lists)"}
# each pass's share of the step's device time in the ncu launch list of this
# workload (gpu__time_duration.sum of ~1000 launches of each of the three
# kernels of a step; profiles/dam_break_2048x512_launch_list.md)
PASS_SHARE_NCU: dict = {"fs234": 0.463, "fs1": 0.284, "stream_collide": 0.252}
# dram__bytes_read.sum + dram__bytes_write.sum per launch (mean of the two
# parities) from one ncu capture of the workload at steps 300-303
# (profiles/dam_break_2048x512_launch_list.md); ncu flushes the caches before
# each launch, so these are cold-start figures for an L2-resident working set
TRAFFIC_NCU: dict = {"fs234": 5356800, "stream_collide": 9796224, "fs1": 13932288}
# the persistent step: one launch runs PERSIST_STEPS lattice steps of every pass
KERNEL_PERSIST = "k_fs_persist (FS_1, stream-collide, FS_2..4 and list build, grid barriers)"
PERSIST_STEPS = 32
TRAFFIC_NCU_PERSIST = None


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def max_over_ranks(value: float, dist=None, device: str = "cuda") -> float:
    """The largest of every rank's value (the job's device time is that of its
    slowest replica); the value itself on one rank."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fp:
            d = json.load(fp)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event reasons sampled during the timed region.

    NVML (read-only queries) polled every 2 ms from a thread when it can be
    opened for the device, so even a timed region of a few hundred
    milliseconds gets many samples; otherwise nvidia-smi every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*)
    NVML_REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                    "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int, uuid: str | None = None):
        self.device = device
        self.uuid = uuid
        self.lines: list[str] = []
        self.samples: list[tuple] = []
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def _open_nvml(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = (pynvml.nvmlDeviceGetHandleByUUID(self.uuid) if self.uuid
                 else pynvml.nvmlDeviceGetHandleByIndex(self.device))
            pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
            return pynvml, h
        except Exception:
            return None

    def __enter__(self):
        opened = self._open_nvml()
        if opened is not None:
            self.nvml = opened
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _poll(self):
        nv, h = self.nvml
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(smax), int(bits)))
            except Exception:
                break
            self.stop.wait(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml is not None:
            self.thread.join(timeout=5)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        if self.nvml is not None:
            for a, b, bits in self.samples:
                sm.append(a)
                smax.append(b)
                reasons.update(name for name, bit in self.NVML_REASONS.items() if bits & bit)
            source = "nvml, 2 ms"
        else:
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
            source = "nvidia-smi, 200 ms"
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": source}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "sm_mhz_min": min(sm), "source": source}


def algorithmic_bytes(counts: dict, pop_bytes: float = 4.0) -> dict:
    """Bytes each free-surface pass must move per launch (populations of
    pop_bytes each: 4 for FP32, 2 for FP16S; FP64 mass), over the cells it
    visits: the listed super-tiles hold the fluid and interface cells (gas
    cells outside them are not touched).
      stream-collide: per fluid/interface cell its flag and wall mask (2 B),
        9 population loads and stores (72 B in FP32), density and velocity
        (12 B); interface cells also read their mass (8 B) and rewrite the
        flag (1 B);
      FS_1: per fluid/interface cell 9 incoming and 8 outgoing populations
        (68 B in FP32), its flag (1 B), mass read and write (16 B) and the
        excess shares it collects (8 B);
      FS_2..4: per fluid/interface cell the flag (1 B), the flag buffer read
        and write (2 B), density (4 B), mass read and write (16 B), excess and
        fill level (16 B)."""
    active = counts["fluid"] + counts["interface"]
    return {"stream_collide": active * (14.0 + 18.0 * pop_bytes) + counts["interface"] * 9.0,
            "fs1": active * (25.0 + 17.0 * pop_bytes), "fs234": active * 39.0}


def _gpu_uuid(torch, device: int):
    """NVML's name ("GPU-<uuid>") of the CUDA device, or None."""
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(device).uuid)
    except Exception:
        return None


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
    case = cases.dam_break(1)
    N = case.cells
    S = args.lattice_steps
    solver = E.Solver(case.flags, free_surface=True, precision=32, mass_precision=64, tau=case.tau, fy=case.fy,
                      bounce_back=E.BB_HALFWAY, fs_mode=E.FS_CONSERVATIVE, device=local_rank, u_max=U_MAX)
    solver.set_step_mode({"auto": E.STEP_AUTO, "kernels": E.STEP_KERNELS,
                          "persistent": E.STEP_PERSISTENT}[args.step_mode])
    stream = torch.cuda.ExternalStream(solver.stream, device=local_rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing (L2 flushed before every step) ------------
    for _ in range(args.warmup):
        solver.step(S)
    solver.sync()
    counts0 = solver.cell_counts()
    m0 = solver.total_mass()
    launches0 = solver.launches
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local_rank, _gpu_uuid(torch, local_rank)) as clocks:
        for a, b in ev:
            flush.zero_()
            torch.cuda.current_stream().synchronize()
            a.record(stream)
            solver.step(S)
            b.record(stream)
        solver.sync()
    barrier()
    elapsed_ms = sum(a.elapsed_time(b) for a, b in ev)
    launches = solver.launches - launches0
    counts1 = solver.cell_counts()
    mass_drift = (solver.total_mass() - m0) / m0
    t_max = max_over_ranks(elapsed_ms, dist)
    value = world * N * S * args.steps / (t_max * 1e-3) / 1e6

    # ---- dominant-kernel roofline ------------------------------------------
    peak, peak_kind = measured_peaks()
    prof_steps = max(32, S // 4)
    step_ms = t_max / (args.steps * S)  # device time per lattice step of the timed region
    if solver.persistent:
        # one kernel runs every pass of the step (32 steps per launch): its
        # launch time is the timed region's per-step time x 32, its bytes the
        # passes' algorithmic bytes over the live-cell census; the phase
        # shares come from the same kernel with a device-clock trace of its
        # grid barriers (they sum to its step time, nothing is serialised)
        ca = solver.cell_counts()
        phases = solver.profile_phases(prof_steps)
        cb = solver.cell_counts()
        counts_avg = {k: 0.5 * (ca[k] + cb[k]) for k in ca}
        pbytes = algorithmic_bytes(counts_avg)
        launch_steps = PERSIST_STEPS
        launch_bytes = sum(pbytes.values()) * launch_steps
        dom_ms = step_ms * launch_steps
        achieved = launch_bytes / (dom_ms * 1e-3) / 1e9
        tot = max(1e-12, sum(phases.values()))
        roofline = {"bound": "hbm", "kernel": KERNEL_PERSIST, "achieved": round(achieved, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                    "traffic": TRAFFIC_NCU_PERSIST, "algorithmic_bytes_per_launch": int(launch_bytes),
                    "lattice_steps_per_launch": launch_steps, "avg_launch_ms": round(dom_ms, 5),
                    "phase_share": {k: round(v / tot, 3) for k, v in phases.items()},
                    "phase_us_per_step": {k: round(v / prof_steps * 1e3, 2) for k, v in phases.items()},
                    "bytes_per_step_by_pass": {k: int(v) for k, v in pbytes.items()}}
    else:
        # per-pass kernels: each pass's share of the production step (four
        # PDL-chained kernels per step, replayed from graphs) is its share of
        # the device time in an ncu launch list of this workload
        # (PASS_SHARE_NCU), applied to the step time measured above, so the
        # pass times add up to the measured step; CUDA events around every
        # pass (serialised, the launches no longer overlap) are reported beside
        ca = solver.cell_counts()
        passes = solver.profile_steps(prof_steps)
        cb = solver.cell_counts()
        counts_avg = {k: 0.5 * (ca[k] + cb[k]) for k in ca}
        pbytes = algorithmic_bytes(counts_avg)
        dom = max(PASS_SHARE_NCU, key=PASS_SHARE_NCU.get)
        dom_ms = PASS_SHARE_NCU[dom] * step_ms
        achieved = pbytes[dom] / (dom_ms * 1e-3) / 1e9
        shares = {k: v / max(1e-12, sum(passes.values())) for k, v in passes.items()}
        per_pass = {k: {"us_per_step": round(PASS_SHARE_NCU[k] * step_ms * 1e3, 2),
                        "achieved_gbs": round(pbytes[k] / (PASS_SHARE_NCU[k] * step_ms * 1e-3) / 1e9, 1)}
                    for k in PASS_SHARE_NCU}
        roofline = {"bound": "hbm", "kernel": KERNEL_OF_PASS[dom], "achieved": round(achieved, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                    "traffic": TRAFFIC_NCU.get(dom), "algorithmic_bytes_per_launch": int(pbytes[dom]),
                    "avg_launch_ms": round(dom_ms, 5), "pass_share": PASS_SHARE_NCU,
                    "pass_share_source": "ncu launch list, profiles/dam_break_2048x512_launch_list.md",
                    "passes": per_pass,
                    "pass_share_serialised_events": {k: round(v, 3) for k, v in shares.items()}}
    step_bytes = sum(pbytes.values())
    roofline["whole_step"] = {"algorithmic_bytes": int(step_bytes), "us": round(step_ms * 1e3, 3),
                              "achieved_gbs": round(step_bytes / (step_ms * 1e-3) / 1e9, 1),
                              "frac": round(step_bytes / (step_ms * 1e-3) / 1e9 / peak, 4)}

    persistent = solver.persistent
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
    e2e_s = max_over_ranks(e2e_s, dist)
    e2e_value = world * N * S * args.steps / e2e_s / 1e6

    # ---- side measurements on rank 0 (FP16 storage, single-phase probe) ---
    extra = {}
    if rank == 0 and not args.no_extra:
        extra = side_measurements(args, local_rank, E, cases, peak, _gpu_uuid(torch, local_rank))

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
                       "step_form": "persistent kernel" if persistent else "per-pass kernels",
                       "timed_lattice_steps": [args.warmup * S, (args.warmup + args.steps) * S],
                       "l2": "working set ~70 MB < 126 MB L2: a 256 MB buffer is zeroed before every timed step "
                             "(outside the timed events)",
                       "cells_by_type_at_start": counts0, "cells_by_type_at_end": counts1,
                       "total_mass_rel_drift": mass_drift},
            "e2e": {"value": round(e2e_value, 1), "unit": "MLUPS", "h2d_bytes_per_step": int(N),
                    "d2h_bytes_per_step": int(N * (4 + 8 + 8 + 1))},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "clocks": clocks.summary(),
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        line.update(extra)
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def _timed(torch, solver, n):
    st = torch.cuda.ExternalStream(solver.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    solver.step(n)
    b.record(st)
    b.synchronize()
    return a.elapsed_time(b)


def side_measurements(args, device, E, cases, peak, uuid):
    """Each side measurement carries the SM clocks sampled while it ran."""
    import torch

    out = {}

    def clocked(key, fn):
        with ClockSampler(device, uuid) as clk:
            r = fn()
        if isinstance(r, dict):
            r["clocks"] = clk.summary()
        out[key] = r

    # plain single phase on 8192x2048 (working set ~1.2 GB): FP32 and FP16S
    p = cases.hbm_probe(8192, 2048)

    def single_phase(prec, bytes_per):
        s = E.Solver(p.flags, free_surface=False, precision=prec, tau=p.tau, fx=p.fx, bounce_back=E.BB_HALFWAY,
                     device=device)
        s.step(50)
        s.sync()
        n = 400
        ms = _timed(torch, s, n)
        s.close()
        mlups = p.cells * n / (ms * 1e-3) / 1e6
        # bytes: the populations of every cell; flag and wall mask only where
        # the plain-fluid chunk map does not cover the cell (about 5 %)
        gbs = p.cells * bytes_per * n / (ms * 1e-3) / 1e9
        return {"value": round(mlups, 1), "unit": "MLUPS", "achieved_gbs": round(gbs, 1),
                "frac_of_measured_hbm": round(gbs / peak, 4), "bytes_per_cell": bytes_per}

    clocked("single_phase_fp32_8192x2048", lambda: single_phase(32, 72.0))
    clocked("single_phase_fp16s_8192x2048", lambda: single_phase(16, 36.0))
    out["fp16s_speedup_single_phase"] = round(out["single_phase_fp16s_8192x2048"]["value"] /
                                              out["single_phase_fp32_8192x2048"]["value"], 3)
    # FP16S accuracy: velocity L2 against FP64 on the 256x64 channel, 10,000 steps
    ch = cases.plain_channel()
    fluid = np.tile(ch.flags.ravel() == cases.FLUID, 2)
    us = {}
    for prec in (64, 32, 16):
        s = E.Solver(ch.flags, precision=prec, tau=ch.tau, fx=ch.fx, bounce_back=E.BB_HALFWAY, device=device)
        s.step(10_000)
        us[prec] = s.u.astype(np.float64)[fluid]
        s.close()
    for prec in (32, 16):
        out[f"velocity_l2_vs_fp64_{'fp32' if prec == 32 else 'fp16s'}_channel_256x64_10000"] = float(
            np.linalg.norm(us[prec] - us[64]) / np.linalg.norm(us[64]))
    # the dam break at 8192x2048 (FP32 and FP16S)
    c = cases.dam_break(4)
    S = args.lattice_steps

    def dam_break_big(prec):
        s = E.Solver(c.flags, free_surface=True, precision=prec, mass_precision=64, tau=c.tau, fy=c.fy,
                     bounce_back=E.BB_HALFWAY, fs_mode=E.FS_CONSERVATIVE, device=device, u_max=U_MAX)
        s.step(S)
        s.sync()
        c0 = s.cell_counts()
        ms = _timed(torch, s, 2 * S)
        c1 = s.cell_counts()
        form = "persistent kernel" if s.persistent else "per-pass kernels"
        s.close()
        # the step's algorithmic bytes from the live-cell census (mean of the
        # window's ends), over the measured copy bandwidth
        cavg = {k: 0.5 * (c0[k] + c1[k]) for k in c0}
        step_bytes = sum(algorithmic_bytes(cavg, 4.0 if prec == 32 else 2.0).values())
        gbs = step_bytes * 2 * S / (ms * 1e-3) / 1e9
        return {"value": round(c.cells * 2 * S / (ms * 1e-3) / 1e6, 1), "unit": "MLUPS", "step_form": form,
                "algorithmic_bytes_per_step": int(step_bytes), "achieved_gbs": round(gbs, 1),
                "frac_of_measured_hbm": round(gbs / peak, 4),
                "live_cells": int(cavg["fluid"] + cavg["interface"])}

    for prec in (32, 16):
        clocked(f"dam_break_8192x2048_fp{prec if prec == 32 else '16s'}", lambda: dam_break_big(prec))
    # storage-precision sweep of the 8192x2048 dam break (FP64 / FP32 / FP16S)
    if args.sweep_steps > 0:
        from flowlb_b200 import precision_sweep

        clocked("precision_sweep_dam_break_8192x2048",
                lambda: precision_sweep.run(4, args.sweep_steps, U_MAX, device))
    # batched ensemble: 512 cases in one launch per call vs a per-case loop,
    # both over the full step count
    ens = cases.ensemble()
    n_b = args.batch_steps
    spec = [(e.flags, e.tau, e.fx, 0.0) for e in ens]
    cells = sum(e.flags.size for e in ens)

    def timed_batch(b):
        b.step(2)
        b.sync()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.step(n_b)
        b.sync()
        tb = time.perf_counter() - t0
        return {"cases_per_s": round(len(ens) / tb, 2), "unit": f"cases/s ({n_b} steps each)",
                "glups": round(cells * n_b / tb / 1e9, 1), "steps_timed": n_b, "config": b.info(), "wall_s": tb}

    def batch():
        # the tuned form (the persistent kernel's shapes and the streams form)
        b = E.Batch(spec, autotune=1, device=device)
        res = timed_batch(b)
        b.close()
        return res

    def batch_persistent():
        # the persistent kernel's best shape alone: one graph-captured launch per flb_batch_step
        b = E.Batch(spec, autotune=0, device=device)
        b.tune(0, E.TUNE_PERSISTENT)
        res = timed_batch(b)
        b.close()
        return res

    def loop():
        sm = torch.cuda.Stream()
        solvers = [E.Solver(e.flags, precision=32, tau=e.tau, fx=e.fx, stream=sm.cuda_stream, device=device)
                   for e in ens]
        for s in solvers:
            s.step(2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in solvers:
            s.step(n_b)
        torch.cuda.synchronize()
        tl = time.perf_counter() - t0
        for s in solvers:
            s.close()
        return {"cases_per_s": round(len(ens) / tl, 2), "wall_s": tl}

    clocked("batch_512_cases", batch)
    clocked("batch_512_cases_persistent_kernel", batch_persistent)
    clocked("per_case_loop_512_cases", loop)
    lt = out["per_case_loop_512_cases"]
    for key in ("batch_512_cases", "batch_512_cases_persistent_kernel"):
        bt = out[key]
        bt["loop_cases_per_s"] = lt["cases_per_s"]
        bt["speedup_vs_per_case_loop"] = round(lt["wall_s"] / bt["wall_s"], 3)

    # adjoint: backward (with checkpoint recomputation) over forward, FP64
    # (the form whose gradient meets the finite-difference check) and FP32
    def adjoint():
        pc = cases.porous_channel()
        r = {}
        for prec in (64, 32):
            a = E.Adjoint(pc.flags, pc.porosity.astype(np.float64), tau=pc.tau, gx=pc.fx, precision=prec,
                          device=device)
            a.forward()
            a.backward()
            a.forward()
            a.backward()
            f_ms, b_ms = a.timing()
            a.close()
            r[f"fp{prec}"] = {"forward_ms": round(f_ms, 2), "backward_ms": round(b_ms, 2),
                              "backward_over_forward": round(b_ms / f_ms, 3)}
        r["backward_over_forward"] = r["fp64"]["backward_over_forward"]
        return r

    clocked("adjoint_1024x256_4096", adjoint)
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
            "sample": f"{case.nx}x{case.ny} dam break, {n} time steps after the first, same storage, modes and "
                      f"arithmetic ({dt:.1f} s)"}


def run_reference(args, rank, world):
    """The reference step restated on the CPU (the oracle, OpenMP on all host
    cores), timed over the same window of lattice steps as the GPU arm:
    W warm-up bench steps and K timed bench steps of S lattice steps each, on
    the same case and in the same modes (half-way walls, conservative free
    surface, limiter 0.25, FP32 populations + FP64 mass), with the reference's
    per-cell expressions (reference arithmetic, as FlowLB's kernels evaluate
    them, lbmKernel2D.cu:306-519).  Rank 0 alone runs and prints it."""
    if rank != 0:
        return
    from flowlb_b200 import cases
    from oracle import oracle as O

    case = cases.dam_break(1)
    threads = os.cpu_count() or 1
    o = O.Oracle(case.flags, O.OracleConfig(variant=O.F32, free_surface=True, bb=O.BB_HALFWAY,
                                            fs_mode=O.FS_CONSERVATIVE, tau=case.tau, fy=case.fy, threads=threads,
                                            u_max=U_MAX, arithmetic=O.ARITH_REFERENCE))
    S = args.lattice_steps
    for _ in range(args.warmup):
        o.step(S)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(S)
    dt = time.perf_counter() - t0
    o.close()
    value = case.cells * S * args.steps / dt / 1e6
    sample = (f"{case.nx}x{case.ny} dam break, lattice steps {args.warmup * S}-{(args.warmup + args.steps) * S} "
              f"timed in {args.steps} chunks of {S} (the GPU arm's window)")
    line = {"metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "nx": case.nx, "ny": case.ny, "cells": case.cells,
                       "lattice_steps_per_step": S, "parallelism": "host cores",
                       "timed_lattice_steps": [args.warmup * S, (args.warmup + args.steps) * S],
                       "arithmetic": "reference (FlowLB's per-cell expressions)"},
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
    ap.add_argument("--cpu-steps", type=int, default=2000)
    ap.add_argument("--batch-steps", type=int, default=5000, help="steps of the batch and per-case-loop measurement")
    ap.add_argument("--sweep-steps", type=int, default=50_000,
                    help="steps of the 8192x2048 storage-precision sweep (0 skips it)")
    ap.add_argument("--step-mode", default="auto", choices=["auto", "kernels", "persistent"],
                    help="free-surface step form (flb_set_step_mode)")
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
