#!/usr/bin/env python
"""Benchmark of ATJUP's time step on B200: one model iteration with the full physics.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload phys|dry] [--precision fp64|mixed]

Workload (default `phys`): the full-physics configuration on the 41 x 181 x 361 shell (2.68 M
cells, FP64). Each step is one iteration of the reference's loop (cJupiterModel.cpp:1032-1381):
on even iterations the red-black pressure pass, mixture density, radiation, the saturation
adjustment of H2O, NH3 and CH4, the NH4SH equilibrium, precipitation, the k-omega SST closure
update, the chemistry fluxes and the output diagnostics (Forces, Latent_Heat); every iteration the four RK4 stages of t, u, v, w, the 11
species and k*, omega*, the boundary passes, the moist convective adjustment, the in-loop
4th-order Shapiro filter of u, v, w, the column balance of v and the species clamp. The initial
state follows the full-physics recipe (atjup_b200/synthetic.py: state + full_physics): vapour at
90 % of saturation with U(0.95, 1.05)
noise, k = 1e-4 m2/s2 x U(0.5, 1.5), omega = 1e-3 1/s x U(0.5, 1.5), the dynamics perturbations of
the dry recipe; it is device-resident when the timed region starts. `--workload dry` times the
dry dynamics iteration instead (microphysics, radiation, closure off). `--precision mixed` runs
the mixed-precision RK step (AtjupParams.precision = ATJUP_PREC_MIXED: FP32 stage inputs and
accumulators of the 17 fields, FP32 species and closure right-hand sides; FP64 time-level-n state,
final update, dynamics right-hand side, pressure, level means, column balance and the loop's
physics).

Prints one JSON line. `value` is seconds per step for the whole job (N replicas: max-over-ranks
device time / (N * K)); `e2e` is the same metric through the public C ABI with host buffers
(pinned), the host->device upload of the step's state and the device->host read of its result
inside the timed region every step: through the asynchronous exchange (atjup_gpu_upload_async,
atjup_gpu_apply_uploads, atjup_gpu_download_async), whose copies of consecutive steps overlap the
compute, and (`e2e_serial`) through the synchronous atjup_gpu_upload / atjup_gpu_download. For the full-physics workload in FP64 the line also carries
`mixed_precision`: the run continued for K more iterations in the mixed-precision RK step, timed
the same way. With --impl reference the line times the reference's own CPU code of the same
iteration (built from its sources into oracle/_ref) on this host's cores.

`roofline` is that of one RK stage. With full physics the species and closure kernels of a stage
run on a second stream beside the dynamics kernel, so the stage (timing class `rk_group`: from the
first start to the last end of its kernels' events) is the unit: the three kernels' algorithmic
bytes over that time. The per-class times
of `device_ms_per_step_by_class` are each class's own event time, so the three concurrent classes
each include the others' share of the GPU, and `rk_group` contains all three.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

IM, JM, KM = 41, 181, 361
N_CELLS = IM * JM * KM
UNIT = "s/step"
METRICS = {
    "phys": "s per RK4 step (full-physics {prec} iteration, 41x181x361: pressure pass, radiation, "
            "saturation adjustment, NH4SH, precipitation, k-omega SST, chemistry, RK4 of 17 fields, "
            "BCs, moist convective adjustment, filters)",
    "dry": "s per RK4 step (dry {prec} dynamics, 41x181x361: one model iteration incl. pressure pass)",
}
PREC_NAMES = {"fp64": "FP64", "mixed": "mixed FP32/FP64"}
PREC_CONFIG = {
    "fp64": "fp64",
    "mixed": "mixed: FP32 stage inputs and accumulators of the RK step, FP32 species and closure "
             "right-hand sides; FP64 state, final update, dynamics right-hand side, pressure, "
             "level means, column balance and microphysics",
}
CONFIGS = {
    "phys": {
        "workload": "full-physics iteration on the 41x181x361 shell (the reference's default "
                    "physics: closure, radiation, precipitation, saturation adjustment, NH4SH "
                    "equilibrium, moist convective adjustment every iteration): the loop's "
                    "schedule, pressure and physics on even iterations (with the Forces and "
                    "Latent_Heat output diagnostics), RK4 of t, u, v, w, 11 species, k*, omega* "
                    "every iteration",
        "grid": "41x181x361", "cells": N_CELLS, "precision": "fp64",
        "l2": "no flush: inputs larger than L2 (each RK stage streams > 1.8 GB)",
        "parallelism": "replicas (the path does not shard)",
    },
    "dry": {
        "workload": "dry dynamics iteration on the 41x181x361 shell (dry knobs: obstacle on, no physics, 4th-order in-loop Shapiro): "
                    "pressure red-black pass on even iterations, RK4 (4 stages), BCs, 4th-order "
                    "Shapiro on u,v,w, column balance of v",
        "grid": "41x181x361", "cells": N_CELLS, "precision": "fp64",
        "l2": "no flush: inputs larger than L2 (each RK stage streams ~0.47 GB)",
        "parallelism": "replicas (the path does not shard)",
    },
}
# Algorithmic bytes per cell of one RK stage launch, averaged over the four stages of a step.
#
# A field of the RK step costs, over the four stages: stage 0 reads its state Y and writes the
# next stage input X and the accumulator; stages 1-2 read X, Y and the accumulator and write X
# and the accumulator; stage 3 reads X, Y and the accumulator and writes Y. With FP64 everywhere
# that is 17 x 8 = 136 B per field and step (the 17F of N b (17F + 4A)); with FP32 X and
# accumulators (mixed) 16 + 24 + 24 + 24 = 88 B. Per stage: 34 B (FP64), 22 B (mixed).
FIELD_STAGE_BYTES = {"fp64": 34.0, "mixed": 22.0}


def rk_stage_bytes(prec, phys):
    # t, u, v, w; A frozen FP64 inputs read every stage (p_dyn, p_hydro, p_stat, rho_mix, wall_nue,
    # and with full physics nue, Q_rad, Q_precip); aux_u, aux_v, aux_w written at stage 3; flags
    a = 8 if phys else 5
    return 4 * FIELD_STAGE_BYTES[prec] + 8 * a + 3 * 8 / 4 + 1


def species_stage_bytes(prec):
    # u, v, w (FP64 at stage 0, the stage buffers' type after), nue and the flag byte; per species
    # the stencil's stage input, the FP64 n copy, the output and the accumulator; the FP64 frozen
    # sources (S_precip of 9 species, the mass fluxes of H2S and NH3, the NH4SH limiter, mass flux
    # and mixture density: 112 B). FP64: 33 + 11 x 36 + 112 = 541 B.
    uvw = 24.0 if prec == "fp64" else (24 + 3 * 12) / 4
    per = 36.0 if prec == "fp64" else 5 + 8 + 5 + 6
    return uvw + 8 + 1 + 11 * per + 112


def closure_stage_bytes(prec):
    # u, v, w; k*, omega*: stage input, n copy, output, accumulator; nue; prod and the two sources
    # written at stage 3 (6 B averaged); flags. FP64: 24 + 48 + 24 + 8 + 6 + 1 = 111 B.
    if prec == "fp64":
        return 24 + 48 + 24 + 8 + 6 + 1
    return (24 + 3 * 12) / 4 + 2 * (5 + 8 + 5) + 2 * 6 + 8 + 6 + 1


def stage_kernels(prec, phys):
    return {"rk_stage": ("rk_stage_kernel", rk_stage_bytes(prec, phys)),
            "species": ("species_stage_kernel", species_stage_bytes(prec)),
            "closure": ("closure_stage_kernel", closure_stage_bytes(prec))}
# (algorithmic bytes per cell and launch; times the cells of the shell)


def stage_roofline(prec, phys, per_class, peak):
    """The roofline of one RK stage. With full physics the species and closure kernels of a stage
    run on a second stream beside the dynamics kernel, so each kernel's event time includes the
    others' share of the GPU: the unit is the stage (timing class rk_group, first kernel start to
    last kernel end) with the three kernels' algorithmic bytes and DRAM traffic. The dry step has the dynamics kernel alone."""
    kernels = stage_kernels(prec, phys)
    parts = [k for k in ("species", "closure", "rk_stage") if k in per_class] if phys else ["rk_stage"]
    names = [kernels[k][0] for k in parts]
    kbytes = sum(kernels[k][1] for k in parts) * N_CELLS
    tpc = [STAGE_TRAFFIC_PER_CELL.get((prec, n)) for n in names]
    traffic = None if None in tpc else sum(tpc) * N_CELLS
    ms, n = per_class["rk_group" if phys else "rk_stage"]
    achieved = kbytes / (ms / n / 1e3) / 1e9
    return {"kernel": " + ".join(names) + (" (one RK stage, two streams)" if len(names) > 1 else ""),
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "algorithmic_bytes_per_launch": kbytes,
            "avg_launch_ms": ms / n, "launches": n}

# DRAM bytes (read + write) per cell and launch, averaged over the four stages of one RK step:
# dram__bytes_read.sum + dram__bytes_write.sum of each stage launch in one ncu capture of this
# workload on the 41x181x361 shell (profiles/stage_traffic_phys_41x181x361.md).
STAGE_TRAFFIC_PER_CELL = {
    ("fp64", "species_stage_kernel"): 560.1, ("fp64", "closure_stage_kernel"): 100.1,
    ("fp64", "rk_stage_kernel"): 199.4,
    ("mixed", "species_stage_kernel"): 406.3, ("mixed", "closure_stage_kernel"): 68.4,
    ("mixed", "rk_stage_kernel"): 153.4,
}

DRY_ENV = {
    "ATJUP_NO_SEAMOUNT": "0", "ATJUP_PRECIP": "0", "ATJUP_RADIATION": "0", "ATJUP_TURB": "0",
    "ATJUP_MCA": "0", "ATJUP_NH4SH_EQ": "0", "ATJUP_CONE_PROJ_STRIDE": "0",
    "ATJUP_VEL_SHAPIRO_ORDER": "4", "ATJUP_VEL_SHAPIRO_INLOOP": "1",
}
# the reference's default full physics: closure, radiation, precipitation, NH4SH equilibrium and
# the moist convective adjustment every iteration
PHYS_ENV = {**DRY_ENV, "ATJUP_TURB": "1", "ATJUP_PRECIP": "1", "ATJUP_RADIATION": "1",
            "ATJUP_NH4SH_EQ": "1", "ATJUP_MCA": "1"}


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in Path(self.path).read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(workload, steps=3, warmup=1):
    """The reference's own CPU iteration (oracle/_ref) timed on this host's cores."""
    cmd = [sys.executable, str(ROOT / "oracle" / "ref_bench.py"), "--steps", str(steps),
           "--warmup", str(warmup)] + (["--phys"] if workload == "phys" else [])
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=600).stdout
        d = json.loads(out.strip().splitlines()[-1])
    except Exception as e:
        return {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                "sample": f"unavailable: {e}"}
    if "unavailable" in d:
        return {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                "sample": "unavailable: " + d["unavailable"]}
    return {"value": d["s_per_step"], "unit": UNIT, "cores": d["threads"], "kind": "reference",
            "sample": f"{d['steps']} {'full-physics' if workload == 'phys' else 'dry'} iterations "
                      f"of the reference (built at -O3 from its sources, OpenMP {d['threads']} "
                      f"threads) after {warmup} warm-up, on its own initial state"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    cb = cpu_baseline(args.workload, steps=args.steps, warmup=args.warmup)
    if cb["value"] is None:
        print(json.dumps({"impl": "reference", "unavailable": cb["sample"]}))
        return
    v = cb["value"]
    line = {"impl": "reference", "metric": METRICS[args.workload].format(prec="FP64"),
            "value": v, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"the reference's own initial state ({args.workload} knobs)",
            "config": CONFIGS[args.workload],
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_adjoint(args):
    """K dry RK4 steps forward and their adjoint through the torch.autograd binding (each step
    keeps its input as the checkpoint and the adjoint recomputes its stages), on the 41x181x361
    shell: the time of forward with checkpoints + backward over the time of K plain forward steps,
    and the device memory the chain holds. One GPU."""
    import numpy as np
    import torch

    from atjup_b200 import synthetic
    from atjup_b200.autograd import rk4_steps
    from atjup_b200.gpu import GpuModel
    from atjup_b200.params import resolve_params

    K = args.steps
    P = resolve_params(DRY_ENV, im=IM, jm=JM, km=KM)
    s = synthetic.state(IM, JM, KM, seed=20261203)
    grid = {k: s[k] for k in ("rad", "the", "solid", "topo", "cell_vbar0", "cell_ubar0")}
    m = GpuModel(P, grid)
    m.upload_state({k: v for k, v in s.items() if k not in grid})
    y0 = m.state_tensors()
    stream = torch.cuda.ExternalStream(m.stream_handle())
    the = torch.tensor(grid["the"], device="cuda")
    a = np.random.Generator(np.random.Philox(key=20261204)).uniform(-50.0, 150.0, 8) / P.u_0
    uref = sum(float(a[n - 1]) * torch.sin(n * the) for n in range(1, 9))

    def forward_plain():
        m.set_state_tensors(y0)
        for _ in range(K):
            m.runge_kutta()

    def chain():
        x = [t.clone().requires_grad_() for t in y0]
        out = rk4_steps(m, *x, steps=K)
        zm = out[3][IM - 2, :, : KM - 1].mean(dim=1)
        J = (torch.sin(the) * (zm - uref) ** 2).sum()
        J.backward()
        return J

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t0 = time.perf_counter()
        fn()
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, e0.elapsed_time(e1) / 1e3

    for _ in range(2):                      # warm-up: library scratch, torch allocator
        forward_plain()
        chain()
    fwd_wall, fwd_dev = timed(forward_plain)
    torch.cuda.reset_peak_memory_stats()
    free0 = torch.cuda.mem_get_info()[0]
    ad_wall, _ = timed(chain)
    torch_peak = torch.cuda.max_memory_allocated()
    lib_scratch = 30 * IM * JM * m.field_ptr("t")[1] * 8
    m.close()
    line = {
        "metric": f"adjoint+forward / forward time, {K} dry RK4 steps (41x181x361, FP64)",
        "value": ad_wall / fwd_wall, "unit": "x", "n_gpus": 1, "steps": K, "warmup": 2,
        "higher_is_better": False, "dtype": "f64", "data": "synthetic (seeded dry state)",
        "config": {"workload": "rk4-adjoint: K RK4 steps of the dry dynamics through "
                               "atjup_b200.autograd.RK4Step, loss = sin-weighted squared error of "
                               "the top level's zonal-mean w against a seeded 8-mode jet",
                   "grid": "41x181x361", "checkpoints": "each step's input (t, u, v, w)"},
        "forward_ms_per_step": fwd_wall / K * 1e3,
        "forward_device_ms_per_step": fwd_dev / K * 1e3,
        "adjoint_and_forward_ms_per_step": ad_wall / K * 1e3,
        "peak_bytes": {"torch_tensors": torch_peak, "library_scratch": lib_scratch,
                       "device_free_at_start": free0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="phys", choices=["phys", "dry", "rk4-adjoint"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--grid", default=None,
                    help="IMxJMxKM of a smaller shell, for profiling only (the metric is quoted "
                         "on 41x181x361)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    args.warmup = max(args.warmup, 3)
    if args.workload == "rk4-adjoint":
        run_adjoint(args)
        return

    import numpy as np
    import torch

    from atjup_b200 import synthetic
    from atjup_b200.gpu import GpuModel
    from atjup_b200.params import (DEFAULT_GASES, FIELD_IDS, PREC_FP64, PREC_MIXED, SCALARS,
                                   resolve_mca, resolve_micro, resolve_params, resolve_physics)
    from atjup_b200.replicas import max_over_ranks, whole_job_seconds_per_step

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist = dist_mod
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    phys = args.workload == "phys"
    global IM, JM, KM, N_CELLS
    if args.grid:
        import math
        IM, JM, KM = (int(x) for x in args.grid.lower().split("x"))
        N_CELLS = IM * JM * KM
    P = resolve_params(PHYS_ENV if phys else DRY_ENV, im=IM, jm=JM, km=KM)
    if args.grid:
        P.dthe = math.pi / (JM - 1)
        P.dphi = 2.0 * math.pi / (KM - 1)
    s = synthetic.state(IM, JM, KM, seed=20261203 + rank)
    grid = {k: s[k] for k in ("rad", "the", "solid", "topo", "cell_vbar0", "cell_ubar0")}
    fields = {k: v for k, v in s.items() if k not in grid}
    if phys:
        P.has_nue = 1
        P.has_heating = 1
        fields.update(synthetic.full_physics(s, DEFAULT_GASES, seed=20261207 + rank))
    m = GpuModel(P, grid)
    if phys:
        m.set_physics(resolve_physics(PHYS_ENV), fields["layer_heights"])
        m.set_micro(resolve_micro(PHYS_ENV))
        m.set_mca(resolve_mca(PHYS_ENV))
    if args.precision == "mixed":
        m.set_precision(PREC_MIXED)
    m.upload_state(fields)
    # events are recorded on the library's own stream; no torch stream is created, so the process
    # holds only the library's streams and each gets a hardware queue of its own
    stream = torch.cuda.ExternalStream(m.stream_handle())

    it = [0]

    def step():
        it[0] += 1
        m.step(it[0], it[0] == 1)

    for _ in range(args.warmup):
        step()
    m.synchronize()
    if m.nonfinite_count() != 0:
        raise SystemExit("non-finite state after warm-up")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-timed region ----
    def timed_region(steps):
        clocks = ClockSampler(local_rank)
        n0 = m.launch_count()
        m.timing(True)
        barrier()
        clocks.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
        ev1.synchronize()
        clk = clocks.stop()
        barrier()
        t_ms = ev0.elapsed_time(ev1)
        launches = m.launch_count() - n0
        per_class = {}
        for ci, cname in enumerate(m.TIMING_CLASSES):
            ms, n = m.timing_read(ci)
            if n:
                per_class[cname] = (ms, n)
        m.timing(False)
        return max_over_ranks(t_ms, device="cuda"), per_class, launches, clk

    t_ms, per_class, launches, clk = timed_region(args.steps)
    value = whole_job_seconds_per_step(t_ms / 1e3, args.steps, world)

    # ---- the same iterations in the mixed-precision RK step, continuing the run ----
    mixed = None
    if phys and args.precision == "fp64":
        m.set_precision(PREC_MIXED)
        for _ in range(2):
            step()
        mt_ms, mper, _, mclk = timed_region(args.steps)
        m.set_precision(PREC_FP64)
        mixed = {"value": whole_job_seconds_per_step(mt_ms / 1e3, args.steps, world),
                 "unit": UNIT, "ms_per_step": mt_ms / args.steps, "dtype": "f32+f64",
                 "precision": PREC_CONFIG["mixed"],
                 "accuracy": "relative L2 vs the FP64 step after 200 iterations of this workload "
                             "<= 1e-5 per prognostic field, except the condensates bounded by "
                             "the FP64 step's own sensitivity to one FP32 rounding of its input "
                             "(tests/test_mixed.py)",
                 "stage_roofline": mper,
                 "device_ms_per_step_by_class": {k: round(v[0] / args.steps, 4) for k, v in
                                                 sorted(mper.items(), key=lambda kv: -kv[1][0])},
                 "clocks": mclk}

    # ---- end to end through the C ABI with pinned host buffers ----
    names = ["t", "u", "v", "w", "p_dyn"] + (list(SCALARS) if phys else [])
    host_in = {n: torch.from_numpy(np.ascontiguousarray(fields[n])).pin_memory() for n in names}
    host_out = {n: torch.empty((IM, JM, KM), dtype=torch.float64).pin_memory() for n in names}
    import ctypes

    def up(n):
        m._rc(m.L.atjup_gpu_upload(m.ctx, FIELD_IDS[n], ctypes.c_void_p(host_in[n].data_ptr())))

    def down(n):
        m._rc(m.L.atjup_gpu_download(m.ctx, FIELD_IDS[n], ctypes.c_void_p(host_out[n].data_ptr())))

    def up_async(n):
        m._rc(m.L.atjup_gpu_upload_async(m.ctx, FIELD_IDS[n], ctypes.c_void_p(host_in[n].data_ptr())))

    def down_async(n):
        m._rc(m.L.atjup_gpu_download_async(m.ctx, FIELD_IDS[n],
                                           ctypes.c_void_p(host_out[n].data_ptr())))

    def e2e_step_async():
        for n in names:
            up_async(n)
        m._rc(m.L.atjup_gpu_apply_uploads(m.ctx))
        step()
        for n in names:
            down_async(n)

    e2e_steps = max(3, min(args.steps, 10))
    # the pipelined exchange (atjup_gpu_upload_async / apply_uploads / download_async): step n+1's
    # uploads and step n's downloads overlap step n's compute; the first round allocates the
    # staging buffers of both rounds, and the untimed rounds fill the pipeline
    for _ in range(2):
        e2e_step_async()
    m.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step_async()
    m.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, device="cuda")
    # the same with the synchronous atjup_gpu_upload / atjup_gpu_download, for comparison
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for n in names:
            up(n)
        step()
        for n in names:
            down(n)
    m.synchronize()
    e2e_serial_s = max_over_ranks(time.perf_counter() - t0, device="cuda")
    nbytes = len(names) * N_CELLS * 8

    peak, peak_kind = measured_peak_hbm()
    roof = stage_roofline(args.precision, phys, per_class, peak)
    roof["peak_kind"] = f"{peak_kind} hbm_gbs (burst copy)"
    line = {
        "metric": METRICS[args.workload].format(prec=PREC_NAMES[args.precision]),
        "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded; shapes and value ranges of the model's initial state"
                + (", full-physics recipe" if phys else "") + ")",
        "config": {**CONFIGS[args.workload], "precision": PREC_CONFIG[args.precision]},
        "roofline": roof,
        "device_ms_per_step_by_class": {k: round(v[0] / args.steps, 4) for k, v in
                                        sorted(per_class.items(), key=lambda kv: -kv[1][0])},
        "e2e": {"value": whole_job_seconds_per_step(e2e_s, e2e_steps, world), "unit": UNIT,
                "steps": e2e_steps,
                "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                "api": "atjup_gpu_upload_async, atjup_gpu_apply_uploads, atjup_gpu_step, "
                       "atjup_gpu_download_async (copies of consecutive steps overlap the compute)"},
        "e2e_serial": {"value": whole_job_seconds_per_step(e2e_serial_s, e2e_steps, world),
                       "unit": UNIT, "api": "atjup_gpu_upload, atjup_gpu_step, atjup_gpu_download"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if mixed is not None:
        mixed["stage_roofline"] = stage_roofline("mixed", phys, mixed["stage_roofline"], peak)
        line["mixed_precision"] = mixed
    if dist is not None:
        dist.barrier()
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.workload)
        print(json.dumps(line))
    m.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
