#!/usr/bin/env python
"""Benchmark of ATJUP's time step on B200: one model iteration with the full physics.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload phys|dry|adjoint|cone] [--precision fp64|mixed] [--no-extras]

Workload (default `phys`): the full-physics configuration on the 41 x 181 x 361 shell (2.68 M
cells, FP64). Each step is one iteration of the reference's loop (cJupiterModel.cpp:1032-1381):
on even iterations the red-black pressure pass, mixture density, radiation, the saturation
adjustment of H2O, NH3 and CH4, the NH4SH equilibrium, precipitation, the k-omega SST closure
update, the chemistry fluxes and the output diagnostics (Forces, Latent_Heat); every iteration
the four RK4 stages of t, u, v, w, the 11 species and k*, omega*, the boundary passes, the moist
convective adjustment, the in-loop 4th-order Shapiro filter of u, v, w, the column balance of v
and the species clamp. `--workload dry` times the dry dynamics iteration instead (microphysics,
radiation, closure off). `--precision mixed` runs the mixed-precision RK step
(AtjupParams.precision = ATJUP_PREC_MIXED: FP32 stage inputs and accumulators of the 17 fields,
FP32 species and closure right-hand sides; FP64 time-level-n state, final update, dynamics
right-hand side, pressure, level means, column balance and the loop's physics).

Initial state: the reference's own initial state with the configuration's seeded recipe applied
(oracle/baseline_state.py: Gaussian noise on t, u, v, w; for full physics vapour at 90 % of
saturation x U(0.95, 1.05), no condensate, seeded k and omega), produced once per run, untimed, by
the reference built from its sources, and handed to this arm byte for byte; the reference arm
and the CPU baseline start from the same bytes. It is device-resident when the timed region
starts. Without the reference library the synthetic state of atjup_b200/synthetic.py stands in
(the line's `data` says which).

Prints one JSON line. `value` is seconds per step for the whole job (N replicas: max-over-ranks
device time / (N * K)); `e2e` is the same metric through the public C ABI with host buffers
(pinned), the host->device upload of the step's state and the device->host read of its result
inside the timed region every step: through the asynchronous exchange (atjup_gpu_upload_async,
atjup_gpu_apply_uploads, atjup_gpu_download_async), whose copies of consecutive steps overlap the
compute, and (`e2e_serial`) through the synchronous atjup_gpu_upload / atjup_gpu_download. With
--impl reference the line times the reference's own CPU code of the same iteration (built from
its sources into oracle/_ref) on this host's cores.

Sections of the default line besides the headline (N = 1; --no-extras drops them):
* `mixed_precision`: the same K iterations from the same state in the mixed-precision RK step,
  and the relative L2 per prognostic field of 200 mixed iterations against 200 FP64 iterations
  from that state.
* `poisson`: the isolated Poisson solve on the shell (seeded smoothed N(0, 1) right-hand side):
  FP64 PCG, mixed PCG (FP32 preconditioner) and point red-black SOR with omega = 1.7 --
  iterations, seconds per solve, relative residual, its FP64 rounding floor, HBM GB/s.
* `adjoint`: adjoint+forward over forward time of 50 whole dry iterations through the
  torch.autograd binding (IterationStep), from the dry configuration's state, with the memory it
  holds.

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
                    "every iteration, the projection around the obstacle every 10 iterations "
                    "(the reference's default stride)",
        "grid": "41x181x361", "cells": N_CELLS, "precision": "fp64",
        "l2": "no flush: inputs larger than L2 (each RK stage streams > 1.8 GB)",
        "parallelism": "replicas (the path does not shard)",
    },
    "dry": {
        "workload": "dry dynamics iteration on the 41x181x361 shell (dry knobs: obstacle on, no physics, 4th-order in-loop Shapiro): "
                    "pressure red-black pass on even iterations, RK4 (4 stages), BCs, 4th-order "
                    "Shapiro on u,v,w, column balance of v, the projection around the obstacle "
                    "every 10 iterations (the reference's default stride)",
        "grid": "41x181x361", "cells": N_CELLS, "precision": "fp64",
        "l2": "no flush: inputs larger than L2 (each RK stage streams ~0.47 GB)",
        "parallelism": "replicas (the path does not shard)",
    },
}
# The roofline's numerator: the algorithmic bytes of one RK stage by the scope's formula,
# B_rk = N b (17 F + 4 A) + 4 N per RK step (a quarter per stage). F = fields integrated (dry 4:
# t, u, v, w; full physics 17: with the 11 species and k*, omega*), A = frozen per-cell inputs the
# right-hand sides read (dry 5: p_dyn, p_hydro, p_stat, rho_mix, wall_nue; full physics 21: with
# nue, Q_rad, Q_precip, 9 S_precip, 3 mass fluxes, the NH4SH flux limiter), b = 8 (FP64) or 4
# (the mixed step, whose stage buffers are FP32), the mask one byte per stage. Per field the 17 b
# is the classic bookkeeping: stage 0 reads Y and writes X1 and the accumulator, stages 1-2 read
# X, Y and the accumulator and write X and the accumulator, stage 3 reads X, Y and the accumulator
# and writes Y.
def formula_bytes_per_cell_stage(prec, phys):
    F, A = (17, 21) if phys else (4, 5)
    b = 8 if prec == "fp64" else 4
    return (b * (17 * F + 4 * A) + 4) / 4


# The bytes this implementation moves per cell and stage launch, averaged over the four stages.
# FP64: the species keep no accumulator (stage 3 recovers the stage right-hand sides from X1, X2,
# X3 and y_n: 3 + 3 + 3 + 5 = 14 accesses of 8 B per species and step, 28 B per stage), the
# dynamics write it once at stage 2 (2 + 3 + 5 + 4 = 14 per field and step, 28 B per stage), the
# closure keeps the classic 17 (34 B). Mixed (FP32 X and accumulators, FP64 y_n): 16 + 24 + 24 + 24
# = 88 B per field and step, 22 B per stage.
FIELD_STAGE_BYTES = {"fp64": 28.0, "mixed": 22.0}


def rk_stage_bytes(prec, phys):
    # t, u, v, w; A frozen FP64 inputs read every stage (p_dyn, p_hydro, p_stat, rho_mix, wall_nue,
    # and with full physics nue, Q_rad, Q_precip); aux_u, aux_v, aux_w written at stage 3; flags
    a = 8 if phys else 5
    return 4 * FIELD_STAGE_BYTES[prec] + 8 * a + 3 * 8 / 4 + 1


def species_stage_bytes(prec):
    # u, v, w (FP64 at stage 0, the stage buffers' type after), nue and the flag byte; per species
    # the stencil's stage input, the FP64 n copy and the output (and X1, X2 at stage 3, or the
    # accumulator in the mixed step); the FP64 frozen sources (S_precip of 9 species, the mass
    # fluxes of H2S and NH3, the NH4SH limiter, mass flux and mixture density: 112 B).
    # FP64: 33 + 11 x 28 + 112 = 453 B.
    uvw = 24.0 if prec == "fp64" else (24 + 3 * 12) / 4
    per = 28.0 if prec == "fp64" else 5 + 8 + 5 + 6
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
# (bytes moved per cell and launch; times the cells of the shell)


def stage_roofline(prec, phys, per_class, peak):
    """The roofline of one RK stage. With full physics the species and closure kernels of a stage
    run on a second stream beside the dynamics kernel, so each kernel's event time includes the
    others' share of the GPU: the unit is the stage (timing class rk_group, first kernel start to
    last kernel end). `achieved` is the stage's algorithmic bytes by the scope's formula over that
    time; `moved_*` the bytes this implementation moves, and `traffic` the DRAM bytes ncu measured.
    The dry step has the dynamics kernel alone."""
    kernels = stage_kernels(prec, phys)
    parts = [k for k in ("species", "closure", "rk_stage") if k in per_class] if phys else ["rk_stage"]
    names = [kernels[k][0] for k in parts]
    moved = sum(kernels[k][1] for k in parts) * N_CELLS
    fbytes = formula_bytes_per_cell_stage(prec, phys) * N_CELLS
    tpc = [STAGE_TRAFFIC_PER_CELL.get((prec, n)) for n in names]
    traffic = None if None in tpc else sum(tpc) * N_CELLS
    ms, n = per_class["rk_group" if phys else "rk_stage"]
    t = ms / n / 1e3
    achieved = fbytes / t / 1e9
    F, A = (17, 21) if phys else (4, 5)
    return {"kernel": " + ".join(names) + (" (one RK stage, two streams)" if len(names) > 1 else ""),
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "algorithmic_bytes_per_launch": fbytes,
            "algorithmic_bytes_formula": "(N b (17 F + 4 A) + 4 N) / 4 per stage, N = %d, F = %d, "
                                         "A = %d, b = %d" % (N_CELLS, F, A, 8 if prec == "fp64" else 4),
            "moved_bytes_per_launch": moved, "moved_gbs": moved / t / 1e9,
            "moved_frac": moved / t / 1e9 / peak,
            "avg_launch_ms": ms / n, "launches": n}


# DRAM bytes (read + write) per cell and launch, averaged over the four stages of one RK step:
# dram__bytes_read.sum + dram__bytes_write.sum of each stage launch in one ncu capture of this
# workload on the 41x181x361 shell.
STAGE_TRAFFIC_PER_CELL = {
    ("fp64", "species_stage_kernel"): 449.2, ("fp64", "closure_stage_kernel"): 106.8,
    ("fp64", "rk_stage_kernel"): 178.5,
    ("mixed", "species_stage_kernel"): 406.3, ("mixed", "closure_stage_kernel"): 68.4,
    ("mixed", "rk_stage_kernel"): 153.4,
}

DRY_ENV = {
    "ATJUP_NO_SEAMOUNT": "0", "ATJUP_PRECIP": "0", "ATJUP_RADIATION": "0", "ATJUP_TURB": "0",
    "ATJUP_MCA": "0", "ATJUP_NH4SH_EQ": "0", "ATJUP_CONE_PROJ_STRIDE": "10",
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


REF_LIB = ROOT / "oracle" / "_ref" / "libatjup_ref.so"
STATE_RECIPE = {
    "phys": "the reference's own initial state (its initialisation, phys knobs) with the "
            "full-physics recipe: Philox(20261203) noise on w, v, u, t; Philox(20261207) vapour at "
            "90 % of saturation x U(0.95, 1.05), k, omega (oracle/baseline_state.py)",
    "dry": "the reference's own initial state (its initialisation, dry knobs) with the dry "
           "recipe: Philox(20261203) noise on w, v, u, t (oracle/baseline_state.py)",
}


def cpu_baseline(workload, steps=10, warmup=2):
    """The reference's own CPU iteration (oracle/_ref) timed on this host's cores, from the same
    seeded initial state as the GPU arm."""
    cmd = [sys.executable, str(ROOT / "oracle" / "ref_bench.py"), "--steps", str(steps),
           "--warmup", str(warmup)] + (["--phys"] if workload == "phys" else [])
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=900).stdout
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
                      f"threads) after {warmup} warm-up, from {d['state']}",
            "state": d["state"]}


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
            "data": cb["state"],
            "config": CONFIGS[args.workload],
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---- the benchmark state ---------------------------------------------------------------------

MICRO_RENAME = {"rad_F_int": "F_int", "rad_S_solar": "S_solar", "rad_albedo_bond": "albedo_bond",
                "rad_x_H2": "x_H2", "rad_x_He": "x_He"}


def reference_state(workload, rank, dist):
    """The configuration's seeded initial state as a dict of arrays: the reference's own
    initialisation with the seeded recipe applied, produced once per run, untimed, by
    oracle/baseline_state.py (rank 0 writes it, every rank reads it), so that this arm and the
    reference arm start from the same bytes. None when the reference library is not built."""
    import numpy as np
    path = Path(tempfile.gettempdir()) / f"atjup_bench_state_{workload}_{os.getpid() if dist is None else 'dist'}.npz"
    ok = [REF_LIB.exists()]
    if rank == 0 and ok[0]:
        cmd = [sys.executable, str(ROOT / "oracle" / "baseline_state.py"), str(path),
               "--config", workload]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        ok[0] = r.returncode == 0 and path.exists()
    if dist is not None:
        dist.barrier()
    if not ok[0] and rank == 0:
        return None
    if not path.exists():
        return None
    with np.load(path) as z:
        d = {k: z[k] for k in z.files}
    if dist is not None:
        dist.barrier()
    if rank == 0:
        path.unlink(missing_ok=True)
    return d


def model_inputs(d, workload):
    """(params, physics, micro, mca, grid, fields) of a state dict written by
    oracle/baseline_state.py."""
    from atjup_b200.params import resolve_mca, resolve_micro, resolve_params, resolve_physics
    env = PHYS_ENV if workload == "phys" else DRY_ENV
    consts = {k[6:]: float(v) for k, v in d.items() if k.startswith("const_")}
    im, jm, km = d["in_t"].shape
    P = resolve_params(env, im=im, jm=jm, km=km, constants=consts)
    grid = {k[5:]: v for k, v in d.items() if k.startswith("grid_")}
    fields = {k[3:]: v for k, v in d.items() if k.startswith("in_")}
    if workload != "phys":
        return P, None, None, None, grid, fields
    P.has_nue = 1
    P.has_heating = 1
    MC = resolve_micro(env, {MICRO_RENAME.get(k[6:], k[6:]): float(v) for k, v in d.items()
                             if k.startswith("micro_")},
                       {g: tuple(d["gas_" + g]) for g in ("H2O", "NH3", "CH4")})
    pc = {k[5:]: float(v) for k, v in d.items() if k.startswith("phys_")}
    pc["abl_height"] = float(d["knobd_abl_height"])
    return P, resolve_physics(env, pc), MC, resolve_mca(env), grid, fields


def synthetic_inputs(workload, rank):
    """Fallback when the reference is not built: the synthetic state of atjup_b200.synthetic
    (the reference's grid shapes and value ranges, the same seeded recipes)."""
    from atjup_b200 import synthetic
    from atjup_b200.params import (DEFAULT_GASES, resolve_mca, resolve_micro, resolve_params,
                                   resolve_physics)
    phys = workload == "phys"
    P = resolve_params(PHYS_ENV if phys else DRY_ENV, im=IM, jm=JM, km=KM)
    if (IM, JM, KM) != (41, 181, 361):
        import math
        P.dthe = math.pi / (JM - 1)
        P.dphi = 2.0 * math.pi / (KM - 1)
    s = synthetic.state(IM, JM, KM, seed=20261203 + rank)
    grid = {k: s[k] for k in ("rad", "the", "solid", "topo", "cell_vbar0", "cell_ubar0")}
    fields = {k: v for k, v in s.items() if k not in grid}
    if not phys:
        return P, None, None, None, grid, fields
    P.has_nue = 1
    P.has_heating = 1
    fields.update(synthetic.full_physics(s, DEFAULT_GASES, seed=20261207 + rank))
    return (P, resolve_physics(PHYS_ENV), resolve_micro(PHYS_ENV), resolve_mca(PHYS_ENV), grid,
            fields)


def build_model(P, PH, MC, MCA, grid, fields):
    from atjup_b200.gpu import GpuModel
    m = GpuModel(P, grid)
    if PH is not None:
        m.set_physics(PH, fields["layer_heights"])
        m.set_micro(MC)
        m.set_mca(MCA)
    m.upload_state(fields)
    return m


# ---- config 1: the isolated Poisson solve ----------------------------------------------------

def poisson_section(m, stream):
    """The isolated Poisson solve on the model's shell (seeded N(0, 1) right-hand side smoothed by
    3 passes of the 1-2-1 filter per direction, its incompatible part removed by the solver):
    FP64 PCG, mixed PCG (FP32 preconditioner) and point red-black SOR with omega = 1.7, each
    timed with CUDA events on the library's stream."""
    import torch

    from atjup_b200 import synthetic
    from atjup_b200.params import PREC_FP64, PREC_MIXED, SOLVE_RESIDUAL, SOLVE_SOR
    im, jm, km = m.shape
    b = synthetic.poisson_rhs(im, jm, km)
    m.set_solve_rhs(b)
    n = im * jm * km
    peak, kind = measured_peak_hbm()

    def timed(**kw):
        m.pressure_solver(**kw)                      # warm: set-up and first-touch
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m.synchronize()
        ev0.record(stream)
        st = m.pressure_solver(**kw)
        ev1.record(stream)
        ev1.synchronize()
        return st, ev0.elapsed_time(ev1) / 1e3

    out = {"problem": "A p = b on the 41x181x361 shell with the obstacle: the reference's folded "
                      "all-Neumann operator (PressureSolver.h:144-766); b seeded N(0, 1) smoothed "
                      "by 3 passes of 1-2-1 per direction, made compatible by removing its "
                      "component along the operator's left null vector",
           "target": "relative residual 1e-10, or <= 8 x the rounding floor of an FP64 p "
                     "(rel_floor) where that is above 1e-10"}
    # PCG: per iteration the operator, the update, the radial line solve, the inverse DFT and the
    # direction touch N (23 b + 1) bytes in FP64 (b = 8); the mixed form keeps z and the line
    # factors in FP32: N (153 + 1) bytes
    for name, prec, bpc in (("fp64", PREC_FP64, 23 * 8 + 1), ("mixed", PREC_MIXED, 154)):
        st, t = timed(mode=SOLVE_RESIDUAL, rel_tol=1e-10, max_iter=5000, precision=prec,
                      external_rhs=True, allow_not_converged=True)
        gbs = st.iterations * n * bpc / t / 1e9 if t > 0 else None
        out[name] = {"s_per_solve": t, "iterations": st.iterations,
                     "refinement_steps": st.inner_solves, "rel_residual": st.rel_residual,
                     "rel_floor": st.rel_floor,
                     "converged": bool(st.rel_residual <= max(1e-10, 8 * st.rel_floor)),
                     "hbm_gbs": gbs, "hbm_frac": gbs / peak if gbs else None,
                     "algorithmic_bytes_per_iteration": n * bpc}
    # point SOR, omega = 1.7: two sweep caps give the contraction per sweep, hence the sweeps
    # 1e-10 would take; each sweep moves N (3 b + 1) bytes
    res = {}
    for cap in (500, 1000):
        st, t = timed(mode=SOLVE_SOR, omega=1.7, rel_tol=1e-10, max_iter=cap,
                      external_rhs=True, allow_not_converged=True)
        res[cap] = (st, t)
    (s1, _), (s2, t2) = res[500], res[1000]
    import math
    rate = (s2.rel_residual / s1.rel_residual) ** (1.0 / 500) if s1.rel_residual > 0 else None
    proj = (1000 + math.log(1e-10 / s2.rel_residual) / math.log(rate)
            if rate is not None and 0 < rate < 1 else None)
    gbs = s2.iterations * n * 25 / t2 / 1e9
    out["sor_omega_1.7"] = {"sweeps": s2.iterations, "s": t2, "s_per_sweep": t2 / s2.iterations,
                            "rel_residual": s2.rel_residual, "rel_residual_at_500": s1.rel_residual,
                            "contraction_per_sweep": rate, "projected_sweeps_to_1e-10": proj,
                            "hbm_gbs": gbs, "hbm_frac": gbs / peak,
                            "algorithmic_bytes_per_sweep": n * 25}
    out["peak"] = {"hbm_gbs": peak, "kind": kind}
    return out


def cone_section(P, grid, fields, calls=3):
    """The in-loop projection around the obstacle (projectAroundObstacle(in_loop = true), every
    ATJUP_CONE_PROJ_STRIDE = 10 iterations by the reference's default, and so in both arms'
    timed iterations), timed here on its own: `calls` calls on the dry
    configuration's state, the first from zero and the rest warm-started, each timed with CUDA
    events on the library's stream, beside the reference's own per-call time on this host."""
    import torch
    m = build_model(P, None, None, None, grid, fields)
    stream = torch.cuda.ExternalStream(m.stream_handle())
    out = {"what": "per level cutting the obstacle (26 levels), the divergence solve (H = 3) and "
                   "the wall-flux solve by lexicographic SOR to 1e-10, bit-identical to the "
                   "reference; margin 40 cells", "calls": []}
    m.cone_stats()                      # the static part (boxes, flags, buffers) outside the timing
    for c in range(calls):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m.synchronize()
        ev0.record(stream)
        m.cone_project()
        ev1.record(stream)
        ev1.synchronize()
        levels, sweeps = m.cone_stats()
        out["calls"].append({"s": ev0.elapsed_time(ev1) / 1e3, "warm_start": c > 0,
                             "levels": int(levels.size), "sweeps_max": int(sweeps.max()),
                             "sweeps_mean": float(sweeps[sweeps > 0].mean())})
    m.close()
    out["gpu_s_per_call"] = sum(x["s"] for x in out["calls"]) / calls
    cmd = [sys.executable, str(ROOT / "oracle" / "ref_bench.py"), "--cone", "2"]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600).stdout
        d = json.loads(r.strip().splitlines()[-1])
        out["reference_s_per_call"] = d.get("cone_s_per_call")
        out["reference_threads"] = d.get("threads")
    except Exception as e:   # noqa: BLE001 -- the CPU leg is reported, not required
        out["reference_s_per_call"] = None
        out["reference_unavailable"] = str(e)
    return out


# ---- config 4: the adjoint -------------------------------------------------------------------

def adjoint_section(P, grid, fields, K):
    """The dry configuration's adjoint: K whole dry iterations of the reference's loop (the
    pressure pass and mixture density on even iterations, RK4, the boundary passes, the in-loop
    Shapiro filter, the column balance) forward, and their adjoint through the torch.autograd
    binding (atjup_b200.autograd.IterationStep: each iteration's input, the nine fields it reads,
    is its checkpoint; the adjoint recomputes the pressure pass and the RK stages from it). The
    loss is J = sum_theta sin(colatitude) (zonal-mean w at the top integrated level -
    u_ref)^2, u_ref = sum_{n=1..8} a_n sin(n theta), a_n seeded U(-50, 150) m/s. Reports the time
    of forward with checkpoints + backward over the time of K plain forward iterations, and the
    device memory the chain holds. The projection around the obstacle has no linearisation here:
    these iterations run without it (cone_proj_stride 0)."""
    import numpy as np
    import torch

    from atjup_b200.autograd import iterations
    from atjup_b200.gpu import GpuModel
    from atjup_b200.params import LIN_FIELDS

    P = type(P).from_buffer_copy(P)
    P.cone_proj_stride = 0
    m = GpuModel(P, grid)
    m.upload_state(fields)
    im, jm, km = m.shape
    x0 = m.state_tensors(LIN_FIELDS)
    stream = torch.cuda.ExternalStream(m.stream_handle())
    the = torch.tensor(grid["the"], device="cuda")
    a = np.random.Generator(np.random.Philox(key=20261204)).uniform(-50.0, 150.0, 8) / P.u_0
    uref = sum(float(a[n - 1]) * torch.sin(n * the) for n in range(1, 9))

    def forward_plain():
        m.set_state_tensors(x0, names=LIN_FIELDS)
        for n in range(1, K + 1):
            m.step(n, n == 1)

    def chain():
        x = [t.clone().requires_grad_() for t in x0]
        out = iterations(m, x, K)
        zm = out[3][im - 2, :, : km - 1].mean(dim=1)
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
    base = torch.cuda.memory_allocated()
    ad_wall, _ = timed(chain)
    torch_peak = torch.cuda.max_memory_allocated() - base
    pitch = m.field_ptr("t")[1]
    lib_scratch = (30 + 8) * im * jm * pitch * 8
    m.close()
    return {
        "metric": f"adjoint+forward / forward time, {K} dry iterations",
        "ratio": ad_wall / fwd_wall, "steps": K,
        "what": "whole dry iterations (pressure pass and mixture density on even iterations, "
                "RK4, boundary passes, 4th-order Shapiro of u, v, w, column balance of v) "
                "through atjup_b200.autograd.IterationStep (atjup_gpu_iteration_adjoint); "
                "checkpoints: each iteration's input, t, u, v, w, p_dyn, aux_u, aux_v, aux_w, "
                "rho_mix",
        "forward_ms_per_iteration": fwd_wall / K * 1e3,
        "forward_device_ms_per_iteration": fwd_dev / K * 1e3,
        "adjoint_and_forward_ms_per_iteration": ad_wall / K * 1e3,
        "peak_bytes": {"torch_tensors_above_start": torch_peak,
                       "checkpoints": K * len(LIN_FIELDS) * im * jm * pitch * 8,
                       "library_scratch": lib_scratch},
    }


def run_adjoint(args):
    """--workload adjoint: the adjoint section alone, as its own JSON line."""
    d = reference_state("dry", 0, None)
    if d is not None:
        P, _, _, _, grid, fields = model_inputs(d, "dry")
        data = STATE_RECIPE["dry"]
    else:
        P, _, _, _, grid, fields = synthetic_inputs("dry", 0)
        data = "synthetic (seeded dry state; the reference is not built here)"
    a = adjoint_section(P, grid, fields, args.steps)
    line = {"metric": a.pop("metric"), "value": a.pop("ratio"), "unit": "x", "n_gpus": 1,
            "steps": args.steps, "warmup": 2, "higher_is_better": False, "dtype": "f64",
            "data": data, "config": {"workload": "adjoint of whole dry iterations", "grid": "41x181x361"}, **a}
    print(json.dumps(line))


def run_cone(args):
    """--workload cone: the projection around the obstacle alone (cone_section, `steps` calls),
    as its own JSON line."""
    d = reference_state("dry", 0, None)
    if d is None:
        print(json.dumps({"workload": "cone", "unavailable": "needs the reference's initial state"}))
        return
    P, _, _, _, grid, fields = model_inputs(d, "dry")
    c = cone_section(P, grid, fields, calls=max(args.steps, 1))
    line = {"metric": "s per call of the in-loop projection around the obstacle (26 levels, two "
                      "solves each)", "value": c.pop("gpu_s_per_call"), "unit": "s/call",
            "n_gpus": 1, "steps": args.steps, "warmup": 0, "higher_is_better": False,
            "dtype": "f64", "data": STATE_RECIPE["dry"],
            "config": {"workload": "projection around the obstacle", "grid": "41x181x361"}, **c}
    print(json.dumps(line))


PROGNOSTIC = ("t", "u", "v", "w", "p_dyn", "h2o", "h2o_cloud", "h2o_ice", "h2s", "nh3",
              "nh3_cloud", "nh3_ice", "ch4", "ch4_cloud", "ch4_ice", "nh4sh", "tke", "dis")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the Poisson, adjoint and mixed-precision accuracy sections")
    ap.add_argument("--workload", default="phys", choices=["phys", "dry", "adjoint", "cone"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--grid", default=None,
                    help="IMxJMxKM of a smaller synthetic shell, for profiling only (the metric "
                         "is quoted on 41x181x361)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    args.warmup = max(args.warmup, 3)
    if args.workload == "adjoint":
        run_adjoint(args)
        return
    if args.workload == "cone":
        run_cone(args)
        return

    import numpy as np
    import torch

    from atjup_b200.params import FIELD_IDS, PREC_FP64, PREC_MIXED, SCALARS
    from atjup_b200.replicas import max_over_ranks, whole_job_seconds_per_step

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist = dist_mod
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    phys = args.workload == "phys"
    global IM, JM, KM, N_CELLS
    if args.grid:
        IM, JM, KM = (int(x) for x in args.grid.lower().split("x"))
        N_CELLS = IM * JM * KM
    d = None if args.grid else reference_state(args.workload, rank, dist)
    if d is not None:
        P, PH, MC, MCA, grid, fields = model_inputs(d, args.workload)
        data = STATE_RECIPE[args.workload]
    else:
        P, PH, MC, MCA, grid, fields = synthetic_inputs(args.workload, rank)
        data = ("synthetic (seeded; shapes and value ranges of the model's initial state"
                + (", full-physics recipe" if phys else "") + "; the reference is not built here)")
    m = build_model(P, PH, MC, MCA, grid, fields)
    prec0 = PREC_MIXED if args.precision == "mixed" else PREC_FP64
    m.set_precision(prec0)
    # events are recorded on the library's own stream; no torch stream is created, so the process
    # holds only the library's streams and each gets a hardware queue of its own
    stream = torch.cuda.ExternalStream(m.stream_handle())

    it = [0]

    def step():
        it[0] += 1
        m.step(it[0], it[0] == 1)

    def restart(prec, state=None):
        """the state back to the configuration's initial state (or `state`), iteration 1 next"""
        m.set_precision(prec)
        m.upload_state(fields if state is None else state)
        it[0] = 0

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

    def warm_and_time(prec):
        restart(prec)
        for _ in range(args.warmup):
            step()
        m.synchronize()
        if m.nonfinite_count() != 0:
            raise SystemExit("non-finite state after warm-up")
        return timed_region(args.steps)

    t_ms, per_class, launches, clk = warm_and_time(prec0)
    value = whole_job_seconds_per_step(t_ms / 1e3, args.steps, world)

    # ---- the same iterations in the mixed-precision RK step, from the same state ----
    mixed = None
    if phys and args.precision == "fp64":
        mt_ms, mper, _, mclk = warm_and_time(PREC_MIXED)
        mixed = {"value": whole_job_seconds_per_step(mt_ms / 1e3, args.steps, world),
                 "unit": UNIT, "ms_per_step": mt_ms / args.steps, "dtype": "f32+f64",
                 "precision": PREC_CONFIG["mixed"],
                 "stage_roofline": mper,
                 "device_ms_per_step_by_class": {k: round(v[0] / args.steps, 4) for k, v in
                                                 sorted(mper.items(), key=lambda kv: -kv[1][0])},
                 "clocks": mclk}
        if not args.no_extras:
            # accuracy: 200 iterations of each from the configuration's state, relative L2 per
            # field of the mixed run against the FP64 run
            # and the FP64 step's own sensitivity: FP64 from the state rounded once to FP32
            n_acc = 200
            prog = set(PROGNOSTIC) | {n + "n" for n in SCALARS}
            rounded = {k: (v.astype(np.float32).astype(np.float64) if k in prog else v)
                       for k, v in fields.items()}
            snaps = {}
            for key, prec, st in (("fp64", PREC_FP64, None), ("mixed", PREC_MIXED, None),
                                  ("fp64_rounded", PREC_FP64, rounded)):
                restart(prec, st)
                for _ in range(n_acc):
                    step()
                snaps[key] = {n: m.download(n) for n in PROGNOSTIC}

            def rel_l2(a, b):
                nb = float(np.linalg.norm(a))
                return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(b))
            rel = {n: rel_l2(snaps["fp64"][n], snaps["mixed"][n]) for n in PROGNOSTIC}
            sens = {n: rel_l2(snaps["fp64"][n], snaps["fp64_rounded"][n]) for n in PROGNOSTIC}
            mixed["rel_l2_vs_fp64_after_200"] = rel
            mixed["fp64_self_sensitivity_after_200"] = sens
            mixed["fields_above_1e-5"] = {k: {"mixed": v, "fp64_self_sensitivity": sens[k]}
                                          for k, v in rel.items() if v > 1e-5}
            mixed["accuracy_note"] = (
                "relative L2 per prognostic field of 200 mixed iterations against 200 FP64 "
                "iterations from the same state; fp64_self_sensitivity is the FP64 step started "
                "from that state rounded once to FP32, against the exact FP64 run: a field above "
                "1e-5 is one the model itself moves that far from an FP32 rounding of its input")

    # ---- end to end through the C ABI with pinned host buffers ----
    restart(prec0)
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
        "data": data,
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
    if world == 1 and not args.no_extras and not args.grid:
        line["poisson"] = poisson_section(m, stream)
    m.close()
    if world == 1 and not args.no_extras and not args.grid:
        dd = reference_state("dry", 0, None) if d is not None else None
        if dd is not None:
            Pd, _, _, _, gd, fd = model_inputs(dd, "dry")
        else:
            Pd, _, _, _, gd, fd = synthetic_inputs("dry", 0)
        line["adjoint"] = adjoint_section(Pd, gd, fd, 50)
        line["cone_projection"] = cone_section(Pd, gd, fd)
    if dist is not None:
        dist.barrier()
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline and not args.grid:
            line["cpu_baseline"] = cpu_baseline(args.workload)
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
