"""Python binding of the B200 C ABI (include/atjup_gpu.h) -- the host-side mirror of the
reference's model object for the time-step hot path.

The reference exposes the model as ``pyatjup.Jupiter`` (python/pyatjup.pyx.template:35-97) whose
``run()`` calls ``cJupiterModel::Run``; the hot path inside it is a sequence of member functions
(cJupiterModel.cpp:1032-1381). ``GpuModel`` exposes the same routines by their reference names,
on a device-resident state: ``pressure_solver()``, ``runge_kutta()``, ``bc_radius()`` ...,
``step()`` for one whole iteration. Fields move in and out as numpy arrays in the reference's
(i, j, k) order. There is no CPU fallback: construction fails if the CUDA library is missing or
no sm_100 device is present.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import params as _p

_LIB_PATH = Path(__file__).resolve().parent / "libatjup_gpu.so"
_lib = None


class AtjupError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"atjup_gpu error {code}: {msg}")
        self.code = code


def load_library() -> ctypes.CDLL:
    """Load libatjup_gpu.so (built by ``python -m atjup_b200.build``); raise if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise ImportError(f"{_LIB_PATH} is missing: build it with `python -m atjup_b200.build`")
    L = ctypes.CDLL(str(_LIB_PATH))
    vp, i32, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double
    L.atjup_gpu_last_error.restype = ctypes.c_char_p
    L.atjup_gpu_create.argtypes = [ctypes.POINTER(_p.AtjupParams), ctypes.POINTER(vp)]
    L.atjup_gpu_destroy.argtypes = [vp]
    L.atjup_gpu_set_stream.argtypes = [vp, vp]
    L.atjup_gpu_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.atjup_gpu_rk4_tlm.argtypes = [vp, ctypes.POINTER(vp)]
    L.atjup_gpu_copy_field.argtypes = [vp, i32, vp, i32]
    L.atjup_gpu_rk4_adjoint.argtypes = [vp, ctypes.POINTER(vp)]
    L.atjup_gpu_iteration_tlm.argtypes = [vp, i32, i32, i32, ctypes.POINTER(vp)]
    L.atjup_gpu_iteration_adjoint.argtypes = [vp, i32, i32, i32, ctypes.POINTER(vp)]
    L.atjup_gpu_iteration_adjoint_ckpt.argtypes = [vp, i32, i32, i32, ctypes.POINTER(vp),
                                                   ctypes.POINTER(vp)]
    L.atjup_gpu_set_stage_buffers.argtypes = [vp, ctypes.POINTER(vp)]
    L.atjup_gpu_set_grid.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.atjup_gpu_upload.argtypes = [vp, i32, vp]
    L.atjup_gpu_download.argtypes = [vp, i32, vp]
    L.atjup_gpu_field_ptr.argtypes = [vp, i32, ctypes.POINTER(vp), ctypes.POINTER(i32)]
    L.atjup_gpu_rk4_step.argtypes = [vp, i32]
    L.atjup_gpu_pressure_solve.argtypes = [vp, ctypes.POINTER(_p.AtjupSolveOpts),
                                           ctypes.POINTER(_p.AtjupSolveStats)]
    L.atjup_gpu_set_solve_rhs.argtypes = [vp, vp]
    L.atjup_gpu_bc.argtypes = [vp, i32]
    L.atjup_gpu_shapiro.argtypes = [vp, i32, i32, dbl, i32, i32]
    L.atjup_gpu_mixture_density.argtypes = [vp]
    L.atjup_gpu_balance_column_v.argtypes = [vp, ctypes.POINTER(dbl)]
    L.atjup_gpu_cone_project.argtypes = [vp]
    L.atjup_gpu_cone_stats.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i32), i32,
                                       ctypes.POINTER(i32)]
    L.atjup_gpu_step.argtypes = [vp, i32, i32, ctypes.POINTER(_p.AtjupSolveOpts)]
    L.atjup_gpu_nonfinite_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.atjup_gpu_synchronize.argtypes = [vp]
    L.atjup_params_default.argtypes = [ctypes.POINTER(_p.AtjupParams)]
    L.atjup_gpu_timing.argtypes = [vp, i32]
    L.atjup_gpu_timing_read.argtypes = [vp, i32, ctypes.POINTER(dbl), ctypes.POINTER(ctypes.c_int64)]
    L.atjup_gpu_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.atjup_gpu_satadj.argtypes = [vp, i32, ctypes.POINTER(_p.AtjupGasParams),
                                   ctypes.POINTER(_p.AtjupSatStats)]
    L.atjup_gpu_set_physics.argtypes = [vp, ctypes.POINTER(_p.AtjupPhysics), vp]
    L.atjup_gpu_upload_n.argtypes = [vp, i32, vp]
    L.atjup_gpu_download_n.argtypes = [vp, i32, vp]
    L.atjup_gpu_restore_scalars.argtypes = [vp]
    L.atjup_gpu_upload2d.argtypes = [vp, i32, vp]
    L.atjup_gpu_turbulence.argtypes = [vp]
    L.atjup_gpu_set_micro.argtypes = [vp, ctypes.POINTER(_p.AtjupMicro)]
    L.atjup_gpu_set_precision.argtypes = [vp, i32]
    L.atjup_gpu_upload_async.argtypes = [vp, i32, vp]
    L.atjup_gpu_apply_uploads.argtypes = [vp]
    L.atjup_gpu_download_async.argtypes = [vp, i32, vp]
    L.atjup_gpu_set_mca.argtypes = [vp, ctypes.POINTER(_p.AtjupMca)]
    L.atjup_gpu_mca.argtypes = [vp, ctypes.POINTER(_p.AtjupMcaStats)]
    L.atjup_gpu_save_state.argtypes = [vp, ctypes.c_char_p, i32, i32]
    L.atjup_gpu_load_state.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(i32), ctypes.POINTER(i32)]
    for n in ("radiation", "precipitation", "nh4sh_equilibrium", "chemistry", "clamp_species",
              "diagnostics"):
        getattr(L, "atjup_gpu_" + n).argtypes = [vp]
    L.atjup_gpu_download2d.argtypes = [vp, i32, vp]
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise AtjupError(rc, load_library().atjup_gpu_last_error().decode())


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class GpuModel:
    """Device-resident hot-path state of one model (one CUDA context, one stream)."""

    def __init__(self, params: _p.AtjupParams, grid: dict):
        self.L = load_library()
        self.P = params
        self.shape = (params.im, params.jm, params.km)
        self.ctx = ctypes.c_void_p()
        _check(self.L.atjup_gpu_create(ctypes.byref(params), ctypes.byref(self.ctx)))
        self._keep = {}
        self._phys = False
        self.set_grid(grid)

    def close(self):
        if self.ctx:
            self.L.atjup_gpu_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- grid and fields ----
    def set_grid(self, g: dict):
        im, jm, km = self.shape
        rad = np.ascontiguousarray(g["rad"], np.float64)
        the = np.ascontiguousarray(g["the"], np.float64)
        solid = np.ascontiguousarray(g["solid"], np.uint8).reshape(im, jm, km)
        topo = np.ascontiguousarray(g["topo"], np.int32).reshape(jm, km)
        cv = g.get("cell_vbar0")
        cu = g.get("cell_ubar0")
        cv = None if cv is None else np.ascontiguousarray(cv, np.float64)
        cu = None if cu is None else np.ascontiguousarray(cu, np.float64)
        _check(self.L.atjup_gpu_set_grid(self.ctx, _ptr(rad), _ptr(the), _ptr(solid), _ptr(topo),
                                         _ptr(cv) if cv is not None else None,
                                         _ptr(cu) if cu is not None else None))

    def upload(self, name: str, a) -> None:
        a = np.ascontiguousarray(a, np.float64).reshape(self.shape)
        _check(self.L.atjup_gpu_upload(self.ctx, _p.FIELD_IDS[name], _ptr(a)))

    def download(self, name: str) -> np.ndarray:
        out = np.empty(self.shape)
        _check(self.L.atjup_gpu_download(self.ctx, _p.FIELD_IDS[name], _ptr(out)))
        return out

    def upload_async(self, name: str, a) -> None:
        """atjup_gpu_upload_async: queue a field's upload (a contiguous float64 array that must stay
        alive and unchanged until synchronize())."""
        assert a.dtype == np.float64 and a.flags.c_contiguous and a.size == int(np.prod(self.shape))
        _check(self.L.atjup_gpu_upload_async(self.ctx, _p.FIELD_IDS[name], _ptr(a)))

    def apply_uploads(self) -> None:
        _check(self.L.atjup_gpu_apply_uploads(self.ctx))

    def download_async(self, name: str, out) -> None:
        """atjup_gpu_download_async into out (contiguous float64; valid after synchronize())."""
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == int(np.prod(self.shape))
        _check(self.L.atjup_gpu_download_async(self.ctx, _p.FIELD_IDS[name], _ptr(out)))

    def upload_state(self, fields: dict) -> None:
        """Upload every known field in fields; with physics set, also the time-level-n copies
        of the transported scalars (key name + "n", else the live field) and vel_star."""
        for n, a in fields.items():
            if n in _p.FIELD_IDS and a is not None:
                self.upload(n, a)
        if self._phys:
            for n in _p.SCALARS:
                src = fields.get(n + "n", fields.get(n))
                if src is not None:
                    self.upload_n(n, src)
            if fields.get("vel_star") is not None:
                self.upload2d("vel_star", fields["vel_star"])

    # ---- full physics ----
    def set_physics(self, phys: "_p.AtjupPhysics | None", layer_heights=None):
        """atjup_gpu_set_physics: species and k*, omega* join the RK4 step (None: dynamics only).
        layer_heights: the model's m_layer_heights [km] per level (float32)."""
        if phys is None:
            _check(self.L.atjup_gpu_set_physics(self.ctx, None, None))
            self._phys = False
            return
        lh = np.ascontiguousarray(layer_heights, np.float32)
        assert lh.shape == (self.shape[0],)
        _check(self.L.atjup_gpu_set_physics(self.ctx, ctypes.byref(phys), _ptr(lh)))
        self._phys = True

    def set_precision(self, precision: int) -> None:
        """The RK step's precision: params.PREC_FP64, or params.PREC_MIXED (FP32 stage buffers and
        accumulators, FP32 species and closure right-hand sides)."""
        _check(self.L.atjup_gpu_set_precision(self.ctx, int(precision)))

    def set_mca(self, mca: "_p.AtjupMca | None") -> None:
        """atjup_gpu_set_mca: the moist convective adjustment of the iteration (None: off)."""
        _check(self.L.atjup_gpu_set_mca(self.ctx, ctypes.byref(mca) if mca is not None else None))

    def mca(self) -> dict:
        """atjup_gpu_mca: one moist convective adjustment of the device state; its counters."""
        st = _p.AtjupMcaStats()
        _check(self.L.atjup_gpu_mca(self.ctx, ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in st._fields_ if n != "pad"}

    # ---- restart files ----
    def save_state(self, path, iter_n: int, carried: int = 1) -> None:
        """atjup_gpu_save_state: the reference's restart file of the state between steps -- JUP2
        (carried = 1), JUP1 (0), or JUP2 with the trailer of the five arrays the reference's list
        omits (2)."""
        _check(self.L.atjup_gpu_save_state(self.ctx, str(path).encode(), int(iter_n), int(carried)))

    def load_state(self, path) -> tuple[int, int]:
        """atjup_gpu_load_state: (iteration in the header, carried: 0 JUP1, 1 JUP2, 2 JUP2 with
        the trailer)."""
        it, car = ctypes.c_int32(), ctypes.c_int32()
        _check(self.L.atjup_gpu_load_state(self.ctx, str(path).encode(), ctypes.byref(it),
                                           ctypes.byref(car)))
        return it.value, car.value

    def upload_n(self, name: str, a) -> None:
        a = np.ascontiguousarray(a, np.float64).reshape(self.shape)
        _check(self.L.atjup_gpu_upload_n(self.ctx, _p.FIELD_IDS[name], _ptr(a)))

    def download_n(self, name: str) -> np.ndarray:
        out = np.empty(self.shape)
        _check(self.L.atjup_gpu_download_n(self.ctx, _p.FIELD_IDS[name], _ptr(out)))
        return out

    def turbulence(self) -> None:
        """Turbulence<cJupiterModel>::run + turbWallOmega (Turbulence.h:307-882,
        cJupiterModel.cpp:360-377)."""
        _check(self.L.atjup_gpu_turbulence(self.ctx))

    def set_micro(self, micro: "_p.AtjupMicro | None") -> None:
        """atjup_gpu_set_micro: the loop's radiation, precipitation and chemistry."""
        _check(self.L.atjup_gpu_set_micro(self.ctx, ctypes.byref(micro) if micro is not None else None))

    def radiation(self) -> None:
        """Radiation<cJupiterModel>::run (Radiation.h:251-487)."""
        _check(self.L.atjup_gpu_radiation(self.ctx))

    def precipitation(self) -> None:
        """Precipitation<cJupiterModel>::run (Precipitation.h:191-445)."""
        _check(self.L.atjup_gpu_precipitation(self.ctx))

    def diagnostics(self) -> None:
        """cJupiterModel::Forces and Latent_Heat: the force densities and the latent and sensible
        heating (output fields)"""
        _check(self.L.atjup_gpu_diagnostics(self.ctx))

    def nh4sh_eq(self) -> None:
        """ChemistryJup::EquilibriumNH4SH("loop") (ChemistryJup.h:291-373)."""
        _check(self.L.atjup_gpu_nh4sh_equilibrium(self.ctx))

    def chemistry(self) -> None:
        """The loop's chemistry block (ChemistryJup.h:59-543, FluxLimiter.h)."""
        _check(self.L.atjup_gpu_chemistry(self.ctx))

    def clamp_species(self) -> None:
        """clampNegativeSpecies (FileIO_Jup.cpp:494-548)."""
        _check(self.L.atjup_gpu_clamp_species(self.ctx))

    def restore_scalars(self) -> None:
        _check(self.L.atjup_gpu_restore_scalars(self.ctx))

    def upload2d(self, name: str, a) -> None:
        a = np.ascontiguousarray(a, np.float64).reshape(self.shape[1:])
        _check(self.L.atjup_gpu_upload2d(self.ctx, {"vel_star": _p.F2_VEL_STAR}[name], _ptr(a)))

    def download2d(self, name: str) -> np.ndarray:
        out = np.empty(self.shape[1:])
        _check(self.L.atjup_gpu_download2d(self.ctx, {"vel_star": _p.F2_VEL_STAR}[name], _ptr(out)))
        return out

    def field_ptr(self, name: str):
        p = ctypes.c_void_p()
        pitch = ctypes.c_int32()
        _check(self.L.atjup_gpu_field_ptr(self.ctx, _p.FIELD_IDS[name], ctypes.byref(p),
                                          ctypes.byref(pitch)))
        return p.value, pitch.value

    def set_stream(self, stream_handle: int | None):
        _check(self.L.atjup_gpu_set_stream(self.ctx, ctypes.c_void_p(stream_handle or 0)))

    def _ptrs(self, tensors):
        """device pointers of float64 CUDA tensors of shape (im, jm, pitch), contiguous"""
        shape = (self.P.im, self.P.jm, self.field_ptr("t")[1])
        ptrs = (ctypes.c_void_p * len(tensors))()
        for q, x in enumerate(tensors):
            if (not x.is_cuda or str(x.dtype) != "torch.float64" or tuple(x.shape) != shape
                    or not x.is_contiguous()):
                raise ValueError(f"expected contiguous float64 CUDA tensors of shape {shape}")
            ptrs[q] = x.data_ptr()
        return ptrs

    def set_state_tensors(self, tensors, names=("t", "u", "v", "w"), wait=True):
        """copy (im, jm, pitch) float64 CUDA tensors into the named fields; with wait False the
        call returns once the copies are queued (the library's later work is ordered after them,
        but the tensors must not be rewritten before the next synchronize)"""
        import torch
        ptrs = self._ptrs(tensors)
        torch.cuda.current_stream().synchronize()
        for q, n in enumerate(names):
            _check(self.L.atjup_gpu_copy_field(self.ctx, _p.FIELD_IDS[n], ptrs[q], 1))
        if wait:
            self.synchronize()

    def state_tensors(self, names=("t", "u", "v", "w")):
        """the named fields as new (im, jm, pitch) float64 CUDA tensors"""
        import torch
        out = [torch.empty((self.P.im, self.P.jm, self.field_ptr("t")[1]), dtype=torch.float64,
                           device="cuda") for _ in names]
        ptrs = self._ptrs(out)
        torch.cuda.current_stream().synchronize()
        for q, n in enumerate(names):
            _check(self.L.atjup_gpu_copy_field(self.ctx, _p.FIELD_IDS[n], ptrs[q], 0))
        self.synchronize()
        return out

    def _on_tensors(self, fn, tensors):
        # the library issues on its own stream: torch's writes of the inputs must be done before
        # it reads them, and its results before torch reads them
        import torch
        ptrs = self._ptrs(tensors)
        torch.cuda.current_stream().synchronize()
        _check(fn(self.ctx, ptrs))
        self.synchronize()

    def rk4_tlm(self, dt, du, dv, dw):
        """tangent-linear of one RK4 step of the dry dynamics about the current state, in place
        on four (im, jm, pitch) float64 CUDA tensors (t, u, v, w)"""
        self._on_tensors(self.L.atjup_gpu_rk4_tlm, (dt, du, dv, dw))

    def rk4_adjoint(self, at, au, av, aw):
        """adjoint of one RK4 step of the dry dynamics about the current state, in place: the
        adjoint of the step's result in, of its input out"""
        self._on_tensors(self.L.atjup_gpu_rk4_adjoint, (at, au, av, aw))

    def iteration_tlm(self, tensors, iter_n: int, first: bool = False, parts: int = _p.LIN_ALL):
        """tangent-linear of one dry iteration (atjup_gpu_iteration_tlm) about the current state,
        in place on nine (im, jm, pitch) float64 CUDA tensors in the order of LIN_FIELDS"""
        self._on_tensors(lambda ctx, ptrs: self.L.atjup_gpu_iteration_tlm(
            ctx, int(iter_n), int(first), int(parts), ptrs), tensors)

    def iteration_adjoint(self, tensors, iter_n: int, first: bool = False,
                          parts: int = _p.LIN_ALL):
        """adjoint of one dry iteration (atjup_gpu_iteration_adjoint) about the current state, in
        place: the adjoint of the iteration's output in, of its input out (LIN_FIELDS order)"""
        self._on_tensors(lambda ctx, ptrs: self.L.atjup_gpu_iteration_adjoint(
            ctx, int(iter_n), int(first), int(parts), ptrs), tensors)

    def iteration_adjoint_ckpt(self, tensors, stages, iter_n: int, first: bool = False,
                               parts: int = _p.LIN_ALL):
        """iteration_adjoint with the RK step's stage inputs kept by the forward iteration
        (set_stage_buffers): twelve (im, jm, pitch) float64 CUDA tensors, X1, X2, X3 of
        t, u, v, w (atjup_gpu_iteration_adjoint_ckpt)"""
        sp = self._ptrs(stages)
        self._on_tensors(lambda ctx, ptrs: self.L.atjup_gpu_iteration_adjoint_ckpt(
            ctx, int(iter_n), int(first), int(parts), ptrs, sp), tensors)

    def set_stage_buffers(self, stages):
        """the following dry FP64 RK steps write their stage inputs X1, X2, X3 of t, u, v, w into
        the twelve (im, jm, pitch) float64 CUDA tensors `stages`; None: the context's own buffers
        (atjup_gpu_set_stage_buffers)"""
        import torch
        if stages is None:
            _check(self.L.atjup_gpu_set_stage_buffers(self.ctx, None))
            return
        torch.cuda.current_stream().synchronize()   # the tensors' memory is free on torch's stream
        _check(self.L.atjup_gpu_set_stage_buffers(self.ctx, self._ptrs(stages)))

    def stream_handle(self) -> int:
        """the cudaStream_t the context issues its work on, as an integer"""
        s = ctypes.c_void_p()
        _check(self.L.atjup_gpu_stream(self.ctx, ctypes.byref(s)))
        return s.value or 0

    # ---- the hot path, by the reference's routine names ----
    def runge_kutta(self, iter_n: int = 0):
        """cJupiterModel::RungeKuttaJup (RungeKutta_Jup_Turb.cpp:261-583)."""
        _check(self.L.atjup_gpu_rk4_step(self.ctx, iter_n))

    def pressure_solver(self, mode=_p.SOLVE_SWEEPS, sweeps=None, omega=1.0, rel_tol=1e-10,
                        max_iter=2000, precision=_p.PREC_FP64, external_rhs=False,
                        allow_not_converged=False):
        """PressureSolverJup::run (PressureSolver.h:144-766); returns AtjupSolveStats. With
        allow_not_converged an iteration cap reached (ATJUP_ERR_NOT_CONVERGED) returns the stats
        instead of raising."""
        o = _p.AtjupSolveOpts(mode, sweeps if sweeps is not None else self.P.press_sweeps,
                              max_iter, precision, rel_tol, omega, int(external_rhs))
        st = _p.AtjupSolveStats()
        rc = self.L.atjup_gpu_pressure_solve(self.ctx, ctypes.byref(o), ctypes.byref(st))
        if not (allow_not_converged and rc == 4):
            _check(rc)
        return st

    def set_solve_rhs(self, b) -> None:
        b = np.ascontiguousarray(b, np.float64).reshape(self.shape)
        _check(self.L.atjup_gpu_set_solve_rhs(self.ctx, _ptr(b)))

    def bc(self, which=_p.BC_ALL):
        """BC_Jup::bcRadius / bcTheta / bcPhi / bcSolidGround (BC_Jup.h:185-658)."""
        _check(self.L.atjup_gpu_bc(self.ctx, which))

    def shapiro(self, name: str, order: int, strength=1.0, passes=1, use_topo=True):
        """JupiterUtils::damp_wiggles / damp_wiggles_ho (lib/Utils.cpp:227-453)."""
        _check(self.L.atjup_gpu_shapiro(self.ctx, _p.FIELD_IDS[name], order, strength, passes,
                                        int(use_topo)))

    def mixture_density(self):
        """cJupiterModel::computeMixtureDensity (InitValues_Jup.cpp:717-740)."""
        _check(self.L.atjup_gpu_mixture_density(self.ctx))

    def balance_column_v(self) -> float:
        """cJupiterModel::balanceColumnV (InitValues_Jup.cpp:1500-1538); returns the shift."""
        s = ctypes.c_double()
        _check(self.L.atjup_gpu_balance_column_v(self.ctx, ctypes.byref(s)))
        return s.value

    def cone_project(self):
        """cJupiterModel::projectAroundObstacle(in_loop = true) (InitValues_Jup.cpp:1595-1822):
        one call, warm-started from the previous call's phi of each level and solve."""
        _check(self.L.atjup_gpu_cone_project(self.ctx))

    def cone_stats(self):
        """(levels i, sweeps [levels, 2]) of the last projection: SOR sweeps of the divergence
        solve (0 when off) and of the wall-flux solve per level."""
        n = ctypes.c_int32()
        _check(self.L.atjup_gpu_cone_stats(self.ctx, None, None, 0, ctypes.byref(n)))
        lv = (ctypes.c_int32 * max(n.value, 1))()
        sw = (ctypes.c_int32 * max(2 * n.value, 1))()
        _check(self.L.atjup_gpu_cone_stats(self.ctx, lv, sw, n.value, ctypes.byref(n)))
        return (np.array(lv[:n.value], dtype=np.int32),
                np.array(sw[:2 * n.value], dtype=np.int32).reshape(n.value, 2))

    def satadj(self, gas: str, gp: _p.AtjupGasParams, stats: bool = True):
        """SaturationAdjustmentJup(*this).run(gas, ...) (SaturationAdjustment.h:255-746) on the
        device fields of gas ("H2O", "NH3" or "CH4"); returns (adjusted, not converged, dry
        exits) when stats, else None (no synchronisation)."""
        st = _p.AtjupSatStats() if stats else None
        _check(self.L.atjup_gpu_satadj(self.ctx, _p.GAS_IDS[gas], ctypes.byref(gp),
                                       ctypes.byref(st) if st is not None else None))
        return (st.adjusted, st.not_converged, st.dry_exits) if st is not None else None

    def step(self, iter_n: int, first: bool = False, solve: _p.AtjupSolveOpts | None = None):
        """One iteration of cJupiterModel::Run's loop (cJupiterModel.cpp:1032-1381)."""
        _check(self.L.atjup_gpu_step(self.ctx, iter_n, int(first),
                                     ctypes.byref(solve) if solve is not None else None))

    def nonfinite_count(self) -> int:
        n = ctypes.c_int64()
        rc = self.L.atjup_gpu_nonfinite_count(self.ctx, ctypes.byref(n))
        if rc not in (0, 5):
            _check(rc)
        return n.value

    def synchronize(self):
        _check(self.L.atjup_gpu_synchronize(self.ctx))

    # ---- instrumentation ----
    TIMING_CLASSES = ("rk_stage", "rk_aux", "pressure", "bc", "shapiro", "balance_v",
                      "mixture", "solver", "satadj", "species", "closure", "turb", "micro", "mca",
                      "rk_group", "cone")

    def timing(self, on: bool):
        """Start (reset) or stop CUDA-event timing of the library's kernel launches."""
        _check(self.L.atjup_gpu_timing(self.ctx, int(on)))

    def timing_read(self, cls: int):
        """(total ms, launches) of one kernel class since timing(True)."""
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        _check(self.L.atjup_gpu_timing_read(self.ctx, cls, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def launch_count(self) -> int:
        n = ctypes.c_int64()
        _check(self.L.atjup_gpu_launch_count(self.ctx, ctypes.byref(n)))
        return n.value

    @staticmethod
    def _rc(rc: int):
        _check(rc)
