"""Test-side access to the CPU oracle (oracle/liboracle.so) and to the reference harness
(oracle/_ref/libatjup_ref.so). Test infrastructure only: the product never imports this."""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

from atjup_b200.params import AtjupParams, resolve_params

import sys as _sys
_sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
from ref_model import RefModel  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]
ORACLE_SO = ROOT / "oracle" / "liboracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "libatjup_ref.so"

# The dry configuration: obstacle on, microphysics / radiation / turbulence / MCA / cone
# projection off, in-loop 4th-order Shapiro on u, v, w (the dry configuration's knobs).
DRY_ENV = {
    "ATJUP_NO_SEAMOUNT": "0", "ATJUP_PRECIP": "0", "ATJUP_RADIATION": "0", "ATJUP_TURB": "0",
    "ATJUP_MCA": "0", "ATJUP_NH4SH_EQ": "0", "ATJUP_CONE_PROJ_STRIDE": "0",
    "ATJUP_VEL_SHAPIRO_ORDER": "4", "ATJUP_VEL_SHAPIRO_INLOOP": "1",
    "ATJUP_RESTART_STRIDE": "0", "ATJUP_VTK_STRIDE": "100000", "ATJUP_PANORAMA_STRIDE": "100000",
}

# Full physics in the RK step: the dry knobs with the k_omega_SST closure switched on.
PHYS_ENV = {**DRY_ENV, "ATJUP_TURB": "1"}
# The full-physics iteration: the closure, radiation, precipitation and the NH4SH equilibrium on
# (their reference defaults); moist convective adjustment and the cone projection stay off.
MOIST_ENV = {**PHYS_ENV, "ATJUP_PRECIP": "1", "ATJUP_RADIATION": "1", "ATJUP_NH4SH_EQ": "1"}
# the reference's default full physics: MOIST_ENV with the moist convective adjustment every iteration
MCA_ENV = {**MOIST_ENV, "ATJUP_MCA": "1"}

DYN_FIELDS = ["t", "u", "v", "w", "p_dyn", "p_hydro", "p_stat", "rho_mix", "wall_nue",
              "aux_u", "aux_v", "aux_w"]


def build_oracle() -> Path:
    if not ORACLE_SO.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, capture_output=True)
    return ORACLE_SO


_P = ctypes.POINTER


class OraGrid(ctypes.Structure):
    _fields_ = [("rad", _P(ctypes.c_double)), ("the", _P(ctypes.c_double)),
                ("solid", _P(ctypes.c_uint8)), ("topo", _P(ctypes.c_int32)),
                ("cell_vbar0", _P(ctypes.c_double)), ("cell_ubar0", _P(ctypes.c_double))]


_STATE_NAMES = ["t", "u", "v", "w", "tn", "un", "vn", "wn", "p_dyn", "p_hydro", "p_stat",
                "rho_mix", "wall_nue", "nue", "p_baro", "aux_u", "aux_v", "aux_w",
                "acc_t", "acc_u", "acc_v", "acc_w", "rhs_t", "rhs_u", "rhs_v", "rhs_w",
                "Q_rad", "Q_precip", "buoy_ref"]


class OraState(ctypes.Structure):
    _fields_ = [(n, _P(ctypes.c_double)) for n in _STATE_NAMES]


def _dp(a):
    return a.ctypes.data_as(_P(ctypes.c_double)) if a is not None else None


class Oracle:
    """Holds a grid + state as numpy arrays and runs oracle routines on them in place."""

    def __init__(self, params: AtjupParams, grid: dict, fields: dict):
        self.lib = ctypes.CDLL(str(build_oracle()))
        self.P = params
        im, jm, km = params.im, params.jm, params.km
        self.shape = (im, jm, km)
        self.g = {k: np.ascontiguousarray(v) for k, v in grid.items()}
        self.g["rad"] = self.g["rad"].astype(np.float64)
        self.g["the"] = self.g["the"].astype(np.float64)
        self.g["solid"] = self.g["solid"].astype(np.uint8)
        self.g["topo"] = self.g["topo"].astype(np.int32)
        self.G = OraGrid(_dp(self.g["rad"]), _dp(self.g["the"]),
                         self.g["solid"].ctypes.data_as(_P(ctypes.c_uint8)),
                         self.g["topo"].ctypes.data_as(_P(ctypes.c_int32)),
                         _dp(self.g.get("cell_vbar0")), _dp(self.g.get("cell_ubar0")))
        self.f = {}
        for n in _STATE_NAMES:
            if n == "buoy_ref":
                self.f[n] = np.zeros(im)
            elif n in fields and fields[n] is not None:
                self.f[n] = np.ascontiguousarray(fields[n], dtype=np.float64).reshape(self.shape).copy()
            elif n in ("nue", "p_baro", "Q_rad", "Q_precip"):
                self.f[n] = None
            else:
                self.f[n] = np.zeros(self.shape)
        for a, b in (("tn", "t"), ("un", "u"), ("vn", "v"), ("wn", "w")):
            if a not in fields:
                self.f[a][...] = self.f[b]
        self.S = OraState(*[_dp(self.f[n]) for n in _STATE_NAMES])
        self.lib.ora_balance_column_v.restype = ctypes.c_double

    def call(self, name, *args):
        fn = getattr(self.lib, name)
        return fn(ctypes.byref(self.P), ctypes.byref(self.G), ctypes.byref(self.S), *args)

    def rk4(self):
        self.call("ora_rk4")

    def iteration(self, iter_n, first, sweeps=1):
        self.call("ora_iteration_dry", ctypes.c_int(iter_n), ctypes.c_int(first), ctypes.c_int(sweeps))

    def pressure(self, sweeps=1, omega=1.0, b=None):
        self.call("ora_pressure_sweeps", ctypes.c_int(sweeps), ctypes.c_double(omega),
                  _dp(b) if b is not None else None)

    def shapiro(self, name, order, strength=1.0, passes=1, use_topo=1):
        self.lib.ora_shapiro(ctypes.byref(self.P), ctypes.byref(self.G), _dp(self.f[name]),
                             ctypes.c_int(order), ctypes.c_double(strength), ctypes.c_int(passes),
                             ctypes.c_int(use_topo))

    def cone_project(self):
        """One in-loop projection around the obstacle (ora_cone_project), warm-started from the
        previous call on this object; returns the sweep counts [levels, 2]."""
        if not hasattr(self, "_cone_phi"):
            self._cone_phi = (np.zeros(self.shape), np.zeros(self.shape))
        sw = np.zeros(2 * self.shape[0], dtype=np.int32)
        n = self.call("ora_cone_project", _dp(self._cone_phi[0]), _dp(self._cone_phi[1]),
                      sw.ctypes.data_as(_P(ctypes.c_int32)))
        return sw[:2 * n].reshape(n, 2)

    def apply_A(self, p):
        out = np.zeros(self.shape)
        pp = np.ascontiguousarray(p, dtype=np.float64)
        self.lib.ora_pressure_apply(ctypes.byref(self.P), ctypes.byref(self.G), _dp(pp), _dp(out))
        return out

    def source(self):
        out = np.zeros(self.shape)
        self.call("ora_pressure_source", _dp(out))
        return out


class Reference(RefModel):
    """The unmodified reference (oracle/_ref/libatjup_ref.so), one model per process, with the
    conversions the tests need (AtjupParams, grid and field dicts)."""

    def params(self, env: dict | None = None) -> AtjupParams:
        """AtjupParams with the model's own constants (the knobs resolved from env)."""
        consts = {n: self.scalar(n) for n in ("dt", "re", "pr", "g", "omega", "u_0", "t_ref",
                                              "L_atm", "r_mix", "R_mix", "cp_mix", "Coriolis",
                                              "centrifugal", "buoyancy")}
        im, jm, km = self.shape
        return resolve_params(env if env is not None else os.environ, im=im, jm=jm, km=km,
                              constants=consts)

    def grid(self) -> dict:
        im, jm, km = self.shape
        g = {"rad": self.get1("rad"), "the": self.get1("the"),
             "solid": (self.get("SeaMount") == 1.0).astype(np.uint8), "topo": self.topo()}
        if self.scalar("cell_hold") == 1.0:
            g["cell_vbar0"] = self.get1("cell_vbar0")
            g["cell_ubar0"] = self.get1("cell_ubar0")
        return g

    def fields(self, names=DYN_FIELDS) -> dict:
        out = {n: self.get(n) for n in names}
        if self.scalar("has_p_baro") == 1.0:
            out["p_baro"] = self.get1("p_baro").reshape(self.shape)
        return out


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


def oracle_satadj(params: AtjupParams, grid: dict, gas, t, p_stat, rho_mix, c, cloud, ice):
    """ora_satadj on float64 C-contiguous (i, j, k) arrays, in place on t, c, cloud, ice.
    Returns (adjusted, not_converged, dry_exits)."""
    lib = ctypes.CDLL(str(build_oracle()))
    solid = np.ascontiguousarray(grid["solid"], dtype=np.uint8)
    G = OraGrid(None, None, solid.ctypes.data_as(_P(ctypes.c_uint8)), None, None, None)
    for a in (t, p_stat, rho_mix, c, cloud, ice):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    counts = (ctypes.c_longlong * 3)()
    lib.ora_satadj(ctypes.byref(params), ctypes.byref(G), ctypes.byref(gas), _dp(t), _dp(p_stat),
                   _dp(rho_mix), _dp(c), _dp(cloud), _dp(ice), counts)
    return tuple(counts)


class OraPhys(ctypes.Structure):
    _D = _P(ctypes.c_double)
    _fields_ = [("q", _D * 11), ("qn", _D * 11), ("acc_q", _D * 11), ("rhs_q", _D * 11),
                ("tke", _D), ("dis", _D), ("tken", _D), ("disn", _D), ("acc_tke", _D),
                ("acc_dis", _D), ("rhs_tke", _D), ("rhs_dis", _D), ("s_precip", _D * 9),
                ("massflux_h2s", _D), ("massflux_nh3", _D), ("massflux_nh4sh", _D),
                ("fluxlim_nh4sh", _D), ("prod", _D), ("tke_source", _D), ("dis_source", _D),
                ("vel_star", _D), ("nue_out", _D), ("layer_heights", _P(ctypes.c_float)),
                ("difflux", _D * 3)]


def oracle_rk4_phys(params, phys, grid: dict, fields: dict) -> dict:
    """ora_rk4_phys on copies of fields (dynamics as for Oracle, plus the species, k*, omega*,
    their *n copies, the sources, nue, vel_star [jm, km] and layer_heights [im] float32).
    Returns every field after the step."""
    from atjup_b200.params import S_PRECIP, SCALARS, SPECIES
    o = Oracle(params, grid, fields)
    shape = o.shape
    keep = {}

    def arr(name, default_zero=True):
        if name in fields and fields[name] is not None:
            a = np.ascontiguousarray(fields[name], dtype=np.float64).reshape(shape).copy()
        else:
            a = np.zeros(shape)
        keep[name] = a
        return a

    for n in SCALARS:
        arr(n)
        keep[n + "n"] = np.ascontiguousarray(fields.get(n + "n", fields[n]), dtype=np.float64).reshape(shape).copy()
        keep["acc_" + n] = np.zeros(shape)
        keep["rhs_" + n] = np.zeros(shape)
    for n in S_PRECIP + ("massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh"):
        arr(n)
    for n in ("prod", "tke_source", "dis_source"):
        arr(n)       # cells the step does not visit keep their values
    vs = np.ascontiguousarray(fields.get("vel_star", np.zeros(shape[1:])), dtype=np.float64).reshape(shape[1:]).copy()
    lh = np.ascontiguousarray(fields["layer_heights"], dtype=np.float32).copy()
    keep["vel_star"], keep["layer_heights"] = vs, lh
    D = _P(ctypes.c_double)
    X = OraPhys()
    for s_, n in enumerate(SPECIES):
        X.q[s_] = _dp(keep[n])
        X.qn[s_] = _dp(keep[n + "n"])
        X.acc_q[s_] = _dp(keep["acc_" + n])
        X.rhs_q[s_] = _dp(keep["rhs_" + n])
    for a in ("tke", "dis"):
        setattr(X, a, _dp(keep[a]))
        setattr(X, a + "n", _dp(keep[a + "n"]))
        setattr(X, "acc_" + a, _dp(keep["acc_" + a]))
        setattr(X, "rhs_" + a, _dp(keep["rhs_" + a]))
    for s_, n in enumerate(S_PRECIP):
        X.s_precip[s_] = _dp(keep[n])
    for n in ("massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "prod",
              "tke_source", "dis_source", "vel_star"):
        setattr(X, n, _dp(keep[n]))
    X.layer_heights = lh.ctypes.data_as(_P(ctypes.c_float))
    X.nue_out = _dp(o.f["nue"]) if o.f.get("nue") is not None else None
    o.lib.ora_rk4_phys(ctypes.byref(params), ctypes.byref(phys), ctypes.byref(o.G),
                       ctypes.byref(o.S), ctypes.byref(X))
    out = {n: o.f[n] for n in ("t", "u", "v", "w", "p_hydro", "aux_u", "aux_v", "aux_w", "buoy_ref")}
    out.update({n: keep[n] for n in SCALARS + ("prod", "tke_source", "dis_source")})
    return out


def oracle_turbulence(params, phys, grid: dict, fields: dict) -> dict:
    """ora_turbulence on copies of fields (u, v, w, t, tke, dis, tken, disn, nue, prod,
    tke_source, dis_source, vel_star, layer_heights). Returns the fields it writes."""
    o = Oracle(params, grid, fields)
    shape = o.shape
    keep = {}
    for n in ("tke", "dis", "nue", "prod", "tke_source", "dis_source"):
        keep[n] = np.ascontiguousarray(fields[n], dtype=np.float64).reshape(shape).copy()
    for n in ("tke", "dis"):
        keep[n + "n"] = np.ascontiguousarray(fields.get(n + "n", fields[n]), dtype=np.float64).reshape(shape).copy()
    keep["vel_star"] = np.ascontiguousarray(fields["vel_star"], dtype=np.float64).reshape(shape[1:]).copy()
    lh = np.ascontiguousarray(fields["layer_heights"], dtype=np.float32).copy()
    X = OraPhys()
    for n in ("tke", "dis", "tken", "disn", "prod", "tke_source", "dis_source", "vel_star"):
        setattr(X, n, _dp(keep[n]))
    X.nue_out = _dp(keep["nue"])
    X.layer_heights = lh.ctypes.data_as(_P(ctypes.c_float))
    o.lib.ora_turbulence(ctypes.byref(params), ctypes.byref(phys), ctypes.byref(o.G),
                         ctypes.byref(o.S), ctypes.byref(X))
    return keep


def oracle_bc(params, grid: dict, fields: dict, steps=("radius", "theta", "phi", "solid"),
              physics=True) -> dict:
    """The boundary passes in order on copies of fields; returns {step: {field: array}} after
    each step. physics=False: the dynamics fields only (ora_bc_*)."""
    from atjup_b200.params import SPECIES
    o = Oracle(params, grid, fields)
    shape = o.shape
    keep = {}
    X = None
    if physics:
        names = list(SPECIES) + ["tke", "dis", "tken", "disn", "nue", "prod", "tke_source",
                                 "dis_source", "massflux_h2s", "massflux_nh3", "massflux_nh4sh",
                                 "fluxlim_nh4sh"]
        for n in names:
            keep[n] = np.ascontiguousarray(fields[n], dtype=np.float64).reshape(shape).copy()
        X = OraPhys()
        for s_, n in enumerate(SPECIES):
            X.q[s_] = _dp(keep[n])
        for n in ("tke", "dis", "tken", "disn", "prod", "tke_source", "dis_source",
                  "massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh"):
            setattr(X, n, _dp(keep[n]))
        X.nue_out = _dp(keep["nue"])
    out = {}
    for step in steps:
        fn = getattr(o.lib, f"ora_bc_{step}_x")
        fn(ctypes.byref(params), ctypes.byref(o.G), ctypes.byref(o.S),
           ctypes.byref(X) if X is not None else None)
        snap = {n: o.f[n].copy() for n in ("t", "u", "v", "w", "p_stat", "p_dyn")}
        snap.update({n: a.copy() for n, a in keep.items()})
        out[step] = snap
    return out


MICRO_SPECIES_SOURCES = ("S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice", "S_precip_nh3",
                         "S_precip_nh3_cloud", "S_precip_nh3_ice", "S_precip_ch4",
                         "S_precip_ch4_cloud", "S_precip_ch4_ice")
MICRO_DIAGNOSTICS = ("CoriolisForce", "CentrifugalForce", "BuoyancyForce", "PresGradForce",
                     "Q_Latent", "Q_Sensible")
MICRO_FIELDS = ("t", "Q_rad", "Q_precip") + MICRO_SPECIES_SOURCES + (
    "massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "difflux_h2s",
    "difflux_nh3", "difflux_nh4sh") + MICRO_DIAGNOSTICS


def oracle_micro(params, micro, grid: dict, fields: dict, steps) -> dict:
    """The microphysics routines in order on copies of fields (steps from radiation,
    precipitation, nh4sh_eq, chemistry, diagnostics, clamp_species); returns
    {step: {field: array}}."""
    from atjup_b200.params import SPECIES
    f = dict(fields)
    f.setdefault("Q_rad", np.zeros(np.shape(fields["t"])))
    f.setdefault("Q_precip", np.zeros(np.shape(fields["t"])))
    o = Oracle(params, grid, f)
    shape = o.shape
    keep = {}
    names = list(SPECIES) + list(MICRO_SPECIES_SOURCES) + [
        "massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "difflux_h2s",
        "difflux_nh3", "difflux_nh4sh"] + list(MICRO_DIAGNOSTICS)
    for n in names:
        keep[n] = np.ascontiguousarray(fields.get(n, np.zeros(shape)), dtype=np.float64).reshape(shape).copy()
    X = OraPhys()
    for s_, n in enumerate(SPECIES):
        X.q[s_] = _dp(keep[n])
    for s_, n in enumerate(MICRO_SPECIES_SOURCES):
        X.s_precip[s_] = _dp(keep[n])
    for n in ("massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh"):
        setattr(X, n, _dp(keep[n]))
    for q, n in enumerate(("difflux_h2s", "difflux_nh3", "difflux_nh4sh")):
        X.difflux[q] = _dp(keep[n])
    lh = np.ascontiguousarray(fields["layer_heights"], dtype=np.float32).copy()
    X.layer_heights = lh.ctypes.data_as(_P(ctypes.c_float))
    out = {}
    for step in steps:
        fn = getattr(o.lib, "ora_" + step)
        if step == "clamp_species":
            fn(ctypes.byref(params), ctypes.byref(X))
        elif step == "diagnostics":
            outs = (_P(ctypes.c_double) * 6)(*[_dp(keep[n]) for n in MICRO_DIAGNOSTICS])
            fn(ctypes.byref(params), ctypes.byref(micro), ctypes.byref(o.G),
               *[_dp(o.f[n]) for n in ("t", "u", "v", "w", "p_dyn", "p_stat")],
               _dp(keep["h2o"]), _dp(keep["nh3"]), outs)
        else:
            fn(ctypes.byref(params), ctypes.byref(micro), ctypes.byref(o.G), ctypes.byref(o.S),
               ctypes.byref(X))
        snap = {n: o.f[n].copy() for n in ("t", "Q_rad", "Q_precip")}
        snap.update({n: a.copy() for n, a in keep.items()})
        out[step] = snap
    return out


def oracle_mca(params, micro, mca, grid: dict, fields: dict):
    """ora_mca (one moist convective adjustment) on copies of fields; returns (fields, counters)
    with counters {columns, layers, moist_triggers, dry_triggers, unstable_t, held, skipped,
    max_passes}."""
    from atjup_b200.params import SPECIES
    o = Oracle(params, grid, fields)
    shape = o.shape
    keep = {n: np.ascontiguousarray(fields.get(n, np.zeros(shape)), dtype=np.float64).reshape(shape).copy()
            for n in SPECIES}
    X = OraPhys()
    for s_, n in enumerate(SPECIES):
        X.q[s_] = _dp(keep[n])
    lh = np.ascontiguousarray(fields["layer_heights"], dtype=np.float32).copy()
    X.layer_heights = lh.ctypes.data_as(_P(ctypes.c_float))
    st = np.zeros(8, dtype=np.int64)
    o.lib.ora_mca(ctypes.byref(params), ctypes.byref(micro), ctypes.byref(mca), ctypes.byref(o.G),
                  ctypes.byref(o.S), ctypes.byref(X), st.ctypes.data_as(ctypes.c_void_p))
    out = {"t": o.f["t"].copy()}
    out.update(keep)
    names = ("columns", "layers", "moist_triggers", "dry_triggers", "unstable_t", "held",
             "skipped", "max_passes")
    return out, dict(zip(names, (int(x) for x in st)))


def oracle_iteration_phys(params, phys, micro, grid: dict, fields: dict, iters, sweeps=1,
                          snapshots=(), mca=None) -> dict:
    """ora_iteration_phys for iterations 1..iters (the first with first = 1) on copies of fields;
    returns {iteration: {field: array}} for the iterations in snapshots (and the last)."""
    from atjup_b200.params import S_PRECIP, SCALARS, SPECIES
    o = Oracle(params, grid, fields)
    shape = o.shape
    keep = {}
    extra = list(SCALARS) + [n + "n" for n in SCALARS] + ["acc_" + n for n in SCALARS] + \
        ["rhs_" + n for n in SCALARS] + list(S_PRECIP) + [
        "massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "difflux_h2s",
        "difflux_nh3", "difflux_nh4sh", "prod", "tke_source", "dis_source"]
    for n in extra:
        src = fields.get(n)
        if src is None and n.endswith("n") and n[:-1] in SCALARS:
            src = fields.get(n[:-1])
        keep[n] = np.zeros(shape) if src is None else np.ascontiguousarray(src, dtype=np.float64).reshape(shape).copy()
    for n in ("nue", "Q_rad", "Q_precip"):
        if o.f.get(n) is None:
            o.f[n] = np.zeros(shape)
            setattr(o.S, n, _dp(o.f[n]))
    keep["vel_star"] = np.ascontiguousarray(fields["vel_star"], dtype=np.float64).reshape(shape[1:]).copy()
    lh = np.ascontiguousarray(fields["layer_heights"], dtype=np.float32).copy()
    X = OraPhys()
    for s_, n in enumerate(SPECIES):
        X.q[s_] = _dp(keep[n])
        X.qn[s_] = _dp(keep[n + "n"])
        X.acc_q[s_] = _dp(keep["acc_" + n])
        X.rhs_q[s_] = _dp(keep["rhs_" + n])
    for a in ("tke", "dis"):
        setattr(X, a, _dp(keep[a]))
        setattr(X, a + "n", _dp(keep[a + "n"]))
        setattr(X, "acc_" + a, _dp(keep["acc_" + a]))
        setattr(X, "rhs_" + a, _dp(keep["rhs_" + a]))
    for s_, n in enumerate(S_PRECIP):
        X.s_precip[s_] = _dp(keep[n])
    for n in ("massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "prod",
              "tke_source", "dis_source", "vel_star"):
        setattr(X, n, _dp(keep[n]))
    for q, n in enumerate(("difflux_h2s", "difflux_nh3", "difflux_nh4sh")):
        X.difflux[q] = _dp(keep[n])
    X.nue_out = _dp(o.f["nue"])
    X.layer_heights = lh.ctypes.data_as(_P(ctypes.c_float))
    out = {}
    for it in range(1, iters + 1):
        o.lib.ora_iteration_phys(ctypes.byref(params), ctypes.byref(phys), ctypes.byref(micro),
                                 ctypes.byref(mca) if mca is not None else None,
                                 ctypes.byref(o.G), ctypes.byref(o.S), ctypes.byref(X),
                                 ctypes.c_int(it), ctypes.c_int(1 if it == 1 else 0),
                                 ctypes.c_int(sweeps))
        if it in snapshots or it == iters:
            snap = {n: a.copy() for n, a in o.f.items() if a is not None}
            snap.update({n: a.copy() for n, a in keep.items()})
            out[it] = snap
    return out
