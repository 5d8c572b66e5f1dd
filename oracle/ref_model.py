"""The unmodified reference (oracle/_ref/libatjup_ref.so, built from its sources by
oracle/Makefile) as a Python object: one cJupiterModel per process, initialised by the
reference's own Run() with nm = 0, with every field readable and writable by name.

TEST AND CPU-BASELINE INFRASTRUCTURE: used by tests/, by the reference arm and the CPU-baseline
leg of bench.py, and to prepare benchmark input states; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_SO = HERE / "_ref" / "libatjup_ref.so"

SPECIES_AND_COPIES = ("h2o", "h2o_cloud", "h2o_ice", "h2s", "nh3", "nh3_cloud", "nh3_ice",
                      "ch4", "ch4_cloud", "ch4_ice", "nh4sh", "h2on", "h2o_cloudn", "h2o_icen",
                      "h2sn", "nh3n", "nh3_cloudn", "nh3_icen", "ch4n", "ch4_cloudn",
                      "ch4_icen", "nh4shn")


class RefModel:
    """The reference model. The knobs in `env` are put into this process's environment before
    the model is built (the reference reads them once, at first use). With zero_species the
    species and their time-level-n copies are zeroed after the initialisation (the dry
    configuration: the reference has no switch for its saturation adjustment, and with no
    species it has nothing to act on)."""

    def __init__(self, env: dict, out_dir: str, threads: int = 0, zero_species: bool = True):
        os.environ.update(env)
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (make -C oracle ref)")
        L = ctypes.CDLL(str(REF_SO))
        L.ref_scalar.restype = ctypes.c_double
        L.ref_knob_d.restype = ctypes.c_double
        L.ref_balance_v.restype = ctypes.c_double
        self.L = L
        L.ref_quiet(1)
        rc = L.ref_create(out_dir.encode(), threads)
        L.ref_quiet(0)
        if rc != 0:
            raise RuntimeError(f"ref_create failed rc={rc}")
        im, jm, km = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.ref_dims(ctypes.byref(im), ctypes.byref(jm), ctypes.byref(km))
        self.shape = (im.value, jm.value, km.value)
        if zero_species:
            z = np.zeros(self.shape)
            for n in SPECIES_AND_COPIES:
                self.set(n, z)

    def scalar(self, n):
        return self.L.ref_scalar(n.encode())

    def get(self, n):
        a = np.empty(self.shape)
        if self.L.ref_get3(n.encode(), a.ctypes.data_as(ctypes.c_void_p)) != 0:
            raise KeyError(n)
        return a

    def set(self, n, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if self.L.ref_set3(n.encode(), a.ctypes.data_as(ctypes.c_void_p)) != 0:
            raise KeyError(n)

    def get1(self, n):
        cap = self.shape[0] * self.shape[1] * self.shape[2]
        a = np.empty(cap)
        m = self.L.ref_get1(n.encode(), a.ctypes.data_as(ctypes.c_void_p), cap)
        if m < 0:
            raise KeyError(n)
        return a[:m].copy()

    def topo(self):
        a = np.empty(self.shape[1] * self.shape[2], dtype=np.int32)
        self.L.ref_get_topo(a.ctypes.data_as(ctypes.c_void_p))
        return a.reshape(self.shape[1], self.shape[2])

    def gas_consts(self, gas: str) -> np.ndarray:
        """The 14 constants SaturationAdjustmentJup::run takes for `gas` (H2O, NH3, CH4)."""
        cst = np.zeros(14)
        if self.L.ref_gas_consts(gas.encode(), cst.ctypes.data_as(ctypes.c_void_p)) != 0:
            raise KeyError(gas)
        return cst

    def solid(self) -> np.ndarray:
        return (self.get("SeaMount") == 1.0).astype(np.uint8)

    def quiet(self, fn, *args):
        self.L.ref_quiet(1)
        try:
            return fn(*args)
        finally:
            self.L.ref_quiet(0)
