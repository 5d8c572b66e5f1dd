"""Run the drop-in patch of cJupiterModel::Run (oracle/gpu_dropin.cpp) beside the reference's own
loop, in one child process, and save both results.

    python tests/dropin_run.py OUT.npz [--iters N] [--threads T]

The reference's initialisation builds the model (dry knobs, species zeroed); the state is saved;
N iterations of the reference's loop run on it (cJupiterModel.cpp:1032-1381 schedule) and the
state is recorded (ref_*); the saved state is put back into the model's arrays; then
dropin_gpu_run does what the maintainer's patch does -- create a GPU context from the resolved
parameters, upload the model's own double*** arrays, N atjup_gpu_step calls, download into the
same arrays -- and the model's arrays are recorded again (gpu_*). Test infrastructure only.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
import baseline_state as BS  # noqa: E402

LIB = ROOT / "oracle" / "_ref" / "libatjup_dropin.so"
KEEP = ("t", "u", "v", "w", "tn", "un", "vn", "wn", "p_dyn", "p_dynn", "p_hydro", "p_stat",
        "rho_mix", "wall_nue", "aux_u", "aux_v", "aux_w", "acc_t", "acc_u", "acc_v", "acc_w")
COMPARED = ("t", "u", "v", "w", "p_dyn", "p_hydro", "rho_mix")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out")
    ap.add_argument("--iters", type=int, default=6)
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args()
    env = BS.ENVS["dry"]
    os.environ.update(env)
    L = ctypes.CDLL(str(LIB))
    L.ref_scalar.restype = ctypes.c_double
    L.dropin_last_error.restype = ctypes.c_char_p
    L.ref_quiet(1)
    if L.ref_create((tempfile.mkdtemp(prefix="atjup_dropin_") + "/run").encode(),
                    a.threads or os.cpu_count() or 1) != 0:
        raise SystemExit("ref_create failed")
    L.ref_quiet(0)
    im, jm, km = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.ref_dims(ctypes.byref(im), ctypes.byref(jm), ctypes.byref(km))
    shape = (im.value, jm.value, km.value)

    def get(n):
        x = np.empty(shape)
        if L.ref_get3(n.encode(), x.ctypes.data_as(ctypes.c_void_p)) != 0:
            raise KeyError(n)
        return x

    def put(n, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        if L.ref_set3(n.encode(), x.ctypes.data_as(ctypes.c_void_p)) != 0:
            raise KeyError(n)

    zero = np.zeros(shape)
    from ref_model import SPECIES_AND_COPIES
    for n in SPECIES_AND_COPIES:       # the dry configuration
        put(n, zero)
    snap = {n: get(n) for n in KEEP}
    data = {}
    L.ref_quiet(1)
    for it in range(1, a.iters + 1):
        if L.ref_iteration(it, 1 if it == 1 else 0, 1) != 0:
            raise SystemExit("ref_iteration failed")
    L.ref_quiet(0)
    for n in COMPARED:
        data["ref_" + n] = get(n)
    for n in KEEP:
        put(n, snap[n])
    from atjup_b200.params import resolve_params
    consts = {c: L.ref_scalar(c.encode()) for c in BS.CONSTS}
    P = resolve_params(env, im=shape[0], jm=shape[1], km=shape[2], constants=consts)
    rc = L.dropin_gpu_run(ctypes.byref(P), a.iters, None)
    if rc != 0:
        raise SystemExit(f"dropin_gpu_run rc={rc}: {L.dropin_last_error().decode()}")
    for n in COMPARED:
        data["gpu_" + n] = get(n)
    np.savez(a.out, **data)
    sys.stdout.flush()
    os._exit(0)


if __name__ == "__main__":
    main()
