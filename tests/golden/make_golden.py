"""Generate the golden digests in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py

Runs the unmodified reference (oracle/_ref/libatjup_ref.so, built from the reference sources by
`make -C oracle ref`) in child processes on its own dry initial state and records, per case and
field, a digest: the L2 norm, the sum, the maximum magnitude, the SHA-256 of the raw bytes and
4096 values at fixed seeded cell indices. Cases:

  init   the dry initial state (cJupiterModel::Run with nm = 0, species zeroed)
  rk4    one cJupiterModel::RungeKuttaJup on it
  press  one PressureSolverJup::run on it (1 red-black sweep)
  iter3  three iterations of the dry loop schedule (cJupiterModel.cpp:1032-1381)
  satadj SaturationAdjustmentJup for H2O, NH3, CH4 (cJupiterModel.cpp:1060-1080) on the seeded
         synthetic moist shell of atjup_b200.synthetic (state + moist, 41x181x361; its cone is
         set as the reference's SeaMount), with t and the gas's fields after each gas, and the
         14 constants of each gas as the reference derives them

tests/test_oracle_ref.py compares the C oracle with these digests (and with the reference run
live when it is built). This script is the only writer of tests/golden/*.json.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))

N_SAMPLES = 1024
SEED = 20261203


def sample_index(shape):
    rng = np.random.Generator(np.random.Philox(SEED))
    n = int(np.prod(shape))
    return np.sort(rng.choice(n, size=N_SAMPLES, replace=False))


def digest(a: np.ndarray) -> dict:
    a = np.ascontiguousarray(a, dtype=np.float64)
    idx = sample_index(a.shape)
    return {"shape": list(a.shape), "l2": float(np.linalg.norm(a.ravel())), "sum": float(a.sum()),
            "maxabs": float(np.abs(a).max()), "sha256": hashlib.sha256(a.tobytes()).hexdigest(),
            "samples": a.ravel()[idx].tolist()}


CASES = {
    "init": ([], ["t", "u", "v", "w", "p_dyn", "p_stat", "rho_mix", "wall_nue", "aux_u", "aux_v", "aux_w"], "in_"),
    "rk4": (["--rk4"], ["t", "u", "v", "w", "p_hydro", "aux_u", "aux_v", "aux_w"], "out_"),
    "press": (["--pressure"], ["p_dyn", "aux_u", "aux_v", "aux_w"], "out_"),
    "iter3": (["--iters", "3"], ["t", "u", "v", "w", "p_dyn", "p_hydro", "rho_mix"], "out_"),
}


def satadj_case(d: dict) -> dict:
    fields = {}
    for gas in ("H2O", "NH3", "CH4"):
        l = gas.lower()
        for n in ("t", l, l + "_cloud", l + "_ice"):
            fields[f"{gas}/{n}"] = digest(d[f"sat_{gas}_{n}"])
    return {"case": "satadj", "flags": ["--satadj-synthetic"],
            "source": "reference (oracle/_ref) SaturationAdjustmentJup on the synthetic moist shell",
            "gases": {g: [float(x) for x in d["gas_" + g]] for g in ("H2O", "NH3", "CH4")},
            "fields": fields}


def main():
    from helpers import ref_dump
    if "--only-satadj" not in sys.argv:
        write_cases(ref_dump)
    (HERE / "golden_satadj.json").write_text(json.dumps(satadj_case(ref_dump("--satadj-synthetic"))))
    print("satadj written")


def write_cases(ref_dump):
    for name, (flags, fields, prefix) in CASES.items():
        d = ref_dump(*flags)
        out = {"case": name, "flags": flags, "source": "reference (oracle/_ref), dry knobs",
               "fields": {f: digest(d[prefix + f]) for f in fields}}
        (HERE / f"golden_{name}.json").write_text(json.dumps(out))
        print(name, "written")


if __name__ == "__main__":
    main()
