"""The CPU oracle against the reference: bit-exact on the reference's own dry initial state, and
against the golden digests generated from the reference (tests/golden/make_golden.py).
Needs oracle/_ref/libatjup_ref.so for the initial state (built from the reference sources)."""
import json
from pathlib import Path

import numpy as np
import pytest

from golden.make_golden import sample_index
from helpers import dump_fields, dump_grid, dump_params, oracle_from, ref_dump

GOLD = Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.slow


def _check_digest(case, arrays):
    g = json.loads((GOLD / f"golden_{case}.json").read_text())
    for name, dg in g["fields"].items():
        a = arrays[name]
        assert list(a.shape) == dg["shape"]
        scale = max(dg["maxabs"], 1e-300)
        s = a.ravel()[sample_index(a.shape)]
        err = np.abs(s - np.asarray(dg["samples"])).max() / scale
        assert err <= 1e-13, f"{case}/{name}: sampled values off by {err:.3e} (relative to max)"
        l2 = np.linalg.norm(a.ravel())
        assert abs(l2 - dg["l2"]) <= 1e-12 * max(dg["l2"], 1e-300), f"{case}/{name}: L2 {l2} vs {dg['l2']}"


def test_init_state_matches_golden(ref_required):
    d = ref_dump("--rk4")
    _check_digest("init", dump_fields(d))


def test_oracle_rk4_bit_exact(ref_required):
    d = ref_dump("--rk4")
    o = oracle_from(dump_params(d), dump_grid(d), dump_fields(d))
    o.rk4()
    out = dump_fields(d, "out_")
    for n in ("t", "u", "v", "w", "p_hydro", "aux_u", "aux_v", "aux_w"):
        assert np.array_equal(o.f[n], out[n]), f"{n} differs from the reference"
    assert np.array_equal(o.f["buoy_ref"], d["out_buoy_ref"])
    _check_digest("rk4", o.f)


def test_oracle_pressure_sweep_bit_exact(ref_required):
    d = ref_dump("--pressure")
    o = oracle_from(dump_params(d), dump_grid(d), dump_fields(d))
    o.pressure(sweeps=1)
    out = dump_fields(d, "out_")
    for n in ("p_dyn", "aux_u", "aux_v", "aux_w"):
        assert np.array_equal(o.f[n], out[n]), f"{n} differs from the reference"
    _check_digest("press", o.f)


def test_oracle_three_iterations_bit_exact(ref_required):
    d = ref_dump("--iters", "3")
    o = oracle_from(dump_params(d), dump_grid(d), dump_fields(d))
    for it in (1, 2, 3):
        o.iteration(it, it == 1)
    out = dump_fields(d, "out_")
    for n in ("t", "u", "v", "w", "p_dyn", "p_hydro", "rho_mix"):
        assert np.array_equal(o.f[n], out[n]), f"{n} differs from the reference"
    _check_digest("iter3", o.f)


@pytest.mark.parametrize("case", ["init", "rk4", "press", "iter3"])
def test_golden_files_present(case):
    g = json.loads((GOLD / f"golden_{case}.json").read_text())
    assert g["fields"] and all(len(v["samples"]) == 1024 for v in g["fields"].values())
