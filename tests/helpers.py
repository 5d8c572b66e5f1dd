"""Shared test helpers: reference dumps, parameter blocks, oracle / GPU model construction."""
from __future__ import annotations

import math
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

from atjup_b200 import synthetic
from atjup_b200.params import resolve_params
from oracle_bridge import DRY_ENV, DYN_FIELDS, Oracle, rel_l2  # noqa: F401

ROOT = Path(__file__).resolve().parents[1]
_DUMPS: dict = {}


def ref_dump(*flags: str, threads: int = 0) -> dict:
    """Run tests/ref_dump.py in a child process (cached per flag set) and load the result."""
    key = tuple(flags)
    if key in _DUMPS:
        return _DUMPS[key]
    fd, path = tempfile.mkstemp(suffix=".npz", prefix="atjup_dump_")
    os.close(fd)
    cmd = [sys.executable, str(ROOT / "tests" / "ref_dump.py"), path, *flags,
           "--threads", str(threads or os.cpu_count() or 1)]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                   env={**os.environ, **DRY_ENV})
    with np.load(path) as z:
        d = {k: z[k] for k in z.files}
    os.unlink(path)
    _DUMPS[key] = d
    return d


def dump_params(d: dict, env=None, **kw):
    consts = {k[6:]: float(v) for k, v in d.items() if k.startswith("const_")}
    im, jm, km = d["in_t"].shape
    return resolve_params(env if env is not None else DRY_ENV, im=im, jm=jm, km=km,
                          constants=consts, **kw)


def dump_grid(d: dict) -> dict:
    return {k[5:]: v for k, v in d.items() if k.startswith("grid_")}


def dump_fields(d: dict, prefix="in_") -> dict:
    return {k[len(prefix):]: v for k, v in d.items() if k.startswith(prefix)}


def synthetic_case(im=13, jm=37, km=49, seed=7, env=None, **kw):
    """(params, grid, fields) of a small synthetic shell whose spacings match its size."""
    s = synthetic.state(im, jm, km, seed=seed)
    p = resolve_params(env if env is not None else DRY_ENV, im=im, jm=jm, km=km, **kw)
    p.dthe = math.pi / (jm - 1)
    p.dphi = 2.0 * math.pi / (km - 1)
    grid = {k: s[k] for k in ("rad", "the", "solid", "topo", "cell_vbar0", "cell_ubar0")}
    fields = {k: v for k, v in s.items() if k not in grid}
    return p, grid, fields


def oracle_from(p, grid, fields) -> Oracle:
    return Oracle(p, grid, fields)


def gpu_from(p, grid, fields):
    from atjup_b200.gpu import GpuModel
    m = GpuModel(p, grid)
    m.upload_state(fields)
    return m

