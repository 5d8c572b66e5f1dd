"""The drop-in boundary exercised from the reference's side: the maintainer's patch of
cJupiterModel::Run (oracle/gpu_dropin.cpp, compiled against the reference's own headers and linked
with atjup_b200/libatjup_gpu.so) creates a GPU context from the resolved parameters, uploads the
reference model's own double*** arrays, runs atjup_gpu_step and downloads into the same arrays.
Six dry iterations (even and odd, the pressure pass on the even ones) from the reference's own
initial state, against the reference's loop on the same model: relative L2 <= 1e-10 per field,
the bar for the FP64 GPU path."""
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

from helpers import rel_l2

ROOT = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin_lib():
    lib = ROOT / "oracle" / "_ref" / "libatjup_dropin.so"
    if not lib.exists():
        pytest.skip("oracle/_ref/libatjup_dropin.so not built (needs the reference sources)")
    return lib


def test_reference_driver_runs_the_gpu_iteration(dropin_lib):
    fd, path = tempfile.mkstemp(suffix=".npz")
    os.close(fd)
    subprocess.run([sys.executable, str(ROOT / "tests" / "dropin_run.py"), path, "--iters", "6"],
                   check=True, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
    with np.load(path) as z:
        d = {k: z[k] for k in z.files}
    os.unlink(path)
    worst = {n[4:]: rel_l2(d[n], d["ref_" + n[4:]]) for n in d if n.startswith("gpu_")}
    print("drop-in, 6 dry iterations, GPU vs the reference's loop:",
          {k: f"{v:.1e}" for k, v in worst.items()})
    for n, e in worst.items():
        assert np.isfinite(e) and e <= 1e-10, f"{n}: relative L2 {e:.3e}"
