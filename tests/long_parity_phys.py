"""Long full-physics parity run: the reference's own moist state, N iterations of the reference
(oracle/_ref, CPU) against N iterations of atjup_gpu_step in FP64 and in the mixed-precision step,
printing the relative L2 difference of every prognostic field. A measurement, not collected by
pytest (the 200-iteration reference run takes several minutes on the host cores).

    python tests/long_parity_phys.py [--iters 200]

Test infrastructure only (reads the reference through oracle/_ref like the other parity tests).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from moist_cases import PROGNOSTIC, gpu_moist_model, ref_iters_case  # noqa: E402
from oracle_bridge import rel_l2  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=200)
    args = ap.parse_args()
    from atjup_b200.params import PREC_FP64, PREC_MIXED
    t0 = time.time()
    d, P, PH, MC, g, f = ref_iters_case(args.iters)
    t_ref = time.time() - t0
    out = {"iterations": args.iters, "reference_seconds": round(t_ref, 1)}
    for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        m = gpu_moist_model(P, PH, MC, g, f)
        m.set_precision(prec)
        for it in range(1, args.iters + 1):
            m.step(it, first=(it == 1))
        out[name] = {n: float(f"{rel_l2(m.download(n), d[f'it{args.iters}_{n}']):.3e}")
                     for n in PROGNOSTIC}
        m.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
