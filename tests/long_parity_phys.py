"""Long full-physics parity run: the reference's own moist state, N iterations of the reference
(oracle/_ref, CPU) against N iterations of atjup_gpu_step in FP64 and in the mixed-precision step,
printing the relative L2 difference of every prognostic field. A measurement, not collected by
pytest (the 200-iteration reference run takes several minutes on the host cores).

    python tests/long_parity_phys.py [--iters 200] [--mca] [--rate-law]

--mca runs both sides with the moist convective adjustment every iteration (the reference's
default); --rate-law forms NH4SH by the reaction-rate law (ATJUP_NH4SH_EQ=0) on both sides.

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
    ap.add_argument("--mca", action="store_true")
    ap.add_argument("--rate-law", action="store_true")
    args = ap.parse_args()
    from atjup_b200.params import PREC_FP64, PREC_MIXED, resolve_mca
    from oracle_bridge import MCA_ENV
    t0 = time.time()
    extra = ("--env", "ATJUP_MCA=1") if args.mca else ()
    if args.rate_law:
        extra = extra + ("--env", "ATJUP_NH4SH_EQ=0")
    d, P, PH, MC, g, f = ref_iters_case(args.iters, *extra)
    t_ref = time.time() - t0
    out = {"iterations": args.iters, "mca": args.mca, "rate_law": args.rate_law,
           "reference_seconds": round(t_ref, 1)}
    for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        m = gpu_moist_model(P, PH, MC, g, f)
        if args.mca:
            m.set_mca(resolve_mca(MCA_ENV))
        m.set_precision(prec)
        for it in range(1, args.iters + 1):
            m.step(it, first=(it == 1))
        out[name] = {n: float(f"{rel_l2(m.download(n), d[f'it{args.iters}_{n}']):.3e}")
                     for n in PROGNOSTIC}
        m.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
