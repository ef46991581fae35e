"""Run a few device-resident products of one seeded case, for profilers.

    python profile_case.py --N 16384 --bits 868 --reps 3

Each rep enqueues the three kernels of one product (k_dec, k_row, k_crt) on the default
stream; the run ends by checking the last result against the host entry point.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=16384)
    ap.add_argument("--bits", type=int, default=868)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args()

    import numpy as np
    import torch

    import cases
    import negacyclic as nc

    case = cases.make_case(a.N, a.bits, a.seed, edge_frac=0.01)
    dev = torch.device("cuda", 0)
    da = torch.from_numpy(case.a.view(np.int32)).to(dev)
    db = torch.from_numpy(case.b.view(np.int32)).to(dev)
    dc = torch.empty_like(da)
    with nc.Plan(case.N, case.q_limbs, W=case.W) as plan:
        for _ in range(a.reps):
            plan.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), 0)
        torch.cuda.synchronize()
        want = plan.multiply(case.a, case.b)
    ok = np.array_equal(dc.cpu().numpy().view(np.uint32), want)
    print(f"N={a.N} bits={a.bits} reps={a.reps} consistent={ok}")
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
