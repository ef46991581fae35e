"""Run a few device-resident products of one seeded case, for profilers.

    python profile_case.py --N 65536 --bits 868 --reps 3 [--config 12,3,512] [--batch 0]

Each rep enqueues the three kernels of one product (residues: k_dec_tc, or k_dec with
--residue-engine imad; k_row; k_crt_tc) on the default stream, with the given row configuration
(default: the plan's default); with --batch B > 0
each rep is instead one persistent launch (k_persistent) of B products; with --residues
imad|tc each rep is the residue stage alone of both operands (k_residues_imad or k_residues_tc).
The run ends by checking the last result against the host entry point (or, for --residues,
against the other residue engine).
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
    ap.add_argument("--config", type=str, default="")
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--residue-engine", choices=["tc", "imad"], default="tc",
                    help="residue stage of the plan's products: k_dec_tc (tensor cores) or k_dec")
    ap.add_argument("--residues", choices=["", "imad", "tc"], default="",
                    help="run only the residue stage of both operands with this engine (k_residues_imad / "
                         "k_residues_tc), checked against the other engine")
    a = ap.parse_args()

    import numpy as np
    import torch

    if a.residues:
        return residues_only(a)

    import cases
    import negacyclic as nc

    case = cases.make_case(a.N, a.bits, a.seed, edge_frac=0.01)
    dev = torch.device("cuda", 0)
    da = torch.from_numpy(case.a.view(np.int32)).to(dev)
    db = torch.from_numpy(case.b.view(np.int32)).to(dev)
    count = max(1, a.batch)
    dcs = [torch.empty_like(da) for _ in range(count)]
    with nc.Plan(case.N, case.q_limbs, W=case.W) as plan:
        if a.config:
            plan.row_config = tuple(int(x) for x in a.config.split(","))
        if a.residue_engine == "imad" or plan.k > 32:
            plan.residue_engine = nc.RESIDUES_IMAD
        if a.batch > 0:
            with nc.Batch() as batch:
                for dc in dcs:
                    batch.add(plan, da.data_ptr(), db.data_ptr(), dc.data_ptr())
                for _ in range(a.reps):
                    batch.run(0, False)
                batch.synchronize()
        else:
            for _ in range(a.reps):
                plan.multiply_device(da.data_ptr(), db.data_ptr(), dcs[0].data_ptr(), 0)
        torch.cuda.synchronize()
        want = plan.multiply(case.a, case.b)
        cfg = plan.row_config
    ok = all(np.array_equal(dc.cpu().numpy().view(np.uint32), want) for dc in dcs)
    print(f"N={a.N} bits={a.bits} reps={a.reps} batch={a.batch} config={cfg} consistent={ok}")
    return 0 if ok else 1


def residues_only(a) -> int:
    import numpy as np
    import torch

    import cases
    import negacyclic as nc

    case = cases.make_case(a.N, a.bits, a.seed, edge_frac=0.01)
    dev = torch.device("cuda", 0)
    engine = nc.RESIDUES_TC_I8 if a.residues == "tc" else nc.RESIDUES_IMAD
    other = nc.RESIDUES_IMAD if engine == nc.RESIDUES_TC_I8 else nc.RESIDUES_TC_I8
    with nc.Plan(case.N, case.q_limbs, W=case.W) as plan:
        k, N = plan.k, plan.N
        xs = [torch.from_numpy(x.view(np.int32)).to(dev) for x in (case.a, case.b)]
        r = torch.empty(2 * k * N, dtype=torch.int64, device=dev)
        check = torch.empty_like(r)
        for _ in range(a.reps):
            for j, x in enumerate(xs):
                plan.residues(x.data_ptr(), r.data_ptr() + j * k * N * 8, engine)
        for j, x in enumerate(xs):
            plan.residues(x.data_ptr(), check.data_ptr() + j * k * N * 8, other)
        torch.cuda.synchronize()
        ok = bool(torch.equal(r, check)) and not nc.residues_gave_up()
    print(f"residues N={a.N} bits={a.bits} reps={a.reps} engine={a.residues} consistent={ok}")
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
