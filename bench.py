#!/usr/bin/env python
"""Benchmark of the negacyclic product c = a*b mod (X^N + 1, q), N = 65536, 868-bit q.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one product of the single-large-product workload (N = 65536, L = 28, seeded
868-bit prime q, 99% uniform coefficients and 1% edge values). Prints one JSON line on rank 0.

ours (default)
  value        products/s with operands resident in HBM: per-step CUDA events on the
               launching stream, L2 flushed (256 MiB write) before every timed step,
               max over ranks (each rank runs its own products: weak scaling)
  e2e          products/s through the reference-facing entry point fherma_run with host
               buffers, timed by the library's harness runner exactly as the platform's harness
               times it (steady clock around fherma_run: host copies, H2D, kernels, D2H)
  roofline     dominant kernel's algorithmic IMAD rate against the IMAD peak measured live
  cpu_baseline the CPU oracle (multi-prime NTT + CRT, OpenMP over all host cores) on one
               product of the same workload (rank 0, N = 1 only)
  batched      the same products back to back (device-resident, no flush between products)

reference
  the reference's own solution on the same workload, timed by its own generated harness
  main.cpp: solve.cu built for sm_100a with two init-time changes only (kMaxN raised to 65536;
  the L = 28 Barrett self-check throw removed, since that check rejects nearly every 868-bit
  q). Falls back to the CPU oracle when that binary is absent or fails.
"""
from __future__ import annotations

import argparse
import json
import os
import queue
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "engel-cuda-negacyclic-multiply_b200"
sys.path.insert(0, str(PKG))

METRIC = "products/s at N=2^16, 868-bit q, bit-exact: batched vs plain; serve p50/p99 ms"
N_MAIN, BITS, SEED, EDGE = 65536, 868, 20261203, 0.01
MIX_SEED = 4242
WORKLOAD = "single large product: N=65536, L=28, seeded 868-bit prime q, 1% edge coefficients"
FLUSH_BYTES = 256 << 20
RUNNER = PKG / "bin" / "solution"
REF_BINARY = ROOT / "oracle" / "_ref" / "solution_patched"
TRAFFIC_FILE = ROOT / "profiles" / "traffic.json"


def log(msg: str) -> None:
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched / uneven / serving sections")
    ap.add_argument("--row-config", type=str, default="",
                    help="pin the row configuration (log_block,log_radix,threads) instead of autotuning, e.g. to "
                         "profile the configuration a plain run picked")
    pc = ap.add_argument_group("profiling modes (untimed runs for ncu; they print no bench line)")
    pc.add_argument("--profile-case", action="store_true",
                    help="run --profile-reps device-resident products of one seeded case and check the last one")
    pc.add_argument("--profile-N", type=int, default=16384)
    pc.add_argument("--profile-bits", type=int, default=868)
    pc.add_argument("--profile-reps", type=int, default=3)
    pc.add_argument("--profile-seed", type=int, default=7)
    pc.add_argument("--profile-batch", type=int, default=0,
                    help="each rep is one batch of this many products (persistent launch) instead of one product")
    pc.add_argument("--profile-residue-engine", choices=["tc", "imad"], default="tc",
                    help="residue stage of the products: k_dec_tc (tensor cores) or k_dec (integer pipes)")
    pc.add_argument("--profile-word-bits", type=int, choices=[0, 32, 64], default=0,
                    help="the plain path's engine (32: the 30-bit word engine, 64: the 62-bit engine; "
                         "0: the library's default)")
    pc.add_argument("--profile-residues", choices=["", "imad", "tc"], default="",
                    help="run only the residue stage of both operands with this engine (k_residues_imad / "
                         "k_residues_tc), checked against the other engine")
    pc.add_argument("--profile-reference", type=int, default=0, metavar="PRODUCTS",
                    help="run the reference's own binary on this many products of the bench workload")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    a.steps = max(a.steps, 1)
    return a


def config(parallelism: str) -> dict:
    return {
        "workload": WORKLOAD,
        "N": N_MAIN,
        "L": (BITS + 31) // 32,
        "q_bits": BITS,
        "edge_frac": EDGE,
        "seed": SEED,
        "l2": "flushed before every timed step (256 MiB device write)",
        "parallelism": parallelism,
    }


# ----------------------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.file = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=self.file, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.file:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        load = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- roofline


def stage_work(k: int, N: int, L: int, logN2: int | None = None, word_bits: int = 64) -> list[float]:
    """Algorithmic IMAD per stage. 62-bit engine (word_bits 64): 8 per 64-bit mulmod (the four
    32 x 32 partial products of a 64 x 64 product, low and high halves), 2 per u32 x u64 limb MAC;
    whole product 8 k N (1.5 log2 N + 7) + 6 k N L + 4 L N. 30-bit engine (word_bits 32): 3 per
    30-bit mulmod (a Shoup or Montgomery product: one high and two low 32 x 32 products), 1 per
    u32 x u32 limb MAC; whole product 3 k N (1.5 log2 N + 7) + 3 k N L + 4 L N. Both count 4 L per
    coefficient for the final reduction. logN2 is the row block of the plan's row configuration
    (its row kernel runs logN2 stages of each transform; the residue and CRT kernels run the
    other logN1 = log2 N - logN2 column stages); the per-stage split depends on it, the product
    total does not."""
    logN = N.bit_length() - 1
    if logN2 is None:
        logN2 = min(logN, 12)
    if not 0 <= logN2 <= logN:
        raise ValueError("row block larger than the ring degree")
    logN1 = logN - logN2
    mm1 = 2 * k * N + 2 * k * N + 2 * k * (N // 2) * logN1   # residue reductions, twists, column stages
    mac1 = 2 * k * N * L
    mm2 = 3 * k * (N // 2) * logN2 + k * N                    # three row transforms, pointwise
    mm3 = k * (N // 2) * logN1 + k * N + k * N                # inverse column stages, untwist, CRT digit
    mac3 = k * N * L
    mm, mac = (8, 2) if word_bits == 64 else (3, 1)
    return [mm * mm1 + mac * mac1, mm * mm2, mm * mm3 + mac * mac3 + 4 * L * N]


def stage_bytes(k: int, N: int, L: int, word_bits: int = 64) -> list[int]:
    """Compulsory HBM bytes per stage (operands, residues, twiddles read once): residues of
    word_bits / 8 bytes, twiddles with their Shoup companions twice that."""
    r = word_bits // 8
    return [2 * N * L * 4 + 2 * k * N * r,
            2 * k * N * r + k * N * r + 2 * k * N * 2 * r,
            k * N * r + N * L * 4]


# ----------------------------------------------------------------------------- harness runs


def make_case_dir(root: Path, case, count: int) -> None:
    import cases

    cases.write_case_dir(root, case.N, case.W, case.L, case.q, [(case.a, case.b)])
    src = root / "cases" / "000000"
    for i in range(1, count):
        d = root / "cases" / f"{i:06d}"
        d.mkdir(parents=True, exist_ok=True)
        for name in ("a.bin", "b.bin"):
            os.link(src / name, d / name)
    (root / "manifest.json").write_text(json.dumps({"N": case.N, "W": case.W, "L": case.L, "cases": count}))


def run_harness(binary: Path, case, warmup: int, steps: int, timeout: float = 600.0, env: dict | None = None,
                stderr_out: list | None = None):
    """Run a harness binary over warmup + steps copies of one case; per-case seconds of the timed ones."""
    import cases

    with tempfile.TemporaryDirectory(prefix="nc_bench_") as tmp:
        root = Path(tmp)
        make_case_dir(root, case, warmup + steps)
        r = subprocess.run([str(binary), str(root)], capture_output=True, text=True, timeout=timeout,
                           env=None if env is None else {**os.environ, **env})
        if stderr_out is not None:
            stderr_out.append(r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"{binary.name} exited {r.returncode}: {r.stderr[-400:]}")
        res = cases.read_results(root)
        rows = res["cases"]
        if len(rows) != warmup + steps or any(row["status"] != "ok" for row in rows):
            raise RuntimeError(f"{binary.name}: {sum(row['status'] != 'ok' for row in rows)} cases failed")
        secs = [row["seconds"] for row in rows[warmup:]]
        out = cases.read_output(root, warmup + steps - 1, case.N, case.L)
        return secs, res["init_s"], out, rows[0]["seconds"]


# ----------------------------------------------------------------------------- CPU baseline


def cpu_baseline(case, budget_s: float = 20.0) -> dict:
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    threads = oracle.max_threads()
    times = []
    t_all = time.perf_counter()
    while not times or (time.perf_counter() - t_all < budget_s / 2 and len(times) < 3):
        t0 = time.perf_counter()
        oracle.negacyclic(case.N, case.q_limbs, case.a, case.b, threads)
        times.append(time.perf_counter() - t0)
    per = statistics.median(times)
    return {"value": 1.0 / per, "unit": "products/s", "cores": threads, "kind": "port",
            "sample": f"{len(times)} product(s) of the N=65536 868-bit workload by the CPU oracle "
                      f"(C, OpenMP over {threads} threads); median {per:.3f} s/product"}


# ----------------------------------------------------------------------------- arms


def max_over_ranks(pg, values, device) -> list[float]:
    """Element-wise maximum of this rank's timings (ms) over every rank of the process group `pg`
    (None: this process alone). Every rank must call it with the same number of values."""
    if pg is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(x) for x in t]


def whole_job_rate(world: int, products_per_rank: int, max_ms: float) -> float:
    """Products per second of the whole job: every rank's products over the slowest rank's time
    (replicas: each rank runs its own products, no data-path collective)."""
    return world * products_per_rank / (max_ms * 1e-3)


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def ours(args) -> dict | None:
    import numpy as np

    import cases

    world, rank, local = dist_setup(args)
    forms = world == 1 and not args.no_forms
    mix = None
    if forms:  # seeded primes of the uneven mix, found before this process touches CUDA
        mix = cases.uneven_mix(256, seed=MIX_SEED, processes=min(16, os.cpu_count() or 1))

    import torch

    import negacyclic as nc

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        pg = dist

    case = cases.make_case(N_MAIN, BITS, SEED, edge_frac=EDGE)
    plan = nc.Plan(case.N, case.q_limbs, W=case.W)
    if args.row_config:
        plan.row_config = tuple(int(x) for x in args.row_config.split(","))
        tuned_ms = None
    else:
        tuned_ms = plan.autotune(reps=3)  # untimed: picks the row tiling for N = 65536
    # the timed steps run the product as a caller does (no per-stage events: they cost ~10 us a
    # product); the per-stage split comes from a separate pass afterwards
    plan.set_timing(False)
    n_pairs = 8  # distinct operand pairs: 8 x 22 MB of operands and outputs exceed L2
    da = [torch.from_numpy(cases.coeffs(case.q, case.N, case.L, SEED + 10 * i + 1).view(np.int32)).to(dev)
          for i in range(n_pairs)]
    db = [torch.from_numpy(cases.coeffs(case.q, case.N, case.L, SEED + 10 * i + 2).view(np.int32)).to(dev)
          for i in range(n_pairs)]
    da[0].copy_(torch.from_numpy(case.a.view(np.int32)))
    db[0].copy_(torch.from_numpy(case.b.view(np.int32)))
    dc = [torch.empty_like(da[0]) for _ in range(n_pairs)]
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def product(i):
        j = i % n_pairs
        plan.multiply_device(da[j].data_ptr(), db[j].data_ptr(), dc[j].data_ptr(), sh)

    for i in range(args.warmup):
        flush.zero_()
        product(i)
    torch.cuda.synchronize()
    # correctness guard on the measured path: device result == host-entry result
    ref = plan.multiply(case.a, case.b)
    product(0)
    torch.cuda.synchronize()
    if not np.array_equal(dc[0].cpu().numpy().view(np.uint32), ref):
        raise RuntimeError("device-resident product differs from the host entry point")
    if pg:
        pg.barrier()
    torch.cuda.synchronize()

    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev0[i].record(stream)
            product(i)
            ev1[i].record(stream)
            torch.cuda.synchronize()
        # batched: the same products back to back, no flush between them
        eb0 = torch.cuda.Event(enable_timing=True)
        eb1 = torch.cuda.Event(enable_timing=True)
        batch = 4 * n_pairs
        eb0.record(stream)
        for i in range(batch):
            product(i)
        eb1.record(stream)
        torch.cuda.synchronize()
    # per-stage split (roofline): the same steps again with CUDA events between the three stages
    plan.set_timing(True)
    stage = []
    for i in range(args.steps):
        flush.zero_()
        product(i)
        torch.cuda.synchronize()
        stage.append(plan.stage_ms())
    plan.set_timing(False)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in zip(ev0, ev1)]
    total_ms = sum(step_ms)
    batch_ms = eb0.elapsed_time(eb1)
    total_ms, batch_ms = max_over_ranks(pg, [total_ms, batch_ms], dev)

    peak = nc.imad_peak()
    word, k, N, L = plan.word_bits, plan.plain_primes, case.N, case.L
    mean_stage = [statistics.mean(s[i] for s in stage) for i in range(3)]
    work = stage_work(k, N, L, plan.row_config[0], word)
    sbytes = stage_bytes(k, N, L, word)
    dom = max(range(3), key=lambda i: mean_stage[i])
    crt_tc = plan.crt_engine == nc.CRT_TC_I8
    res_tc = plan.residue_engine == nc.RESIDUES_TC_I8
    names = ["residues (contraction on the tensor cores)+forward columns" if res_tc else "residues+forward columns",
             "row NTTs+pointwise",
             "inverse columns+CRT (accumulation on the tensor cores)" if crt_tc else "inverse columns+CRT"]
    if word == 32:
        kernels = ["k_dec_tc32", "k_row32", "k_crt_tc32"]
    else:
        kernels = ["k_dec_tc" if res_tc else "k_dec", "k_row", "k_crt_tc" if crt_tc else "k_crt"]
    traffic = None
    if TRAFFIC_FILE.exists():
        tf = json.loads(TRAFFIC_FILE.read_text())
        traffic = tf.get(kernels[dom], {}).get("bytes_per_launch")
    achieved = work[dom] / (mean_stage[dom] * 1e-3) / 1e9
    result = {
        "metric": METRIC,
        "value": whole_job_rate(world, args.steps, total_ms),
        "unit": "products/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32" if word == 32 else "u64",
        "data": "synthetic (seeded)",
        "config": config(f"replicas{world}"),
        "gpu_launches": 3 * args.steps,
        "engine": {"word_bits": word, "primes": k,
                   "what": ("30-bit word engine: u32 residues modulo primes below 2^30" if word == 32 else
                            "62-bit engine: u64 residues modulo primes 2^62 - m")},
        "row_config": {"log_block": plan.row_config[0], "log_radix": plan.row_config[1],
                       "threads": plan.row_config[2], "autotune_ms": tuned_ms},
        "roofline": {
            "bound": "imad",
            "kernel": f"{kernels[dom]} ({names[dom]})",
            "achieved": achieved,
            "peak": peak / 1e9,
            "unit": "GIMAD/s",
            "frac": achieved * 1e9 / peak,
            "traffic": traffic,
            "frac_recomputed_from": ("stage_imad_alg[dom] / stage_ms[dom] / peak; the stage shares agree with the "
                                     "ncu launch list in profiles/launches_bench_n65536.md, DRAM bytes in "
                                     "profiles/traffic.json"),
            "peak_source": "measured live: mad.lo.u32 chains over every SM (nc_imad_peak)",
            "stage_ms": mean_stage,
            "stage_imad_alg": work,
            "product_imad_alg": sum(work),
            "product_frac": sum(work) / (total_ms / args.steps * 1e-3) / peak,
            "stage_hbm_gbs": [b / (t * 1e-3) / 1e9 for b, t in zip(sbytes, mean_stage)],
            "hbm_peak_gbs": _hbm_peak(),
        },
        "batched": {"products": batch, "value": whole_job_rate(world, batch, batch_ms), "unit": "products/s",
                    "form": "plain launches back to back, device-resident, 8 operand pairs rotated"},
        "clocks": clk.summary(),
    }
    plan.close()

    if rank == 0 and not args.no_e2e and RUNNER.exists():
        # about a millisecond per call: more calls than the device-timed steps, for a stable mean
        e2e_warmup, e2e_steps = max(args.warmup, 10), max(args.steps, 60)
        secs, init_s, out, first_s = run_harness(RUNNER, case, e2e_warmup, e2e_steps)
        if not np.array_equal(out, ref):
            raise RuntimeError("harness runner output differs from the library")
        per = statistics.mean(secs)
        # a separate, shorter run with the library's host-path trace: where one call's time goes
        traced: list = []
        run_harness(RUNNER, case, 5, 20, env={"NC_TRACE": "1"}, stderr_out=traced)
        phases = trace_phases(traced[0], 20)
        h2d_gbs, d2h_gbs = copy_rates(dev, 2 * N * L * 4, N * L * 4)
        h2d_ms = 2 * N * L * 4 / (h2d_gbs * 1e9) * 1e3
        d2h_ms = N * L * 4 / (d2h_gbs * 1e9) * 1e3
        result["e2e"] = {"value": world / per, "unit": "products/s",
                         "h2d_bytes_per_step": 2 * N * L * 4, "d2h_bytes_per_step": N * L * 4,
                         "ms_p50": 1e3 * statistics.median(secs), "ms_p99": 1e3 * sorted(secs)[int(0.99 * (len(secs) - 1))],
                         "first_call_ms": 1e3 * first_s,
                         "floor_ms": h2d_ms + mean_stage[1] + d2h_ms,
                         "floor": {"h2d_gbs": h2d_gbs, "d2h_gbs": d2h_gbs, "h2d_ms": h2d_ms, "row_stage_ms": mean_stage[1],
                                   "d2h_ms": d2h_ms,
                                   "why": ("every input byte crosses PCIe before the row stage can finish (each row "
                                           "block needs residues of coefficients from the whole operand), and every "
                                           "output byte after it; copy rates measured here from pinned memory in the "
                                           "library's chunk sizes (4 MiB up, 2 MiB down), one direction at a time")},
                         "phases_us": phases,
                         "calls": e2e_steps, "warmup_calls": e2e_warmup, "init_s": init_s,
                         "via": "fherma_run in the library's harness runner (pageable std::vector in/out); "
                                "first_call_ms is the first call after fherma_init"}
    if forms:
        # each form checks its own results; a failure is reported in its entry, not hidden
        for key, what, fn in (("batched_n65536", "batched N=65536", lambda: batched_same_shape(dev, case.q, 65536, 16, args)),
                              ("batched_c3", "batched 64 x N=16384", lambda: batched_same_shape(dev, case.q, 16384, 64, args)),
                              ("uneven_c4", "uneven batch", lambda: uneven_batch(dev, mix, args)),
                              ("ablation_residues", "residue ablation", lambda: residue_ablation(dev, case)),
                              ("chained_n65536", "chained products", lambda: chained(dev)),
                              ("serve_c5", "serving", lambda: serving(dev, mix, args))):
            log(what)
            try:
                result[key] = fn()
            except Exception as e:
                result[key] = {"error": f"{type(e).__name__}: {e}"[:500]}
        log("forms done")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(case)
    if pg:
        pg.destroy_process_group()
    return result if rank == 0 else None


def trace_phases(stderr: str, last: int) -> dict | None:
    """Median over the last `last` calls of each field of the library's NC_TRACE lines: device-clock
    ends of a's upload, a's forward transform, b's upload, the product and the download, and host
    times at which a and b were staged, everything was enqueued, and the result was copied out
    (microseconds from the call's start)."""
    rows = []
    for line in stderr.splitlines():
        if line.startswith("nc_trace "):
            rows.append(dict((k, float(v)) for k, v in (f.split("=") for f in line.split()[1:])))
    rows = rows[-last:]
    if not rows:
        return None
    out = {k: round(statistics.median(r[k] for r in rows), 1) for k in rows[0]}
    out["calls"] = len(rows)
    out["what"] = ("device clock (a_uploaded .. downloaded) and host clock (a_staged .. collected), us from the "
                   "call's start, median over calls of a separate traced run (NC_TRACE=1)")
    return out


def copy_rates(dev, up_bytes: int, down_bytes: int, reps: int = 20) -> tuple[float, float]:
    """GB/s of pinned host -> device copies of `up_bytes` in 4 MiB chunks and device -> pinned host
    copies of `down_bytes` in 2 MiB chunks (the host path's chunk sizes), best of `reps`."""
    import torch

    host = torch.empty(max(up_bytes, down_bytes), dtype=torch.uint8, pin_memory=True)
    host.fill_(1)
    devbuf = torch.empty_like(host, device=dev)
    s = torch.cuda.current_stream(dev)

    def timed(fn) -> float:
        best = 1e30
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    def up():
        for o in range(0, up_bytes, 4 << 20):
            devbuf[o:min(up_bytes, o + (4 << 20))].copy_(host[o:min(up_bytes, o + (4 << 20))], non_blocking=True)

    def down():
        for o in range(0, down_bytes, 2 << 20):
            host[o:min(down_bytes, o + (2 << 20))].copy_(devbuf[o:min(down_bytes, o + (2 << 20))], non_blocking=True)

    return up_bytes / (timed(up) * 1e-3) / 1e9, down_bytes / (timed(down) * 1e-3) / 1e9


# ----------------------------------------------------------------------------- batched forms


def _event_ms(fn, warmup: int, reps: int) -> float:
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def residue_ablation(dev, case, reps: int = 20) -> dict:
    """Residue stage alone for both operands of the main workload, by the integer pipes (the
    product path's arithmetic) and by the INT8 tensor-core contraction; L2 flushed before each
    timed pair; both engines' residues compared bit for bit."""
    import numpy as np
    import torch

    import negacyclic as nc

    with nc.Plan(case.N, case.q_limbs, W=case.W) as plan:
        k, N, L = plan.k, plan.N, plan.L
        da = torch.from_numpy(case.a.view(np.int32)).to(dev)
        db = torch.from_numpy(case.b.view(np.int32)).to(dev)
        flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
        outs, ms = {}, {}
        for name, engine in (("imad", nc.RESIDUES_IMAD), ("tc_i8", nc.RESIDUES_TC_I8)):
            r = torch.empty(2 * k * N, dtype=torch.int64, device=dev)
            ra, rb = r.data_ptr(), r.data_ptr() + k * N * 8

            def pair():
                plan.residues(da.data_ptr(), ra, engine)
                plan.residues(db.data_ptr(), rb, engine)

            for _ in range(3):
                pair()
            times = []
            for _ in range(reps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                pair()
                e1.record()
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
            if nc.residues_gave_up():
                raise RuntimeError("a tensor-core residue launch gave up its wait")
            outs[name] = r
            ms[name] = statistics.median(times)
        exact = bool(torch.equal(outs["imad"], outs["tc_i8"]))
    if not exact:
        raise RuntimeError("the two residue engines disagree")
    hbm_bytes = 2 * (N * L * 4 + k * N * 8)
    macs = 2 * k * N * L  # u32 x u64 limb MACs of the integer engine
    return {"what": "residues x mod p_i of both operands (k x N u64 each), N=65536, 868-bit q, k=29",
            "imad_us": 1e3 * ms["imad"], "tc_i8_us": 1e3 * ms["tc_i8"], "speedup": ms["imad"] / ms["tc_i8"],
            "bit_exact": exact, "tc_i8_hbm_gbs": hbm_bytes / (ms["tc_i8"] * 1e-3) / 1e9,
            "tc_i8_int8_tops": 2 * 2 * 128 * (8 * ((k + 1) & ~1)) * N / (ms["tc_i8"] * 1e-3) / 1e12,
            "imad_limb_macs_per_s": macs / (ms["imad"] * 1e-3), "hbm_bytes": hbm_bytes,
            "l2": "flushed (256 MiB write) before each timed pair"}


def _flushed_ms(fn, flush, reps: int) -> float:
    """Median CUDA-event milliseconds of fn() over `reps` runs, L2 flushed before each."""
    import torch

    for _ in range(3):
        fn()
    times = []
    for _ in range(reps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return statistics.median(times)


def chained(dev, reps: int = 10) -> dict:
    """x_0 x_1 ... x_{m-1} at N=65536 as one chained product (one residue stage per operand, one
    row launch with every forward transform and pointwise product, one inverse transform and CRT)
    against m - 1 plain products where each feeds the next, device-resident, L2 flushed before each
    timed run; both outputs compared."""
    import numpy as np
    import torch

    import cases
    import negacyclic as nc

    N = 65536
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    out = {}
    for m, bits in ((3, 868), (4, 731), (4, 434)):
        L = (bits + 31) // 32
        q = cases.gen_prime(bits, 4000 + bits)
        ql = cases.limbs_of(q, L)
        xs = [torch.from_numpy(cases.coeffs(q, N, L, 4100 + f).view(np.int32)).to(dev) for f in range(m)]
        c_chain, c_pair, tmp = (torch.empty_like(xs[0]) for _ in range(3))
        with nc.Plan(N, ql, factors=m) as chain, nc.Plan(N, ql) as pair:
            chain.autotune(reps=2)
            pair.autotune(reps=2)
            ptrs = [x.data_ptr() for x in xs]

            def run_chain():
                chain.multiply_chain_device(ptrs, c_chain.data_ptr(), 0)

            # ping-pong so that the last product lands in c_pair
            bufs = [c_pair.data_ptr() if (m - 2 - i) % 2 == 0 else tmp.data_ptr() for i in range(m - 1)]

            def run_pairs():
                pair.multiply_device(ptrs[0], ptrs[1], bufs[0], 0)
                for i, x in enumerate(ptrs[2:], start=1):
                    pair.multiply_device(bufs[i - 1], x, bufs[i], 0)

            ms_chain = _flushed_ms(run_chain, flush, reps)
            ms_pairs = _flushed_ms(run_pairs, flush, reps)
            exact = bool(torch.equal(c_chain, c_pair))
            k_chain, k_pair, word_pair = chain.k, pair.plain_primes, pair.word_bits
        if not exact:
            raise RuntimeError(f"chained and pairwise products differ (m={m}, {bits}-bit q)")
        out[f"m{m}_q{bits}"] = {"chain_us": 1e3 * ms_chain, "pairwise_us": 1e3 * ms_pairs,
                                "speedup": ms_pairs / ms_chain, "primes_chain": k_chain,
                                "primes_pairwise": k_pair, "pairwise_word_bits": word_pair,
                                "bit_exact_vs_pairwise": exact}
    out["form"] = ("N=65536, device-resident; pairwise = m - 1 plain products (the plan's engine: 30-bit "
                   "where it runs), each output the next product's operand; the chain runs the 62-bit engine "
                   "(its bound needs more than 64 primes below 2^30); L2 flushed before each timed run; "
                   "median of 10")
    return out


def batched_same_shape(dev, q: int, N: int, count: int, args) -> dict:
    """`count` products of one (N, q): one batch replayed from a CUDA graph (below N = 2^15: a residue
    launch, a persistent launch for the rows and a CRT launch; from 2^15: each product's own
    launches over two streams), against the same products as back-to-back plain per-call launches.
    Operands (> L2) stay in HBM."""
    import numpy as np
    import torch

    import cases
    import negacyclic as nc

    L = (BITS + 31) // 32
    ql = cases.limbs_of(q, L)
    rng = np.random.default_rng(N + count)
    a = [torch.from_numpy(cases.coeffs(q, N, L, 9000 + i).view(np.int32)).to(dev) for i in range(min(count, 8))]
    b = [torch.from_numpy(cases.coeffs(q, N, L, 9100 + i).view(np.int32)).to(dev) for i in range(min(count, 8))]
    ops = [(a[i % len(a)], b[(i * 5 + 3) % len(b)]) for i in range(count)]
    outs_b = [torch.empty_like(a[0]) for _ in range(count)]
    outs_p = [torch.empty_like(a[0]) for _ in range(count)]
    del rng
    with nc.Plan(N, ql) as plan, nc.Batch() as batch:
        plan.autotune(reps=2)
        for (x, y), z in zip(ops, outs_b):
            batch.add(plan, x.data_ptr(), y.data_ptr(), z.data_ptr())

        def run_batch():
            batch.run(0, True)

        def run_plain():
            for (x, y), z in zip(ops, outs_p):
                plan.multiply_device(x.data_ptr(), y.data_ptr(), z.data_ptr(), 0)

        ms_batch = _event_ms(run_batch, 2, 5)
        batch.synchronize()
        ms_plain = _event_ms(run_plain, 2, 5)
        exact = all(torch.equal(p, q_) for p, q_ in zip(outs_b, outs_p))
        info = batch.query()
    if not exact:
        raise RuntimeError(f"batched and plain products differ at N={N}")
    if N >= 1 << 15:
        launches, form = 3 * count, ("per product: tensor-core residues, rows with the tuned configuration, "
                                     "tensor-core CRT; products alternate over two streams inside one CUDA graph")
    else:
        launches, form = 3, ("one tensor-core residue launch, one persistent launch for the row stage, one "
                             "tensor-core CRT launch; CUDA graph replay")
    return {"products": count, "N": N, "q_bits": BITS,
            "batched": {"value": count / (ms_batch * 1e-3), "unit": "products/s", "ms_per_launch": ms_batch,
                        "ctas": info["ctas"], "gpu_launches_per_batch": launches, "form": form},
            "plain": {"value": count / (ms_plain * 1e-3), "unit": "products/s",
                      "gpu_launches_per_batch": 3 * count, "form": "3 launches per product, back to back"},
            "speedup": ms_plain / ms_batch, "bit_exact_vs_plain": exact}


def uneven_batch(dev, mix, args) -> dict:
    """The 256-product uneven mix (N log-uniform 2^10..2^16, 434- and 868-bit seeded q) in one
    persistent launch, against per-product plain launches of the same products."""
    import numpy as np
    import torch

    import cases
    import negacyclic as nc

    plans, bufs, engines = [], [], []
    for i, (N, bits, q) in enumerate(mix):
        L = (bits + 31) // 32
        p = nc.Plan(N, cases.limbs_of(q, L))
        engines.append((p.plain_primes, p.word_bits))
        x = torch.from_numpy(cases.coeffs(q, N, L, 11000 + i).view(np.int32)).to(dev)
        y = torch.from_numpy(cases.coeffs(q, N, L, 12000 + i).view(np.int32)).to(dev)
        plans.append(p)
        bufs.append((x, y, torch.empty_like(x), torch.empty_like(x)))
    try:
        with nc.Batch() as batch:
            for p, (x, y, z, _) in zip(plans, bufs):
                batch.add(p, x.data_ptr(), y.data_ptr(), z.data_ptr())
            ms_batch = _event_ms(lambda: batch.run(0, True), 2, 5)
            batch.synchronize()

            def plain():
                for p, (x, y, _, w) in zip(plans, bufs):
                    p.multiply_device(x.data_ptr(), y.data_ptr(), w.data_ptr(), 0)

            ms_plain = _event_ms(plain, 1, 3)
            exact = all(torch.equal(z, w) for _, _, z, w in bufs)
            info = batch.query()
    finally:
        for p in plans:
            p.close()
    if not exact:
        raise RuntimeError("uneven batch differs from plain products")
    total_imad = 0.0
    for (N, bits, _), (k, word) in zip(mix, engines):
        total_imad += sum(stage_work(k, N, (bits + 31) // 32, None, word))
    return {"products": len(mix), "mix": "N log-uniform 2^10..2^16, q 434- or 868-bit (seeded per product)",
            "batched": {"value": len(mix) / (ms_batch * 1e-3), "unit": "products/s", "ms_per_launch": ms_batch,
                        "ctas": info["ctas"], "imad_alg_rate_gops": total_imad / (ms_batch * 1e-3) / 1e9},
            "plain": {"value": len(mix) / (ms_plain * 1e-3), "unit": "products/s", "ms": ms_plain},
            "speedup": ms_plain / ms_batch, "bit_exact_vs_plain": exact}


def serving(dev, mix, args, rates=(2000, 8000, 16000), requests=600, streams=3, max_batch=64) -> dict:
    """Poisson arrivals of the uneven mix at each rate; 30% of requests reuse one of 8 registered
    operands (NTT form cached on the device); admission by a 40 GB HBM budget. The same arrival
    schedule is also served by the plain per-call form (one worker, fherma_run-style host calls)."""
    import random
    import threading

    import numpy as np

    import cases
    import negacyclic as nc

    rng = random.Random(MIX_SEED)
    sub = mix[:64]  # 64 distinct (N, q) plans serve the requests
    plans = []
    for N, bits, q in sub:
        L = (bits + 31) // 32
        plans.append((nc.Plan(N, cases.limbs_of(q, L)), q, L))
    host = [(cases.coeffs(q, p.N, L, 13000 + i), cases.coeffs(q, p.N, L, 14000 + i)) for i, (p, q, L) in
            enumerate(plans)]
    out = {"budget_bytes": 40 << 30, "requests_per_rate": requests, "reuse_fraction": 0.3, "streams": streams,
           "max_batch": max_batch, "rates": []}
    try:
        # every request of plan i multiplies host[i]: one expected product per plan (this also
        # allocates each plan's staging before any timing)
        want = [p.multiply(a, b) for (p, _, _), (a, b) in zip(plans, host)]
        for rate in rates:
            sched = []
            t = 0.0
            for _ in range(requests):
                t += rng.expovariate(rate)
                pi = rng.randrange(len(plans))
                sched.append((t, pi, rng.random() < 0.3 and pi < 8))
            row = {"rate_per_s": rate}
            with nc.Server(hbm_budget=40 << 30, staging=2 << 30, max_batch=max_batch, streams=streams) as srv:
                opids = {i: srv.register_operand(plans[i][0], host[i][0]) for i in range(8)}
                clients = 8  # independent Poisson clients (their superposition is Poisson at `rate`)
                t0 = time.perf_counter()

                def producer(c, pending):
                    for ta, pi, reuse in sched[c::clients]:
                        while time.perf_counter() - t0 < ta:
                            time.sleep(0)
                        p = plans[pi][0]
                        a, b = host[pi]
                        pending.put((pi, srv.submit(p, None if reuse else a, b, operand=opids[pi] if reuse else -1)))
                    pending.put(None)

                wrong, failed, lat_srv = [], [], []

                def consumer(pending):  # each client collects and checks its results as they come
                    while (item := pending.get()) is not None:
                        try:
                            c, ms = srv.wait(item[1], plans[item[0]][0])
                        except nc.NegacyclicError as e:  # keep draining so staging is released
                            failed.append(str(e))
                            continue
                        lat_srv.append(ms)
                        if not np.array_equal(c, want[item[0]]):
                            wrong.append(item[0])

                threads = []
                for c in range(clients):
                    qq = queue.Queue()
                    threads += [threading.Thread(target=producer, args=(c, qq)), threading.Thread(target=consumer, args=(qq,))]
                for th in threads:
                    th.start()
                for th in threads:
                    th.join()
                st = srv.stats()
                io = srv.io_stats()
            if wrong or failed:
                raise RuntimeError(f"served products differ from the plain path for plans {sorted(set(wrong))[:8]}; "
                                   f"{len(failed)} requests failed: {failed[:2]}")
            win = io["device_window_ms"] * 1e-3
            row["server"] = {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": max(lat_srv),
                             "products_per_s": st["products_per_s"], "batches": st["batches"],
                             "timeouts": st["timeouts"], "verified": len(lat_srv),
                             "h2d_gbs": io["h2d_bytes"] / win / 1e9 if win else None,
                             "d2h_gbs": io["d2h_bytes"] / win / 1e9 if win else None,
                             "device_busy_frac": io["device_busy_ms"] / io["device_window_ms"]
                             if io["device_window_ms"] else None,
                             "batch_size_mean": len(lat_srv) / st["batches"] if st["batches"] else None,
                             "scheduler_busy_frac": io["scheduler_ms"] / io["device_window_ms"]
                             if io["device_window_ms"] else None}
            # plain per-call form on the same schedule: one worker, host operands in and out
            lat = []
            t0 = time.perf_counter()
            for ta, pi, _ in sched:
                while time.perf_counter() - t0 < ta:
                    pass
                p = plans[pi][0]
                a, b = host[pi]
                p.multiply(a, b)
                lat.append(1e3 * (time.perf_counter() - t0 - ta))
            wall = time.perf_counter() - t0
            row["plain_per_call"] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                                     "products_per_s": requests / wall}
            out["rates"].append(row)
    finally:
        for p, _, _ in plans:
            p.close()
    return out


REF_KERNELS_FILE = ROOT / "profiles" / "reference_kernels_n65536.json"


def _reference_device_time() -> dict | None:
    """The reference's kernel time per product (sum of its launches' ncu durations over whole
    products, from the committed launch-list summary), beside its wall-clock value."""
    try:
        tf = json.loads(REF_KERNELS_FILE.read_text())
    except Exception:
        return None
    ms = tf.get("device_ms_per_product")
    if not ms:
        return None
    return {"value": 1e3 / ms, "unit": "products/s", "ms_per_product": ms,
            "source": f"{REF_KERNELS_FILE.relative_to(ROOT)} (ncu gpu__time_duration.sum per launch, "
                      f"serialised and cold-cache)"}


def _hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return json.loads(p.read_text()).get("hbm_gbs")
    except Exception:
        return None


def reference(args) -> dict | None:
    import cases

    world, rank, _ = dist_setup(args)
    if rank != 0:
        return None
    case = cases.make_case(N_MAIN, BITS, SEED, edge_frac=EDGE)
    N, L = case.N, case.L
    base = {"metric": METRIC, "unit": "products/s", "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64", "data": "synthetic (seeded)", "config": config(f"replicas{world}")}
    why = None
    if REF_BINARY.exists():
        try:
            secs, init_s, _, first_s = run_harness(REF_BINARY, case, args.warmup, args.steps)
            per = statistics.mean(secs)
            v = 1.0 / per
            # fherma_run of the reference copies both operands in and the product out inside the
            # timed call (solve.cu:1499-1520), so its wall clock is an end-to-end figure
            base.update({"value": v, "ms_per_step": 1e3 * per, "init_s": init_s,
                         "cpu_baseline": {"value": v, "unit": "products/s", "cores": 1, "kind": "reference",
                                          "sample": f"reference solve.cu (sm_100a; kMaxN raised to 65536 and the "
                                                    f"L=28 init self-check throw removed, kernels unmodified) "
                                                    f"with its own harness main.cpp, "
                                                    f"{args.steps} timed products after {args.warmup} warm-up; "
                                                    f"its kernels run on the GPU, one host thread drives them"},
                         "e2e": {"value": v, "unit": "products/s", "h2d_bytes_per_step": 2 * N * L * 4,
                                 "d2h_bytes_per_step": N * L * 4, "ms_p50": 1e3 * statistics.median(secs),
                                 "first_call_ms": 1e3 * first_s,
                                 "via": "fherma_run in the reference's own harness main.cpp (wall clock)"},
                         "gpu_launches": None})
            dev_ref = _reference_device_time()
            if dev_ref:
                base["device"] = dev_ref
            return base
        except Exception as e:  # fall back to the CPU oracle
            why = str(e)[:300]
    cb = cpu_baseline(case)
    base.update({"value": cb["value"], "ms_per_step": 1e3 / cb["value"], "cpu_baseline": cb,
                 "e2e": {"value": cb["value"], "unit": "products/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                 "note": f"reference binary unavailable ({why or 'not built'}); CPU oracle timed instead"})
    return base


# ----------------------------------------------------------------------------- profiling modes


def profile_case(a) -> int:
    """Device-resident products of one seeded case for a profiler: each rep enqueues the three
    kernels of one product (k_dec_tc or k_dec, k_row, k_crt_tc) on the default stream with the
    --row-config configuration (default: the plan's default); with --profile-batch B each rep is
    one batch of B products (k_persistent and the batched residue / CRT launches); with
    --profile-residues each rep is the residue stage alone of both operands (k_residues_imad or
    k_residues_tc). The run ends by checking the last result against the host entry point (or,
    for --profile-residues, against the other residue engine)."""
    import numpy as np
    import torch

    import cases
    import negacyclic as nc

    case = cases.make_case(a.profile_N, a.profile_bits, a.profile_seed, edge_frac=0.01)
    dev = torch.device("cuda", 0)
    da = torch.from_numpy(case.a.view(np.int32)).to(dev)
    db = torch.from_numpy(case.b.view(np.int32)).to(dev)
    if a.profile_residues:
        engine = nc.RESIDUES_TC_I8 if a.profile_residues == "tc" else nc.RESIDUES_IMAD
        other = nc.RESIDUES_IMAD if engine == nc.RESIDUES_TC_I8 else nc.RESIDUES_TC_I8
        with nc.Plan(case.N, case.q_limbs, W=case.W) as plan:
            k, N = plan.k, plan.N
            r = torch.empty(2 * k * N, dtype=torch.int64, device=dev)
            check = torch.empty_like(r)
            for _ in range(a.profile_reps):
                for j, x in enumerate((da, db)):
                    plan.residues(x.data_ptr(), r.data_ptr() + j * k * N * 8, engine)
            for j, x in enumerate((da, db)):
                plan.residues(x.data_ptr(), check.data_ptr() + j * k * N * 8, other)
            torch.cuda.synchronize()
            ok = bool(torch.equal(r, check)) and not nc.residues_gave_up()
        print(f"residues N={case.N} bits={a.profile_bits} reps={a.profile_reps} engine={a.profile_residues} "
              f"consistent={ok}")
        return 0 if ok else 1
    count = max(1, a.profile_batch)
    dcs = [torch.empty_like(da) for _ in range(count)]
    with nc.Plan(case.N, case.q_limbs, W=case.W) as plan:
        if a.profile_word_bits:
            plan.word_bits = a.profile_word_bits
        if a.row_config:
            plan.row_config = tuple(int(x) for x in a.row_config.split(","))
        if a.profile_residue_engine == "imad" or plan.k > 32:
            plan.residue_engine = nc.RESIDUES_IMAD
        if a.profile_batch > 0:
            with nc.Batch() as batch:
                for dc in dcs:
                    batch.add(plan, da.data_ptr(), db.data_ptr(), dc.data_ptr())
                for _ in range(a.profile_reps):
                    batch.run(0, False)
                batch.synchronize()
        else:
            for _ in range(a.profile_reps):
                plan.multiply_device(da.data_ptr(), db.data_ptr(), dcs[0].data_ptr(), 0)
        torch.cuda.synchronize()
        want = plan.multiply(case.a, case.b)
        cfg = plan.row_config
    ok = all(np.array_equal(dc.cpu().numpy().view(np.uint32), want) for dc in dcs)
    print(f"N={case.N} bits={a.profile_bits} reps={a.profile_reps} batch={a.profile_batch} config={cfg} consistent={ok}")
    return 0 if ok else 1


def profile_reference(a) -> int:
    """The reference's own binary (its harness main.cpp) on `--profile-reference` products of the
    bench workload, for a launch list of its kernels; its last product is checked against the
    library's product of the same case."""
    import numpy as np

    import cases

    case = cases.make_case(N_MAIN, BITS, SEED, edge_frac=EDGE)
    if not REF_BINARY.exists():
        print(f"no reference binary at {REF_BINARY.relative_to(ROOT)}")
        return 1
    _, _, out, _ = run_harness(REF_BINARY, case, 0, a.profile_reference)
    import negacyclic as nc

    with nc.Plan(case.N, case.q_limbs, W=case.W) as plan:
        want = plan.multiply(case.a, case.b)
    ok = bool(np.array_equal(out, want))
    print(f"reference products={a.profile_reference} N={case.N} matches_library={ok}")
    return 0 if ok else 1


def main() -> int:
    args = parse_args()
    if args.profile_case:
        return profile_case(args)
    if args.profile_reference:
        return profile_reference(args)
    out = reference(args) if args.impl == "reference" else ours(args)
    if out is not None:
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
