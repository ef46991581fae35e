"""Seeded synthetic cases for the negacyclic product, and the harness's case-directory format.

Moduli: a seeded prime q of `bits` bits, top bit set, odd, 40 rounds of Miller-Rabin with
seeded bases. Coefficients: uniform in [0, q) by rejection over raw PCG64 words, optionally
with a fraction replaced by edge values {0, 1, q-1, 2^j mod q (j uniform in [0, 1000))}.
Every draw is a pure function of its seed.

Case directory (the reference harness's format, main.cpp:47-86):
    manifest.json            {"N": .., "W": .., "L": .., "cases": ..}
    point/q.bin              L little-endian u32
    cases/000000/a.bin       N*L little-endian u32, coefficient-major
    cases/000000/b.bin
    out/000000/c.bin         written by the runner
    out/results.json         {"init_s": .., "cases": [{"i":..,"seconds":..,"status":..}]}
"""
from __future__ import annotations

import json
import random
from dataclasses import dataclass
from pathlib import Path

import numpy as np


# ----------------------------------------------------------------------------- integers


def is_probable_prime(n: int, rounds: int, rng: random.Random) -> bool:
    if n < 2:
        return False
    for sp in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % sp == 0:
            return n == sp
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for _ in range(rounds):
        a = rng.randrange(2, n - 1)
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def gen_prime(bits: int, seed: int, rounds: int = 40) -> int:
    """Seeded `bits`-bit prime with the top bit set."""
    rng = random.Random(seed)
    while True:
        x = rng.getrandbits(bits) | (1 << (bits - 1)) | 1
        if is_probable_prime(x, rounds, rng):
            return x


def _primorial(limit: int) -> int:
    sieve = bytearray([1]) * limit
    sieve[0:2] = b"\x00\x00"
    for i in range(2, int(limit ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = bytearray(len(sieve[i * i::i]))
    out = 1
    for i, s in enumerate(sieve):
        if s:
            out *= i
    return out


_PRIMORIAL = None


def gen_prime_fast(bits: int, seed: int, rounds: int = 40) -> int:
    """Seeded `bits`-bit prime (top bit set, Miller-Rabin `rounds` rounds with seeded bases).
    Candidates sharing a factor below 10000 are dropped by one gcd before any Miller-Rabin
    round, so it is several times faster than gen_prime; it yields different primes for the
    same seed (its own seeded sequence)."""
    global _PRIMORIAL
    import math

    if _PRIMORIAL is None:
        _PRIMORIAL = _primorial(10000)
    rng = random.Random(seed)
    while True:
        x = rng.getrandbits(bits) | (1 << (bits - 1)) | 1
        if math.gcd(x, _PRIMORIAL) != 1:
            continue
        if is_probable_prime(x, rounds, rng):
            return x


def _prime_job(args):
    return gen_prime_fast(*args)


def uneven_mix(count: int, seed: int, log_n=(10, 16), widths=(434, 868),
               processes: int = 0) -> list[tuple[int, int, int]]:
    """(N, bits, q) per product: N log-uniform over 2^log_n[0]..2^log_n[1], width uniform over
    `widths`, a seeded prime q of that width per product. With processes > 1 the primes are
    found by a spawn-context process pool (create it before the process initialises CUDA)."""
    rng = random.Random(seed)
    shape = []
    for i in range(count):
        N = 1 << rng.randint(*log_n)
        shape.append((N, rng.choice(list(widths))))
    jobs = [(bits, seed * 100003 + i) for i, (_, bits) in enumerate(shape)]
    if processes > 1:
        import multiprocessing as mp

        with mp.get_context("spawn").Pool(processes) as pool:
            qs = pool.map(_prime_job, jobs, chunksize=4)
    else:
        qs = [gen_prime_fast(*j) for j in jobs]
    return [(N, bits, q) for (N, bits), q in zip(shape, qs)]


def limbs_of(x: int, L: int) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(L)], dtype=np.uint32)


def int_of(limbs) -> int:
    v = 0
    for i, w in enumerate(np.asarray(limbs, dtype=np.uint64).tolist()):
        v |= int(w) << (32 * i)
    return v


def ints_of_rows(arr: np.ndarray) -> list[int]:
    """Rows of an (n, L) u32 array as Python integers."""
    arr = np.ascontiguousarray(arr, dtype=np.uint32)
    n, L = arr.shape
    raw = arr.tobytes()
    step = 4 * L
    return [int.from_bytes(raw[i * step:(i + 1) * step], "little") for i in range(n)]


def rows_of_ints(values, L: int) -> np.ndarray:
    buf = b"".join(int(v).to_bytes(4 * L, "little") for v in values)
    return np.frombuffer(buf, dtype=np.uint32).reshape(len(values), L).copy()


# ----------------------------------------------------------------------------- coefficients


def _less_than(rows: np.ndarray, q: np.ndarray) -> np.ndarray:
    """Lexicographic rows < q over little-endian limbs."""
    less = np.zeros(rows.shape[0], dtype=bool)
    decided = np.zeros(rows.shape[0], dtype=bool)
    for l in range(rows.shape[1] - 1, -1, -1):
        lt = rows[:, l] < q[l]
        gt = rows[:, l] > q[l]
        less |= ~decided & lt
        decided |= lt | gt
    return less


def uniform_coeffs(q: int, N: int, L: int, seed: int) -> np.ndarray:
    """(N, L) u32 limbs, each row uniform in [0, q)."""
    gen = np.random.PCG64(seed)
    qbits = q.bit_length()
    ql = limbs_of(q, L)
    top = (qbits - 1) // 32
    top_mask = np.uint32((1 << (qbits - 32 * top)) - 1) if qbits - 32 * top < 32 else np.uint32(0xFFFFFFFF)
    out = np.zeros((N, L), dtype=np.uint32)
    todo = np.arange(N)
    while todo.size:
        words = (todo.size * L + 1) // 2
        raw = gen.random_raw(words).astype(np.uint64)
        limbs = np.empty(words * 2, dtype=np.uint32)
        limbs[0::2] = (raw & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        limbs[1::2] = (raw >> np.uint64(32)).astype(np.uint32)
        rows = limbs[: todo.size * L].reshape(todo.size, L)
        rows[:, top + 1:] = 0
        rows[:, top] &= top_mask
        ok = _less_than(rows, ql)
        out[todo[ok]] = rows[ok]
        todo = todo[~ok]
    return out


def edge_values(q: int, count: int, seed: int) -> list[int]:
    rng = random.Random(seed)
    vals = []
    for _ in range(count):
        kind = rng.randrange(4)
        if kind == 0:
            vals.append(0)
        elif kind == 1:
            vals.append(1)
        elif kind == 2:
            vals.append(q - 1)
        else:
            vals.append(pow(2, rng.randrange(1000), q))
    return vals


def coeffs(q: int, N: int, L: int, seed: int, edge_frac: float = 0.0) -> np.ndarray:
    """Uniform coefficients with a seeded fraction of edge values."""
    out = uniform_coeffs(q, N, L, seed)
    n_edge = int(round(N * edge_frac))
    if n_edge:
        rng = random.Random(seed ^ 0x5EED)
        idx = rng.sample(range(N), n_edge)
        out[idx] = rows_of_ints(edge_values(q, n_edge, seed ^ 0xED6E), L)
    return out


@dataclass
class Case:
    N: int
    L: int
    W: int
    q: int
    a: np.ndarray
    b: np.ndarray

    @property
    def q_limbs(self) -> np.ndarray:
        return limbs_of(self.q, self.L)


def make_case(N: int, bits: int, seed: int, edge_frac: float = 0.0, q: int | None = None) -> Case:
    """One seeded product: q from `seed`, a and b from derived seeds."""
    L = (bits + 31) // 32
    if q is None:
        q = gen_prime(bits, seed)
    a = coeffs(q, N, L, seed * 2 + 1, edge_frac)
    b = coeffs(q, N, L, seed * 2 + 2, edge_frac)
    return Case(N=N, L=L, W=bits, q=q, a=a, b=b)


# ----------------------------------------------------------------------------- harness format


def write_case_dir(root: Path, N: int, W: int, L: int, q: int, pairs) -> None:
    root = Path(root)
    (root / "point").mkdir(parents=True, exist_ok=True)
    limbs_of(q, L).tofile(root / "point" / "q.bin")
    pairs = list(pairs)
    for i, (a, b) in enumerate(pairs):
        d = root / "cases" / f"{i:06d}"
        d.mkdir(parents=True, exist_ok=True)
        np.ascontiguousarray(a, dtype=np.uint32).tofile(d / "a.bin")
        np.ascontiguousarray(b, dtype=np.uint32).tofile(d / "b.bin")
    (root / "manifest.json").write_text(json.dumps({"N": N, "W": W, "L": L, "cases": len(pairs)}))


def read_output(root: Path, i: int, N: int, L: int) -> np.ndarray:
    return np.fromfile(Path(root) / "out" / f"{i:06d}" / "c.bin", dtype=np.uint32).reshape(N, L)


def read_results(root: Path) -> dict:
    return json.loads((Path(root) / "out" / "results.json").read_text())
