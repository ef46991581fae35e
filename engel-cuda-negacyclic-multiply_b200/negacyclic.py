"""Python binding of libnegacyclic_b200.so (ctypes over the C ABI in include/negacyclic_b200.h).

The functions fherma_init / fherma_run / fherma_free mirror the reference's C++ contract
(fherma.h:45-47): same names, same argument meaning (Point{N, W, L, q}, Inputs{a, b},
Outputs{c} with N x L little-endian u32 limbs) and the same error behaviour (a RuntimeError
with a message where the reference throws std::runtime_error).

There is no fallback: if the shared library is missing or fails to load, every entry point
raises. Build it with `python build.py` in this directory.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libnegacyclic_b200.so"

NC_OK, NC_EINVAL, NC_ECUDA, NC_ENOMEM, NC_ETIMEOUT, NC_EBUSY, NC_ESELFCHECK = 0, -1, -2, -3, -4, -5, -6

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p

# (name, restype, argtypes) of every symbol include/negacyclic_b200.h declares.
C_SYMBOLS = [
    ("nc_last_error", ctypes.c_char_p, []),
    ("nc_version", ctypes.c_int, []),
    ("nc_plan_create", ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p, ctypes.POINTER(_vp)]),
    ("nc_self_check", ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p]),
    ("nc_plan_destroy", ctypes.c_int, [_vp]),
    ("nc_multiply", ctypes.c_int, [_vp, _u32p, _u32p, _u32p]),
    ("nc_multiply_device", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    ("nc_multiply_device_noalloc", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    ("nc_plan_create_chain", ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p, ctypes.c_int,
                                            ctypes.POINTER(_vp)]),
    ("nc_plan_factors", ctypes.c_int, [_vp]),
    ("nc_multiply_chain", ctypes.c_int, [_vp, ctypes.POINTER(_u32p), _u32p]),
    ("nc_multiply_chain_device", ctypes.c_int, [_vp, ctypes.POINTER(_vp), _vp, _vp]),
    ("nc_plan_set_crt_engine", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nc_plan_get_crt_engine", ctypes.c_int, [_vp]),
    ("nc_plan_synchronize", ctypes.c_int, [_vp]),
    ("nc_plan_query", ctypes.c_int, [_vp, _u32p, _u32p, _u32p, _u32p]),
    ("nc_plan_last_kernel_ms", ctypes.c_float, [_vp]),
    ("nc_plan_set_timing", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nc_plan_stage_ms", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float)]),
    ("nc_imad_peak", ctypes.c_int, [ctypes.POINTER(ctypes.c_double)]),
    ("nc_primes", ctypes.c_int, [_u64p, ctypes.c_int]),
    ("nc_primes32", ctypes.c_int, [_u32p, ctypes.c_int]),
    ("nc_residues", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    ("nc_residues_status", ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    ("nc_plan_set_residue_engine", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nc_plan_get_residue_engine", ctypes.c_int, [_vp]),
    ("nc_row_variants", ctypes.c_int, [ctypes.c_uint32, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    ("nc_plan_set_row_config", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("nc_plan_get_row_config", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int)]),
    ("nc_plan_autotune", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    ("nc_row_variants32", ctypes.c_int, [ctypes.c_uint32, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    ("nc_plan_set_word_bits", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nc_plan_word_bits", ctypes.c_int, [_vp, _u32p]),
    ("nc_batch_create", ctypes.c_int, [ctypes.POINTER(_vp)]),
    ("nc_batch_destroy", ctypes.c_int, [_vp]),
    ("nc_batch_add", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    ("nc_batch_add_cached", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    ("nc_batch_add_forward", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("nc_batch_clear", ctypes.c_int, [_vp]),
    ("nc_batch_run", ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    ("nc_batch_synchronize", ctypes.c_int, [_vp]),
    ("nc_batch_query", ctypes.c_int, [_vp, _u32p, _u32p, _u64p]),
    ("nc_plan_hat_words", ctypes.c_uint64, [_vp]),
    ("nc_server_create", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(_vp)]),
    ("nc_server_destroy", ctypes.c_int, [_vp]),
    ("nc_server_register_operand", ctypes.c_int, [_vp, _vp, _u32p, ctypes.POINTER(ctypes.c_int)]),
    ("nc_server_release_operand", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nc_server_submit", ctypes.c_int, [_vp, _vp, _u32p, ctypes.c_int, _u32p, _u64p]),
    ("nc_server_poll", ctypes.c_int, [_vp, ctypes.c_uint64]),
    ("nc_server_wait", ctypes.c_int, [_vp, ctypes.c_uint64, _u32p, ctypes.POINTER(ctypes.c_double)]),
    ("nc_server_stats", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), _u64p,
                                       ctypes.POINTER(ctypes.c_double), _u64p, _u64p, _u64p]),
    ("nc_server_io_stats", ctypes.c_int, [_vp, _u64p, _u64p, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
]

_lib: ctypes.CDLL | None = None


class NegacyclicError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{message} (status {code})")
        self.code = code


def load(path: str | Path | None = None) -> ctypes.CDLL:
    """Load the library (once) and declare every C entry point."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: build it with `python build.py` (no CPU fallback exists)")
    lib = ctypes.CDLL(str(p))
    for name, res, args in C_SYMBOLS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _check(status: int) -> None:
    if status != NC_OK:
        msg = load().nc_last_error().decode(errors="replace")
        raise NegacyclicError(status, msg)


def _u32(arr: np.ndarray):
    return arr.ctypes.data_as(_u32p)


def imad_peak() -> float:
    """Measured mad.lo.u32 throughput of the current device (ops/s)."""
    v = ctypes.c_double()
    _check(load().nc_imad_peak(ctypes.byref(v)))
    return float(v.value)


def primes(count: int = 48) -> list[int]:
    out = (ctypes.c_uint64 * count)()
    _check(load().nc_primes(out, count))
    return list(out)


def primes32(count: int = 64) -> list[int]:
    """The 30-bit word engine's primes (below 2^30, 1 mod 2^17, descending)."""
    out = (ctypes.c_uint32 * count)()
    _check(load().nc_primes32(out, count))
    return list(out)


def self_check(N: int, q_limbs: np.ndarray, W: int = 0) -> None:
    """The init-time checks of plan creation that need no device (nc_self_check); raises
    NegacyclicError (NC_EINVAL for an invalid point, NC_ESELFCHECK for a failed check)."""
    q = np.ascontiguousarray(q_limbs, dtype=np.uint32)
    _check(load().nc_self_check(N, W, len(q), _u32(q)))


RESIDUES_IMAD, RESIDUES_TC_I8 = 0, 1
CRT_IMAD, CRT_TC_I8 = 0, 1


def residues_gave_up() -> bool:
    """True if a tensor-core residue launch on the current device gave up its bounded wait since the
    last call (read after the work has finished)."""
    v = ctypes.c_int()
    _check(load().nc_residues_status(ctypes.byref(v)))
    return bool(v.value)


class Plan:
    """One (N, q) configuration on the current CUDA device."""

    def __init__(self, N: int, q_limbs: np.ndarray, W: int = 0, factors: int = 2, word_bits: int | None = None):
        """factors > 2 makes a chain plan: its primes cover products of that many operands
        (multiply_chain); it still runs ordinary two-operand products. word_bits (32 or 64) picks
        the plain path's residue engine (default: the library's choice; see word_bits)."""
        q = np.ascontiguousarray(q_limbs, dtype=np.uint32)
        self.N, self.L = int(N), int(q.size)
        self._h = _vp()
        if factors == 2:
            _check(load().nc_plan_create(self.N, int(W), self.L, _u32(q), ctypes.byref(self._h)))
        else:
            _check(load().nc_plan_create_chain(self.N, int(W), self.L, _u32(q), int(factors), ctypes.byref(self._h)))
        self.factors = int(load().nc_plan_factors(self._h))
        n, l, k, qb = (ctypes.c_uint32() for _ in range(4))
        _check(load().nc_plan_query(self._h, ctypes.byref(n), ctypes.byref(l), ctypes.byref(k), ctypes.byref(qb)))
        self.k, self.qbits = int(k.value), int(qb.value)
        if word_bits is not None:
            self.word_bits = word_bits

    @property
    def word_bits(self) -> int:
        """32 (the 30-bit engine: u32 residues modulo primes below 2^30) or 64 (the 62-bit engine)
        for this plan's plain-path products; the engine in use."""
        v = load().nc_plan_word_bits(self._h, None)
        if v < 0:
            _check(v)
        return v

    @word_bits.setter
    def word_bits(self, bits: int) -> None:
        _check(load().nc_plan_set_word_bits(self._h, int(bits)))

    @property
    def plain_primes(self) -> int:
        """Residue primes of the plain path's engine in use (k of the 62-bit engine, or the
        30-bit engine's count)."""
        k = ctypes.c_uint32()
        v = load().nc_plan_word_bits(self._h, ctypes.byref(k))
        if v < 0:
            _check(v)
        return int(k.value)

    @property
    def handle(self) -> int:
        return int(self._h.value or 0)

    def multiply(self, a: np.ndarray, b: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        """Host arrays (N, L) u32 in, product out (nc_multiply: copies both ways)."""
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = np.ascontiguousarray(b, dtype=np.uint32)
        if a.size != self.N * self.L or b.size != self.N * self.L:
            raise NegacyclicError(NC_EINVAL, "a and b must contain N*L limbs")
        c = out if out is not None else np.empty((self.N, self.L), dtype=np.uint32)
        _check(load().nc_multiply(self._h, _u32(a), _u32(b), _u32(c)))
        return c

    def multiply_device(self, d_a: int, d_b: int, d_c: int, stream: int = 0) -> None:
        """Device pointers (e.g. torch tensor .data_ptr()), enqueued on `stream` (0: default stream)."""
        _check(load().nc_multiply_device(self._h, _vp(d_a), _vp(d_b), _vp(d_c), _vp(stream or None)))

    def multiply_chain(self, xs, out: np.ndarray | None = None) -> np.ndarray:
        """Product of the plan's `factors` host operands (N, L) u32 (nc_multiply_chain)."""
        if len(xs) != self.factors:
            raise NegacyclicError(NC_EINVAL, f"the plan multiplies {self.factors} operands")
        xs = [np.ascontiguousarray(x, dtype=np.uint32) for x in xs]
        if any(x.size != self.N * self.L for x in xs):
            raise NegacyclicError(NC_EINVAL, "every operand must contain N*L limbs")
        ptrs = (_u32p * len(xs))(*[_u32(x) for x in xs])
        c = out if out is not None else np.empty((self.N, self.L), dtype=np.uint32)
        _check(load().nc_multiply_chain(self._h, ptrs, _u32(c)))
        return c

    def multiply_chain_device(self, d_xs, d_c: int, stream: int = 0) -> None:
        """Device pointers of the plan's `factors` operands, enqueued on `stream`."""
        if len(d_xs) != self.factors:
            raise NegacyclicError(NC_EINVAL, f"the plan multiplies {self.factors} operands")
        ptrs = (_vp * len(d_xs))(*[_vp(int(x)) for x in d_xs])
        _check(load().nc_multiply_chain_device(self._h, ptrs, _vp(d_c), _vp(stream or None)))

    def multiply_device_noalloc(self, d_a: int, d_b: int, d_c: int, stream: int = 0) -> None:
        """Like multiply_device, but allocates nothing: for callers that must not allocate device
        memory at call time. Its residue scratch is one 8 MiB array inside the library shared by
        all calls (so overlapping calls race); limit k * N <= 2^19 (N <= 16384 at an 868-bit q)."""
        _check(load().nc_multiply_device_noalloc(self._h, _vp(d_a), _vp(d_b), _vp(d_c), _vp(stream or None)))

    def residues(self, d_x: int, d_r: int, engine: int = 0, stream: int = 0) -> None:
        """Residue stage alone (an ablation): d_r[i * N + n] = x_n mod p_i, k * N u64, by the integer
        pipes (RESIDUES_IMAD) or an exact INT8 tensor-core contraction (RESIDUES_TC_I8)."""
        _check(load().nc_residues(self._h, _vp(d_x), _vp(d_r), int(engine), _vp(stream or None)))

    @property
    def crt_engine(self) -> int:
        """CRT_TC_I8 (tensor cores, the default for <= 32 primes) or CRT_IMAD (integer pipes)."""
        v = load().nc_plan_get_crt_engine(self._h)
        if v < 0:
            _check(v)
        return v

    @crt_engine.setter
    def crt_engine(self, engine: int) -> None:
        _check(load().nc_plan_set_crt_engine(self._h, int(engine)))

    @property
    def residue_engine(self) -> int:
        """RESIDUES_TC_I8 (the default) or RESIDUES_IMAD for this plan's products."""
        e = load().nc_plan_get_residue_engine(self._h)
        if e < 0:
            _check(e)
        return e

    @residue_engine.setter
    def residue_engine(self, engine: int) -> None:
        _check(load().nc_plan_set_residue_engine(self._h, int(engine)))

    def synchronize(self) -> None:
        _check(load().nc_plan_synchronize(self._h))

    def set_timing(self, enable: bool = True) -> None:
        _check(load().nc_plan_set_timing(self._h, int(enable)))

    def stage_ms(self) -> list[float]:
        out = (ctypes.c_float * 3)()
        _check(load().nc_plan_stage_ms(self._h, out))
        return list(out)

    @property
    def last_kernel_ms(self) -> float:
        return float(load().nc_plan_last_kernel_ms(self._h))

    @property
    def row_config(self) -> tuple[int, int, int]:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(load().nc_plan_get_row_config(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    @row_config.setter
    def row_config(self, cfg: tuple[int, int, int]) -> None:
        _check(load().nc_plan_set_row_config(self._h, *map(int, cfg)))

    def autotune(self, reps: int = 5) -> float:
        """Time every compiled row configuration for this N, keep the fastest; ms per product."""
        ms = ctypes.c_float()
        _check(load().nc_plan_autotune(self._h, int(reps), ctypes.byref(ms)))
        return float(ms.value)

    @property
    def hat_words(self) -> int:
        """u64 words that hold one operand's NTT-domain form on either engine (k * N u64 on the
        62-bit one, k32 * N u32 on the 30-bit one)."""
        return int(load().nc_plan_hat_words(self._h))

    def close(self) -> None:
        if self._h:
            _check(load().nc_plan_destroy(self._h))
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def row_variants(log_n: int, word_bits: int = 64) -> list[tuple[int, int, int]]:
    """Compiled row configurations (log_block, log_radix, threads) valid for N = 2^log_n, of the
    62-bit engine (word_bits 64) or the 30-bit engine (32)."""
    fn = load().nc_row_variants if word_bits == 64 else load().nc_row_variants32
    n = fn(int(log_n), None, 0)
    if n < 0:
        _check(n)
    buf = (ctypes.c_int * (3 * max(n, 1)))()
    got = fn(int(log_n), buf, n)
    return [(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]) for i in range(got)]


class Batch:
    """Many products (any mix of plans) run together (nc_batch_*): tensor-core residue launches, one
    persistent launch for the row stage, one CRT launch per engine; products of N >= 2^15 as plain
    launches on two graph branches. Device pointers."""

    def __init__(self):
        self._h = _vp()
        _check(load().nc_batch_create(ctypes.byref(self._h)))

    def add(self, plan: Plan, d_a: int, d_b: int, d_c: int) -> None:
        _check(load().nc_batch_add(self._h, plan._h, _vp(d_a), _vp(d_b), _vp(d_c)))

    def add_cached(self, plan: Plan, d_a_hat: int, d_b: int, d_c: int) -> None:
        _check(load().nc_batch_add_cached(self._h, plan._h, _vp(d_a_hat), _vp(d_b), _vp(d_c)))

    def add_forward(self, plan: Plan, d_a: int, d_a_hat: int) -> None:
        _check(load().nc_batch_add_forward(self._h, plan._h, _vp(d_a), _vp(d_a_hat)))

    def clear(self) -> None:
        _check(load().nc_batch_clear(self._h))

    def run(self, stream: int = 0, use_graph: bool = True) -> None:
        _check(load().nc_batch_run(self._h, _vp(stream or None), int(use_graph)))

    def synchronize(self) -> None:
        _check(load().nc_batch_synchronize(self._h))

    def query(self) -> dict:
        n, c, s = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint64()
        _check(load().nc_batch_query(self._h, ctypes.byref(n), ctypes.byref(c), ctypes.byref(s)))
        return {"products": n.value, "ctas": c.value, "scratch_bytes": s.value}

    def close(self) -> None:
        if self._h:
            _check(load().nc_batch_destroy(self._h))
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching server (nc_server_*): host operands in, products out."""

    def __init__(self, hbm_budget: int = 1 << 30, staging: int = 1 << 28, max_batch: int = 64, streams: int = 2):
        self._h = _vp()
        _check(load().nc_server_create(int(hbm_budget), int(staging), int(max_batch), int(streams),
                                       ctypes.byref(self._h)))

    def register_operand(self, plan: Plan, a: np.ndarray) -> int:
        a = np.ascontiguousarray(a, dtype=np.uint32)
        oid = ctypes.c_int()
        _check(load().nc_server_register_operand(self._h, plan._h, _u32(a), ctypes.byref(oid)))
        return oid.value

    def release_operand(self, oid: int) -> None:
        _check(load().nc_server_release_operand(self._h, int(oid)))

    def submit(self, plan: Plan, a: np.ndarray | None, b: np.ndarray, operand: int = -1) -> int:
        b = np.ascontiguousarray(b, dtype=np.uint32)
        a_ptr = None
        if a is not None:
            a = np.ascontiguousarray(a, dtype=np.uint32)
            a_ptr = _u32(a)
        rid = ctypes.c_uint64()
        _check(load().nc_server_submit(self._h, plan._h, a_ptr, int(operand), _u32(b), ctypes.byref(rid)))
        return rid.value

    def poll(self, rid: int) -> bool:
        st = load().nc_server_poll(self._h, int(rid))
        if st < 0:
            _check(st)
        return st == 1

    def wait(self, rid: int, plan: Plan) -> tuple[np.ndarray, float]:
        c = np.empty((plan.N, plan.L), dtype=np.uint32)
        ms = ctypes.c_double()
        _check(load().nc_server_wait(self._h, int(rid), _u32(c), ctypes.byref(ms)))
        return c, ms.value

    def stats(self) -> dict:
        p50, p99, pps = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        done, hbm, batches, tmo = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(load().nc_server_stats(self._h, ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(done),
                                      ctypes.byref(pps), ctypes.byref(hbm), ctypes.byref(batches), ctypes.byref(tmo)))
        return {"p50_ms": p50.value, "p99_ms": p99.value, "completed": done.value, "products_per_s": pps.value,
                "hbm_in_use": hbm.value, "batches": batches.value, "timeouts": tmo.value}

    def io_stats(self) -> dict:
        """Bytes each way of finished batches, the device-clock time any batch had copies or kernels
        in flight within the window from the first batch's start to the last one's end, and the host
        time the scheduler thread spent enqueueing batches."""
        up, down = ctypes.c_uint64(), ctypes.c_uint64()
        busy, window, sched = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(load().nc_server_io_stats(self._h, ctypes.byref(up), ctypes.byref(down), ctypes.byref(busy),
                                         ctypes.byref(window), ctypes.byref(sched)))
        return {"h2d_bytes": up.value, "d2h_bytes": down.value, "device_busy_ms": busy.value,
                "device_window_ms": window.value, "scheduler_ms": sched.value}

    def close(self) -> None:
        if self._h:
            _check(load().nc_server_destroy(self._h))
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ the reference's interface


@dataclass
class Tensor:
    shape: list
    data: np.ndarray

    def count(self) -> int:
        n = 1
        for d in self.shape:
            n *= int(d)
        return n


@dataclass
class Point:
    N: int
    W: int
    L: int
    q: Tensor


@dataclass
class Inputs:
    a: Tensor
    b: Tensor


@dataclass
class Outputs:
    c: Tensor = field(default_factory=lambda: Tensor([], np.zeros(0, dtype=np.uint32)))


def fherma_init(p: Point) -> Plan:
    """Setup for one point; raises RuntimeError on an invalid point (fherma.h:45)."""
    q = np.ascontiguousarray(p.q.data, dtype=np.uint32).reshape(-1)
    if q.size != p.L:
        raise RuntimeError("q must hold L limbs")
    return Plan(p.N, q, W=p.W)


def fherma_run(state: Plan, inputs: Inputs) -> Outputs:
    """c = a * b mod (X^N + 1, q); raises RuntimeError on bad sizes (fherma.h:46)."""
    if state is None:
        raise RuntimeError("null state")
    count = state.N * state.L
    a = np.ascontiguousarray(inputs.a.data, dtype=np.uint32).reshape(-1)
    b = np.ascontiguousarray(inputs.b.data, dtype=np.uint32).reshape(-1)
    if a.size != count or b.size != count:
        raise RuntimeError("a and b must contain N*L limbs")
    c = state.multiply(a.reshape(state.N, state.L), b.reshape(state.N, state.L))
    return Outputs(Tensor([state.N, state.L], c.reshape(-1)))


def fherma_free(state: Plan | None) -> None:
    """Releases the state; None is a no-op (fherma.h:47)."""
    if state is not None:
        state.close()
