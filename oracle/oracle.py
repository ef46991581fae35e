"""ctypes wrapper of the CPU oracle (negacyclic_oracle.c) and the Python big-integer schoolbook.

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke test and bench.py's cpu_baseline leg to
check or time the reference algorithm on the CPU. The product path never imports this module.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None


def build() -> Path:
    if not LIB.exists() or LIB.stat().st_mtime < (HERE / "negacyclic_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True, capture_output=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        u64 = ctypes.c_uint64
        L.oracle_negacyclic.restype = ctypes.c_int
        L.oracle_negacyclic.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p, _u32p, _u32p, ctypes.c_int]
        L.oracle_schoolbook.restype = ctypes.c_int
        L.oracle_schoolbook.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p, _u32p, _u32p]
        L.oracle_primes.restype = ctypes.c_int
        L.oracle_primes.argtypes = [ctypes.c_uint32, ctypes.c_int, _u64p, ctypes.c_int]
        for name, args in [
            ("oracle_mul_mod", [u64, u64, u64]),
            ("oracle_pow_mod", [u64, u64, u64]),
            ("oracle_neg_inv64", [u64]),
            ("oracle_mont_mul", [u64, u64, u64, u64]),
            ("oracle_shoup_companion", [u64, u64]),
            ("oracle_shoup_mul", [u64, u64, u64, u64]),
            ("oracle_barrett_mu96", [u64]),
            ("oracle_barrett_reduce", [u64, u64, u64, u64]),
            ("oracle_mod128", [u64, u64, u64]),
            ("oracle_find_psi", [u64, ctypes.c_uint32]),
            ("oracle_limbs_mod_u64", [_u32p, ctypes.c_int, u64]),
        ]:
            fn = getattr(L, name)
            fn.restype = u64
            fn.argtypes = args
        L.oracle_div_pow2_64.restype = u64
        L.oracle_div_pow2_64.argtypes = [u64, _u64p]
        L.oracle_magic128.restype = None
        L.oracle_magic128.argtypes = [u64, _u64p, _u64p]
        L.oracle_is_prime_u64.restype = ctypes.c_int
        L.oracle_is_prime_u64.argtypes = [u64]
        L.oracle_mod_q.restype = None
        L.oracle_mod_q.argtypes = [_u32p, ctypes.c_int, _u32p, ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        L.oracle_max_threads.argtypes = []
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


def negacyclic(N: int, q_limbs: np.ndarray, a: np.ndarray, b: np.ndarray, threads: int = 0) -> np.ndarray:
    """CPU multi-prime NTT + CRT following the reference algorithm."""
    q = np.ascontiguousarray(q_limbs, dtype=np.uint32)
    L = q.size
    a = np.ascontiguousarray(a, dtype=np.uint32).reshape(N, L)
    b = np.ascontiguousarray(b, dtype=np.uint32).reshape(N, L)
    c = np.empty((N, L), dtype=np.uint32)
    rc = lib().oracle_negacyclic(N, L, _p(q), _p(a), _p(b), _p(c), threads)
    if rc != 0:
        raise ValueError(f"oracle rejected the point (code {rc})")
    return c


def schoolbook_c(N: int, q_limbs: np.ndarray, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """O(N^2) schoolbook in C (exact integers, reduced mod q)."""
    q = np.ascontiguousarray(q_limbs, dtype=np.uint32)
    L = q.size
    a = np.ascontiguousarray(a, dtype=np.uint32).reshape(N, L)
    b = np.ascontiguousarray(b, dtype=np.uint32).reshape(N, L)
    c = np.empty((N, L), dtype=np.uint32)
    if lib().oracle_schoolbook(N, L, _p(q), _p(a), _p(b), _p(c)) != 0:
        raise ValueError("bad L")
    return c


def reference_primes(N: int, q_bits: int) -> list[int]:
    out = (ctypes.c_uint64 * 48)()
    k = lib().oracle_primes(N, q_bits, out, 48)
    if k < 0:
        raise ValueError("bound does not fit 48 primes")
    return list(out[:k])


def max_threads() -> int:
    return int(lib().oracle_max_threads())


# ----------------------------------------------------------------------------- pure Python


def schoolbook_py(a: list[int], b: list[int], q: int) -> list[int]:
    """c_k = sum_{i+j=k} a_i b_j - sum_{i+j=k+N} a_i b_j mod q, with Python integers."""
    N = len(a)
    out = []
    for k in range(N):
        s = 0
        for i in range(N):
            j = k - i
            if j >= 0:
                s += a[i] * b[j]
            else:
                s -= a[i] * b[j + N]
        out.append(s % q)
    return out


def coefficient_py(a: list[int], b: list[int], q: int, k: int) -> int:
    """One output coefficient in O(N) (spot checks at large N)."""
    N = len(a)
    s = 0
    for i in range(N):
        j = k - i
        if j >= 0:
            s += a[i] * b[j]
        else:
            s -= a[i] * b[j + N]
    return s % q
