"""CPU oracle loader — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this. It
wraps liboracle.so (the C restatement, cs_oracle.c) and, when present,
_ref/libcsref.so (the reference's own CPU code compiled from its sources by the
Makefile here). The product path never touches it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libcsref.so"

_c_u64 = ctypes.c_uint64
_c_u32 = ctypes.c_uint32
_vp = ctypes.c_void_p


def build() -> None:
    """Compile liboracle.so (and _ref/libcsref.so when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Oracle:
    def __init__(self) -> None:
        if not ORACLE_SO.exists():
            build()
        lib = ctypes.CDLL(str(ORACLE_SO), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        sig = {
            "oracle_compact": (_c_u64, [_vp, _vp, _vp, _c_u64, _c_u32]),
            "oracle_compact_mt": (_c_u64, [_vp, _vp, _vp, _c_u64, _c_u32, ctypes.c_int]),
            "oracle_count": (_c_u64, [_vp, _c_u64]),
            "oracle_popc_chunks": (None, [_vp, _c_u64, _c_u32, _vp]),
            "oracle_exclusive_scan": (_c_u64, [_vp, _c_u64, _vp]),
            "oracle_mix64": (_c_u64, [_c_u64, _c_u64]),
            "oracle_gen_payload": (None, [_vp, _c_u64, _c_u32, _c_u64, ctypes.c_int]),
            "oracle_gen_mask_bernoulli": (None, [_vp, _c_u64, ctypes.c_double, _c_u64]),
            "oracle_gen_mask_runs": (None, [_vp, _c_u64, ctypes.c_double, _c_u64]),
            "oracle_gen_mask_dense_prefix": (_c_u64, [_vp, _c_u64, ctypes.c_float]),
            "oracle_gen_mask_pattern": (_c_u64, [_vp, _c_u64, _c_u32, _c_u32]),
            "oracle_ref_mask_uniform_msb": (_c_u64, [_vp, _c_u64, ctypes.c_double, _c_u64]),
            "oracle_rev8": (None, [_vp, _c_u64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        self.lib = lib

    # --- compaction -------------------------------------------------------------------
    def compact(self, data: np.ndarray, mask_words: np.ndarray, n: int, threads: int = 1) -> np.ndarray:
        data = np.ascontiguousarray(data)
        mask_words = np.ascontiguousarray(mask_words, dtype=np.uint32)
        out = np.empty(max(n, 1), dtype=data.dtype)
        w = data.dtype.itemsize
        if threads > 1:
            k = self.lib.oracle_compact_mt(_ptr(data), _ptr(mask_words), _ptr(out), n, w, threads)
        else:
            k = self.lib.oracle_compact(_ptr(data), _ptr(mask_words), _ptr(out), n, w)
        return out[:k].copy()

    def count(self, mask_words: np.ndarray, n: int) -> int:
        mask_words = np.ascontiguousarray(mask_words, dtype=np.uint32)
        return int(self.lib.oracle_count(_ptr(mask_words), n))

    def popc_chunks(self, mask_words: np.ndarray, n: int, chunk_length: int) -> np.ndarray:
        mask_words = np.ascontiguousarray(mask_words, dtype=np.uint32)
        c = (n + chunk_length - 1) // chunk_length
        out = np.zeros(max(c, 1), dtype=np.uint32)
        self.lib.oracle_popc_chunks(_ptr(mask_words), n, chunk_length, _ptr(out))
        return out[:c]

    def exclusive_scan(self, counts: np.ndarray) -> tuple[np.ndarray, int]:
        counts = np.ascontiguousarray(counts, dtype=np.uint32)
        out = np.zeros(max(len(counts), 1), dtype=np.uint64)
        total = self.lib.oracle_exclusive_scan(_ptr(counts), len(counts), _ptr(out))
        return out[: len(counts)], int(total)

    # --- generators -------------------------------------------------------------------
    def payload(self, n: int, elem_bytes: int, seed: int, float_unit: bool = False) -> np.ndarray:
        dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[elem_bytes]
        out = np.empty(max(n, 1), dtype=dt)
        self.lib.oracle_gen_payload(_ptr(out), n, elem_bytes, seed, int(float_unit))
        return out[:n]

    def mask_bernoulli(self, n: int, p: float, seed: int) -> np.ndarray:
        out = np.zeros(max((n + 31) // 32, 1), dtype=np.uint32)
        self.lib.oracle_gen_mask_bernoulli(_ptr(out), n, p, seed)
        return out[: (n + 31) // 32]

    def mask_runs(self, n: int, mean_run: float, seed: int) -> np.ndarray:
        out = np.zeros(max((n + 31) // 32, 1), dtype=np.uint32)
        self.lib.oracle_gen_mask_runs(_ptr(out), n, mean_run, seed)
        return out[: (n + 31) // 32]

    def mask_dense_prefix(self, n: int, frac: float) -> np.ndarray:
        out = np.zeros(max((n + 31) // 32, 1), dtype=np.uint32)
        self.lib.oracle_gen_mask_dense_prefix(_ptr(out), n, frac)
        return out[: (n + 31) // 32]

    def mask_pattern(self, n: int, pattern: int, length: int) -> np.ndarray:
        """LSB-first words of the periodic mask: bit i = bit (i % length) of pattern."""
        out = np.zeros(max((n + 31) // 32, 1), dtype=np.uint32)
        self.lib.oracle_gen_mask_pattern(_ptr(out), n, pattern, length)
        return out[: (n + 31) // 32]

    def mix64(self, seed: int, i: int) -> int:
        return int(self.lib.oracle_mix64(seed, i))

    def ref_mask_uniform_msb(self, length: int, selectivity: float, seed: int = 42) -> tuple[np.ndarray, int]:
        out = np.zeros(max(length, 1), dtype=np.uint8)
        ones = self.lib.oracle_ref_mask_uniform_msb(_ptr(out), length, selectivity, seed)
        return out[:length], int(ones)

    def rev8(self, b: np.ndarray) -> np.ndarray:
        b = np.ascontiguousarray(b, dtype=np.uint8).copy()
        self.lib.oracle_rev8(_ptr(b), len(b))
        return b


def lsb_words_to_msb_bytes(mask_words: np.ndarray) -> np.ndarray:
    """The reference's MSB-first byte mask that selects the same elements."""
    o = Oracle.instance()
    return o.rev8(np.ascontiguousarray(mask_words, dtype=np.uint32).view(np.uint8))


class Reference:
    """The reference's own CPU code (oracle/_ref/libcsref.so), when it was built."""

    def __init__(self) -> None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference sources)")
        lib = ctypes.CDLL(str(REF_SO), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        sig = {
            "ref_generate_validation": (_c_u64, [_vp, _vp, _vp, _c_u64, _c_u32]),
            "ref_generate_validation_mt": (_c_u64, [_vp, _vp, _vp, _vp, _c_u64, _c_u32, ctypes.c_int]),
            "ref_generate_mask_uniform": (_c_u64, [_vp, _c_u64, _c_u64, ctypes.c_double]),
            "ref_generate_mask_clustering": (_c_u64, [ctypes.c_float, _c_u64, _c_u64, _vp]),
            "ref_generate_mask_pattern": (_c_u64, [_vp, _c_u64, _c_u32, _c_u32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        self.lib = lib

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def generate_validation(self, data: np.ndarray, mask_msb: np.ndarray, count: int) -> np.ndarray:
        data = np.ascontiguousarray(data)
        mask_msb = np.ascontiguousarray(mask_msb, dtype=np.uint8)
        out = np.empty(max(count, 1), dtype=data.dtype)
        k = self.lib.ref_generate_validation(_ptr(data), _ptr(mask_msb), _ptr(out), count, data.dtype.itemsize)
        return out[:k].copy()

    def generate_mask_uniform(self, length: int, selectivity: float) -> tuple[np.ndarray, int]:
        out = np.zeros(max(length, 1), dtype=np.uint8)
        ones = self.lib.ref_generate_mask_uniform(_ptr(out), 0, length, selectivity)
        return out[:length], int(ones)

    def generate_mask_pattern(self, nbytes: int, pattern_msb: int, length: int) -> tuple[np.ndarray, int]:
        out = np.zeros(max(nbytes, 1), dtype=np.uint8)
        ones = self.lib.ref_generate_mask_pattern(_ptr(out), nbytes, pattern_msb, length)
        return out[:nbytes], int(ones)

    def generate_mask_clustering(self, selectivity: float, clusters: int, total: int) -> tuple[np.ndarray, int]:
        out = np.zeros(max(total // 8, 1), dtype=np.uint8)
        ones = self.lib.ref_generate_mask_clustering(selectivity, clusters, total, _ptr(out))
        return out[: total // 8], int(ones)


_instance: Oracle | None = None


def _get() -> Oracle:
    global _instance
    if _instance is None:
        _instance = Oracle()
    return _instance


Oracle.instance = staticmethod(_get)  # type: ignore[attr-defined]
