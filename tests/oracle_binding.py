"""ctypes view of the CPU oracle (oracle/liboracle.so) -- test infrastructure.

The oracle restates the reference CPU path (cpu_trials.hpp:56-127,
cuckoo_bench.cu:86-99,150-193,393-404,483-526) in C, generalised to k copies.
Only tests, __graft_entry__.smoke() and bench.py's CPU baseline use it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
MODES = {"bgh25": 1, "drrt18": 2}
INPUT_MODES = {"sequential": 0, "affine": 1}


class OrcParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in
                ("mode", "input_mode", "pnum", "ell_i", "k", "buckets", "kick", "half_bits")] + \
               [(n, ctypes.c_uint64) for n in ("bucket_size", "domain", "mask", "range_mask")]


class OrcStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("probes", "evaluations", "distinct", "aes_blocks")]


class Oracle:
    def __init__(self, path: Path | None = None):
        path = path or ORACLE_DIR / "liboracle.so"
        if not path.exists():
            subprocess.run(["make", "-C", str(ORACLE_DIR), "all"], check=True,
                           stdout=subprocess.DEVNULL)
        lib = ctypes.CDLL(str(path))
        u32, u64, P = ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER
        lib.orc_params_derive.argtypes = [u32, u32, u32, u32, u32, u32, u32, P(OrcParams)]
        lib.orc_params_derive.restype = ctypes.c_int
        lib.orc_batch.argtypes = [P(OrcParams), u64, u64, u32, u32, ctypes.c_int, P(u32),
                                  P(OrcStats)]
        lib.orc_batch.restype = u32
        lib.orc_batch_key.argtypes = [u64, u64, P(u32)]
        lib.orc_aes128.argtypes = [P(u32), u32, u32, u32, u32, P(u32)]
        lib.orc_expand_key.argtypes = [u64, u64, P(u32)]
        lib.orc_trial.argtypes = [P(OrcParams), P(u32), u32, P(u32), P(OrcStats)]
        lib.orc_trial.restype = ctypes.c_int
        lib.orc_trial_map.argtypes = [P(OrcParams), P(u32), u32, P(u32)]
        self.lib = lib

    def params(self, mode="bgh25", pnum=16, ell_i=8, k=3, buckets=0, kick=0,
               input_mode="sequential") -> OrcParams:
        p = OrcParams()
        rc = self.lib.orc_params_derive(MODES[mode], pnum, ell_i, k, buckets, kick,
                                        INPUT_MODES[input_mode], ctypes.byref(p))
        assert rc == 0
        return p

    def batch(self, p: OrcParams, seed: int, batch: int, first: int, count: int,
              threads: int = 8, stats: bool = False):
        out = (ctypes.c_uint32 * max(count, 1))()
        st = OrcStats()
        n = self.lib.orc_batch(ctypes.byref(p), seed, batch, first, count, threads, out,
                               ctypes.byref(st) if stats else None)
        failures = list(out[:n])
        return (failures, st) if stats else failures

    def batch_key(self, seed: int, batch: int) -> list[int]:
        w = (ctypes.c_uint32 * 44)()
        self.lib.orc_batch_key(seed, batch, w)
        return list(w)

    def aes(self, rk, block) -> list[int]:
        out = (ctypes.c_uint32 * 4)()
        self.lib.orc_aes128((ctypes.c_uint32 * 44)(*rk), *block, out)
        return list(out)

    def expand_key(self, lo: int, hi: int) -> list[int]:
        w = (ctypes.c_uint32 * 44)()
        self.lib.orc_expand_key(lo, hi, w)
        return list(w)

    def trial_map(self, p: OrcParams, seed: int, batch: int, offset: int) -> list[int]:
        out = (ctypes.c_uint32 * (p.pnum * p.k))()
        self.lib.orc_trial_map(ctypes.byref(p), (ctypes.c_uint32 * 44)(*self.batch_key(seed, batch)),
                               offset, out)
        return list(out)
