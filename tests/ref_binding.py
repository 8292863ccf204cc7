"""ctypes view of the reference's own CPU code (oracle/_ref/libcmcref.so) --
test infrastructure.

oracle/ref_harness.cpp exposes the reference's cpu_trial / cpu_trial_cached
(cpu_trials.hpp:69-149) with Params.buckets and Params.kick overridden.  The
library is built from the reference sources by `make -C oracle ref REF=<dir>`
and travels with the repository tree; when it is absent the C restatement
(oracle/liboracle.so) stands in, at the sizes it finishes quickly.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
REF_LIB = ROOT / "oracle" / "_ref" / "libcmcref.so"


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class Reference:
    """The reference's CPU trial functions, or None when not built."""

    def __init__(self):
        lib = ctypes.CDLL(str(REF_LIB))
        u32, u64 = ctypes.c_uint32, ctypes.c_uint64
        lib.ref_batch.argtypes = [ctypes.c_char_p, ctypes.c_char_p, u32, u32, u32, u32, u64, u64,
                                  u32, u32, ctypes.c_int, ctypes.c_int, ctypes.POINTER(u32)]
        lib.ref_batch.restype = u32
        lib.ref_has_aesni.restype = ctypes.c_int
        self.lib = lib

    @staticmethod
    def load():
        if not REF_LIB.exists():
            return None
        r = Reference()
        return r if r.lib.ref_has_aesni() else None

    def batch(self, mode: str, input_mode: str, pnum: int, ell_i: int, buckets: int, kick: int,
              seed: int, batch: int, first: int, count: int, threads: int = 0,
              cached: bool = True) -> list[int]:
        """Sorted failing offsets of trials [first, first+count) of `batch`
        (k = 3, the only copy count the reference supports)."""
        out = (ctypes.c_uint32 * max(count, 1))()
        n = self.lib.ref_batch(mode.encode(), input_mode.encode(), pnum, ell_i, buckets, kick,
                               seed, batch, first, count, threads or host_threads(),
                               1 if cached else 0, out)
        return list(out[:n])
