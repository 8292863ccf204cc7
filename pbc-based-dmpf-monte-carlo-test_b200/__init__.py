"""B200 cuckoo-hashing Monte Carlo estimator: Python view of libcmc.so.

The product is the C ABI in ``include/cmc.h`` (kernels for sm_100a plus the
host-side parameter and batch-key logic).  This module binds it with ctypes
so that tests, the benchmark and Python callers use exactly the functions a
C, C++ or FFI caller would.  It adds no computation of its own and has no
fallback: if ``libcmc.so`` is missing or fails to load, every call raises.

Names follow the reference (``cuckoo_bench.cu``): ``parameters`` derives B,
kick, bucket size, PRP domain and half width; ``batch_key`` is the per-batch
AES key schedule; ``Context.launch`` is the ``Launch`` seam that
``process_batch`` calls (cuckoo_bench.cu:724-736).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
LIB_PATH = PACKAGE_DIR / "libcmc.so"

MODES = {"bgh25": 1, "drrt18": 2}
INPUT_MODES = {"sequential": 0, "affine": 1}

CMC_OK = 0
CMC_EINVAL = -1
CMC_ECUDA = -2
CMC_EKAT = -3
CMC_ETIMEOUT = -4
CMC_ERANGE = -5
CMC_ENOMEM = -6

# every function include/cmc.h declares
EXPORTS = (
    "cmc_derive_params", "cmc_batch_key", "cmc_host_aes128", "cmc_init", "cmc_destroy",
    "cmc_last_error", "cmc_launch", "cmc_launch_device", "cmc_check",
    "cmc_last_kernel_count", "cmc_last_plan", "cmc_plan_describe", "cmc_set_option",
    "cmc_set_stream", "cmc_last_engine_ms", "cmc_last_stats", "cmc_launch_static",
    "cmc_run_jobs", "cmc_autotune", "cmc_server_create", "cmc_server_submit", "cmc_server_step",
    "cmc_server_status", "cmc_server_pending", "cmc_server_error", "cmc_server_destroy",
    "cmc_server_policy", "cmc_server_get_stats", "cmc_server_set_option",
)


class CmcError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"cmc error {code}: {message}")
        self.code = code


class Params(ctypes.Structure):
    """cmc_params: Options+Params of the reference with k generalised."""

    _fields_ = [
        ("mode", ctypes.c_uint32),
        ("input_mode", ctypes.c_uint32),
        ("pnum", ctypes.c_uint32),
        ("ell_i", ctypes.c_uint32),
        ("k", ctypes.c_uint32),
        ("buckets", ctypes.c_uint32),
        ("kick", ctypes.c_uint32),
        ("half_bits", ctypes.c_uint32),
        ("bucket_size", ctypes.c_uint64),
        ("domain", ctypes.c_uint64),
        ("mask", ctypes.c_uint64),
        ("range_mask", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Job(ctypes.Structure):
    """cmc_job: one parameter set and a run of trials of one batch."""

    _fields_ = [
        ("params", Params),
        ("seed", ctypes.c_uint64),
        ("batch", ctypes.c_uint64),
        ("first", ctypes.c_uint32),
        ("count", ctypes.c_uint32),
    ]


_lib = None


def load_library(path: os.PathLike | str | None = None) -> ctypes.CDLL:
    """Load libcmc.so (built by ``make`` in this directory); raise if absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise CmcError(CMC_EINVAL, f"{p} is missing: build it with `make -C {PACKAGE_DIR}`")
    lib = ctypes.CDLL(str(p))
    u32, u64, vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
    P = ctypes.POINTER
    lib.cmc_derive_params.argtypes = [u32, u32, u32, u32, u32, u32, u32, P(Params)]
    lib.cmc_derive_params.restype = ctypes.c_int
    lib.cmc_batch_key.argtypes = [u64, u64, P(u32)]
    lib.cmc_batch_key.restype = None
    lib.cmc_host_aes128.argtypes = [P(u32), P(u32), P(u32)]
    lib.cmc_host_aes128.restype = None
    lib.cmc_init.argtypes = [ctypes.c_int, P(vp)]
    lib.cmc_init.restype = ctypes.c_int
    lib.cmc_destroy.argtypes = [vp]
    lib.cmc_destroy.restype = ctypes.c_int
    lib.cmc_last_error.argtypes = [vp]
    lib.cmc_last_error.restype = ctypes.c_char_p
    lib.cmc_launch.argtypes = [vp, P(Params), P(u32), u32, u32, P(u32), P(u32)]
    lib.cmc_launch.restype = ctypes.c_int
    lib.cmc_launch_device.argtypes = [vp, P(Params), vp, u32, u32, vp, vp, vp]
    lib.cmc_launch_device.restype = ctypes.c_int
    lib.cmc_check.argtypes = [vp]
    lib.cmc_check.restype = ctypes.c_int
    lib.cmc_last_kernel_count.argtypes = [vp]
    lib.cmc_last_kernel_count.restype = u32
    lib.cmc_set_option.argtypes = [vp, ctypes.c_char_p, ctypes.c_int64]
    lib.cmc_set_option.restype = ctypes.c_int
    lib.cmc_set_stream.argtypes = [vp, vp]
    lib.cmc_set_stream.restype = ctypes.c_int
    lib.cmc_last_engine_ms.argtypes = [vp]
    lib.cmc_last_engine_ms.restype = ctypes.c_double
    lib.cmc_last_stats.argtypes = [vp, P(u64)]
    lib.cmc_last_stats.restype = ctypes.c_int
    lib.cmc_launch_static.argtypes = [P(Params), vp, u32, u32, vp, vp, vp]
    lib.cmc_launch_static.restype = ctypes.c_int
    lib.cmc_run_jobs.argtypes = [vp, P(Job), u32, P(u64), P(u32), P(u32), u64, P(u64)]
    lib.cmc_run_jobs.restype = ctypes.c_int
    lib.cmc_autotune.argtypes = [vp, P(Job), u32, u32, P(ctypes.c_char_p)]
    lib.cmc_autotune.restype = ctypes.c_int
    lib.cmc_server_create.argtypes = [vp, u32, u64, u32, u64, P(vp)]
    lib.cmc_server_create.restype = ctypes.c_int
    lib.cmc_server_submit.argtypes = [vp, P(Params), u64, u64, ctypes.c_char_p, P(u32)]
    lib.cmc_server_submit.restype = ctypes.c_int
    lib.cmc_server_step.argtypes = [vp, u64, P(u32), u32, P(u32)]
    lib.cmc_server_step.restype = ctypes.c_int
    lib.cmc_server_status.argtypes = [vp, u32, P(u64), P(u64), P(ctypes.c_int)]
    lib.cmc_server_status.restype = ctypes.c_int
    lib.cmc_server_policy.argtypes = [vp, ctypes.c_double]
    lib.cmc_server_policy.restype = ctypes.c_int
    lib.cmc_server_pending.argtypes = [vp]
    lib.cmc_server_pending.restype = u32
    lib.cmc_server_get_stats.argtypes = [vp, vp]
    lib.cmc_server_get_stats.restype = ctypes.c_int
    lib.cmc_server_set_option.argtypes = [vp, ctypes.c_char_p, ctypes.c_double]
    lib.cmc_server_set_option.restype = ctypes.c_int
    lib.cmc_server_error.argtypes = [vp]
    lib.cmc_server_error.restype = ctypes.c_char_p
    lib.cmc_server_destroy.argtypes = [vp]
    lib.cmc_server_destroy.restype = ctypes.c_int
    lib.cmc_last_plan.argtypes = [vp]
    lib.cmc_last_plan.restype = ctypes.c_char_p
    lib.cmc_plan_describe.argtypes = [ctypes.POINTER(Params), u32, u32, ctypes.c_uint64,
                                      ctypes.c_char_p, u32]
    lib.cmc_plan_describe.restype = ctypes.c_int
    if path is None:
        _lib = lib
    return lib


def parameters(mode: str = "bgh25", pnum: int = 16, ell_i: int = 32, k: int = 3,
               buckets: int = 0, kick: int = 0, input_mode: str = "sequential") -> Params:
    """Reference parameters() (cuckoo_bench.cu:500-526); buckets/kick 0 = derived."""
    lib = load_library()
    p = Params()
    rc = lib.cmc_derive_params(MODES[mode], pnum, ell_i, k, buckets, kick,
                               INPUT_MODES[input_mode], ctypes.byref(p))
    if rc:
        raise CmcError(rc, "invalid parameters")
    return p


def plan_describe(params: Params, count: int, sms: int = 148, smem_optin: int = 232448) -> str:
    """Planner dry run without a device: the plan cmc_launch would choose for
    `count` trials (defaults: B200's SM count and opt-in shared memory)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(512)
    rc = lib.cmc_plan_describe(ctypes.byref(params), count, sms, smem_optin, buf, len(buf))
    if rc:
        raise CmcError(rc, buf.value.decode())
    return buf.value.decode()


def batch_key(seed: int, batch_id: int) -> list[int]:
    """44-word AES key schedule of batch `batch_id` (cuckoo_bench.cu:393-404)."""
    lib = load_library()
    out = (ctypes.c_uint32 * 44)()
    lib.cmc_batch_key(seed & (2**64 - 1), batch_id & (2**64 - 1), out)
    return list(out)


def host_aes128(rk: list[int], block: list[int]) -> list[int]:
    lib = load_library()
    out = (ctypes.c_uint32 * 4)()
    lib.cmc_host_aes128((ctypes.c_uint32 * 44)(*rk), (ctypes.c_uint32 * 4)(*block), out)
    return list(out)


class Context:
    """One device context (cmc_init); use from one host thread."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.cmc_init(device, ctypes.byref(h))
        if rc:
            raise CmcError(rc, self.lib.cmc_last_error(None).decode())
        self.handle = h

    def close(self) -> None:
        if self.handle:
            self.lib.cmc_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _raise(self, rc: int):
        raise CmcError(rc, self.lib.cmc_last_error(self.handle).decode())

    def launch(self, params: Params, key: list[int], first: int, count: int) -> list[int]:
        """The Launch seam: failing within-batch offsets of trials [first, first+count)."""
        out = (ctypes.c_uint32 * max(count, 1))()
        nf = ctypes.c_uint32()
        rc = self.lib.cmc_launch(self.handle, ctypes.byref(params), (ctypes.c_uint32 * 44)(*key),
                                 first, count, out, ctypes.byref(nf))
        if rc:
            self._raise(rc)
        return list(out[: nf.value])

    def launch_device(self, params: Params, d_key: int, first: int, count: int,
                      d_offsets: int, d_nfailed: int, stream: int = 0) -> None:
        """Device-resident form (pointers are device addresses); asynchronous."""
        rc = self.lib.cmc_launch_device(self.handle, ctypes.byref(params), ctypes.c_void_p(d_key),
                                        first, count, ctypes.c_void_p(d_offsets),
                                        ctypes.c_void_p(d_nfailed), ctypes.c_void_p(stream))
        if rc:
            self._raise(rc)

    def check(self) -> None:
        rc = self.lib.cmc_check(self.handle)
        if rc:
            self._raise(rc)

    def run_jobs(self, jobs: list[tuple], cap: int | None = None):
        """Batched launch.  jobs: (params, seed, batch, first, count) tuples.
        Returns (failed counts per job, {job index: sorted failing offsets})."""
        n = len(jobs)
        arr = (Job * n)()
        total_trials = 0
        for i, (p, seed, batch, first, count) in enumerate(jobs):
            arr[i] = Job(p, seed, batch, first, count)
            total_trials += count
        cap = total_trials if cap is None else cap
        failed = (ctypes.c_uint64 * n)()
        offs = (ctypes.c_uint32 * max(cap, 1))()
        which = (ctypes.c_uint32 * max(cap, 1))()
        total = ctypes.c_uint64()
        rc = self.lib.cmc_run_jobs(self.handle, arr, n, failed, offs, which, cap, ctypes.byref(total))
        if rc:
            self._raise(rc)
        per_job: dict[int, list[int]] = {i: [] for i in range(n)}
        for i in range(min(total.value, cap)):
            per_job[which[i]].append(offs[i])
        return list(failed), per_job

    def autotune(self, jobs: list[tuple], sample_div: int = 64) -> str:
        n = len(jobs)
        arr = (Job * n)()
        for i, (p, seed, batch, first, count) in enumerate(jobs):
            arr[i] = Job(p, seed, batch, first, count)
        choice = ctypes.c_char_p()
        rc = self.lib.cmc_autotune(self.handle, arr, n, sample_div, ctypes.byref(choice))
        if rc:
            self._raise(rc)
        return choice.value.decode()

    def set_option(self, name: str, value: int) -> None:
        rc = self.lib.cmc_set_option(self.handle, name.encode(), value)
        if rc:
            self._raise(rc)

    def set_stream(self, stream: int) -> None:
        rc = self.lib.cmc_set_stream(self.handle, ctypes.c_void_p(stream))
        if rc:
            self._raise(rc)

    def last_engine_ms(self) -> float:
        return self.lib.cmc_last_engine_ms(self.handle)

    def last_stats(self) -> dict:
        out = (ctypes.c_uint64 * 6)()
        self.lib.cmc_last_stats(self.handle, out)
        keys = ("walks", "probes", "slot_wait_cycles", "walker_idle_cycles", "walker_cycles", "error")
        return dict(zip(keys, list(out)))

    @property
    def last_plan(self) -> str:
        return self.lib.cmc_last_plan(self.handle).decode()

    @property
    def last_kernel_count(self) -> int:
        return self.lib.cmc_last_kernel_count(self.handle)


class ServerStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint64), ("trials", ctypes.c_uint64),
                ("engine_ms", ctypes.c_double), ("busy_ms", ctypes.c_double),
                ("span_ms", ctypes.c_double)]


class Server:
    """Serving loop (cmc_server_*): jobs submitted as they arrive, continuously
    batched into the persistent engine; state and counts stay on the device."""

    def __init__(self, ctx: Context, max_jobs: int = 1024, mem_budget: int = 4 << 30,
                 batch_bits: int = 20, max_iteration_trials: int = 1 << 22):
        self.ctx = ctx
        self.lib = ctx.lib
        h = ctypes.c_void_p()
        rc = self.lib.cmc_server_create(ctx.handle, max_jobs, mem_budget, batch_bits,
                                        max_iteration_trials, ctypes.byref(h))
        if rc:
            raise CmcError(rc, self.lib.cmc_last_error(ctx.handle).decode())
        self.handle = h

    def _raise(self, rc: int):
        raise CmcError(rc, self.lib.cmc_server_error(self.handle).decode())

    def submit(self, params: Params, seed: int, trials: int, journal_dir: str | None = None) -> int:
        out = ctypes.c_uint32()
        rc = self.lib.cmc_server_submit(self.handle, ctypes.byref(params), seed, trials,
                                        journal_dir.encode() if journal_dir else None,
                                        ctypes.byref(out))
        if rc:
            self._raise(rc)
        return out.value

    def step(self, work_blocks: int) -> list[int]:
        cap = 4096
        fin = (ctypes.c_uint32 * cap)()
        n = ctypes.c_uint32()
        rc = self.lib.cmc_server_step(self.handle, work_blocks, fin, cap, ctypes.byref(n))
        if rc:
            self._raise(rc)
        return list(fin[: min(n.value, cap)])

    def status(self, job: int) -> tuple[int, int, int]:
        done, failed, state = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int()
        rc = self.lib.cmc_server_status(self.handle, job, ctypes.byref(done), ctypes.byref(failed),
                                        ctypes.byref(state))
        if rc:
            self._raise(rc)
        return done.value, failed.value, state.value

    def pending(self) -> int:
        return self.lib.cmc_server_pending(self.handle)

    def stats(self) -> dict:
        """Device-time accounting of the iterations read back so far."""
        out = ServerStats()
        rc = self.lib.cmc_server_get_stats(self.handle, ctypes.byref(out))
        if rc:
            self._raise(rc)
        return {name: getattr(out, name) for name, _ in ServerStats._fields_}

    def set_option(self, name: str, value: float) -> None:
        rc = self.lib.cmc_server_set_option(self.handle, name.encode(), float(value))
        if rc:
            self._raise(rc)

    def policy(self, fifo_share: float) -> None:
        rc = self.lib.cmc_server_policy(self.handle, fifo_share)
        if rc:
            self._raise(rc)

    def close(self) -> None:
        """Commits the iterations still in flight, then frees the server."""
        if self.handle:
            rc = self.lib.cmc_server_destroy(self.handle)
            self.handle = None
            if rc:
                raise CmcError(rc, self.lib.cmc_last_error(self.ctx.handle).decode())

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_journal(path: os.PathLike | str) -> dict[int, list[int]]:
    """Committed records of a v3/v4 journal file: {batch: sorted failing offsets}."""
    import struct
    data = Path(path).read_bytes()
    version = struct.unpack_from("<I", data, 4)[0]
    at = 56 + (8 if version == 4 else 0)
    out: dict[int, list[int]] = {}
    while at + 16 <= len(data):
        batch, tried, failed = struct.unpack_from("<QII", data, at)
        end = at + 16 + 4 * failed + 8
        if end > len(data):
            break
        out[batch] = list(struct.unpack_from(f"<{failed}I", data, at + 16))
        at = end
    return out


STATIC_MAX_TRIALS = 1 << 20


def launch_static(params: Params, d_key: int, first: int, count: int, d_offsets: int,
                  d_nfailed: int, stream: int = 0) -> None:
    """cmc_launch_static: the Launch seam without any device allocation by the
    library (device pointers in and out, current device, asynchronous)."""
    lib = load_library()
    rc = lib.cmc_launch_static(ctypes.byref(params), ctypes.c_void_p(d_key), first, count,
                               ctypes.c_void_p(d_offsets), ctypes.c_void_p(d_nfailed),
                               ctypes.c_void_p(stream))
    if rc:
        raise CmcError(rc, lib.cmc_last_error(None).decode())


def process_batch(ctx: Context, params: Params, seed: int, batch_id: int, batch_trials: int,
                  micro: int) -> list[int]:
    """Host loop of process_batch (cuckoo_bench.cu:724-745) without the journal:
    micro-launches over the batch, sorted failing offsets."""
    key = batch_key(seed, batch_id)
    failures: list[int] = []
    offset = 0
    while offset < batch_trials:
        n = min(micro, batch_trials - offset)
        failures += ctx.launch(params, key, offset, n)
        offset += n
    return sorted(failures)
