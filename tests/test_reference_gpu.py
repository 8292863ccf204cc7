"""The reference's own CUDA path, built unmodified for sm_100a (oracle/_ref),
against this engine on the same B200: the stock `cuckoo_bench` CLI of the
reference and this repository's CLI given the same flags write the same
journal and failure list, and the reference's gpu_worker with B and the
eviction limit overridden (oracle/ref_gpu_harness.cu) fails the same trials
as cmc_launch.  Bit-exact: outcomes are integer decisions."""
import ctypes
import json
import subprocess
import tempfile
from pathlib import Path

import pytest

from conftest import PKG_DIR, ROOT

pytestmark = pytest.mark.gpu
OURS = PKG_DIR / "cuckoo_bench"
REF_GPU_CLI = ROOT / "oracle" / "_ref" / "cuckoo_bench_ref"
REF_GPU_LIB = ROOT / "oracle" / "_ref" / "librefgpu.so"


def cli(binary, out, args):
    r = subprocess.run([str(binary), *args, "--workers", "1", "--out", str(out)],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (binary.name, r.stdout[-2000:], r.stderr[-2000:])
    return json.loads((out / "summary.json").read_text())


# configs 1 and 2 as the reference CLI expresses them: B and the eviction
# limit derived from PNUM (B = 1.5 t, kick = 3 t for t >= 30)
CLI_CASES = {
    "config1": ["--mode", "bgh25", "--et", "16", "--bt", "14", "--pnum", "64", "--ell-i", "16",
                "--seed", "1", "--input-mode", "affine"],
    "config2": ["--mode", "bgh25", "--et", "17", "--bt", "16", "--pnum", "1024", "--ell-i", "20",
                "--seed", "2", "--input-mode", "affine"],
    "config1_drrt18": ["--mode", "drrt18", "--et", "14", "--bt", "12", "--pnum", "64",
                       "--ell-i", "16", "--seed", "1", "--input-mode", "affine"],
}


@pytest.mark.skipif(not REF_GPU_CLI.exists(), reason="oracle/_ref/cuckoo_bench_ref not built")
@pytest.mark.parametrize("case", sorted(CLI_CASES))
def test_stock_cli_matches_reference_gpu_cli(tmp_path, case):
    args = CLI_CASES[case] + ["--stop-after", str(1 << 20)]
    a = cli(REF_GPU_CLI, tmp_path / "ref", args)
    b = cli(OURS, tmp_path / "ours", args)
    assert a["status"] == b["status"] == "complete"
    for key in ("completed", "failed", "BUCKETS_NUM", "MAX_KICK_TIMES", "PRP_DOMAIN"):
        assert a[key] == b[key], key
    # one worker commits batches in claim order: the journals agree byte for byte
    assert (tmp_path / "ref" / "worker_0.bin").read_bytes() == \
        (tmp_path / "ours" / "worker_0.bin").read_bytes()
    assert (tmp_path / "ref" / "failures.csv").read_bytes() == \
        (tmp_path / "ours" / "failures.csv").read_bytes()


def ref_gpu_batch(lib, mode, im, pnum, ell, buckets, kick, seed, bt):
    with tempfile.TemporaryDirectory(prefix="cmc-refgpu-") as d:
        secs, done, failed = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_uint64()
        info = ctypes.create_string_buffer(256)
        rc = lib.ref_gpu_run(0, mode.encode(), im.encode(), pnum, ell, buckets, kick, seed, bt, bt,
                             b"auto", d.encode(), ctypes.byref(secs), ctypes.byref(done),
                             ctypes.byref(failed), info, 256)
        assert rc == 0, info.value.decode()
        rows = (Path(d) / "failures.csv").read_text().split()[1:]
        return sorted(int(r.split(",")[1]) for r in rows), info.value.decode()


@pytest.mark.skipif(not REF_GPU_LIB.exists(), reason="oracle/_ref/librefgpu.so not built")
@pytest.mark.parametrize("shape", [
    # mode, input, t, ell_i, B, kick, seed, log2 trials  (reference layout)
    ("bgh25", "affine", 1024, 20, 1250, 250, 2, 16),    # shared-map, ~1 % fail
    ("bgh25", "affine", 1024, 20, 1536, 500, 2, 16),    # config 2 (benchmark limit)
    ("bgh25", "affine", 64, 16, 96, 100, 1, 16),        # config 1: direct, per-thread bins
    ("drrt18", "affine", 64, 16, 80, 20, 1, 14),        # direct, ~12 % fail
    ("bgh25", "affine", 600, 16, 720, 150, 6, 14),      # cached-global (h = 9)
    ("bgh25", "affine", 500, 24, 640, 100, 3, 12),      # sweep-like h = 13: direct, global bins
])
def test_reference_kernels_with_overrides_match_engine(ctx, cmc, shape):
    lib = ctypes.CDLL(str(REF_GPU_LIB))
    u32, u64, P = ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER
    lib.ref_gpu_run.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, u32, u32, u32, u32,
                                u64, u32, u32, ctypes.c_char_p, ctypes.c_char_p,
                                P(ctypes.c_double), P(u64), P(u64), ctypes.c_char_p, u32]
    mode, im, pnum, ell, buckets, kick, seed, bt = shape
    want, layout = ref_gpu_batch(lib, mode, im, pnum, ell, buckets, kick, seed, bt)
    p = cmc.parameters(mode, pnum, ell, 3, buckets, kick, im)
    got = ctx.launch(p, cmc.batch_key(seed, 0), 0, 1 << bt)
    assert got == want, (layout, ctx.last_plan)
