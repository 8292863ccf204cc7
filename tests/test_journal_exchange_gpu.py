"""Journal exchange with the reference's own tool.  The v3 journal
(cuckoo_bench.cu:565-698) is the drop-in contract: a run directory started by
the reference's cpu_bench (oracle/_ref, built from its sources) resumes under
this cuckoo_bench and ends on the reference's golden lists, the reverse too,
and a complete single-worker run writes byte-identical worker_0.bin,
failures.csv and experiment fields of summary.json in both tools."""
import csv
import json
import subprocess

import pytest

from conftest import PKG_DIR, ROOT

pytestmark = pytest.mark.gpu
OURS = PKG_DIR / "cuckoo_bench"
REF_CPU = ROOT / "oracle" / "_ref" / "cpu_bench"

# the golden experiment of cpu_golden.hpp: seed 123, PNUM 16, ell_i 8, ET 15, BT 8
GOLDEN_ARGS = ["--et", "15", "--bt", "8", "--pnum", "16", "--ell-i", "8", "--seed", "123",
               "--input-mode", "sequential"]
SUMMARY_KEYS = ["status", "seed_scheme", "mode", "algorithm", "input_mode", "seed", "ET", "BT",
                "batch_size", "PNUM_T", "ELL_I", "BUCKETS_NUM", "MAX_KICK_TIMES", "BUCKET_SIZE",
                "PRP_DOMAIN", "planned", "completed", "failed", "completed_batches",
                "pending_batches", "failed_ratio", "threshold_exceeded"]


@pytest.fixture(autouse=True)
def _need_reference():
    if not REF_CPU.exists():
        pytest.skip("oracle/_ref/cpu_bench not built (make -C oracle ref REF=<reference dir>)")


def tool(binary, out, mode, *extra):
    cmd = [str(binary), "--mode", mode, *GOLDEN_ARGS, "--workers", "1", "--out", str(out), *extra]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (cmd, r.stdout, r.stderr)
    return json.loads((out / "summary.json").read_text())


def trials(out, bt=8):
    with open(out / "failures.csv", newline="") as f:
        return sorted(int(r["batch_id"]) * (1 << bt) + int(r["offset"]) for r in csv.DictReader(f))


@pytest.mark.parametrize("mode", ["bgh25", "drrt18"])
def test_reference_started_run_resumes_here(tmp_path, golden, mode):
    # the reference stops on its failure threshold (deterministic: batches run
    # in order) part-way; this tool finishes the directory
    out = tmp_path / "run"
    stop = {"bgh25": 2, "drrt18": 100}[mode]
    part = tool(REF_CPU, out, mode, "--stop-after", str(stop))
    assert part["status"] == "threshold" and 0 < part["completed"] < 1 << 15
    before = (out / "worker_0.bin").read_bytes()
    done = tool(OURS, out, mode, "--stop-after", str(1 << 15))
    assert done["status"] == "complete" and done["completed"] == 1 << 15
    assert trials(out) == golden["golden_32768"]["failures"][mode]
    # the reference's committed records are kept as they were
    assert (out / "worker_0.bin").read_bytes()[:len(before)] == before


@pytest.mark.parametrize("mode", ["bgh25", "drrt18"])
def test_run_started_here_resumes_in_reference(tmp_path, golden, mode):
    out = tmp_path / "run"
    stop = {"bgh25": 2, "drrt18": 100}[mode]
    part = tool(OURS, out, mode, "--stop-after", str(stop), "--micro", "256")
    assert part["status"] == "threshold" and 0 < part["completed"] < 1 << 15
    done = tool(REF_CPU, out, mode, "--stop-after", str(1 << 15))
    assert done["status"] == "complete" and done["completed"] == 1 << 15
    assert trials(out) == golden["golden_32768"]["failures"][mode]


@pytest.mark.parametrize("mode", ["bgh25", "drrt18"])
def test_single_worker_files_byte_identical(tmp_path, mode):
    a = tool(REF_CPU, tmp_path / "ref", mode, "--stop-after", str(1 << 15))
    b = tool(OURS, tmp_path / "ours", mode, "--stop-after", str(1 << 15))
    assert (tmp_path / "ref" / "worker_0.bin").read_bytes() == \
        (tmp_path / "ours" / "worker_0.bin").read_bytes()
    assert (tmp_path / "ref" / "failures.csv").read_bytes() == \
        (tmp_path / "ours" / "failures.csv").read_bytes()
    assert {k: a[k] for k in SUMMARY_KEYS} == {k: b[k] for k in SUMMARY_KEYS}
