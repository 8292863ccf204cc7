"""End-to-end CLI runs on the GPU, after the reference's smoke_test.py:
2^15 trials per mode compared with the golden failure list, a run with two
workers and an odd micro size, a real mid-run PAUSE followed by a resume with
different workers/micro, and a re-run of a completed directory."""
import csv
import json
import subprocess
import time

import pytest

from conftest import PKG_DIR

pytestmark = pytest.mark.gpu
BENCH = PKG_DIR / "cuckoo_bench"


def run(out, mode, *extra, et=15, bt=8, timeout=600):
    cmd = [str(BENCH), "--mode", mode, "--et", str(et), "--bt", str(bt), "--pnum", "16",
           "--ell-i", "8", "--seed", "123", "--input-mode", "sequential",
           "--stop-after", str(1 << et), "--out", str(out)] + list(extra)
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)


def failures(out, bt=8):
    with open(out / "failures.csv", newline="") as f:
        rows = list(csv.DictReader(f))
    trials = sorted(int(r["batch_id"]) * (1 << bt) + int(r["offset"]) for r in rows)
    assert len(trials) == len(set(trials))
    return trials


@pytest.mark.parametrize("mode", ["bgh25", "drrt18"])
def test_cli_golden(tmp_path, golden, mode):
    out = tmp_path / mode
    r = run(out, mode, "--workers", "1", "--micro", "256")
    assert r.returncode == 0, r.stderr
    s = json.loads((out / "summary.json").read_text())
    assert s["status"] == "complete" and s["completed"] == 1 << 15
    assert failures(out) == golden["golden_32768"]["failures"][mode]
    assert s["failed"] == len(golden["golden_32768"]["failures"][mode])
    # a completed directory adds no work
    r = run(out, mode)
    assert r.returncode == 0 and "Status: complete" in r.stdout


def test_cli_two_workers_global_table(tmp_path, golden):
    out = tmp_path / "w2"
    r = run(out, "drrt18", "--workers", "2", "--micro", "37", "--global-table",
            "--table-layout", "global")
    assert r.returncode == 0, r.stderr
    assert failures(out) == golden["golden_32768"]["failures"]["drrt18"]
    assert len(list(out.glob("worker_*.bin"))) == 2


def test_cli_pause_and_resume(tmp_path, golden):
    out = tmp_path / "pause"
    cmd = [str(BENCH), "--mode", "bgh25", "--et", "15", "--bt", "8", "--pnum", "16", "--ell-i",
           "8", "--seed", "123", "--workers", "1", "--micro", "1", "--stop-after", str(1 << 15),
           "--out", str(out)]
    proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    deadline = time.monotonic() + 300
    try:
        while proc.poll() is None:
            # 56-byte header + one empty record (24 bytes) = first committed batch
            if any(p.stat().st_size >= 80 for p in out.glob("worker_*.bin")):
                (out / "PAUSE").touch()
                break
            assert time.monotonic() < deadline
            time.sleep(0.005)
        proc.wait(timeout=300)
    finally:
        if proc.poll() is None:
            proc.kill()
            proc.wait()
    assert proc.returncode == 0
    s = json.loads((out / "summary.json").read_text())
    assert s["status"] == "paused" and 0 < s["completed"] < 1 << 15
    (out / "PAUSE").unlink()
    r = run(out, "bgh25", "--workers", "2", "--micro", "113")
    assert r.returncode == 0, r.stderr
    s = json.loads((out / "summary.json").read_text())
    assert s["status"] == "complete"
    assert failures(out) == golden["golden_32768"]["failures"]["bgh25"]


def test_cli_extensions_k_and_overrides(tmp_path, oracle):
    # --k / --buckets / --max-kicks: parity against the oracle (k != 3 is an
    # extension without a reference counterpart)
    out = tmp_path / "k4"
    cmd = [str(BENCH), "--mode", "bgh25", "--et", "12", "--bt", "10", "--pnum", "64", "--ell-i",
           "16", "--seed", "7", "--input-mode", "affine", "--k", "4", "--buckets", "72",
           "--max-kicks", "40", "--out", str(out), "--stop-after", "4096"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    p = oracle.params("bgh25", 64, 16, 4, 72, 40, "affine")
    want = []
    for b in range(4):
        want += [b * 1024 + o for o in oracle.batch(p, 7, b, 0, 1024)]
    assert failures(out, bt=10) == want
    s = json.loads((out / "summary.json").read_text())
    assert s["K_COPIES"] == 4 and s["BUCKETS_NUM"] == 72 and s["MAX_KICK_TIMES"] == 40


def test_cli_large_table_checkpoint_resume(tmp_path, golden):
    # config 4's table (t=16384, N=2^28) under a tighter load (B=19500, kick
    # 300, ~20% failures): a run stopped after 3 of 8 batches and resumed with
    # two workers matches an uninterrupted run, and batch 2's first trials
    # match the reference's own CPU run of the same shape
    def cli(out, *extra):
        cmd = [str(BENCH), "--mode", "bgh25", "--et", "14", "--bt", "11", "--pnum", "16384",
               "--ell-i", "28", "--buckets", "19500", "--max-kicks", "300", "--seed", "4",
               "--input-mode", "affine", "--stop-after", str(1 << 20), "--out", str(out)]
        r = subprocess.run(cmd + list(extra), capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        return json.loads((out / "summary.json").read_text())

    clean = cli(tmp_path / "clean", "--workers", "1")
    assert clean["status"] == "complete" and clean["completed"] == 1 << 14
    part = cli(tmp_path / "resumed", "--workers", "1", "--max-batches", "3")
    assert part["status"] == "budget" and part["completed"] == 3 << 11
    done = cli(tmp_path / "resumed", "--workers", "2")
    assert done["status"] == "complete" and done["failed"] == clean["failed"]
    want = failures(tmp_path / "clean", bt=11)
    assert failures(tmp_path / "resumed", bt=11) == want and len(want) > 1000
    ref = next(r for r in golden["reference_runs"] if r["name"] == "config4_stress")
    assert ref["batch"] == 2 and ref["first"] == 0
    got = [t - (2 << 11) for t in want if (2 << 11) <= t < (2 << 11) + ref["count"]]
    assert got == ref["failures"]
