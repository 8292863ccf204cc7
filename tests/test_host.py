"""Host controller, journal and CLI behaviour without a GPU."""
import json
import subprocess

import pytest

from conftest import PKG_DIR

BENCH = PKG_DIR / "cuckoo_bench"
HOST_TESTS = PKG_DIR / "host_tests"


@pytest.fixture(scope="module", autouse=True)
def built(cmc):
    subprocess.run(["make", "-C", str(PKG_DIR), "-j4"], check=True, stdout=subprocess.DEVNULL)


def test_host_tests_binary(tmp_path):
    r = subprocess.run([str(HOST_TESTS), str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "ALL HOST TESTS PASSED" in r.stdout


@pytest.mark.parametrize("args", [
    ["--pnum", "2"], ["--et", "41"], ["--bt", "8", "--et", "7"], ["--ell-i", "62"],
    ["--mode", "cuckoo"], ["--input-mode", "random"], ["--block-threads", "96"],
    ["--prp-cache", "maybe"], ["--warps-per-block", "33"], ["--k", "1"], ["--micro", "0"],
    ["--pnum", "300", "--ell-i", "8"],
])
def test_cli_rejects_invalid_config(tmp_path, args):
    r = subprocess.run([str(BENCH), "--out", str(tmp_path / "o")] + args, capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1
    assert "FATAL: Invalid config" in r.stderr


def test_cli_unknown_option_and_missing_value(tmp_path):
    r = subprocess.run([str(BENCH), "--bogus", "1"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Unknown option --bogus" in r.stderr
    r = subprocess.run([str(BENCH), "--seed"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Missing value after --seed" in r.stderr


def test_cli_help():
    r = subprocess.run([str(BENCH), "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.startswith("Usage: ./cuckoo_bench")


def test_cli_status_summary_keys(tmp_path):
    out = tmp_path / "status"
    r = subprocess.run([str(BENCH), "--mode", "bgh25", "--et", "10", "--bt", "8", "--pnum", "16",
                        "--ell-i", "8", "--seed", "123", "--out", str(out), "--status"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert "Status: ready; pending batches=4" in r.stdout
    s = json.loads((out / "summary.json").read_text())
    for key, value in dict(status="ready", seed_scheme="aes-batch-v1", mode="bgh25", ET=10, BT=8,
                           PNUM_T=16, ELL_I=8, BUCKETS_NUM=32, MAX_KICK_TIMES=48, planned=1024,
                           completed=0, failed=0, pending_batches=4, seed_decimal="123").items():
        assert s[key] == value, key
    assert (out / "failures.csv").read_text() == "batch_id,offset\n"


def test_cli_lock(tmp_path):
    import fcntl
    out = tmp_path / "locked"
    out.mkdir()
    with open(out / ".run.lock", "w") as f:
        fcntl.flock(f, fcntl.LOCK_EX | fcntl.LOCK_NB)
        r = subprocess.run([str(BENCH), "--out", str(out), "--status"], capture_output=True,
                           text=True, timeout=60)
    assert r.returncode == 1 and "Another process is using the output directory" in r.stderr
