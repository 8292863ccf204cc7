#!/usr/bin/env python3
"""Generate tests/golden/golden.json from the reference.

Sources (read from the reference tree, given with --ref):
  * cpu_golden.hpp:3-4        -- 32,768-trial failure lists (seed 123, PNUM 16, ell_i 8,
                                 ET 15, BT 8, sequential) for BGH25 and DRRT18
  * smoke_expected.json        -- the first 8,192 trials of the same set
  * cpu_tests.cpp:30-39        -- affine PNUM 3 known answers of batch 0
  * host_tests.cpp:37-46       -- AES(batch_key(123, {0, 7}), 0^128) vectors
  * host_tests.cpp:158-159     -- B derivations (DRRT18 23, BGH25 32)
  * cuckoo_bench.cu:341        -- the FIPS-197 AES-128 vector
and, run here, the reference's own CPU implementation compiled from its sources
into oracle/_ref/libcmcref.so (oracle/Makefile target `ref`): cpu_trial
(cpu_trials.hpp:69-127) over the benchmark shapes with B/kick overrides,
parameters() over a grid, and batch_key() schedules.

The JSON is committed; tests never read the reference tree.
Usage: python tests/golden/make_golden.py --ref <directory of the reference sources>
"""
import argparse
import ctypes
import json
import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]


def ints(text):
    return [int(x, 0) for x in re.findall(r"0x[0-9a-fA-F]+|\d+", text)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="directory of the reference sources")
    args = ap.parse_args()
    ref = Path(args.ref)
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "all", "ref", f"REF={ref}"], check=True,
                   stdout=subprocess.DEVNULL)
    lib = ctypes.CDLL(str(ROOT / "oracle/_ref/libcmcref.so"))
    u32, u64 = ctypes.c_uint32, ctypes.c_uint64
    lib.ref_batch.argtypes = [ctypes.c_char_p, ctypes.c_char_p, u32, u32, u32, u32, u64, u64, u32,
                              u32, ctypes.c_int, ctypes.c_int, ctypes.POINTER(u32)]
    lib.ref_batch.restype = u32
    lib.ref_params.argtypes = [ctypes.c_char_p, u32, u32, u32, u32, ctypes.POINTER(u64)]
    lib.ref_batch_key.argtypes = [u64, u64, ctypes.POINTER(u32)]
    lib.ref_host_aes.argtypes = [ctypes.POINTER(u32)] * 3

    out = {"generated_by": "tests/golden/make_golden.py"}

    golden = (ref / "cpu_golden.hpp").read_text()
    sets = {}
    for name in ("golden_bgh25", "golden_drrt18"):
        body = re.search(name + r"=\{([^}]*)\}", golden).group(1)
        sets[name.split("_")[1]] = ints(body)
    out["golden_32768"] = {"seed": 123, "pnum": 16, "ell_i": 8, "et": 15, "bt": 8,
                           "input_mode": "sequential", "failures": sets,
                           "source": "cpu_golden.hpp:3-4"}
    smoke = json.loads((ref / "smoke_expected.json").read_text())
    out["smoke_8192"] = dict(smoke, source="smoke_expected.json")

    cpu_tests = (ref / "cpu_tests.cpp").read_text()
    m = re.search(r'mode=="bgh25"\?std::vector<uint32_t>\{([^}]*)\}:std::vector<uint32_t>\{([^}]*)\}',
                  cpu_tests)
    out["affine_pnum3"] = {"seed": 123, "pnum": 3, "ell_i": 8, "batch": 0, "count": 256,
                           "input_mode": "affine",
                           "failures": {"bgh25": ints(m.group(1)), "drrt18": ints(m.group(2))},
                           "source": "cpu_tests.cpp:30-39"}

    host_tests = (ref / "host_tests.cpp").read_text()
    m = re.search(r"expected\[2\]\[4\]=\{\{([^}]*)\},\s*\{([^}]*)\}\}", host_tests)
    out["batch_key_vectors"] = {"seed": 123, "batches": [0, 7],
                                "aes_of_zero": [ints(m.group(1)), ints(m.group(2))],
                                "source": "host_tests.cpp:37-46"}
    out["param_pins"] = [
        {"mode": "drrt18", "pnum": 16, "ell_i": 8, "buckets": 23, "source": "host_tests.cpp:158"},
        {"mode": "bgh25", "pnum": 16, "ell_i": 8, "buckets": 32, "source": "host_tests.cpp:159"},
    ]
    out["fips197"] = {"key_lo": 0x0706050403020100, "key_hi": 0x0f0e0d0c0b0a0908,
                      "plain": [0x00112233, 0x44556677, 0x8899aabb, 0xccddeeff],
                      "cipher": [0x69c4e0d8, 0x6a7b0430, 0xd8cdb780, 0x70b4c55a],
                      "source": "cuckoo_bench.cu:332-344"}

    # parameters() over a grid, including the float-log DRRT18 derivation
    grid = []
    for mode in ("bgh25", "drrt18"):
        for pnum in (3, 4, 5, 7, 16, 29, 30, 31, 64, 100, 255, 256, 1000, 1024, 4096, 10000,
                     16000, 16384, 30000, 65534):
            for ell in (8, 14, 16, 20, 24, 28, 32, 40, 61):
                if ell < 16 and (1 << ell) < pnum:
                    continue
                for b_over, k_over in ((0, 0), (int(pnum * 1.5), 500)):
                    o = (u64 * 6)()
                    lib.ref_params(mode.encode(), pnum, ell, b_over, k_over, o)
                    grid.append({"mode": mode, "pnum": pnum, "ell_i": ell, "buckets_override": b_over,
                                 "kick_override": k_over, "buckets": o[0], "kick": o[1],
                                 "bucket_size": o[2], "domain": o[3], "mask": o[4],
                                 "half_bits": o[5]})
    out["params_grid"] = grid

    keys = []
    for seed, batch in ((1, 0), (2, 0), (2, 5), (123, 0), (123, 127), (4, 15), (2**64 - 1, 2**40 + 3)):
        w = (u32 * 44)()
        lib.ref_batch_key(seed, batch, w)
        keys.append({"seed": seed, "batch": batch, "schedule": list(w)})
    out["batch_key_schedules"] = keys

    # Reference cpu_trial runs at the benchmark shapes and stress shapes.
    cases = [
        # config 1 shape: t=64, N=2^16, B=96, kick 100, seed 1
        ("config1", "bgh25", "affine", 64, 16, 96, 100, 1, 0, 0, 16384),
        ("config1_b1", "bgh25", "affine", 64, 16, 96, 100, 1, 1, 0, 4096),
        ("config1_seq", "bgh25", "sequential", 64, 16, 96, 100, 1, 0, 0, 4096),
        ("config1_drrt", "drrt18", "affine", 64, 16, 96, 100, 1, 0, 0, 4096),
        # config 2 shape: t=1024, N=2^20, B=1536, kick 500, seed 2, BT 20
        ("config2", "bgh25", "affine", 1024, 20, 1536, 500, 2, 0, 0, 1024),
        ("config2_tail", "bgh25", "affine", 1024, 20, 1536, 500, 2, 0, (1 << 20) - 512, 512),
        ("config2_drrt", "drrt18", "affine", 1024, 20, 1536, 500, 2, 0, 0, 512),
        # stress: tight loads so that failures are frequent
        ("stress_t64", "bgh25", "affine", 64, 16, 80, 50, 11, 0, 0, 4096),
        ("stress_t1024", "bgh25", "affine", 1024, 20, 1200, 200, 12, 3, 0, 512),
        ("stress_drrt_t256", "drrt18", "affine", 256, 18, 290, 50, 13, 0, 0, 2048),
        ("stress_seq_t200", "bgh25", "sequential", 200, 24, 230, 60, 14, 0, 100, 1024),
        # h = 13 / 14 shapes of the sweep, and a large-table shape (config 4 size)
        ("sweep_h13", "bgh25", "affine", 300, 24, 400, 100, 3, 0, 0, 512),
        ("sweep_h13_drrt", "drrt18", "affine", 150, 24, 190, 100, 3, 0, 0, 512),
        ("config4", "bgh25", "affine", 16384, 28, 24576, 1000, 4, 0, 0, 16),
        ("config4_stress", "bgh25", "affine", 16384, 28, 19500, 300, 4, 2, 0, 16),
    ]
    runs = []
    for name, mode, im, pnum, ell, b, kick, seed, batch, first, count in cases:
        buf = (u32 * count)()
        n = lib.ref_batch(mode.encode(), im.encode(), pnum, ell, b, kick, seed, batch, first, count,
                          8, 0, buf)
        runs.append({"name": name, "mode": mode, "input_mode": im, "pnum": pnum, "ell_i": ell,
                     "buckets": b, "kick": kick, "k": 3, "seed": seed, "batch": batch,
                     "first": first, "count": count, "failures": list(buf[:n])})
        print(f"{name}: {n} failures of {count}")
    out["reference_runs"] = runs

    dst = Path(__file__).resolve().parent / "golden.json"
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", dst, dst.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
