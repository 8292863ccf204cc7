"""The CPU oracle is pinned to the reference's golden vectors and to the
reference's own CPU code (fixtures in tests/golden/golden.json)."""
import pytest


def test_fips197(oracle, golden):
    g = golden["fips197"]
    rk = oracle.expand_key(g["key_lo"], g["key_hi"])
    assert oracle.aes(rk, g["plain"]) == g["cipher"]


def test_batch_key_vectors(oracle, golden):
    g = golden["batch_key_vectors"]
    for batch, expect in zip(g["batches"], g["aes_of_zero"]):
        assert oracle.aes(oracle.batch_key(g["seed"], batch), [0, 0, 0, 0]) == expect


def test_batch_key_schedules(oracle, golden):
    for case in golden["batch_key_schedules"]:
        assert oracle.batch_key(case["seed"], case["batch"]) == case["schedule"]


def test_param_pins(oracle, golden):
    for pin in golden["param_pins"]:
        assert oracle.params(pin["mode"], pin["pnum"], pin["ell_i"]).buckets == pin["buckets"]


def test_params_grid(oracle, golden):
    for g in golden["params_grid"]:
        p = oracle.params(g["mode"], g["pnum"], g["ell_i"], 3, g["buckets_override"],
                          g["kick_override"])
        got = (p.buckets, p.kick, p.bucket_size, p.domain, p.mask, p.half_bits)
        want = (g["buckets"], g["kick"], g["bucket_size"], g["domain"], g["mask"], g["half_bits"])
        assert got == want, g


@pytest.mark.parametrize("mode", ["bgh25", "drrt18"])
def test_golden_32768(oracle, golden, mode):
    g = golden["golden_32768"]
    p = oracle.params(mode, g["pnum"], g["ell_i"])
    per = 1 << g["bt"]
    failed = []
    for batch in range(1 << (g["et"] - g["bt"])):
        failed += [batch * per + o for o in oracle.batch(p, g["seed"], batch, 0, per)]
    assert failed == g["failures"][mode]


def test_smoke_prefix_consistent(golden):
    s = golden["smoke_8192"]
    full = golden["golden_32768"]["failures"]
    for mode, fails in s["failures"].items():
        assert fails == [x for x in full[mode] if x < (1 << s["ET"])]


@pytest.mark.parametrize("mode", ["bgh25", "drrt18"])
def test_affine_pnum3(oracle, golden, mode):
    g = golden["affine_pnum3"]
    p = oracle.params(mode, g["pnum"], g["ell_i"], input_mode="affine")
    assert oracle.batch(p, g["seed"], g["batch"], 0, g["count"]) == g["failures"][mode]


def test_reference_runs(oracle, golden):
    for r in golden["reference_runs"]:
        p = oracle.params(r["mode"], r["pnum"], r["ell_i"], r["k"], r["buckets"], r["kick"],
                          r["input_mode"])
        got = oracle.batch(p, r["seed"], r["batch"], r["first"], r["count"])
        assert got == r["failures"], r["name"]


def test_k_generalisation_changes_only_k(oracle):
    # k=3 is the reference; k=2 and k=4 are extensions (parity unpinned).
    # Their derived domain follows D = B * ceil(k 2^ell / B).
    for k in (2, 3, 4):
        p = oracle.params("bgh25", 64, 16, k, 96, 100, "affine")
        assert p.bucket_size == -(-(k << 16) // 96)
        assert p.domain == 96 * p.bucket_size
        assert len(oracle.batch(p, 1, 0, 0, 64)) <= 64
