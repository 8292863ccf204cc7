"""GPU parity: the sm_100a path through the C ABI against the reference's
golden vectors, the reference's own CPU code (fixtures) and the oracle.
Outcomes are integer decisions, so the bar is bit-exact equality."""
import random

import pytest

pytestmark = pytest.mark.gpu

ENGINE_VARIANTS = [
    {},                                        # automatic plan
    {"method": 0},                             # direct AES passes
    {"method": 1},                             # shared-memory round cache (h <= 12)
    {"global_slots": 1},                       # walk slots in global memory
    {"warps_per_group": 1},
    {"warps_per_group": 4, "groups": 2},
    {"walker_ctas": 8},                        # split engine: 8 SMs walk, the rest build maps
    {"walker_ctas": 20, "warps_per_group": 8, "method": 0},
    {"walkers": 2, "warps_per_group": 7, "isolate_walkers": 0},
    {"isolate_walkers": 1, "warps_per_group": 6, "walkers": 3},
    {"isolate_walkers": 1, "warps_per_group": 1, "global_slots": 1},
    {"method": 2},                             # round cache in global memory (h <= 16)
    {"method": 2, "isolate_walkers": 1, "global_slots": 1, "warps_per_group": 4},
    {"method": 1, "map_chains": 2},            # two lookup chains per lane (shared cache)
    {"method": 2, "map_chains": 1},
    {"method": 2, "map_chains": 4},
    {"pool": 1, "warps_per_group": 1, "method": 0},   # pooled direct passes (three trials per warp)
]


DEFAULTS = {"method": -1, "global_slots": 0, "warps_per_group": 0, "groups": 0, "walkers": 0,
            "walker_ctas": -1, "isolate_walkers": -1, "map_chains": 0, "pool": -1}


def apply(ctx, opts):
    for name, default in DEFAULTS.items():
        ctx.set_option(name, opts.get(name, default))


@pytest.fixture(autouse=True)
def _reset(ctx):
    apply(ctx, {})
    yield
    apply(ctx, {})


def test_selftest_and_plan(ctx, cmc):
    p = cmc.parameters("bgh25", 16, 8)
    assert ctx.launch(p, cmc.batch_key(123, 16), 146, 1) == [146]   # golden trial 4242
    assert "engine=group" in ctx.last_plan
    assert ctx.last_kernel_count == 2


@pytest.mark.parametrize("mode", ["bgh25", "drrt18"])
@pytest.mark.parametrize("micro", [256, 37])
def test_golden_32768(ctx, cmc, golden, mode, micro):
    g = golden["golden_32768"]
    p = cmc.parameters(mode, g["pnum"], g["ell_i"])
    per = 1 << g["bt"]
    failed = []
    for batch in range(1 << (g["et"] - g["bt"])):
        failed += [batch * per + o for o in cmc.process_batch(ctx, p, g["seed"], batch, per, micro)]
    assert failed == g["failures"][mode]


@pytest.mark.parametrize("variant", range(len(ENGINE_VARIANTS)))
def test_golden_engine_variants(ctx, cmc, golden, variant):
    apply(ctx, ENGINE_VARIANTS[variant])
    g = golden["golden_32768"]
    per = 1 << g["bt"]
    for mode in ("bgh25", "drrt18"):
        p = cmc.parameters(mode, g["pnum"], g["ell_i"])
        failed = []
        for batch in range(32):   # first 8192 trials
            failed += [batch * per + o for o in ctx.launch(p, cmc.batch_key(g["seed"], batch), 0, per)]
        assert failed == [x for x in g["failures"][mode] if x < 32 * per], (mode, ctx.last_plan)


@pytest.mark.parametrize("mode", ["bgh25", "drrt18"])
def test_affine_pnum3(ctx, cmc, golden, mode):
    g = golden["affine_pnum3"]
    p = cmc.parameters(mode, g["pnum"], g["ell_i"], input_mode="affine")
    assert ctx.launch(p, cmc.batch_key(g["seed"], g["batch"]), 0, g["count"]) == g["failures"][mode]


def reference_cases(golden):
    return [r["name"] for r in golden["reference_runs"]]


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 6, 7, 9, 10, 11, 12, 13, 14, 15])
def test_reference_runs(ctx, cmc, golden, variant):
    apply(ctx, ENGINE_VARIANTS[variant])
    for r in golden["reference_runs"]:
        p = cmc.parameters(r["mode"], r["pnum"], r["ell_i"], r["k"], r["buckets"], r["kick"],
                           r["input_mode"])
        got = ctx.launch(p, cmc.batch_key(r["seed"], r["batch"]), r["first"], r["count"])
        assert got == r["failures"], (r["name"], ctx.last_plan)


def random_shapes(n, seed):
    rng = random.Random(seed)
    out = []
    for _ in range(n):
        k = rng.choice([2, 3, 3, 4])
        pnum = rng.choice([3, 5, 16, 40, 64, 100, 257, 600, 1024])
        ell = rng.choice([e for e in (8, 12, 16, 20, 24, 28, 33, 40) if e >= 16 or (1 << e) >= pnum])
        load = rng.choice([1.05, 1.15, 1.3, 1.6])
        buckets = max(pnum + 1, int(pnum * load))
        kick = rng.choice([5, 20, 100, 500])
        mode = rng.choice(["bgh25", "drrt18"])
        im = rng.choice(["sequential", "affine"])
        out.append((mode, im, pnum, ell, k, buckets, kick, rng.randrange(1 << 40), rng.randrange(64)))
    return out


@pytest.mark.parametrize("shape", random_shapes(24, 7))
def test_vs_oracle_random_shapes(ctx, cmc, oracle, shape):
    mode, im, pnum, ell, k, buckets, kick, seed, batch = shape
    apply(ctx, ENGINE_VARIANTS[[0, 6, 7, 9, 10, 11, 12, 13, 15, 16][seed % 10]])
    p = cmc.parameters(mode, pnum, ell, k, buckets, kick, im)
    op = oracle.params(mode, pnum, ell, k, buckets, kick, im)
    count = 512 if pnum <= 100 else 96
    first = 1000
    want = oracle.batch(op, seed, batch, first, count)
    got = ctx.launch(p, cmc.batch_key(seed, batch), first, count)
    assert got == want, (shape, ctx.last_plan)


def test_wide_entries(ctx, cmc, oracle):
    # B > 65535 forces 32-bit map and table entries
    p = cmc.parameters("bgh25", 50000, 20, 3, 70000, 50, "affine")
    op = oracle.params("bgh25", 50000, 20, 3, 70000, 50, "affine")
    want = oracle.batch(op, 9, 0, 0, 8)
    assert ctx.launch(p, cmc.batch_key(9, 0), 0, 8) == want
    assert "variant=wide" in ctx.last_plan


def test_wide_domain(ctx, cmc, oracle):
    # ell_i = 33 puts the PRP domain above 2^32 (64-bit Feistel halves)
    p = cmc.parameters("drrt18", 40, 33, 3, 60, 30, "affine")
    assert p.domain > 2**32
    op = oracle.params("drrt18", 40, 33, 3, 60, 30, "affine")
    want = oracle.batch(op, 5, 1, 0, 256)
    assert ctx.launch(p, cmc.batch_key(5, 1), 0, 256) == want
    assert "wide-domain" in ctx.last_plan


@pytest.mark.parametrize("method", [0, 2])
def test_global_round_cache_h13_to_16(ctx, cmc, oracle, method):
    # half widths 13..16: direct passes and the L2-resident round cache agree
    # with the oracle trial for trial
    for mode, pnum, ell, k, buckets, kick, seed in [
            ("bgh25", 3000, 24, 3, 3900, 100, 21),      # h = 13
            ("drrt18", 1500, 24, 4, 1900, 60, 22),      # h = 14
            ("bgh25", 600, 28, 3, 700, 200, 23),        # h = 15
            ("bgh25", 200, 28, 4, 260, 100, 24)]:       # h = 16
        p = cmc.parameters(mode, pnum, ell, k, buckets, kick, "affine")
        op = oracle.params(mode, pnum, ell, k, buckets, kick, "affine")
        ctx.set_option("method", method)
        want = oracle.batch(op, seed, 1, 50, 64)
        assert ctx.launch(p, cmc.batch_key(seed, 1), 50, 64) == want, (p.half_bits, ctx.last_plan)
        assert ("cache=global" in ctx.last_plan) == (method == 2)


def test_launch_device_matches_host(ctx, cmc):
    import torch
    p = cmc.parameters("bgh25", 64, 16, 3, 80, 50, "affine")
    key = cmc.batch_key(11, 0)
    want = ctx.launch(p, key, 0, 4096)
    d_key = torch.tensor(key, dtype=torch.int64).to(torch.int32).cuda()
    d_out = torch.zeros(4096, dtype=torch.int32, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    ctx.launch_device(p, d_key.data_ptr(), 0, 4096, d_out.data_ptr(), d_n.data_ptr(), stream)
    torch.cuda.synchronize()
    ctx.check()
    n = int(d_n.item())
    assert d_out[:n].cpu().tolist() == want


def test_full_batch_properties(ctx, cmc):
    # config 2 shape, one whole batch of 2^20 trials: sorted, unique, in range,
    # and identical when the batch is split into micro-launches.
    p = cmc.parameters("bgh25", 1024, 20, 3, 1200, 200, "affine")
    key = cmc.batch_key(2, 0)
    n = 1 << 17
    whole = ctx.launch(p, key, 0, n)
    assert whole == sorted(set(whole)) and all(0 <= x < n for x in whole)
    parts = []
    for off in range(0, n, 3 << 14):
        parts += ctx.launch(p, key, off, min(3 << 14, n - off))
    assert parts == whole
    assert len(whole) > 0


@pytest.mark.parametrize("shape", [
    # mode, input, t, ell_i, k, B, kick  (direct passes, shared walk slots)
    ("bgh25", "affine", 64, 16, 3, 96, 100),       # config-1 table
    ("bgh25", "affine", 64, 16, 3, 70, 20),        # failing often
    ("drrt18", "affine", 64, 16, 3, 80, 20),
    ("bgh25", "sequential", 27, 12, 2, 30, 5),
    ("bgh25", "affine", 300, 20, 4, 330, 50),
    ("drrt18", "sequential", 5, 8, 3, 6, 5),       # fewer candidates than lanes
    ("bgh25", "affine", 100, 18, 3, 130, 100),     # h = 10: 4 fold entries per round
    ("bgh25", "affine", 40, 17, 2, 50, 30),        # h = 10, k = 2
])
def test_pooled_direct_passes_vs_oracle(ctx, cmc, oracle, shape):
    # three trials in flight per one-warp group, maps staged and copied into
    # slots at publish time, rounds 1-2 from the trial's fold table when
    # h <= 10 (the t = 300 shape, h = 11, takes unfolded passes): every
    # trial's outcome as the oracle has it
    mode, im, pnum, ell, k, buckets, kick = shape
    apply(ctx, {"pool": 1, "warps_per_group": 1, "method": 0})
    p = cmc.parameters(mode, pnum, ell, k, buckets, kick, im)
    op = oracle.params(mode, pnum, ell, k, buckets, kick, im)
    want = oracle.batch(op, 11, 2, 5, 3000)
    got = ctx.launch(p, cmc.batch_key(11, 2), 5, 3000)
    assert "pooled" in ctx.last_plan, ctx.last_plan
    assert got == want, (shape, ctx.last_plan)


@pytest.mark.parametrize("shape", [
    # mode, input, t, ell_i, k, B, kick: direct passes in 4-warp groups with
    # shared walk slots, rounds 1-2 from the word-split fold table (h <= 13)
    ("bgh25", "affine", 1000, 24, 3, 1300, 200),   # h = 13: 32 fold entries per round
    ("drrt18", "sequential", 800, 20, 3, 1000, 50),
    ("bgh25", "affine", 700, 24, 4, 900, 500),      # h = 14: unfolded passes
])
def test_folded_direct_passes_vs_oracle(ctx, cmc, oracle, shape):
    mode, im, pnum, ell, k, buckets, kick = shape
    apply(ctx, {"method": 0, "warps_per_group": 4, "groups": 3, "pool": 0})
    p = cmc.parameters(mode, pnum, ell, k, buckets, kick, im)
    op = oracle.params(mode, pnum, ell, k, buckets, kick, im)
    want = oracle.batch(op, 13, 1, 7, 200)
    got = ctx.launch(p, cmc.batch_key(13, 1), 7, 200)
    assert "slots_in=smem" in ctx.last_plan, ctx.last_plan
    assert got == want, (shape, ctx.last_plan)

