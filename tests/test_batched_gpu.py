"""Batched launches (cmc_run_jobs): every job's failures are identical alone
(one cmc_launch per job) and in the mix, whatever the plan."""
import random

import pytest

pytestmark = pytest.mark.gpu


def random_mix(cmc, n, seed, small=False):
    rng = random.Random(seed)
    jobs = []
    for _ in range(n):
        pnum = rng.choice([16, 30, 64, 150, 300] if small else [16, 64, 300, 1024, 2500])
        k = rng.choice([2, 3, 3, 4])
        ell = rng.choice([16, 20, 24])
        b = int(pnum * rng.choice([1.1, 1.25, 1.5]))
        kick = rng.choice([50, 100, 500])
        mode = rng.choice(["bgh25", "bgh25", "drrt18"])
        im = rng.choice(["affine", "sequential"])
        p = cmc.parameters(mode, pnum, ell, k, b, kick, im)
        count = rng.choice([1, 7, 100, 513]) if pnum > 1000 else rng.choice([1, 33, 1000, 2048])
        jobs.append((p, rng.randrange(1 << 32), rng.randrange(16), rng.randrange(1000), count))
    return jobs


@pytest.mark.parametrize("seed", [1, 2])
def test_alone_equals_mix(ctx, cmc, seed):
    jobs = random_mix(cmc, 12, seed)
    failed, per_job = ctx.run_jobs(jobs)
    for i, (p, s, b, first, count) in enumerate(jobs):
        alone = ctx.launch(p, cmc.batch_key(s, b), first, count)
        assert per_job[i] == alone, (i, ctx.last_plan)
        assert failed[i] == len(alone)


def test_autotuned_plan_keeps_results(ctx, cmc):
    jobs = random_mix(cmc, 8, 5, small=True)
    before, per_before = ctx.run_jobs(jobs)
    choice = ctx.autotune(jobs, sample_div=8)
    assert "engine=" in choice
    after, per_after = ctx.run_jobs(jobs)
    assert after == before and per_after == per_before


def test_capacity_limits_offsets_not_counts(ctx, cmc):
    jobs = [(cmc.parameters("bgh25", 64, 16, 3, 70, 20, "affine"), 3, 0, 0, 2000)]
    failed, per_job = ctx.run_jobs(jobs, cap=5)
    assert failed[0] > 5 and len(per_job[0]) == 5
    full = ctx.launch(jobs[0][0], cmc.batch_key(3, 0), 0, 2000)
    assert failed[0] == len(full)


def plan_class_jobs(cmc):
    # long-walk sets (global walk slots) and short ones (shared-memory slots):
    # several plan classes of one entry width
    return [(cmc.parameters("bgh25", 8000, 24, 3, 11200, 500, "affine"), 5, 0, 0, 96),
            (cmc.parameters("bgh25", 64, 16, 3, 80, 50, "affine"), 11, 1, 10, 3000),
            (cmc.parameters("drrt18", 3000, 24, 2, 3600, 100, "affine"), 6, 2, 0, 64),
            (cmc.parameters("bgh25", 300, 20, 4, 340, 100, "sequential"), 7, 0, 5, 700)]


@pytest.mark.parametrize("fused", [1, 0])
def test_plan_classes(ctx, cmc, fused):
    # each class runs under its own plan: all of them in one persistent launch
    # (fused, the default) or one launch per class
    jobs = plan_class_jobs(cmc)
    ctx.set_option("fused", fused)
    ctx.set_option("pool", 0)   # the t = 64 class would take pooled passes, unfused
    try:
        failed, per_job = ctx.run_jobs(jobs)
    finally:
        ctx.set_option("fused", 1)
        ctx.set_option("pool", -1)
    assert " | " in ctx.last_plan
    if fused:
        # classes of one entry width and walk-slot placement share a launch:
        # here shared-slot and global-slot classes, two launches + compaction
        assert ctx.last_plan.startswith("fused(") and ctx.last_kernel_count == 3
    else:
        assert ctx.last_kernel_count == 4   # three classes + compaction
    for i, (p, s, b, first, count) in enumerate(jobs):
        assert per_job[i] == ctx.launch(p, cmc.batch_key(s, b), first, count), i
        assert failed[i] == len(per_job[i])


def test_fused_with_other_entry_width(ctx, cmc):
    # a class with 32-bit entries (B > 65535) runs in a launch of its own
    # beside the fused launch of the 16-bit shared-slot classes (t = 64 and
    # t = 300); the 16-bit global-slot class (t = 3000) is alone in its kind
    # and runs by itself too; every job as alone
    jobs = plan_class_jobs(cmc)[1:] + [
        (cmc.parameters("bgh25", 50000, 20, 3, 70000, 50, "affine"), 9, 0, 0, 8)]
    ctx.set_option("pool", 0)
    try:
        failed, per_job = ctx.run_jobs(jobs)
    finally:
        ctx.set_option("pool", -1)
    assert ctx.last_plan.startswith("fused(") and ctx.last_kernel_count == 4
    for i, (p, s, b, first, count) in enumerate(jobs):
        assert per_job[i] == ctx.launch(p, cmc.batch_key(s, b), first, count), i


def test_fused_uneven_classes_share_ctas(ctx, cmc):
    # one heavy class and many light ones: CTAs that finish a light class move
    # to the heavy one; the result equals the launches one class at a time
    jobs = [(cmc.parameters("bgh25", 2500, 24, 3, 3300, 300, "affine"), 21, 0, 0, 600),
            (cmc.parameters("bgh25", 40, 16, 3, 50, 20, "affine"), 22, 0, 0, 20000),
            (cmc.parameters("bgh25", 200, 20, 2, 260, 60, "affine"), 23, 3, 7, 5000)]
    want = ctx.run_jobs(jobs)
    plan = ctx.last_plan
    ctx.set_option("fused", 0)
    try:
        assert ctx.run_jobs(jobs) == want
    finally:
        ctx.set_option("fused", 1)
    if " | " in plan:
        assert plan.startswith("fused(")


def test_graph_capture_and_replay(ctx, cmc):
    # the same call shape runs eagerly, is captured, then replayed; other keys
    # (other seeds and offsets, same shapes and counts) replay the same graph
    jobs = random_mix(cmc, 10, 9)
    results, states = [], []
    for rnd in range(4):
        js = [(p, s + rnd, b, first, count) for (p, s, b, first, count) in jobs]
        results.append((ctx.run_jobs(js), js))
        states.append(ctx.last_plan.rsplit("graph=", 1)[-1])
        assert ctx.last_engine_ms() > 0     # timing works across capture and replay
    assert states == ["eager", "captured", "replayed", "replayed"], states
    for (failed, per_job), js in results:
        for i, (p, s, b, first, count) in enumerate(js):
            assert per_job[i] == ctx.launch(p, cmc.batch_key(s, b), first, count), i
    ctx.set_option("graph", 0)
    try:
        assert ctx.run_jobs(results[-1][1]) == results[-1][0]
        assert "graph=" not in ctx.last_plan
    finally:
        ctx.set_option("graph", 1)


def test_pooled_class_runs_unfused(ctx, cmc):
    # the t = 64 class takes pooled direct passes in a kernel of its own; the
    # two global-slot classes share a fused launch and the t = 300 class, alone
    # in its kind, runs by itself: four kernels with the compaction, and every
    # job as alone
    jobs = plan_class_jobs(cmc)
    failed, per_job = ctx.run_jobs(jobs)
    assert "pooled" in ctx.last_plan
    assert ctx.last_kernel_count == 4
    for i, (p, s, b, first, count) in enumerate(jobs):
        assert per_job[i] == ctx.launch(p, cmc.batch_key(s, b), first, count), i

