"""Serving loop: jobs of different sizes arrive over several steps and run
continuously batched; each job's per-batch failures (from its v3 journal) are
identical to the job run alone, and a served job resumes from its journal."""
import random

import pytest

pytestmark = pytest.mark.gpu


def alone(ctx, cmc, p, seed, budget, bt):
    per = 1 << bt
    out = {}
    for b in range(-(-budget // per)):
        out[b] = ctx.launch(p, cmc.batch_key(seed, b), 0, per)
    return out


def make_jobs(cmc, n, seed):
    rng = random.Random(seed)
    jobs = []
    for _ in range(n):
        pnum = rng.choice([16, 40, 100, 300, 1024])
        k = rng.choice([2, 3])
        b = int(pnum * rng.choice([1.1, 1.2, 1.4]))
        p = cmc.parameters("bgh25", pnum, 24, k, b, rng.choice([30, 500]), "affine")
        jobs.append((p, rng.randrange(1 << 40), rng.choice([1, 300, 1024, 2500, 4096])))
    return jobs


@pytest.mark.parametrize("resident", [0, 1])
def test_served_equals_alone(ctx, cmc, tmp_path, resident):
    bt = 10
    srv = cmc.Server(ctx, max_jobs=16, mem_budget=1 << 30, batch_bits=bt, max_iteration_trials=1 << 16)
    srv.set_option("resident", resident)
    jobs = make_jobs(cmc, 14, 3)
    ids = []
    finished = set()
    for i, (p, seed, budget) in enumerate(jobs):      # arrivals interleaved with steps
        ids.append(srv.submit(p, seed, budget, str(tmp_path / f"job{i}")))
        if i % 3 == 2:
            finished.update(srv.step(2_000_000))
    steps = 0
    while srv.pending():
        finished.update(srv.step(2_000_000))
        steps += 1
        assert steps < 10000
    assert finished == set(ids)
    st = srv.stats()
    total = sum(-(-b // (1 << min(bt, max(1, (b - 1).bit_length())))) << min(bt, max(1, (b - 1).bit_length()))
                for _, _, b in jobs)
    assert st["trials"] == total and st["iterations"] >= 1
    assert 0 < st["busy_ms"] <= st["engine_ms"] + 1e-3 and st["busy_ms"] <= st["span_ms"] + 1e-3
    for i, (p, seed, budget) in enumerate(jobs):
        per = 1 << min(bt, max(1, (budget - 1).bit_length()))
        got = cmc.read_journal(tmp_path / f"job{i}" / "worker_0.bin")
        want = alone(ctx, cmc, p, seed, budget, per.bit_length() - 1)
        assert got == want, i
        done, failed, state = srv.status(ids[i])
        assert state == 2 and failed == sum(len(v) for v in want.values())
        assert done == len(want) * per
    srv.close()


@pytest.mark.parametrize("resident", [0, 1])
def test_served_job_resumes_from_journal(ctx, cmc, tmp_path, resident):
    p = cmc.parameters("bgh25", 64, 16, 3, 70, 20, "affine")
    seed, budget, bt = 77, 4096, 8            # 16 batches of 256
    d = str(tmp_path / "j")
    srv = cmc.Server(ctx, max_jobs=4, batch_bits=bt, max_iteration_trials=1 << 12)
    srv.set_option("resident", resident)
    srv.submit(p, seed, budget, d)
    srv.step(3 * 256 * 800)                   # a few batches only
    srv.close()
    part = cmc.read_journal(tmp_path / "j" / "worker_0.bin")
    assert 0 < len(part) < 16
    srv = cmc.Server(ctx, max_jobs=4, batch_bits=bt, max_iteration_trials=1 << 12)
    srv.set_option("resident", resident)
    job = srv.submit(p, seed, budget, d)
    while srv.pending():
        srv.step(1 << 22)
    full = cmc.read_journal(tmp_path / "j" / "worker_0.bin")
    assert full == alone(ctx, cmc, p, seed, budget, bt)
    assert srv.status(job)[2] == 2
    srv.close()


def test_resident_larger_table_relaunches(ctx, cmc):
    # a job whose walk slots exceed the running launch's plan closes that
    # launch and runs in the next one; results stay those of the job alone
    srv = cmc.Server(ctx, max_jobs=8, mem_budget=1 << 31, batch_bits=12, max_iteration_trials=1 << 16)
    srv.set_option("resident", 1)
    small = cmc.parameters("bgh25", 64, 16, 3, 80, 50, "affine")
    big = cmc.parameters("bgh25", 3000, 24, 3, 3900, 100, "affine")
    a = srv.submit(small, 3, 4096)
    srv.step(1 << 20)
    b = srv.submit(big, 4, 300)
    steps = 0
    while srv.pending():
        srv.step(1 << 20)
        steps += 1
        assert steps < 100000
    assert srv.status(a)[1] == len(alone_flat(ctx, cmc, small, 3, 4096, 12))
    assert srv.status(b)[1] == len(alone_flat(ctx, cmc, big, 4, 300, 9))
    assert srv.stats()["iterations"] >= 1
    srv.close()


def alone_flat(ctx, cmc, p, seed, budget, bt):
    return [x for v in alone(ctx, cmc, p, seed, budget, bt).values() for x in v]
