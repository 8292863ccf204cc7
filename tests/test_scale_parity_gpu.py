"""Bit-exact parity at benchmark scale: whole batches of the benchmark shapes,
at loads where trials do fail, against the reference's own CPU code
(cpu_trials.hpp:69-149 via oracle/_ref) -- or, without that build, against
the C restatement at a size it finishes in seconds.  Outcomes are integer
decisions: the bar is equality of the full failure lists."""
import pytest

from ref_binding import Reference, host_threads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def reference():
    return Reference.load()


def cpu_failures(reference, oracle, shape, seed, batch, first, count, port_count):
    """(failures, trials checked): the reference's code over `count` trials,
    or the restatement over the first `port_count` of them."""
    mode, im, pnum, ell, buckets, kick = shape
    if reference is not None:
        return reference.batch(mode, im, pnum, ell, buckets, kick, seed, batch, first, count), count
    op = oracle.params(mode, pnum, ell, 3, buckets, kick, im)
    return oracle.batch(op, seed, batch, first, port_count, host_threads()), port_count


def test_config2_shape_full_batch_stressed(ctx, cmc, oracle, reference):
    # N = 2^20, t = 1024, k = 3 as in the benchmark, B lowered to 1250 and the
    # eviction limit to 250 so that ~1.2 % of trials fail: one whole batch of
    # 2^20 trials, every failing offset compared.
    shape = ("bgh25", "affine", 1024, 20, 1250, 250)
    want, n = cpu_failures(reference, oracle, shape, 2, 0, 0, 1 << 20, 1 << 13)
    p = cmc.parameters("bgh25", 1024, 20, 3, 1250, 250, "affine")
    got = ctx.launch(p, cmc.batch_key(2, 0), 0, n)
    assert got == want
    assert len(want) > n // 200, len(want)   # the case exercises failures


def test_config2_full_batch(ctx, cmc, oracle, reference):
    # the benchmark workload itself (B = 1536, kick 500): one whole batch
    shape = ("bgh25", "affine", 1024, 20, 1536, 500)
    want, n = cpu_failures(reference, oracle, shape, 2, 1, 0, 1 << 20, 1 << 13)
    p = cmc.parameters("bgh25", 1024, 20, 3, 1536, 500, "affine")
    assert ctx.launch(p, cmc.batch_key(2, 1), 0, n) == want


@pytest.mark.parametrize("buckets,kick", [(24576, 1000), (19500, 300)])
def test_config4_table_launch(ctx, cmc, oracle, reference, buckets, kick):
    # full-size config-4 tables (N = 2^28, t = 16384, h = 15: global round
    # cache and global walk slots), 2^12 trials of batch 3; B = 19500 with
    # kick 300 fails about a fifth of the trials.
    shape = ("bgh25", "affine", 16384, 28, buckets, kick)
    want, n = cpu_failures(reference, oracle, shape, 4, 3, 0, 1 << 12, 64)
    p = cmc.parameters("bgh25", 16384, 28, 3, buckets, kick, "affine")
    got = ctx.launch(p, cmc.batch_key(4, 3), 0, n)
    assert got == want, ctx.last_plan
    if buckets == 19500:
        assert len(want) > n // 20


def test_config1_full_batch_drrt18(ctx, cmc, oracle, reference):
    # config-1 table (N = 2^16, t = 64, B = 96) under DRRT18 cycling eviction
    # with a short limit: a whole 2^16-trial batch
    shape = ("drrt18", "affine", 64, 16, 80, 20)
    want, n = cpu_failures(reference, oracle, shape, 1, 0, 0, 1 << 16, 1 << 14)
    p = cmc.parameters("drrt18", 64, 16, 3, 80, 20, "affine")
    assert ctx.launch(p, cmc.batch_key(1, 0), 0, n) == want
    assert len(want) > 0
