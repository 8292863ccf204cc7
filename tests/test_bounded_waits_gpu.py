"""Bounded device waits, exercised without a fault: a resident launch waits for
work that the host never publishes.  The wait gives up after spin_limit
microseconds, the kernel returns, the host reads CMC_ETIMEOUT, and the
context stays usable for later launches."""
import time

import pytest

pytestmark = pytest.mark.gpu


def test_resident_wait_gives_up_and_context_survives(ctx, cmc, oracle):
    p = cmc.parameters("bgh25", 64, 16, 3, 80, 50, "affine")
    ctx.set_option("spin_limit", 200_000)  # 0.2 s
    try:
        srv = cmc.Server(ctx, max_jobs=4, batch_bits=16, max_iteration_trials=1 << 16)
        srv.set_option("resident", 1)
        srv.submit(p, 5, 1 << 16)
        srv.step(200_000)      # publishes a first small chunk and starts the launch
        time.sleep(1.0)        # nobody publishes the rest: the launch's waits run out
        with pytest.raises(cmc.CmcError) as e:
            for _ in range(100):
                srv.step(200_000)
        assert e.value.code == cmc.CMC_ETIMEOUT
        try:
            srv.close()
        except cmc.CmcError:
            pass
    finally:
        ctx.set_option("spin_limit", 0)  # back to the default
    # the context still works
    op = oracle.params("bgh25", 64, 16, 3, 80, 50, "affine")
    assert ctx.launch(p, cmc.batch_key(5, 0), 0, 2048) == oracle.batch(op, 5, 0, 0, 2048)
