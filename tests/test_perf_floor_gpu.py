"""Throughput floors on B200: half of the rates measured for these shapes, so a
plan or engine change that costs a large factor fails here.  Walks over
global walk slots have twice turned ~4-5x slower after changes that passed
every correctness test (a value held across the walker loop; a change of the
kernel's register allocation): config 4 and the global-slot plan of config 2
guard that.  Run-to-run spread on B200 is about 1 %."""
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [
    # name, shape, seed, trials, planner options, measured trials/s
    ("config2", ("bgh25", 1024, 20, 3, 1536, 500, "affine"), 2, 1 << 18, {}, 3.47e6),
    ("config2_global_slots", ("bgh25", 1024, 20, 3, 1536, 500, "affine"), 2, 1 << 18,
     {"warps_per_group": 3, "groups": 4}, 3.44e6),
    ("config1", ("bgh25", 64, 16, 3, 96, 100, "affine"), 1, 1 << 20, {}, 3.0e7),
    ("config4", ("bgh25", 16384, 28, 3, 24576, 1000, "affine"), 4, 1 << 16, {}, 1.62e5),
    ("t8000_global_slots", ("bgh25", 8000, 24, 3, 11200, 500, "affine"), 5, 1 << 16, {}, 4.2e5),
]


@pytest.mark.parametrize("name,shape,seed,n,options,measured", SHAPES, ids=[s[0] for s in SHAPES])
def test_throughput_floor(ctx, cmc, name, shape, seed, n, options, measured):
    p = cmc.parameters(*shape)
    for k, v in options.items():
        ctx.set_option(k, v)
    try:
        ctx.launch(p, cmc.batch_key(seed, 0), 0, n)          # warm
        ctx.launch(p, cmc.batch_key(seed, 1), 0, n)
        rate = n / (ctx.last_engine_ms() / 1e3)
    finally:
        for k in options:
            ctx.set_option(k, 0)
    assert rate >= 0.5 * measured, (name, rate, ctx.last_plan)
