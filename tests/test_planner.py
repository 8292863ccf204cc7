"""Launch planner decisions on CPU (cmc_plan_describe needs no device), pinned
to the plans measured fastest on B200: shared walk slots and a shared round
cache where walks keep up with the producers, global slots with four isolated
walkers and an L2 round cache for long walks, the u32 and 64-bit-domain
variants where the shape needs them."""
import pytest

B200 = dict(sms=148, smem_optin=232448)


def plan(cmc, shape, count):
    return cmc.plan_describe(cmc.parameters(*shape), count, **B200)


@pytest.mark.parametrize("shape,count,expect", [
    # config 2 (measured 2.81 M trials/s with this plan)
    (("bgh25", 1024, 20, 3, 1536, 500, "affine"), 1 << 20,
     ["groups=2 warps_per_group=6 walkers=1(isolated)", "slots_in=smem", "cache=smem", "variant=narrow"]),
    # config 1 (28.8 M trials/s): many one-warp groups, no cache, three trials
    # per warp (pooled direct passes)
    (("bgh25", 64, 16, 3, 96, 100, "affine"), 1 << 16,
     ["groups=14 warps_per_group=1", "slots_in=smem", "cache=off pooled"]),
    # direct passes up to 1,536 candidates per trial: one-warp groups, pooled
    # (t=300: 6.75 M trials/s against 5.14 M in 4-warp groups)
    (("bgh25", 300, 20, 3, 400, 100, "affine"), 1 << 18, ["warps_per_group=1", "pooled"]),
    # beyond it 4-warp groups, one trial at a time (t=1000: 1.61 M against 1.57 M)
    (("bgh25", 1000, 24, 3, 1300, 200, "affine"), 1 << 16,
     ["warps_per_group=4", "slots=15 slots_in=smem", "cache=off"]),
    # config 4 and long walks: global slots walked by four isolated warps
    (("bgh25", 16384, 28, 3, 24576, 1000, "affine"), 1 << 16,
     ["walkers=4(isolated)", "slots=128 slots_in=global", "cache=global"]),
    (("bgh25", 8000, 24, 3, 11200, 500, "affine"), 1 << 16, ["slots_in=global", "cache=global"]),
    (("bgh25", 3000, 24, 3, 3900, 500, "affine"), 1 << 17, ["slots_in=global", "cache=global"]),
    # walker beside producers would not keep up with four shared slots
    (("bgh25", 500, 20, 4, 640, 100, "affine"), 1 << 19, ["slots_in=global", "cache=smem"]),
    # walks keep up: shared slots
    (("bgh25", 400, 24, 2, 520, 500, "affine"), 1 << 19, ["slots_in=smem"]),
    (("bgh25", 1500, 24, 4, 2025, 100, "affine"), 1 << 17, ["slots_in=smem", "cache=global"]),
    # entry width and PRP domain
    (("bgh25", 50000, 20, 3, 70000, 50, "affine"), 8, ["variant=wide"]),
    (("drrt18", 40, 33, 3, 60, 30, "affine"), 256, ["variant=wide-domain", "cache=off"]),
])
def test_plan_choices(cmc, shape, count, expect):
    text = plan(cmc, shape, count)
    for e in expect:
        assert e in text, (e, text)
    smem = int(text.split("smem=")[1].split()[0])
    assert smem <= B200["smem_optin"]


def test_plan_respects_the_device_limits(cmc):
    # fewer SMs: one persistent CTA per SM; less shared memory: fewer slots
    small = plan(cmc, ("bgh25", 1024, 20, 3, 1536, 500, "affine"), 1 << 20)
    assert "ctas=148" in small
    text = cmc.plan_describe(cmc.parameters("bgh25", 1024, 20, 3, 1536, 500, "affine"), 1 << 20,
                             sms=20, smem_optin=164 * 1024)
    assert "ctas=20" in text and int(text.split("smem=")[1].split()[0]) <= 164 * 1024


def test_plan_describe_rejects_bad_arguments(cmc):
    p = cmc.parameters("bgh25", 64, 16, 3, 96, 100, "affine")
    with pytest.raises(cmc.CmcError):
        cmc.plan_describe(p, 0)
    with pytest.raises(cmc.CmcError):
        cmc.plan_describe(p, 16, sms=148, smem_optin=4096)


def test_direct_fold_tables_yield_to_walk_slots(cmc):
    # direct passes at h = 13 keep their 4 KB fold tables while 4 or more
    # shared slots per group remain (t=1000: 15 slots, 1.74 M trials/s against
    # 1.59 M with 18 slots and no tables) and give them up below (t=2000: 9
    # slots, not 6: 0.83 M against 0.72 M)
    t1000 = plan(cmc, ("bgh25", 1000, 24, 3, 1300, 200, "affine"), 1 << 16)
    t2000 = plan(cmc, ("bgh25", 2000, 24, 3, 2600, 100, "affine"), 1 << 15)
    assert "groups=3 warps_per_group=4" in t1000 and "slots=15 slots_in=smem" in t1000
    assert "groups=3 warps_per_group=4" in t2000 and "slots=9 slots_in=smem" in t2000
    assert "pooled" not in t1000 + t2000

