"""cmc_launch_static: the Launch seam for callers that cannot let this library
allocate device memory (for instance a process whose device memory belongs to
another framework's caching allocator, or a serving loop that must avoid
cudaMalloc/cudaFree synchronisation).  Its working memory is a fixed device
array shared by every call; these checks compare it with cmc_launch and with
the oracle on two calls in a row (the second must not see the first call's
failures) and check its limits.  Integer decisions: equality is exact."""
import pytest

pytestmark = pytest.mark.gpu

SHAPES = {
    # load 0.85: frequent failures; 16-bit entries
    "narrow": (("bgh25", 1024, 20, 3, 1200, 200, "affine"), 2, 4096),
    # ell_i = 33 puts the PRP domain above 2^32: 64-bit Feistel halves and
    # 32-bit entries (the other 32-bit-entry shapes, B > 65535 or t > 16384,
    # never fit shared-memory slots and are rejected below)
    "wide_domain": (("drrt18", 40, 33, 3, 48, 20, "affine"), 5, 512),
    # one-warp groups with pooled, folded direct passes (cmc_engine_pooled)
    "pooled": (("bgh25", 64, 16, 3, 70, 20, "affine"), 3, 8192),
}


def device_key(torch, key):
    return torch.tensor(key, dtype=torch.int64).to(torch.int32).cuda()


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_static_matches_launch_and_oracle_on_two_calls(cmc, ctx, oracle, name):
    import torch
    shape, seed, n = SHAPES[name]
    p = cmc.parameters(*shape)
    op = oracle.params(shape[0], shape[1], shape[2], shape[3], shape[4], shape[5], shape[6])
    first = 17
    batches = (3, 4)
    keys = [cmc.batch_key(seed, b) for b in batches]
    want = [oracle.batch(op, seed, b, first, n) for b in batches]
    assert [ctx.launch(p, k, first, n) for k in keys] == want
    assert all(len(w) > 0 for w in want)
    d_keys = [device_key(torch, k) for k in keys]
    outs = [torch.full((n,), -1, dtype=torch.int32, device="cuda") for _ in keys]
    counts = [torch.zeros(1, dtype=torch.int32, device="cuda") for _ in keys]
    stream = torch.cuda.current_stream().cuda_stream
    for d_key, d_out, d_n in zip(d_keys, outs, counts):     # back to back, same stream
        cmc.launch_static(p, d_key.data_ptr(), first, n, d_out.data_ptr(), d_n.data_ptr(), stream)
    torch.cuda.synchronize()
    for w, d_out, d_n in zip(want, outs, counts):
        nf = int(d_n.item()) & 0xffffffff
        assert nf != 0xffffffff, "a bounded device wait gave up"
        assert d_out[:nf].cpu().tolist() == w


def test_static_count_zero_and_limits(cmc):
    import torch
    p = cmc.parameters(*SHAPES["narrow"][0])
    d_key = device_key(torch, cmc.batch_key(2, 0))
    d_out = torch.zeros(16, dtype=torch.int32, device="cuda")
    d_n = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    # no trials: the count is written as 0, as cmc_launch_device does
    cmc.launch_static(p, d_key.data_ptr(), 0, 0, d_out.data_ptr(), d_n.data_ptr())
    torch.cuda.synchronize()
    assert int(d_n.item()) == 0
    with pytest.raises(cmc.CmcError) as e:
        cmc.launch_static(p, d_key.data_ptr(), 0, cmc.STATIC_MAX_TRIALS + 1, d_out.data_ptr(),
                          d_n.data_ptr())
    assert e.value.code == cmc.CMC_EINVAL and "1048576" in str(e.value)
    # tables too large for shared-memory walk slots would need an allocation:
    # the config-4 table, and 32-bit entries from B > 65535
    for shape in (("bgh25", 16384, 28, 3, 24576, 1000, "affine"),
                  ("bgh25", 50000, 20, 3, 70000, 50, "affine")):
        big = cmc.parameters(*shape)
        with pytest.raises(cmc.CmcError) as e:
            cmc.launch_static(big, d_key.data_ptr(), 0, 16, d_out.data_ptr(), d_n.data_ptr())
        assert e.value.code == cmc.CMC_EINVAL and "global memory" in str(e.value)
