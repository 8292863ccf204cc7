"""cmc_launch_static: the Launch seam for callers that cannot let this library
allocate device memory (for instance a process whose device memory belongs to
another framework's caching allocator, or a serving loop that must avoid
cudaMalloc/cudaFree synchronisation).  Its working memory is a fixed device
array shared by every call; these checks compare it with cmc_launch on two
calls in a row (the second must not see the first call's failures) and check
its limits.  Integer decisions: equality is exact."""
import pytest

pytestmark = pytest.mark.gpu

SHAPE = ("bgh25", 1024, 20, 3, 1200, 200, "affine")   # load 0.85: frequent failures


def device_key(torch, key):
    return torch.tensor(key, dtype=torch.int64).to(torch.int32).cuda()


def test_static_matches_launch_on_two_calls(cmc, ctx):
    import torch
    p = cmc.parameters(*SHAPE)
    n, first = 4096, 17
    keys = [cmc.batch_key(2, b) for b in (3, 4)]
    want = [ctx.launch(p, k, first, n) for k in keys]
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


def test_static_rejects_sizes_beyond_its_memory(cmc):
    import torch
    p = cmc.parameters(*SHAPE)
    d_key = device_key(torch, cmc.batch_key(2, 0))
    d_out = torch.zeros(16, dtype=torch.int32, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(cmc.CmcError) as e:
        cmc.launch_static(p, d_key.data_ptr(), 0, cmc.STATIC_MAX_TRIALS + 1, d_out.data_ptr(),
                          d_n.data_ptr())
    assert e.value.code == cmc.CMC_EINVAL and "1048576" in str(e.value)
    # a table too large for shared-memory walk slots would need an allocation
    big = cmc.parameters("bgh25", 16384, 28, 3, 24576, 1000, "affine")
    with pytest.raises(cmc.CmcError) as e:
        cmc.launch_static(big, d_key.data_ptr(), 0, 16, d_out.data_ptr(), d_n.data_ptr())
    assert e.value.code == cmc.CMC_EINVAL and "global memory" in str(e.value)
