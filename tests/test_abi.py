"""The C ABI library: it loads, exports what include/cmc.h declares, and its
host-side functions (parameters, batch keys, host AES) match the reference."""
import ctypes
import re

import pytest

from conftest import ROOT


def declared_functions():
    text = (ROOT / "include/cmc.h").read_text()
    return sorted(set(re.findall(r"\b(cmc_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(cmc):
    lib = ctypes.CDLL(str(cmc.LIB_PATH))
    declared = declared_functions()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(cmc.EXPORTS)


def test_build_targets_sm100a_only():
    # every nvcc line of the product build compiles for sm_100a and nothing else
    # (no PTX for JIT, no other architecture)
    make = (ROOT / "pbc-based-dmpf-monte-carlo-test_b200" / "Makefile").read_text()
    arch = re.findall(r"^ARCH\s*:=\s*(.+)$", make, re.M)
    assert arch == ["-gencode arch=compute_100a,code=sm_100a"]
    assert "$(ARCH)" in make.split("CUFLAGS", 1)[1].split("\n", 1)[0]
    assert re.findall(r"-arch[= ]|compute_\d+(?![\da])|code=compute", make) == []


def test_params_grid(cmc, golden):
    for g in golden["params_grid"]:
        p = cmc.parameters(g["mode"], g["pnum"], g["ell_i"], 3, g["buckets_override"],
                           g["kick_override"])
        got = (p.buckets, p.kick, p.bucket_size, p.domain, p.mask, p.half_bits)
        want = (g["buckets"], g["kick"], g["bucket_size"], g["domain"], g["mask"], g["half_bits"])
        assert got == want, g


def test_param_pins(cmc, golden):
    for pin in golden["param_pins"]:
        assert cmc.parameters(pin["mode"], pin["pnum"], pin["ell_i"]).buckets == pin["buckets"]


@pytest.mark.parametrize("args", [
    dict(mode="bgh25", pnum=2, ell_i=8),          # PNUM < 3
    dict(mode="bgh25", pnum=65535, ell_i=20),     # PNUM > 65534
    dict(mode="bgh25", pnum=16, ell_i=62),        # ell_i > 61
    dict(mode="bgh25", pnum=300, ell_i=8),        # 2^ell_i < PNUM
    dict(mode="bgh25", pnum=16, ell_i=8, k=5),    # k outside 2..4
])
def test_invalid_params_rejected(cmc, args):
    with pytest.raises(cmc.CmcError):
        cmc.parameters(**args)


def test_batch_keys(cmc, golden, oracle):
    for case in golden["batch_key_schedules"]:
        assert cmc.batch_key(case["seed"], case["batch"]) == case["schedule"]
    g = golden["batch_key_vectors"]
    for batch, expect in zip(g["batches"], g["aes_of_zero"]):
        assert cmc.host_aes128(cmc.batch_key(g["seed"], batch), [0, 0, 0, 0]) == expect


def test_host_aes_fips(cmc, golden, oracle):
    g = golden["fips197"]
    rk = oracle.expand_key(g["key_lo"], g["key_hi"])
    assert cmc.host_aes128(rk, g["plain"]) == g["cipher"]


def test_init_without_gpu_fails_cleanly(cmc):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(cmc.CmcError) as e:
        cmc.Context(0)
    assert e.value.code in (cmc.CMC_ECUDA, cmc.CMC_EINVAL)
