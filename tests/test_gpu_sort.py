"""The frontier dedupe's radix sort (cz_sort_pairs) against a stable reference sort: below 2^22 keys one launch
per 8-bit digit pass with decoupled look-back, from 2^22 keys per-tile histograms, a scan and the same staged
scatter per pass. The dedupe relies on stability (equal class keys keep the
order of their child indices) and on the bit ranges it sorts by: the top 32 bits of the class key, and the low
bytes of the child index when the kept classes are put back in order."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    import cheese_b200 as cz
    e = cz.Engine(0)
    yield e
    e.close()


def stable_reference(keys, vals, lo, hi):
    """(keys, vals) stably sorted by bits [lo, hi) of the key, with torch on the device"""
    import torch
    k = keys.clone()
    if hi - lo < 64:
        k = (k >> lo) & ((1 << (hi - lo)) - 1) if hi - lo < 63 else (k >> lo)
    u = k ^ torch.iinfo(torch.int64).min if hi - lo == 64 else k      # unsigned order of the full 64-bit key
    _, order = torch.sort(u, stable=True)
    return keys[order], vals[order]


@pytest.mark.parametrize("n,lo,hi,spread", [
    (2, 0, 64, 64), (2047, 32, 64, 64), (2048, 32, 64, 64), (2049, 32, 64, 64), (100000, 32, 64, 64),
    (100000, 32, 64, 3), (300001, 0, 64, 64), (1 << 20, 0, 24, 24), (3 << 20, 32, 64, 9), (1 << 22, 32, 64, 12),
    (5000000, 32, 64, 64), (9000001, 0, 40, 64)])
def test_sort_matches_stable_reference(engine, n, lo, hi, spread):
    """few distinct keys (spread = random bits in the key) exercise long equal runs across many tiles"""
    import torch
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(n + lo + spread)
    r = torch.randint(0, 1 << 62, (n,), dtype=torch.int64, device=dev, generator=g)
    keys = (r & ((1 << spread) - 1)) << (64 - spread) if spread < 64 else r * 4 + (r >> 60)
    vals = torch.arange(n, dtype=torch.int32, device=dev)
    want_k, want_v = stable_reference(keys, vals, lo, hi)
    k, v = keys.clone(), vals.clone()
    torch.cuda.synchronize()                  # the sort runs on the engine's stream, not torch's
    engine.sort_pairs(k.data_ptr(), v.data_ptr(), n, lo, hi)
    torch.cuda.synchronize()
    assert torch.equal(v, want_v)
    assert torch.equal(k, want_k)


def test_sort_refuses_partial_bytes(engine):
    import torch
    k = torch.zeros(4, dtype=torch.int64, device="cuda")
    v = torch.zeros(4, dtype=torch.int32, device="cuda")
    with pytest.raises(RuntimeError):
        engine.sort_pairs(k.data_ptr(), v.data_ptr(), 4, 0, 12)
