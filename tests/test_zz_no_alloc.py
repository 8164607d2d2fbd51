"""The allocation-free bound evaluation (cz_eval_bounds_noalloc) against the allocating one (cz_eval_bounds).

The entry point exists for callers that cannot allocate device memory themselves: code whose device memory is
owned by a fixed-size pool or by another runtime's allocator, or a memory-capped service that must not grow its
footprint. They hand in device buffers for the residuals, exponents and results, and the library stages the
spec's tables in a static device array instead of allocating. Here the test owns the device buffers (allocated
with torch, outside the call) and checks calls in a row on one stream, on specs of different qubit counts, so
each call must fully replace the tables the previous one staged.

The file name sorts last so that pytest collects it after every other test file: a run that stops at the first
failure (-x) has then already run the rest of the suite before this addition can stop it. Each test also passes
in a fresh process on its own.
"""
import ctypes as C
import random

import pytest

import cheese_b200 as cz
from cheese_b200 import workloads
from conftest import spec_text

pytestmark = pytest.mark.gpu

# the no-alloc kernel's grid is capped at (SM count x 8) blocks of 8 warps, one residual per warp per step: more
# residuals than that run through its grid-stride loop (148 SMs on a B200)
GRID_STRIDE = 148 * 8 * 8


def residuals(seed, n, count):
    rng = random.Random(seed)
    out = []
    for _ in range(count):
        circ = []
        for _ in range(rng.randint(0, 14)):
            g = rng.choice(["h", "t", "tdg", "s", "sdg", "x", "z", "cx"])
            circ.append((g, tuple(rng.sample(range(n), 2)) if g == "cx" else (rng.randrange(n),)))
        out.append(workloads.unitary(n, circ))
    return out


def rotations(seed, count):
    """3-qubit residuals whose limbs exceed int32: (H T)^m on one qubit (an irrational rotation, so the sqrt2
    exponent grows with m and stays after normalisation), then a few random gates"""
    rng = random.Random(seed)
    out = []
    for _ in range(count):
        q = rng.randrange(3)
        circ = [("h", (q,)), ("t", (q,))] * rng.randint(130, 150)
        for _ in range(8):
            g = rng.choice(["h", "t", "cx", "s"])
            circ.append((g, tuple(rng.sample(range(3), 2)) if g == "cx" else (rng.randrange(3),)))
        out.append(workloads.unitary(3, circ))
    return out


def call_noalloc(L, spec, res, stream, dev):
    import torch
    count = len(res)
    ent = torch.tensor([v for _, M in res for row in M for x in row for v in x], dtype=torch.int64, device=dev)
    ks = torch.tensor([k for k, _ in res], dtype=torch.int32, device=dev)
    out = torch.full((count, 4), -7, dtype=torch.int32, device=dev)
    err = C.create_string_buffer(256)
    rc = L.cz_eval_bounds_noalloc(spec._h, count, ent.data_ptr(), ks.data_ptr(), out.data_ptr(), stream, err, 256)
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize(dev)
    return [tuple(r) for r in out.cpu().tolist()]


def test_noalloc_bounds_match_allocating_entry_point():
    import torch
    eng = cz.Engine(0)
    L = cz.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call, (stem, n, count) in enumerate([("toffoli", 3, 257), ("cs", 2, 130), ("toffoli", 3, 33)]):
        spec = cz.Spec(spec_text(stem))
        res = residuals(100 + call, n, count)
        want = eng.eval_bounds(spec, res)                      # the existing entry point (it allocates)
        got = call_noalloc(L, spec, res, stream, dev)
        assert got == want, (stem, [i for i, (a, b) in enumerate(zip(got, want)) if a != b][:5])
    eng.close()


def test_noalloc_wide_limbs_and_grid_stride():
    """residuals with limbs beyond int32 (the allocating path then computes in int64 too, like this one), and more
    residuals than one pass of the kernel's grid covers"""
    import torch
    eng = cz.Engine(0)
    L = cz.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    spec = cz.Spec(spec_text("toffoli"))
    wide = rotations(7, 6)
    assert max(abs(v) for _, M in wide for row in M for x in row for v in x) > 2 ** 31
    want = eng.eval_bounds(spec, wide)
    assert call_noalloc(L, spec, wide, stream, dev) == want
    base = residuals(11, 3, 97)
    many = (base * (GRID_STRIDE // len(base) + 2))[:GRID_STRIDE + 1]
    want = eng.eval_bounds(spec, many)
    got = call_noalloc(L, spec, many, stream, dev)
    assert got == want, [i for i, (a, b) in enumerate(zip(got, want)) if a != b][:5]
    eng.close()


def test_noalloc_refuses_what_does_not_fit():
    import torch
    L = cz.lib()
    dev = torch.device("cuda", 0)
    text = spec_text("toffoli")
    big = text.split("cxtable")[0] + "cxtable 5000\n" + " ".join(["0"] * 5000) + "\nend\n"
    spec = cz.Spec(big)
    ent = torch.zeros(64 * 4, dtype=torch.int64, device=dev)
    ks = torch.zeros(1, dtype=torch.int32, device=dev)
    out = torch.zeros(4, dtype=torch.int32, device=dev)
    err = C.create_string_buffer(256)
    rc = L.cz_eval_bounds_noalloc(spec._h, 1, ent.data_ptr(), ks.data_ptr(), out.data_ptr(), None, err, 256)
    assert rc == cz.ERR_USAGE and b"4096" in err.value
    rc = L.cz_eval_bounds_noalloc(spec._h, 1, ent.data_ptr() + 8, ks.data_ptr(), out.data_ptr(), None, err, 256)
    assert rc == cz.ERR_USAGE and b"aligned" in err.value
    # no residuals: nothing to do, so null buffers are accepted
    rc = L.cz_eval_bounds_noalloc(cz.Spec(text)._h, 0, None, None, None, None, err, 256)
    assert rc == 0
    # state-target specs have their own row bounds: refused by both entry points
    st = cz.Spec(spec_text("cs-states"))
    rc = L.cz_eval_bounds_noalloc(st._h, 1, ent.data_ptr(), ks.data_ptr(), out.data_ptr(), None, err, 256)
    assert rc == cz.ERR_USAGE and b"state" in err.value
    eng = cz.Engine(0)
    with pytest.raises(RuntimeError):
        eng.eval_bounds(st, [(0, [[(1, 0, 0, 0) if i == j else (0, 0, 0, 0) for j in range(4)] for i in range(4)])])
    eng.close()
