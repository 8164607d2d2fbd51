"""The allocation-free bound evaluation (cz_eval_bounds_noalloc) against the allocating one (cz_eval_bounds).

The entry point exists for callers that cannot allocate device memory themselves (a fixed-size or foreign
allocator owns the GPU): they hand in device buffers for the residuals, exponents and results, and the library
stages the spec's tables in a static device array instead of allocating. Here the test owns the device buffers
(allocated with torch, outside the call) and checks two calls in a row, on specs of different qubit counts, so the
second call must fully replace the staged tables of the first. This file is collected last on purpose.
"""
import ctypes as C
import random

import pytest

import cheese_b200 as cz
from cheese_b200 import workloads
from conftest import spec_text

pytestmark = pytest.mark.gpu


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


def test_noalloc_bounds_match_allocating_entry_point():
    import torch
    eng = cz.Engine(0)
    L = cz.lib()
    dev = torch.device("cuda", 0)
    for call, (stem, n, count) in enumerate([("toffoli", 3, 257), ("cs", 2, 130)]):
        spec = cz.Spec(spec_text(stem))
        res = residuals(100 + call, n, count)
        want = eng.eval_bounds(spec, res)                      # the existing entry point (it allocates)
        ent = torch.tensor([v for _, M in res for row in M for x in row for v in x], dtype=torch.int64, device=dev)
        ks = torch.tensor([k for k, _ in res], dtype=torch.int32, device=dev)
        out = torch.full((count, 4), -7, dtype=torch.int32, device=dev)
        err = C.create_string_buffer(256)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = L.cz_eval_bounds_noalloc(spec._h, count, ent.data_ptr(), ks.data_ptr(), out.data_ptr(), stream, err, 256)
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize(dev)
        got = [tuple(r) for r in out.cpu().tolist()]
        assert got == want, (stem, [i for i, (a, b) in enumerate(zip(got, want)) if a != b][:5])
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
