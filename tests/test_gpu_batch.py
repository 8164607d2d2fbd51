"""Batched searches on the GPU: every job of a batch session gives the same level lines, exit code and circuit as
the plain search on its own, whether it runs alone, in a mix of uneven jobs, or joins while others are running."""
import random

import pytest

from conftest import golden_cases, spec_text

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from cheese_b200 import Engine
    return Engine()


def _jobs(seed, count):
    from cheese_b200 import workloads
    return [(n, workloads.make_spec(n, circ, d)) for n, circ, d in workloads.batch(seed, count)]


def _plain(eng, spec):
    return eng.search(spec)


def _same(a, b):
    assert a.rc == b.rc
    assert a.lines() == b.lines()
    assert a.circuit == b.circuit


def test_mixed_batch_matches_plain(eng):
    """64 seeded uneven jobs (2 and 3 qubits, budgets 6..12) in two sessions, every result equal to the plain path"""
    from cheese_b200 import Batch, verify
    jobs = _jobs(11, 64)
    plain = [_plain(eng, s) for _, s in jobs]
    sessions = {n: Batch(eng, n) for n in (2, 3)}
    ids = [sessions[n].submit(s) for n, s in jobs]
    for b in sessions.values():
        b.run()
    for (n, s), jid, p in zip(jobs, ids, plain):
        r = sessions[n].result(jid)
        _same(r, p)
        if r.rc == 0 and r.circuit:
            assert verify.equivalent(s, r.circuit)


def test_memory_bound_session_matches_plain(eng):
    """a budget too small for every job at once makes jobs wait steps (nodes carried over); results unchanged"""
    from cheese_b200 import Batch
    jobs = [(n, s) for n, s in _jobs(15, 48) if n == 3]
    b = Batch(eng, 3, memory_gb=0.05)
    ids = [b.submit(s) for _, s in jobs]
    b.run()
    assert b.info()["waits"] > 0
    for (n, s), jid in zip(jobs, ids):
        _same(b.result(jid), _plain(eng, s))


def test_alone_equals_in_mix(eng):
    from cheese_b200 import Batch
    jobs = _jobs(12, 24)
    n3 = [s for n, s in jobs if n == 3]
    mix = Batch(eng, 3)
    ids = [mix.submit(s) for s in n3]
    mix.run()
    for s, jid in zip(n3, ids):
        alone = Batch(eng, 3)
        a = alone.submit(s)
        alone.run()
        _same(alone.result(a), mix.result(jid))


def test_late_joiners(eng):
    """jobs submitted after the session has stepped (continuous batching) still match the plain path"""
    from cheese_b200 import Batch
    jobs = [(n, s) for n, s in _jobs(13, 40) if n == 3]
    b = Batch(eng, 3)
    ids = {}
    rng = random.Random(5)
    pending = list(enumerate(jobs))
    while True:
        for _ in range(rng.randint(0, 3)):
            if pending:
                i, (n, s) = pending.pop(0)
                ids[i] = b.submit(s)
        running = b.step()
        if not pending and running == 0:
            break
    for i, (n, s) in enumerate(jobs):
        _same(b.result(ids[i]), _plain(eng, s))


def test_golden_cases_in_one_batch(eng):
    """the reference golden cases with default flags (3 qubits), all in one session"""
    from cheese_b200 import Batch, Spec
    cases = [c for c in golden_cases()
             if (not c["flags"] or c["flags"] == ["--depth", c["flags"][-1]]) and c["rc"] in (0, 1)
             and c["name"] not in ("toffoli-12",)]
    b = Batch(eng, 3)
    ids = []
    for c in cases:
        sp = Spec(spec_text(c["spec"]))
        if sp.n != 3:
            continue
        depth = int(c["flags"][1]) if c["flags"] else -1
        ids.append((c, b.submit(sp, depth=depth)))
    b.run()
    assert ids
    for c, jid in ids:
        r = b.result(jid)
        assert r.rc == c["rc"], c["name"]
        assert r.lines() == c["stdout"], c["name"]


def test_session_info(eng):
    from cheese_b200 import Batch
    b = Batch(eng, 2)
    for _, s in [j for j in _jobs(14, 16) if j[0] == 2]:
        b.submit(s)
    b.run()
    info = b.info()
    assert info["running"] == 0 and info["steps"] >= 1 and info["kernel_launches"] > 0


def test_tuning_changes_time_not_results(eng):
    """the autotuner returns a tuning from its search space, and sessions run under extreme tunings (small chunks,
    few or many blocks) give the plain path's results"""
    import cheese_b200 as cz
    jobs = [(n, s) for n, s in _jobs(23, 40) if n == 3]
    t = cz.autotune(eng, 3, [s for _, s in jobs[:8]])
    assert t.chunk_bytes in (8 << 30, 1 << 30, 2 << 30, 4 << 30)
    assert t.expand_blocks_per_sm in (16, 4, 8, 32) and t.tbound_blocks_per_sm in (4, 1, 2, 8)
    assert t.trials == 10 and t.best_seconds > 0
    plain = [_plain(eng, s) for _, s in jobs]
    for chunk, eb, tb in ((1 << 20, 1, 1), (1 << 30, 32, 8)):
        b = cz.Batch(eng, 3)
        b.set_tuning(cz.BatchTuning(chunk, eb, tb, 0, (0.0,) * 16, 0.0))
        ids = [b.submit(s) for _, s in jobs]
        b.run()
        for i, p in zip(ids, plain):
            _same(b.result(i), p)
        b.close()
