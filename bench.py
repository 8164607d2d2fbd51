"""Benchmark of the gate-count search: the deep-proof workload, 3 qubits, default Clifford+T candidates (27).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = the three proofs of the deep-proof configuration: Toffoli at budgets 11 and 12 and CCZ at budget 8
(every one exits 1: no circuit of at most that many gates exists). Metric: prefixes/s, the sum of the per-level
"prefixes" fields of the reference's JSON statistics over the step, divided by the step time; the Toffoli budget-12
proof time is reported beside it. Inputs are the reference's own targets (tests/golden/specs, written by its spec
generator); nothing is random.

value: device-timed (CUDA events on the engine's stream), specs parsed and their tables resident on the device,
L2 flushed (256 MiB write) between steps. e2e: the same metric through the C ABI's text entry point
(cz_search_text: parse, upload, search, read-back) timed on the host. Multi-GPU: replicas (every rank runs the
whole workload on its own GPU; the search has no collective), value = all ranks' prefixes / max over ranks.

--impl reference times the reference's own CPU build (oracle/_ref/cheese-cpu, compiled from the reference sources
with its OpenMP recipe) on the host cores, on a bounded sample of the same workload per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
SPECS = ROOT / "tests" / "golden" / "specs"
REF_CPU = ROOT / "oracle" / "_ref" / "cheese-cpu"
WORKLOAD = [("toffoli", 11), ("toffoli", 12), ("ccz", 8)]
SAMPLE = [("ccz", 8), ("toffoli", 11)]   # the reference CPU arm's per-step sample when the host allows it
METRIC = "prefixes/s"
# algorithmic int32 operations (a multiply or an add counts 1) per unit of work of the level kernel, 3 qubits, as
# the kernel computes them:
#  T-bound evaluation (conjugate-pair form): 63 pairs (fa, fb) != 0 x [32 products x (4 four-term dot products:
#  16 mul + 12 add, + 4 adds of operand combinations) + 4 real 32-point transforms (4 x 80 butterflies x 2) + 32 x 2
#  OR words] + the (0, 0) pair [64 x (8 mul + 6 add) + 2 real 64-point transforms (2 x 192 x 2) + 64 x 2 OR]
#  child whose residual is computed: update (<= 2 unit-multiple terms: 4 adds per entry), sqrt2-divisibility test
#  (2 per entry), goal / support tests (4 per entry) over 64 entries
OPS_T_EVAL = 63 * (32 * 32 + 640 + 64) + (64 * 14 + 768 + 128)
OPS_CHILD = 64 * (4 + 2 + 4)
CLOCK_Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
           "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
           "clocks_event_reasons.sw_power_cap")


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def allreduce(vals, op):
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return t.tolist()


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs"""

    def __init__(self, device):
        self.device, self.rows, self.p = device, [], None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={CLOCK_Q}", "--format=csv,noheader,nounits",
                                       "-lms", "100", "-i", str(self.device)], stdout=subprocess.PIPE, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait()
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows),
                "power_w_max": max((float(r[3]) for r in self.rows if r[3].replace(".", "").isdigit()), default=None)}


def run_ref_cpu(cases, threads):
    """the reference CPU build on (spec, budget) cases: (prefixes, seconds)"""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    pre, t0 = 0, time.perf_counter()
    for stem, d in cases:
        p = subprocess.run([str(REF_CPU), str(SPECS / f"{stem}.spec"), "--depth", str(d)], capture_output=True,
                           text=True, env=env, timeout=3600)
        if p.returncode not in (0, 1):
            raise RuntimeError(f"reference CPU build failed on {stem} {d}: {p.stderr[-300:]}")
        pre += sum(json.loads(l).get("prefixes", 0) for l in p.stdout.splitlines() if '"prefixes"' in l)
    return pre, time.perf_counter() - t0


REF_GPU = ROOT / "oracle" / "_ref" / "cheese-gpu-ref"
# large-frontier instances pinned to the reference (tests/golden/heavy_cases.json): (name, spec, budget, classes on)
LARGE = [("toffoli-12-nosym", "toffoli", 12, False), ("heavy-28", "heavy-28", 12, True),
         ("heavy-17", "heavy-17", 12, True), ("heavy-6", "heavy-6", 12, True), ("heavy-24", "heavy-24", 12, True)]


def reference_gpu(eng, specs):
    """The reference's own GPU build (src/cheese.cu compiled for sm_100a with its build.sh "cuda" flags) on the same
    B200: each search of the workload as one process (its CLI; the last level line's "seconds" is its search time
    without CUDA start-up), every JSON line compared with this library's (seconds excluded); then its --table 8 path
    to the Toffoli optimum, one process per budget as the reference's run.sh does (the first builds the table and
    writes its cache file, the others load it)."""
    import shutil
    import tempfile
    if not REF_GPU.exists():
        return {"unavailable": "oracle/_ref/cheese-gpu-ref not built (make -C oracle REF=<reference tree> refgpu)"}
    out, tot_pre, tot_s = {}, 0, 0.0
    d = Path(tempfile.mkdtemp())
    try:
        (d / "build").mkdir()
        for stem, dd in WORKLOAD:
            t0 = time.perf_counter()
            p = subprocess.run([str(REF_GPU), str(SPECS / f"{stem}.spec"), "--depth", str(dd)], cwd=d,
                               capture_output=True, text=True, timeout=900)
            wall = time.perf_counter() - t0
            lines = p.stdout.splitlines()
            lv = [json.loads(l) for l in lines if '"prefixes"' in l]
            search_s = lv[-1]["seconds"] if lv else None
            mine = eng.search(specs[stem], depth=dd)
            import re
            same = [re.sub(r'"seconds": [0-9.]+', '"seconds": 0.00', l) for l in lines] == mine.lines()
            pre = sum(x["prefixes"] for x in lv)
            out[f"{stem}-{dd}"] = {"rc": p.returncode, "process_s": wall, "search_s": search_s, "prefixes": pre,
                                   "same_lines": same}
            tot_pre += pre
            tot_s += search_s or 0.0
        out["prefixes_per_s"] = tot_pre / tot_s if tot_s else None
        out["toffoli12_proof_s"] = out.get("toffoli-12", {}).get("search_s")
        # the large-frontier regime (levels of 1e7-4.4e7 prefixes, millions of survivors): long enough for the
        # reference's 10 ms "seconds" resolution; this library device-timed on the same specs
        import torch
        stream = torch.cuda.ExternalStream(eng.stream, device=f"cuda:{eng.device}")
        large, r_s, o_s, r_pre = {}, 0.0, 0.0, 0
        for name, stem, dd, sym in LARGE:
            t0 = time.perf_counter()
            p = subprocess.run([str(REF_GPU), str(SPECS / f"{stem}.spec"), "--depth", str(dd)] +
                               ([] if sym else ["--no-sym"]), cwd=d, capture_output=True, text=True, timeout=900)
            wall = time.perf_counter() - t0
            lines = p.stdout.splitlines()
            lv = [json.loads(l) for l in lines if '"prefixes"' in l]
            text = (SPECS / f"{stem}.spec").read_text()
            eng.search(text, depth=dd, sym=sym)                      # warm (buffers grown)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            mine = eng.search(text, depth=dd, sym=sym)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            import re
            same = [re.sub(r'"seconds": [0-9.]+', '"seconds": 0.00', l) for l in lines] == mine.lines()
            ref_search = max((x["seconds"] for x in lv), default=None)
            large[name] = {"rc": p.returncode, "same_lines": same, "prefixes": sum(x["prefixes"] for x in lv),
                           "reference_search_s": ref_search, "reference_process_s": wall, "ours_ms": ms}
            r_s += ref_search or 0.0
            o_s += ms / 1e3
            r_pre += large[name]["prefixes"]
        out["large_frontier"] = {"cases": large, "reference_prefixes_per_s": r_pre / r_s if r_s else None,
                                 "ours_prefixes_per_s": r_pre / o_s if o_s else None,
                                 "ours_vs_reference": (r_s / o_s) if o_s else None}
        t0 = time.perf_counter()
        budgets = {}
        for dd in range(1, 16):
            a = time.perf_counter()
            p = subprocess.run([str(REF_GPU), str(SPECS / "toffoli.spec"), "--depth", str(dd), "--table", "8"], cwd=d,
                               capture_output=True, text=True, timeout=900)
            budgets[str(dd)] = {"rc": p.returncode, "s": time.perf_counter() - a}
            if p.returncode != 1:
                break
        out["table8_toffoli_optimum"] = {"total_s": time.perf_counter() - t0, "budgets": budgets,
                                         "found_at": next((int(k) for k, v in budgets.items() if v["rc"] == 0), None)}
    finally:
        shutil.rmtree(d, ignore_errors=True)   # its distance-table cache file
    return out


def reference_sample(steps, warmup, threads):
    """bounded per-step sample of the workload for the reference CPU arm, sized so K + W steps take ~2.5 min"""
    _, t10 = run_ref_cpu([("toffoli", 10)], threads)          # calibration (~2.4 s on 8 cores)
    f = t10 / 2.4
    budget = 150.0 / max(1, steps + warmup)
    for cases, est in ([WORKLOAD, (17 + 72 + 0.1) * f], [[("ccz", 8), ("toffoli", 11)], (17 + 0.1) * f],
                       [[("ccz", 8), ("toffoli", 10)], 2.5 * f]):
        if est <= budget:
            return cases
    return [("ccz", 8), ("toffoli", 9)]


def reference_arm(args, ws, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if not REF_CPU.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cheese-cpu not built (make -C oracle)"}))
        return
    cases = reference_sample(args.steps, args.warmup, threads)
    for _ in range(args.warmup):
        run_ref_cpu(cases, threads)
    pre = secs = 0.0
    for _ in range(args.steps):
        p, s = run_ref_cpu(cases, threads)
        pre += p
        secs += s
    v = pre / secs
    sample = " + ".join(f"{a}-{b}" for a, b in cases)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "prefixes/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "reference targets",
        "config": {"workload": "deep proofs, 3 qubits, 27 Clifford+T candidates", "sample": sample,
                   "threads": threads},
        "cpu_baseline": {"value": v, "unit": "prefixes/s", "cores": threads, "kind": "reference",
                         "sample": f"{sample} per step, reference CPU build (OpenMP, Thrust OMP backend)"},
        "e2e": {"value": v, "unit": "prefixes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def reference_gpu_tcount(eng):
    """the reference's own sm_100a builds of tcount and cliffopt (oracle/_ref, compiled from its sources) on this
    GPU, one process per query as its scripts run them, beside this library on the same inputs: the 3-qubit K = 4
    coset table build, eight seeded T-count queries (table loaded from the cache file by each process), and six
    zero-T Clifford-segment jobs (each reference process builds the 92,897,280-element table first)"""
    import subprocess
    import tempfile
    tc, co = ROOT / "oracle" / "_ref" / "tcount-ref", ROOT / "oracle" / "_ref" / "cliffopt-ref"
    if not tc.exists() or not co.exists():
        return {"unavailable": "oracle/_ref/tcount-ref or cliffopt-ref not built (make -C oracle)"}
    gold = ROOT / "tests" / "golden"
    tmp = Path(tempfile.mkdtemp())
    (tmp / "build").mkdir()
    qs = [gold / "tcount" / f"q3-{i}.tspec" for i in range(8)]
    out = {}
    try:
        t0 = time.perf_counter()
        p = subprocess.run([str(tc), str(qs[0]), "--table", "4"], cwd=tmp, capture_output=True, text=True, timeout=900)
        out["tcount_table_and_first_query_s"] = time.perf_counter() - t0
        ok = p.returncode == 0
        t0 = time.perf_counter()
        for q in qs:
            p = subprocess.run([str(tc), str(q), "--table", "4"], cwd=tmp, capture_output=True, text=True, timeout=900)
            ok = ok and p.returncode == 0
        out["tcount_per_query_s"] = (time.perf_counter() - t0) / len(qs)
        out["tcount_ok"] = ok
        t0 = time.perf_counter()
        for q in qs:
            eng.tcount(q.read_text(), table_k=4, cache_dir=None)
        out["ours_tcount_per_query_s"] = (time.perf_counter() - t0) / len(qs)
        jobs = [gold / "cliffopt" / f"c3-{i}.job" for i in range(6)]
        t0 = time.perf_counter()
        for j in jobs:
            p = subprocess.run([str(co), str(j)], cwd=tmp, capture_output=True, text=True, timeout=900)
            ok = ok and p.returncode == 0
        out["cliffopt_per_job_s"] = (time.perf_counter() - t0) / len(jobs)
        t0 = time.perf_counter()
        for j in jobs:
            eng.cliffopt(j.read_text())
        out["ours_cliffopt_per_job_s"] = (time.perf_counter() - t0) / len(jobs)
        out["ok"] = ok
    except subprocess.TimeoutExpired as e:
        out["unavailable"] = f"timed out: {e.cmd[0]}"
    return out


def rus_spec(target):
    """a committed rus-spec fixture (written by the reference's rus.py): shared blocks joined with the target's roots"""
    import gzip
    gold = ROOT / "tests" / "golden" / "rus"
    with gzip.open(gold / "common.rspec.gz", "rt") as f:
        root_blk, rest = f.read().split("\n@@\n")
    return "rus-spec 1\n" + root_blk + (gold / f"{target}.roots").read_text() + rest + "end\n"


def rus_leg(eng):
    """RUS T-count with measurement (the reference's build/rus) on its 0229 regression target: the K = 8 table
    (5.7M cosets) built in the library, then queries with it resident; beside it the reference's own sm_100a build,
    one process per query as rus.sh runs it (cold: builds and writes its table; cached: loads it)"""
    import tempfile
    try:
        rspec = rus_spec("ricotta-rus-0229")
        t0 = time.perf_counter()
        rc, _, r = eng.rus(rspec, table_k=8, maxt=11, cache_dir=None)
        first = time.perf_counter() - t0
        q = []
        for _ in range(5):
            t0 = time.perf_counter()
            rc, _, r2 = eng.rus(rspec, table_k=8, maxt=11, cache_dir=None)
            q.append(time.perf_counter() - t0)
        out = {"workload": "ricotta-rus-0229 (the reference's RUS regression target), --table 8 --max 11",
               "rc": rc, "tcount": r2["tcount"], "split": [r2["split_j"], r2["split_c"]],
               "table_cosets": r["table_cosets"], "table_build_s": r["table_seconds"], "first_call_s": first,
               "query_ms_median": 1e3 * statistics.median(q)}
        ref = ROOT / "oracle" / "_ref" / "rus-ref"
        if ref.exists():
            import shutil
            d = Path(tempfile.mkdtemp())
            try:
                (d / "build").mkdir()
                (d / "t.rspec").write_text(rspec)
                for rep in ("cold", "cached"):
                    t0 = time.perf_counter()
                    p = subprocess.run([str(ref), "t.rspec", "--table", "8", "--max", "11"], cwd=d,
                                       capture_output=True, text=True, timeout=600)
                    last = json.loads(p.stdout.splitlines()[-1]) if p.stdout.strip() else {}
                    out[f"reference_gpu_{rep}"] = {"rc": p.returncode, "process_s": time.perf_counter() - t0,
                                                   "seconds": last.get("seconds"), "tcount": last.get("tcount"),
                                                   "split": last.get("split")}
            finally:
                shutil.rmtree(d, ignore_errors=True)      # its K = 8 table file (about 140 MB), on every path
        eng.trim()
        return out
    except Exception as e:                     # a failed side leg must not lose the headline line
        return {"error": str(e)[:300]}


def sort_leg(eng, n, device):
    """the dedupe's radix sort at scale: n (u64 key, u32 value) pairs resident in HBM, sorted stably by the keys'
    top 32 bits (cz_sort_pairs, four 8-bit passes), device time on the engine's stream; inputs (12n bytes) are larger
    than L2 for n = 1e8, and each timed sort starts from a fresh copy of the unsorted pairs"""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(7)
    keys = torch.randint(-(1 << 62), 1 << 62, (n,), dtype=torch.int64, device=device, generator=g)
    vals = torch.arange(n, dtype=torch.int32, device=device)
    k, v = torch.empty_like(keys), torch.empty_like(vals)
    times = []
    for rep in range(4):                      # one warm-up sort, three timed
        k.copy_(keys)
        v.copy_(vals)
        torch.cuda.synchronize()              # the sort runs on the engine's stream
        ms = eng.sort_pairs(k.data_ptr(), v.data_ptr(), n, 32, 64)
        if rep:
            times.append(ms)
    top = (k >> 32) & 0xFFFFFFFF
    ok = bool((top[1:] >= top[:-1]).all()) and bool((keys[v.long()] == k).all())
    same = top[1:] == top[:-1]                # stability: equal digits keep their input order
    ok = ok and bool((v[1:][same] > v[:-1][same]).all())
    ms = min(times)
    alg = 8 * n + 4 * 24 * n                  # digit counts read once, then 12-byte pairs read and written per pass
    peak = None
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peak = json.loads(pk.read_text()).get("hbm_gbs")
    del keys, vals, k, v
    return {"workload": f"{n} (u64, u32) pairs, top 32 key bits, random keys", "ms": ms, "ms_all": times,
            "algorithmic_bytes": alg, "achieved_gbs": alg / (ms * 1e-3) / 1e9,
            "hbm_peak_gbs": peak, "frac": (alg / (ms * 1e-3) / 1e9 / peak) if peak else None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (copy bandwidth)", "sorted_stable_permutation": ok}


def systems(eng, args):
    """the batched, served and table-driven workloads beside the headline metric (one GPU)"""
    import statistics
    import torch
    import cheese_b200 as cz
    from cheese_b200 import tcwork, workloads
    out = {}
    out["sort"] = sort_leg(eng, 10 ** 8, f"cuda:{eng.device}")
    # batched search: 512 seeded targets, plain job by job vs one batch session per qubit count. Both arms run once
    # untimed first, so both are timed warm: the engine's buffers and the sessions' device memory already grown (the
    # sessions live across both passes, as a server's do).
    jobs = workloads.batch(1, 512)
    specs = [cz.Spec(workloads.make_spec(n, c, d)) for n, c, d in jobs]
    # the autotuner: per qubit count, probe jobs from another seed of the same generator
    probe = [(n, cz.Spec(workloads.make_spec(n, c, d))) for n, c, d in workloads.batch(2, 96)]
    t0 = time.perf_counter()
    tuning = {n: cz.autotune(eng, n, [s for m, s in probe if m == n][:48]) for n in (2, 3)}
    t_tune = time.perf_counter() - t0
    sess = {n: cz.Batch(eng, n) for n in (2, 3)}
    for n, b in sess.items():
        b.set_tuning(tuning[n])
    tps, tbs = [], []
    for rep in range(4):                       # pass 0 warms both arms up; passes 1-3 are timed (median reported)
        t0 = time.perf_counter()
        per_job = []
        plain = []
        for s in specs:
            a = time.perf_counter()
            plain.append(eng.search(s))
            per_job.append(time.perf_counter() - a)
        tp = time.perf_counter() - t0
        l0 = sum(b.info()["kernel_launches"] for b in sess.values())
        s0 = sum(b.info()["steps"] for b in sess.values())
        w0 = sum(b.info()["waits"] for b in sess.values())
        t0 = time.perf_counter()
        ids = [sess[s.n].submit(s) for s in specs]
        for b in sess.values():
            b.run()
        tb = time.perf_counter() - t0
        if rep:
            tps.append(tp)
            tbs.append(tb)
    tp, tb = statistics.median(tps), statistics.median(tbs)
    bad = sum(1 for s, i, p in zip(specs, ids, plain)
              if (lambda r: r.rc != p.rc or r.lines() != p.lines() or r.circuit != p.circuit)(sess[s.n].result(i)))
    launches = sum(b.info()["kernel_launches"] for b in sess.values()) - l0
    steps = sum(b.info()["steps"] for b in sess.values()) - s0
    waits = sum(b.info()["waits"] for b in sess.values()) - w0
    # the light jobs alone (plain time under 5 ms each): the part of the mix that is launch and sync bound
    light = [s for s, t in zip(specs, per_job) if t < 5e-3]
    heavy_plain = sum(t for t in per_job if t >= 5e-3)
    t0 = time.perf_counter()
    for s in light:
        eng.search(s)
    tpl = time.perf_counter() - t0
    t0 = time.perf_counter()
    for s in light:
        sess[s.n].submit(s)
    for b in sess.values():
        b.run()
    tbl = time.perf_counter() - t0
    for b in sess.values():
        b.close()
    out["batched"] = {"workload": "512 seeded targets: random circuits of L in [6,12] gates over 2-3 qubits "
                                  "(T/Tdg with prob 0.3), budget L", "plain_jobs_s": 512 / tp, "batched_jobs_s": 512 / tb,
                      "speedup": tp / tb, "mismatches": bad,
                      "timing": "warm: median of passes 2-4 of both arms (pass 1 untimed)",
                      "plain_s_passes": tps, "batched_s_passes": tbs,
                      "launches": launches, "steps": steps, "memory_waits": waits,
                      "heavy_plain_s": heavy_plain,
                      "light_subset": {"jobs": len(light), "rule": "plain time under 5 ms",
                                       "plain_jobs_s": len(light) / tpl if tpl else None,
                                       "batched_jobs_s": len(light) / tbl if tbl else None,
                                       "speedup": tpl / tbl if tbl else None},
                      "autotune": {"probe": "48 jobs per qubit count from seed 2 of the same generator",
                                   "search_space": {"chunk_gib": [8, 1, 2, 4], "expand_blocks_per_sm": [16, 4, 8, 32],
                                                    "tbound_blocks_per_sm": [4, 1, 2, 8]},
                                   "seconds": t_tune,
                                   "chosen": {str(n): {"chunk_gib": t.chunk_bytes / 2 ** 30,
                                                       "expand_blocks_per_sm": t.expand_blocks_per_sm,
                                                       "tbound_blocks_per_sm": t.tbound_blocks_per_sm,
                                                       "probe_s": t.best_seconds,
                                                       "trial_s": list(t.trial_seconds[:t.trials])}
                                              for n, t in tuning.items()}}}
    del sess, plain
    # table-driven T count: Clifford BFS table + K = 4 coset table (3 qubits), then seeded queries, each verified
    t0 = time.perf_counter()
    ct = eng.clifford_table(3)
    t_cl = time.perf_counter() - t0
    qs = tcwork.table_queries(eng, 4, 1024)
    nq = len(qs)
    specs_t = [tcwork.tspec_of_circuit(3, c) for c, _ in qs[:nq]]
    t0 = time.perf_counter()
    rc, lv, r0 = eng.tcount(specs_t[0], table_k=4, cache_dir=None)
    t_tab = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = [eng.tcount(t, table_k=4, cache_dir=None) for t in specs_t]
    t_q = time.perf_counter() - t0
    ver = sum(1 for (c, k), (rc, _, r) in zip(qs[:nq], res)
              if rc == 0 and r["tcount"] <= k and tcwork.verify_decomposition(3, tcwork.unitary_np(3, c), r["rotations"]))
    out["table_tcount"] = {"workload": f"{nq} of 1024 seeded queries C0 T C1 .. T Ck, k in [1,7], Ci uniform 3-qubit "
                                       "Cliffords (uniform index into the BFS table, its optimal word)",
                           "clifford_table_s": ct["seconds"] if ct["built"] else t_cl,
                           "clifford_elements": ct["elements"], "coset_table_s": r0["table_seconds"],
                           "coset_table_cosets": r0["table_cosets"], "queries": nq, "queries_s": nq / t_q,
                           "ms_per_query": 1e3 * t_q / nq, "verified": ver}
    out["table_tcount"]["reference_gpu"] = reference_gpu_tcount(eng)
    # distance table (--table 8, 17.9M classes): the optimum of Toffoli (15 gates, budgets 1..14 proved) and the
    # Fredkin proofs of budgets 15 and 16, through the library (table built once, resident) and as the reference's
    # run.sh does it (one drop-in process per budget, the table cached on disk by the first)
    import tempfile
    from cheese_b200 import verify
    eng.trim()                                # the batched and headline buffers go back to the device
    eng_t = cz.Engine()
    tsp = {nm: (SPECS / f"{nm}.spec").read_text() for nm in ("toffoli", "fredkin")}
    t0 = time.perf_counter()
    r = eng_t.search(tsp["toffoli"], depth=1, table_k=8, cache_dir=None)
    t_build = time.perf_counter() - t0
    classes = r.table["table_classes"]
    budgets = {}
    t0 = time.perf_counter()
    for d in range(1, 16):
        a = time.perf_counter()
        r = eng_t.search(tsp["toffoli"], depth=d, table_k=8, cache_dir=None)
        budgets[d] = (r.rc, time.perf_counter() - a)
        if r.rc == 0:
            break
    t_loop = time.perf_counter() - t0
    opt_ok = r.rc == 0 and len(r.circuit) == 15 and verify.equivalent(tsp["toffoli"], r.circuit)
    fred = {}
    for d in (15, 16, 17):
        free_gb = torch.cuda.mem_get_info()[0] / 1e9
        a = time.perf_counter()
        rf = eng_t.search(tsp["fredkin"], depth=d, table_k=8, cache_dir=None)
        fred[str(d)] = {"rc": rf.rc, "s": time.perf_counter() - a, "error": rf.error, "free_gb_before": free_gb}
        if rf.rc == 0:
            fred[str(d)]["verified"] = bool(verify.equivalent(tsp["fredkin"], rf.circuit))
            fred[str(d)]["gates"] = len(rf.circuit)
        eng_t.trim()
    del eng_t
    tmp = Path(tempfile.mkdtemp())
    (tmp / "build").mkdir()
    t0 = time.perf_counter()
    cli = {}
    for d in range(1, 16):
        a = time.perf_counter()
        p = subprocess.run([str(cz.BIN_DIR / "cheese"), str(SPECS / "toffoli.spec"), "--depth", str(d), "--table", "8"],
                           cwd=tmp, capture_output=True, text=True, timeout=600)
        cli[str(d)] = {"rc": p.returncode, "s": time.perf_counter() - a}
        if p.returncode != 1:
            break
    t_cli = time.perf_counter() - t0
    out["table_gatecount"] = {
        "workload": "--table 8, 3 qubits, 27 Clifford+T candidates: Toffoli budgets 1..15 (optimum 15), Fredkin "
                    "budgets 15 and 16 (proofs) and 17 (optimum 17)",
        "table_classes": classes, "table_build_s": t_build,
        "toffoli_optimum_s": t_loop, "toffoli_budget14_s": budgets.get(14, (None, None))[1],
        "toffoli_budget15_s": budgets.get(15, (None, None))[1], "toffoli_optimum_verified": bool(opt_ok),
        "fredkin": fred,
        "toffoli_optimum_cli_s": t_cli, "cli_budgets": cli,
        "reference_published": "RTX 3060 Ti: K=8 table 17.9M classes in 30 s; Toffoli optimum 27 s (budget 14 1.5 s, "
                               "15 11.1 s); Fredkin budget 15 11.3 s, 16 91 s, 17 out of memory at level 8 "
                               "(docs/PLAN.md:87-95)"}
    # state targets (RUS without measurement): the reference's GPU binary refuses them, its CPU build searches them;
    # both on the same three specs (budgets where the optimum is found or proved), the CPU build on all host cores
    st = {}
    cases = [("rus1-states", 11), ("rus3-states", 11), ("rus8-states", 9)]
    t0 = time.perf_counter()
    for stem, d in cases:
        r = eng.search((SPECS / f"{stem}.spec").read_text(), depth=d)
        st[f"{stem}-{d}"] = r.rc
    st["ours_s"] = time.perf_counter() - t0
    if REF_CPU.exists():
        env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
        t0 = time.perf_counter()
        for stem, d in cases:
            subprocess.run([str(REF_CPU), str(SPECS / f"{stem}.spec"), "--depth", str(d)], capture_output=True,
                           env=env, timeout=900)
        st["reference_cpu_s"] = time.perf_counter() - t0
        st["reference_cpu_threads"] = os.cpu_count()
    out["state_targets"] = {"workload": "RUS 1 budget 11, RUS 3 budget 11, RUS 8 budget 9 (ancillas in |0>)", **st}
    out["rus"] = rus_leg(eng)
    # serving: seeded Poisson streams of the mixed workload, against the same requests run one by one
    N = args.serve_requests
    reqs = tcwork.serve_requests(eng, 5, N)

    def sequential():
        for kind, text, depth, _ in reqs:
            if kind == 0:
                eng.search(text, depth=depth)
            elif kind == 1:
                eng.tcount(text, table_k=4, cache_dir=None)
            else:
                eng.cliffopt(text)
    sequential()                               # warm, as the server's engines are: buffers grown, tables resident
    t0 = time.perf_counter()
    sequential()
    t_seq = time.perf_counter() - t0
    # the same requests through the drop-in binaries, one process per request (how the reference's scripts run
    # them), on a subset: the T-count table cache is written once beforehand and loaded by every process
    tmp = Path(tempfile.mkdtemp())
    (tmp / "build").mkdir()
    exes = [cz.BIN_DIR / "cheese", cz.BIN_DIR / "tcount", cz.BIN_DIR / "cliffopt"]
    sfx = ["spec", "tspec", "job"]
    first_t = next(r for r in reqs if r[0] == 1)
    (tmp / "w.tspec").write_text(first_t[1])
    subprocess.run([str(exes[1]), str(tmp / "w.tspec")], cwd=tmp, capture_output=True, timeout=600)
    sub = reqs[:24]
    t0 = time.perf_counter()
    for i, (kind, text, depth, _) in enumerate(sub):
        f = tmp / f"r{i}.{sfx[kind]}"
        f.write_text(text)
        subprocess.run([str(exes[kind]), str(f)], cwd=tmp, capture_output=True, timeout=600)
    t_cli = time.perf_counter() - t0
    eng.trim()                                     # the server runs its own engines: give them this one's buffers
    srv = cz.Server(memory_gb=180.0)               # the admission limit of the serving configuration
    for k, t, d, _ in [next(r for r in reqs if r[0] == kind) for kind in (0, 1, 2)]:   # one request of each kind
        srv.submit(k, t, d)                        # first: its engines, tables and batch session set up
    srv.wait(3, 900)
    rates = {}
    for rate in (10, 30, 100, 300, 1000):
        arr = tcwork.poisson_arrivals(rate, N, rate)
        t0 = time.perf_counter()
        rid = srv.replay([(k, t, d) for k, t, d, _ in reqs], arr)
        wall = time.perf_counter() - t0
        lat = sorted(srv.poll(i)["latency_s"] for i in rid)
        rates[str(rate)] = {"jobs_s": N / wall, "p50_ms": 1e3 * lat[len(lat) // 2],
                            "p99_ms": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))]}
    st = srv.stats()
    srv.close()
    out["served"] = {"workload": f"{N} requests per rate: 60% gate-count searches (2-3 qubits, budgets 4..11), 30% "
                                 "T-count queries, 10% Clifford-segment minimisations; seeded Poisson arrivals",
                     "sequential_jobs_s": N / t_seq, "sequential_cli_jobs_s": len(sub) / t_cli,
                     "sequential_cli_sample": f"first {len(sub)} requests, one drop-in process each", "rates": rates,
                     "peak_jobs_s_vs_sequential": max(v["jobs_s"] for v in rates.values()) / (N / t_seq),
                     "peak_jobs_s_vs_sequential_cli": max(v["jobs_s"] for v in rates.values()) / (len(sub) / t_cli),
                     "batch_peak_running": st["batch_peak_running"], "batch_steps": st["batch_steps"]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-systems", action="store_true", help="skip the batched / served / table-driven lines")
    ap.add_argument("--serve-requests", type=int, default=120)
    ap.add_argument("--sort-pairs", type=int, default=0, help="only time the dedupe sort on this many pairs")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    ws, rank, local = dist_init() if args.impl == "ours" else (int(os.environ.get("WORLD_SIZE", "1")),
                                                                 int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        return reference_arm(args, ws, rank)

    import torch
    import cheese_b200 as cz
    torch.cuda.set_device(local)
    eng = cz.Engine(local)
    if args.sort_pairs:
        print(json.dumps(sort_leg(eng, args.sort_pairs, f"cuda:{local}")))
        return
    stream = torch.cuda.ExternalStream(eng.stream, device=f"cuda:{local}")
    texts = {stem: (SPECS / f"{stem}.spec").read_text() for stem, _ in WORKLOAD}
    specs = {stem: cz.Spec(t) for stem, t in texts.items()}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def step(timed):
        """the three proofs; returns (prefixes, device ms, toffoli-12 ms, per-search results)"""
        outs, t12 = [], 0.0
        tot = 0.0
        for stem, d in WORKLOAD:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            o = eng.search(specs[stem], depth=d, profile=True)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            if o.rc != 1:
                raise RuntimeError(f"{stem} {d}: exit {o.rc} ({o.error}), expected a proof")
            tot += ms
            if (stem, d) == ("toffoli", 12):
                t12 = ms
            outs.append(o)
        return sum(o.raw.prefixes for o in outs), tot, t12, outs

    for _ in range(args.warmup):
        step(False)
    peak_int = eng.int32_peak()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    prefixes = 0
    dev_ms = t12_ms = 0.0
    exp_ms = ops = 0.0
    launches = exp_launches = parents = 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)                     # L2 (126 MB) flushed between steps
            torch.cuda.synchronize()
            p, ms, t12, outs = step(True)
            prefixes += p
            dev_ms += ms
            t12_ms += t12
            for o in outs:
                parents += sum(l["parents"] for l in o.levels)
                r = o.raw
                exp_ms += r.expand_ms
                exp_launches += r.expand_launches
                launches += r.kernel_launches
                ops += r.t_evals * OPS_T_EVAL + r.children_full * OPS_CHILD
    torch.cuda.synchronize()
    # end to end through the C ABI's text entry point: parse + upload + search + read-back, host-timed
    h2d = d2h = 0
    e2e_pre = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for stem, d in WORKLOAD:
            o = eng.search(texts[stem], depth=d)
            e2e_pre += o.raw.prefixes
            h2d += o.raw.h2d_bytes + len(texts[stem])
            d2h += o.raw.d2h_bytes
    e2e_s = time.perf_counter() - t0
    step_ms = dev_ms / args.steps
    if ws > 1:
        step_ms, e2e_s = allreduce([step_ms, e2e_s], "max")
        prefixes, e2e_pre = allreduce([float(prefixes), float(e2e_pre)], "sum")
    value = prefixes / args.steps / (step_ms / 1e3)
    launch_ms = exp_ms / max(1, exp_launches)
    achieved = (ops / max(1, exp_launches)) / (launch_ms * 1e-3) if launch_ms > 0 else 0.0
    traffic = None
    tf = ROOT / "profiles" / "level-kernels-toffoli11-level6.md"
    if tf.exists():   # ncu DRAM bytes per parent of a captured launch, scaled to this run's average launch
        import re
        m = re.search(r"bytes per parent \(for bench.py scaling\): (\d+)", tf.read_text())
        if m and exp_launches:
            traffic = int(m.group(1)) * parents / exp_launches
    # this library's rate on the reference arm's per-step sample (ccz 8 + toffoli 11), device-timed like value, so
    # the two arms can be compared on the same work
    s_pre, s_ms = 0, 0.0
    for _ in range(3):
        for stem, d in SAMPLE:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            flush.fill_(1)
            e0.record(stream)
            o = eng.search(specs[stem], depth=d)
            e1.record(stream)
            e1.synchronize()
            s_pre += o.raw.prefixes
            s_ms += e0.elapsed_time(e1)
    cpu = None
    ref_gpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and REF_CPU.exists():
        threads = os.cpu_count() or 1
        cp, cs = run_ref_cpu(SAMPLE, threads)
        tp, ts = run_ref_cpu([("toffoli", 12)], threads)
        cpu = {"value": cp / cs, "unit": "prefixes/s", "cores": threads, "kind": "reference",
               "sample": "ccz-8 + toffoli-11 once, reference CPU build (OpenMP), %.1f s" % cs,
               "toffoli12_proof_s": ts, "toffoli12_prefixes_per_s": tp / ts}
    if rank == 0 and ws == 1 and not args.no_systems:
        try:
            ref_gpu = reference_gpu(eng, specs)
        except Exception as e:               # a failed side leg must not lose the headline line
            ref_gpu = {"error": str(e)[:300]}
    extra = systems(eng, args) if (rank == 0 and ws == 1 and not args.no_systems) else {}
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "prefixes/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "reference targets (Toffoli, CCZ specs from its generator)",
            "config": {"workload": "deep proofs, 3 qubits, 27 Clifford+T candidates: toffoli budget 11 + toffoli "
                                   "budget 12 + ccz budget 8 per step", "parallelism": f"replicas x{ws}",
                       "l2": "flushed between steps (256 MiB write)", "toffoli12_proof_ms": t12_ms / args.steps,
                       "prefixes_per_step": prefixes / args.steps / ws,
                       "sample_rate": s_pre / (s_ms / 1e3) if s_ms else None,
                       "sample": "ccz-8 + toffoli-11 (the reference arm's per-step sample), device-timed"},
            "e2e": {"value": e2e_pre / e2e_s, "unit": "prefixes/s", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps},
            "gpu_launches": launches,
            "roofline": {"bound": "int32", "kernel": "k_expand + k_tbound (one level)", "achieved": achieved / 1e12, "peak": peak_int / 1e12,
                         "unit": "Tops/s", "frac": achieved / peak_int if peak_int else None, "traffic": traffic,
                         "peak_source": "measured in this run: IMAD loop (multiply-add = 2 ops)",
                         "launch_ms": launch_ms, "ops_per_launch": ops / max(1, exp_launches)},
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "clocks": clk.summary(),
        }
        out.update(extra)
        print(json.dumps(out))
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    eng.close()


if __name__ == "__main__":
    main()
