"""cheese_b200: B200-native rebuild of cheese's level-synchronous branch-and-bound search.

The product is the sm_100a library behind include/cheese_b200.h (cheese_b200/lib/libcheese_b200.so) and the
drop-in binary cheese_b200/bin/cheese. This module is a thin ctypes host over that C ABI, with the same
interface as the reference's process boundary (src/cheese.cu:1851-1895): a spec text in, the per-level JSON
statistics, the found circuit and the exit code out. There is no CPU fallback: without the compiled library
every call raises.
"""
import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libcheese_b200.so"
BIN_DIR = PKG / "bin"
MAX_DEPTH = 48

CIRCUIT, PROOF, ERR_SPEC, ERR_USAGE, ERR_OVERFLOW, ERR_CUDA = 0, 1, 2, 3, 4, 5


class LevelStats(C.Structure):
    _fields_ = [("t", C.c_int), ("parents", C.c_int64), ("prefixes", C.c_int64), ("cut_w3", C.c_int64),
                ("cut_lb", C.c_int64), ("survivors", C.c_int64), ("distinct", C.c_int64),
                ("proved_unsat", C.c_int), ("seconds", C.c_double), ("dir", C.c_int)]


class Options(C.Structure):
    _fields_ = [("depth", C.c_int), ("dedupe", C.c_int), ("sym", C.c_int), ("store64", C.c_int),
                ("profile", C.c_int), ("table_k", C.c_int), ("cache_dir", C.c_char_p), ("mitm", C.c_int)]


class Result(C.Structure):
    _fields_ = [("rc", C.c_int), ("depth0", C.c_int), ("found_len", C.c_int), ("found", C.c_int * MAX_DEPTH),
                ("n_found", C.c_int64), ("nsym", C.c_int), ("store64", C.c_int), ("levels", C.c_int),
                ("prefixes", C.c_int64), ("kernel_launches", C.c_int64), ("t_evals", C.c_int64),
                ("children", C.c_int64), ("expand_ms", C.c_double), ("dedupe_ms", C.c_double),
                ("total_ms", C.c_double), ("expand_launches", C.c_int64), ("h2d_bytes", C.c_int64),
                ("d2h_bytes", C.c_int64), ("children_full", C.c_int64), ("table_k", C.c_int),
                ("table_split", C.c_int * 2), ("table_proof", C.c_int), ("table_classes", C.c_int64),
                ("table_levels", C.c_int), ("table_loaded", C.c_int), ("table_built", C.c_int),
                ("table_seconds", C.c_double), ("table_path", C.c_char * 256), ("mitm_join", C.c_int),
                ("mitm_forward", C.c_int64), ("mitm_backward", C.c_int64), ("mitm_hash_matches", C.c_int64),
                ("mitm_seconds", C.c_double), ("mitm_split", C.c_int * 2), ("mitm_found", C.c_int),
                ("mitm_proof", C.c_int), ("error", C.c_char * 256)]


LEVEL_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(LevelStats))


class SpecGenInfo(C.Structure):
    _fields_ = [("n", C.c_int), ("gates", C.c_int), ("candidates", C.c_int), ("w2_pairs", C.c_int),
                ("w3_triples", C.c_int)]


class TcOptions(C.Structure):
    _fields_ = [("table_k", C.c_int), ("maxt", C.c_int), ("cache_dir", C.c_char_p)]


class TcLevel(C.Structure):
    _fields_ = [("table", C.c_int), ("t", C.c_int), ("parents", C.c_int64), ("children", C.c_int64),
                ("cosets", C.c_int64), ("fresh", C.c_int64), ("seconds", C.c_double)]


class TcResult(C.Structure):
    _fields_ = [("rc", C.c_int), ("tcount", C.c_int), ("split_j", C.c_int), ("split_c", C.c_int), ("maxt", C.c_int),
                ("nrot", C.c_int), ("rot_p", C.c_int * 64), ("rot_inv", C.c_int * 64), ("table_cosets", C.c_int64),
                ("table_levels", C.c_int), ("table_loaded", C.c_int), ("table_built", C.c_int),
                ("table_resident", C.c_int), ("table_seconds", C.c_double), ("total_seconds", C.c_double),
                ("kernel_launches", C.c_int64), ("table_path", C.c_char * 256), ("error", C.c_char * 256)]


TC_LEVEL_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(TcLevel))


class RspecInfo(C.Structure):
    _fields_ = [("outcome", C.c_int), ("roots", C.c_int), ("rescalings", C.c_int), ("failure_amplitudes", C.c_int),
                ("p", C.c_int64 * 3)]


class RusResult(C.Structure):
    _fields_ = [("rc", C.c_int), ("tcount", C.c_int), ("split_j", C.c_int), ("split_c", C.c_int), ("maxt", C.c_int),
                ("root", C.c_uint32), ("cliff", C.c_int), ("fw", C.c_int * 32), ("tb", C.c_int * 32),
                ("table_cosets", C.c_int64), ("table_levels", C.c_int), ("table_loaded", C.c_int),
                ("table_built", C.c_int), ("table_resident", C.c_int), ("table_seconds", C.c_double),
                ("total_seconds", C.c_double), ("kernel_launches", C.c_int64), ("table_path", C.c_char * 256),
                ("error", C.c_char * 256)]


class CliffTableInfo(C.Structure):
    _fields_ = [("n", C.c_int), ("order", C.c_int64), ("elements", C.c_int64), ("max_distance", C.c_int),
                ("per_distance", C.c_int64 * 32), ("built", C.c_int), ("seconds", C.c_double)]


class CliffResult(C.Structure):
    _fields_ = [("rc", C.c_int), ("clifford_gates", C.c_int), ("clifford_gates_before", C.c_int),
                ("t_gates", C.c_int), ("seconds", C.c_double), ("table", CliffTableInfo),
                ("kernel_launches", C.c_int64), ("text_len", C.c_size_t), ("error", C.c_char * 256)]


CLIFF_STEP_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_int64, C.c_int)


class ServerOptions(C.Structure):
    _fields_ = [("device", C.c_int), ("memory_gb", C.c_double), ("max_jobs", C.c_int), ("tcount_table_k", C.c_int),
                ("beam", C.c_int), ("cache_dir", C.c_char_p)]


class ServerResult(C.Structure):
    _fields_ = [("rc", C.c_int), ("kind", C.c_int), ("latency_s", C.c_double), ("queued_s", C.c_double),
                ("gpu_work", C.c_int64), ("text_len", C.c_size_t), ("error", C.c_char * 256)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("batch_steps", C.c_int64),
                ("batch_admitted", C.c_int64), ("batch_deferred", C.c_int64), ("batch_peak_running", C.c_int64),
                ("batch_peak_bytes", C.c_int64), ("queued", C.c_int64 * 3)]


class BatchInfo(C.Structure):
    _fields_ = [("nq", C.c_int), ("jobs", C.c_int), ("running", C.c_int), ("frontier", C.c_int64),
                ("steps", C.c_int64), ("kernel_launches", C.c_int64), ("device_bytes", C.c_int64),
                ("waits", C.c_int64)]

class BatchTuning(C.Structure):
    _fields_ = [("chunk_bytes", C.c_int64), ("expand_blocks_per_sm", C.c_int), ("tbound_blocks_per_sm", C.c_int),
                ("trials", C.c_int), ("trial_seconds", C.c_double * 16), ("best_seconds", C.c_double)]


# every C entry point of include/cheese_b200.h with its ctypes signature
SIGNATURES = {
    "cz_spec_parse": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "cz_spec_free": (None, [C.c_void_p]),
    "cz_spec_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "cz_spec_gate_name": (C.c_char_p, [C.c_void_p, C.c_int]),
    "cz_spec_is_states": (C.c_int, [C.c_void_p]),
    "cz_engine_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "cz_engine_destroy": (None, [C.c_void_p]),
    "cz_engine_trim": (C.c_int64, [C.c_void_p]),
    "cz_options_default": (None, [C.POINTER(Options)]),
    "cz_search": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Options), LEVEL_FN, C.c_void_p, C.POINTER(Result)]),
    "cz_search_text": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(Options), LEVEL_FN, C.c_void_p,
                                 C.POINTER(Result)]),
    "cz_eval_bounds": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)]),
    "cz_eval_bounds_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_char_p, C.c_size_t]),
    "cz_engine_stream": (C.c_void_p, [C.c_void_p]),
    "cz_int32_peak": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "cz_batch_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(BatchTuning)]),
    "cz_batch_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(Options),
                                    C.POINTER(BatchTuning)]),
    "cz_sort_pairs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int,
                                C.POINTER(C.c_float)]),
    "cz_tcount_options_default": (None, [C.POINTER(TcOptions)]),
    "cz_tspec_check": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_int), C.c_char_p, C.c_size_t]),
    "cz_spec_generate": (C.c_int, [C.c_char_p, C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_char_p),
                                   C.POINTER(C.c_int), C.c_int, C.c_int, C.c_char_p, C.c_size_t,
                                   C.POINTER(C.c_size_t), C.POINTER(SpecGenInfo), C.c_char_p, C.c_size_t]),
    "cz_spec_generate_states": (C.c_int, [C.c_char_p, C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_char_p),
                                          C.POINTER(C.c_int), C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int,
                                          C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(SpecGenInfo),
                                          C.c_char_p, C.c_size_t]),
    "cz_rspec_generate": (C.c_int, [C.c_char_p, C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_char_p),
                                    C.POINTER(C.c_int), C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t),
                                    C.POINTER(RspecInfo), C.c_char_p, C.c_size_t]),
    "cz_tspec_generate": (C.c_int, [C.c_char_p, C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_char_p),
                                    C.POINTER(C.c_int), C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t), C.c_char_p,
                                    C.c_size_t]),
    "cz_tcount": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(TcOptions), TC_LEVEL_FN, C.c_void_p,
                            C.POINTER(TcResult)]),
    "cz_rus_options_default": (None, [C.POINTER(TcOptions)]),
    "cz_rspec_check": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_int), C.c_char_p, C.c_size_t]),
    "cz_rus": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(TcOptions), TC_LEVEL_FN, C.c_void_p,
                         C.POINTER(RusResult)]),
    "cz_clifford_table": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(CliffTableInfo), C.c_char_p, C.c_size_t]),
    "cz_clifford_dist": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_size_t, C.POINTER(C.c_int)]),
    "cz_clifford_element": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_size_t,
                                      C.POINTER(C.c_uint64)]),
    "cz_clifford_words": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_size_t, C.POINTER(C.c_int),
                                    C.POINTER(C.c_int)]),
    "cz_cliffjob_check": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p,
                                    C.c_size_t]),
    "cz_cliffopt": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.c_int, CLIFF_STEP_FN, C.c_void_p, C.c_char_p,
                              C.c_size_t, C.POINTER(CliffResult)]),
    "cz_batch_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "cz_batch_destroy": (None, [C.c_void_p]),
    "cz_batch_submit": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Options)]),
    "cz_batch_set_memory": (C.c_int, [C.c_void_p, C.c_double]),
    "cz_batch_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "cz_batch_info_get": (C.c_int, [C.c_void_p, C.POINTER(BatchInfo)]),
    "cz_batch_error": (C.c_char_p, [C.c_void_p]),
    "cz_batch_done": (C.c_int, [C.c_void_p, C.c_int]),
    "cz_batch_result": (C.c_int, [C.c_void_p, C.c_int, LEVEL_FN, C.c_void_p, C.POINTER(Result)]),
    "cz_server_options_default": (None, [C.POINTER(ServerOptions)]),
    "cz_server_create": (C.c_int, [C.POINTER(ServerOptions), C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "cz_server_destroy": (None, [C.c_void_p]),
    "cz_server_submit": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_size_t, C.c_int]),
    "cz_server_poll": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(ServerResult), C.c_char_p, C.c_size_t]),
    "cz_server_wait": (C.c_int, [C.c_void_p, C.c_longlong, C.c_double]),
    "cz_server_stats_get": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "cz_server_replay": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_char_p),
                                   C.POINTER(C.c_size_t), C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_double,
                                   C.POINTER(C.c_int)]),
    "cz_version": (C.c_char_p, []),
}

_lib = None


def lib():
    """the compiled library (raises when it has not been built: there is no fallback path)"""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m cheese_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


class Spec:
    """a parsed spec (the reference's text grammar)"""

    def __init__(self, text):
        if isinstance(text, str):
            text = text.encode()
        self._h = C.c_void_p()
        err = C.create_string_buffer(256)
        rc = lib().cz_spec_parse(text, len(text), C.byref(self._h), err, 256)
        if rc:
            raise SpecError(rc, err.value.decode())
        n, g, d = C.c_int(), C.c_int(), C.c_int()
        lib().cz_spec_info(self._h, C.byref(n), C.byref(g), C.byref(d))
        self.n, self.gates, self.depth = n.value, g.value, d.value
        self.names = [lib().cz_spec_gate_name(self._h, i).decode() for i in range(self.gates)]
        self.states = bool(lib().cz_spec_is_states(self._h))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.cz_spec_free(self._h)
            self._h = None


class SpecError(Exception):
    def __init__(self, rc, msg):
        super().__init__(msg)
        self.rc = rc


def _gen_args(circ, qasm):
    if qasm is not None:
        q = qasm.encode() if isinstance(qasm, str) else qasm
        return q, len(q), 0, None, None
    names = (C.c_char_p * max(1, len(circ)))(*[g.encode() for g, _ in circ])
    qs = (C.c_int * max(3, 3 * len(circ)))(*[v for _, q in circ for v in (list(q) + [-1, -1, -1])[:3]])
    return None, 0, len(circ), names, qs


def _gen_call(fn, *args):
    cap = 1 << 16
    while True:
        out = C.create_string_buffer(cap)
        need = C.c_size_t()
        err = C.create_string_buffer(256)
        rc = fn(*args, out, cap, C.byref(need), err, 256)
        if rc == 3 and need.value + 1 > cap:
            cap = need.value + 1
            continue
        if rc:
            raise SpecError(rc, err.value.decode())
        return out.value.decode()


def spec_generate(n=None, circ=None, depth=1, w3=True, qasm=None, inputs=None):
    """the gate-count spec text of a target circuit (gate list [(name, qubits)] on n qubits, or QASM text), as the
    reference's spec generator writes it; with `inputs` (basis states, bit q = qubit q) the state-target spec of
    those inputs (`--inputs`; `state_inputs(n, ancilla)` gives the `--ancilla` list). Returns (text, info dict)."""
    q, ql, ng, names, qs = _gen_args(circ, qasm)
    info = SpecGenInfo()
    inputs = list(inputs or [])
    arr = (C.c_int * max(1, len(inputs)))(*inputs)

    def fn(*a):
        *head, out, cap, need, err, errlen = a
        return lib().cz_spec_generate_states(*head, arr, len(inputs), out, cap, need, C.byref(info), err, errlen)
    text = _gen_call(fn, q, ql, n or 0, ng, names, qs, depth, 0 if w3 else 1)
    return text, {k: getattr(info, k) for k, _ in SpecGenInfo._fields_}


def state_inputs(n, ancilla):
    """the input basis states of a state target whose `ancilla` qubits start in |0> (spec.py state_inputs)"""
    mask = sum(1 << a for a in ancilla)
    return [x for x in range(1 << n) if not x & mask]


def rspec_generate(n=None, circ=None, qasm=None, outcome=-1):
    """the rus-spec of a two-qubit RUS circuit, as the reference's rus.py writes it; returns (text, info dict)"""
    q, ql, ng, names, qs = _gen_args(circ, qasm)
    info = RspecInfo()

    def fn(*a):
        *head, out, cap, need, err, errlen = a
        return lib().cz_rspec_generate(*head, out, cap, need, C.byref(info), err, errlen)
    text = _gen_call(fn, q, ql, n or 0, ng, names, qs, outcome)
    d = {k: getattr(info, k) for k, _ in RspecInfo._fields_ if k != "p"}
    d["p"] = list(info.p)
    return text, d


def tspec_generate(n=None, circ=None, qasm=None):
    """the T-count spec text of a target circuit, as the reference's tcount.py writes it"""
    q, ql, ng, names, qs = _gen_args(circ, qasm)
    return _gen_call(lib().cz_tspec_generate, q, ql, n or 0, ng, names, qs)


def tspec_check(text):
    """qubit count of a tcount-spec, parsed on the host; raises SpecError (rc 2 or 3) like the reference's reader"""
    if isinstance(text, str):
        text = text.encode()
    n = C.c_int()
    err = C.create_string_buffer(256)
    rc = lib().cz_tspec_check(text, len(text), C.byref(n), err, 256)
    if rc:
        raise SpecError(rc, err.value.decode())
    return n.value


class Engine:
    """one CUDA device and stream; searches run one at a time on it"""

    def __init__(self, device=0):
        self._h = C.c_void_p()
        self.device = device
        err = C.create_string_buffer(256)
        rc = lib().cz_engine_create(device, C.byref(self._h), err, 256)
        if rc:
            raise RuntimeError(f"engine on device {device}: {err.value.decode()}")

    def close(self):
        lib_ = _lib                           # (at interpreter exit the module's globals may already be gone)
        if self._h and lib_ is not None:
            lib_.cz_engine_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        if getattr(self, "_h", None):
            self.close()

    def trim(self):
        """release the cached device work buffers (kept at peak size between calls otherwise); resident tables stay.
        Returns the bytes released."""
        return lib().cz_engine_trim(self._h)

    @property
    def stream(self):
        """the cudaStream_t the engine launches on (an integer handle)"""
        return lib().cz_engine_stream(self._h)

    def sort_pairs(self, keys_ptr, vals_ptr, n, lo=0, hi=64):
        """the dedupe's radix sort on device buffers (u64 keys, u32 values), in place; returns device ms"""
        ms = C.c_float()
        rc = lib().cz_sort_pairs(self._h, C.c_void_p(keys_ptr), C.c_void_p(vals_ptr), n, lo, hi, C.byref(ms))
        if rc:
            raise RuntimeError(f"cz_sort_pairs failed: {rc}")
        return ms.value

    def int32_peak(self):
        v = C.c_double()
        if lib().cz_int32_peak(self._h, C.byref(v)):
            raise RuntimeError("int32 probe failed")
        return v.value

    def eval_bounds(self, spec, residuals):
        """[(k, rows)] -> [(T bound, CX bound, H structure, support)] computed on the device"""
        if not isinstance(spec, Spec):
            spec = Spec(spec)
        n = len(residuals)
        flat = [v for _, M in residuals for row in M for x in row for v in x]
        ent = (C.c_int64 * len(flat))(*flat)
        ks = (C.c_int * n)(*[k for k, _ in residuals])
        out = (C.c_int * (4 * n))()
        rc = lib().cz_eval_bounds(self._h, spec._h, n, ent, ks, out)
        if rc:
            raise RuntimeError(f"cz_eval_bounds failed: {rc}")
        return [tuple(out[4 * i:4 * i + 4]) for i in range(n)]

    def tcount(self, tspec, table_k=4, maxt=16, cache_dir="build", on_level=None):
        """`tcount TSPEC --table K --max T`: (rc, level dicts, result dict)"""
        if isinstance(tspec, str):
            tspec = tspec.encode()
        opt = TcOptions(table_k, maxt, cache_dir.encode() if cache_dir else None)
        levels = []

        def cb(_u, p):
            l = p.contents
            d = {k: getattr(l, k) for k, _ in TcLevel._fields_}
            levels.append(d)
            if on_level:
                on_level(d)

        res = TcResult()
        rc = lib().cz_tcount(self._h, tspec, len(tspec), C.byref(opt), TC_LEVEL_FN(cb), None, C.byref(res))
        out = {k: getattr(res, k) for k, _ in TcResult._fields_ if k not in ("rot_p", "rot_inv")}
        out["rotations"] = [[res.rot_p[i], res.rot_inv[i]] for i in range(res.nrot)]
        out["error"] = res.error.decode()
        out["table_path"] = res.table_path.decode()
        return rc, levels, out

    def rus(self, rspec, table_k=8, maxt=16, cache_dir="build", on_level=None):
        """`rus SPEC --table K --max T`: (rc, level dicts, result dict); `lines()` of the result are the drop-in's
        stdout lines with "seconds" 0.00"""
        if isinstance(rspec, str):
            rspec = rspec.encode()
        opt = TcOptions(table_k, maxt, cache_dir.encode() if cache_dir else None)
        levels = []

        def cb(_u, p):
            l = p.contents
            d = {k: getattr(l, k) for k, _ in TcLevel._fields_}
            levels.append(d)
            if on_level:
                on_level(d)

        res = RusResult()
        rc = lib().cz_rus(self._h, rspec, len(rspec), C.byref(opt), TC_LEVEL_FN(cb), None, C.byref(res))
        out = {k: getattr(res, k) for k, _ in RusResult._fields_ if k not in ("fw", "tb")}
        out["fw"] = [res.fw[i] for i in range(res.split_j)] if rc == 0 else []
        out["tb"] = [res.tb[i] for i in range(res.split_c)] if rc == 0 else []
        out["error"] = res.error.decode()
        out["table_path"] = res.table_path.decode()
        return rc, levels, out

    @staticmethod
    def rus_lines(rc, levels, out):
        """the drop-in's stdout lines of a `rus` call, "seconds" printed as 0.00"""
        lines = [f'{{"dir": "{"table" if l["table"] else "search"}", "t": {l["t"]}, "parents": {l["parents"]}, '
                 f'"children": {l["children"]}, "cosets": {l["cosets"]}, "new": {l["fresh"]}, "seconds": 0.00}}'
                 for l in levels]
        if rc == 0:
            lines.append(f'{{"tcount": {out["tcount"]}, "root": {out["root"]}, "fw": [{", ".join(map(str, out["fw"]))}], '
                         f'"cliff": {out["cliff"]}, "tb": [{", ".join(map(str, out["tb"]))}], '
                         f'"split": [{out["split_j"]}, {out["split_c"]}], "seconds": 0.00}}')
        elif rc == 1:
            lines.append(f'{{"tcount_above": {out["maxt"]}, "seconds": 0.00}}')
        return lines

    def clifford_table(self, n):
        """the resident BFS table of the n-qubit Clifford group: info dict (per_distance as a list)"""
        info = CliffTableInfo()
        err = C.create_string_buffer(256)
        rc = lib().cz_clifford_table(self._h, n, C.byref(info), err, 256)
        if rc:
            raise RuntimeError(f"cz_clifford_table failed ({rc}): {err.value.decode()}")
        d = {k: getattr(info, k) for k, _ in CliffTableInfo._fields_ if k != "per_distance"}
        d["per_distance"] = [info.per_distance[i] for i in range(info.max_distance + 1)]
        return d

    def clifford_dist(self, n, tableaux):
        m = len(tableaux)
        arr = (C.c_uint64 * max(m, 1))(*tableaux)
        out = (C.c_int * max(m, 1))()
        rc = lib().cz_clifford_dist(self._h, n, arr, m, out)
        if rc:
            raise RuntimeError(f"cz_clifford_dist failed: {rc}")
        return list(out[:m])

    def clifford_element(self, n, indices):
        m = len(indices)
        arr = (C.c_uint64 * max(m, 1))(*indices)
        out = (C.c_uint64 * max(m, 1))()
        rc = lib().cz_clifford_element(self._h, n, arr, m, out)
        if rc:
            raise RuntimeError(f"cz_clifford_element failed: {rc}")
        return list(out[:m])

    def clifford_words(self, n, tableaux):
        """optimal words [(gate name, qubits)] of tableaux (from the resident Clifford table)"""
        m = len(tableaux)
        arr = (C.c_uint64 * max(m, 1))(*tableaux)
        words = (C.c_int * (max(m, 1) * 32 * 3))()
        lens = (C.c_int * max(m, 1))()
        rc = lib().cz_clifford_words(self._h, n, arr, m, words, lens)
        if rc:
            raise RuntimeError(f"cz_clifford_words failed: {rc}")
        names = ["h", "s", "sdg", "x", "z", "cx", "y"]
        out = []
        for i in range(m):
            w = []
            for j in range(lens[i]):
                k, a, b = words[(i * 32 + j) * 3:(i * 32 + j) * 3 + 3]
                w.append((names[k], (a, b) if k == 5 else (a,)))
            out.append(w)
        return out

    def cliffopt(self, job, beam=16, on_step=None):
        """`cliffopt JOB --beam B`: (rc, result dict, output lines after the JSON line, step tuples)"""
        if isinstance(job, str):
            job = job.encode()
        steps = []

        def cb(_u, j, placements, best):
            steps.append((j, placements, best))
            if on_step:
                on_step(j, placements, best)

        cap = 1 << 16
        while True:
            buf = C.create_string_buffer(cap)
            res = CliffResult()
            steps.clear()
            rc = lib().cz_cliffopt(self._h, job, len(job), beam, CLIFF_STEP_FN(cb), None, buf, cap, C.byref(res))
            if rc or res.text_len < cap:
                break
            cap = res.text_len + 1
        out = {k: getattr(res, k) for k, _ in CliffResult._fields_ if k not in ("table", "error")}
        out["error"] = res.error.decode()
        out["table_built"] = res.table.built
        return rc, out, buf.value.decode().splitlines(), list(steps)

    def search(self, spec, depth=-1, dedupe=True, sym=True, store64=False, profile=False, on_level=None,
               table_k=0, cache_dir="build", mitm=False):
        """run `cheese SPEC [--depth D] [--no-dedupe] [--no-sym] [--table K] [--mitm]`; returns a SearchOutcome
        (cache_dir: where the distance table of --table K is cached, None for no cache)"""
        if not isinstance(spec, Spec):
            spec = Spec(spec)
        opt = Options(depth, int(dedupe), int(sym), int(store64), int(profile), int(table_k),
                      cache_dir.encode() if cache_dir else None, int(mitm))
        levels = []

        def cb(_user, p):
            s = p.contents
            d = {k: getattr(s, k) for k, _ in LevelStats._fields_}
            d["proved_unsat"] = bool(d["proved_unsat"])
            levels.append(d)
            if on_level:
                on_level(d)

        res = Result()
        rc = lib().cz_search(self._h, spec._h, C.byref(opt), LEVEL_FN(cb), None, C.byref(res))
        return SearchOutcome(spec, rc, levels, res)


def autotune(engine, nq, probe_specs):
    """the batch autotuner (cz_batch_autotune) on probe specs of nq qubits: a BatchTuning with the probe times"""
    specs = [s if isinstance(s, Spec) else Spec(s) for s in probe_specs]
    arr = (C.c_void_p * len(specs))(*[s._h.value for s in specs])
    out = BatchTuning()
    opt = Options(-1, 1, 1, 0, 0, 0, None, 0)
    rc = lib().cz_batch_autotune(engine._h, nq, arr, len(specs), C.byref(opt), C.byref(out))
    if rc:
        raise RuntimeError(f"cz_batch_autotune failed: {rc}")
    return out


class Batch:
    """a batch session of one qubit count on an engine: submit specs, step, collect SearchOutcomes"""

    def __init__(self, engine, nq, memory_gb=None):
        self.engine = engine
        self._h = C.c_void_p()
        rc = lib().cz_batch_create(engine._h, nq, C.byref(self._h))
        if rc:
            raise RuntimeError(f"cz_batch_create failed: {rc}")
        if memory_gb is not None:
            lib().cz_batch_set_memory(self._h, memory_gb)
        self.specs = {}

    def set_tuning(self, tuning):
        """apply a BatchTuning (e.g. from autotune)"""
        rc = lib().cz_batch_set_tuning(self._h, C.byref(tuning))
        if rc:
            raise RuntimeError(f"cz_batch_set_tuning failed: {rc}")

    def submit(self, spec, depth=-1, dedupe=True, sym=True, store64=False):
        if not isinstance(spec, Spec):
            spec = Spec(spec)
        opt = Options(depth, int(dedupe), int(sym), int(store64), 0, 0, None, 0)
        jid = lib().cz_batch_submit(self._h, spec._h, C.byref(opt))
        if jid < 0:
            raise RuntimeError(f"cz_batch_submit failed: {-jid}")
        self.specs[jid] = spec
        return jid

    def step(self):
        r = C.c_int()
        rc = lib().cz_batch_step(self._h, C.byref(r))
        if rc:
            raise RuntimeError(f"cz_batch_step failed ({rc}): {lib().cz_batch_error(self._h).decode()}")
        return r.value

    def run(self):
        while self.step():
            pass

    def info(self):
        i = BatchInfo()
        lib().cz_batch_info_get(self._h, C.byref(i))
        return {k: getattr(i, k) for k, _ in BatchInfo._fields_}

    def done(self, jid):
        return bool(lib().cz_batch_done(self._h, jid))

    def result(self, jid):
        levels = []

        def cb(_user, p):
            s = p.contents
            d = {k: getattr(s, k) for k, _ in LevelStats._fields_}
            d["proved_unsat"] = bool(d["proved_unsat"])
            levels.append(d)

        res = Result()
        rc = lib().cz_batch_result(self._h, jid, LEVEL_FN(cb), None, C.byref(res))
        if rc:
            raise RuntimeError(f"cz_batch_result failed: {rc}")
        return SearchOutcome(self.specs[jid], res.rc, levels, res)

    def close(self):
        """free the session's device buffers now"""
        if getattr(self, "_h", None) and _lib is not None:
            _lib.cz_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


REQ_GATES, REQ_TCOUNT, REQ_CLIFFORD, REQ_GATES_QASM, REQ_TCOUNT_QASM = 0, 1, 2, 3, 4


class Server:
    """the persistent request server (gate-count searches batched continuously, T-count and Clifford requests on
    their own streams); results are the reference programs' stdout for each request"""

    def __init__(self, device=0, memory_gb=150.0, max_jobs=4096, tcount_table_k=4, beam=16, cache_dir=None):
        o = ServerOptions()
        lib().cz_server_options_default(C.byref(o))
        o.device, o.memory_gb, o.max_jobs, o.tcount_table_k, o.beam = device, memory_gb, max_jobs, tcount_table_k, beam
        o.cache_dir = cache_dir.encode() if cache_dir else None
        self._opt = o
        self._h = C.c_void_p()
        err = C.create_string_buffer(256)
        rc = lib().cz_server_create(C.byref(o), C.byref(self._h), err, 256)
        if rc:
            raise RuntimeError(f"cz_server_create failed ({rc}): {err.value.decode()}")

    def submit(self, kind, text, depth=-1):
        b = text.encode() if isinstance(text, str) else text
        rid = lib().cz_server_submit(self._h, kind, b, len(b), depth)
        if rid < 0:
            raise RuntimeError(f"cz_server_submit failed: {-rid}")
        return rid

    def poll(self, rid, cap=1 << 20):
        res = ServerResult()
        buf = C.create_string_buffer(cap)
        st = lib().cz_server_poll(self._h, rid, C.byref(res), buf, cap)
        if st < 0:
            raise KeyError(rid)
        if st == 0:
            return None
        if res.text_len >= cap:
            return self.poll(rid, res.text_len + 1)
        return {"rc": res.rc, "kind": res.kind, "latency_s": res.latency_s, "queued_s": res.queued_s,
                "gpu_work": res.gpu_work, "text": buf.value.decode(), "error": res.error.decode()}

    def wait(self, count, timeout=600.0):
        return lib().cz_server_wait(self._h, count, timeout) == 0

    def stats(self):
        s = ServerStats()
        lib().cz_server_stats_get(self._h, C.byref(s))
        d = {k: getattr(s, k) for k, _ in ServerStats._fields_ if k != "queued"}
        d["queued"] = list(s.queued)
        return d

    def replay(self, requests, arrivals, timeout=1800.0):
        """requests [(kind, text, depth)], arrival offsets in seconds: submitted on time by the library; ids"""
        n = len(requests)
        kinds = (C.c_int * n)(*[k for k, _, _ in requests])
        blobs = [t.encode() if isinstance(t, str) else t for _, t, _ in requests]
        texts = (C.c_char_p * n)(*blobs)
        lens = (C.c_size_t * n)(*[len(b) for b in blobs])
        depths = (C.c_int * n)(*[d for _, _, d in requests])
        arr = (C.c_double * n)(*arrivals)
        ids = (C.c_int * n)()
        rc = lib().cz_server_replay(self._h, n, kinds, texts, lens, depths, arr, timeout, ids)
        if rc:
            raise TimeoutError("replay did not finish")
        return list(ids)

    def close(self):
        if getattr(self, "_h", None):
            lib().cz_server_destroy(self._h)
            self._h = None

    def __del__(self):
        if _lib is not None:
            self.close()


class SearchOutcome:
    def __init__(self, spec, rc, levels, res):
        self.rc, self.levels, self.raw = rc, levels, res
        self.depth0 = bool(res.depth0)
        self.circuit = [spec.names[res.found[i]] for i in range(res.found_len)]
        self.n_found = res.n_found
        self.error = res.error.decode()
        self.table_split = (res.table_split[0], res.table_split[1])
        self.table = {k: getattr(res, k) for k in ("table_k", "table_proof", "table_classes", "table_levels",
                                                   "table_loaded", "table_built", "table_seconds")}
        self.table["table_path"] = res.table_path.decode()
        self.mitm = {k: getattr(res, k) for k in ("mitm_join", "mitm_forward", "mitm_backward", "mitm_hash_matches",
                                                  "mitm_seconds", "mitm_found", "mitm_proof")}
        self.mitm["mitm_split"] = (res.mitm_split[0], res.mitm_split[1])

    def lines(self, seconds=False, depth=None):
        """stdout of the reference binary for this search (seconds as 0.00 unless asked for; depth: the --depth
        of a --table run, for its proof line)"""
        out = []
        for s in self.levels:
            sec = f"{s['seconds']:.2f}" if seconds else "0.00"
            pre = {1: '"dir": "table", ', 2: '"dir": "fwd", ', 3: '"dir": "bwd", '}.get(s.get("dir", 0), "")
            out.append(f'{{{pre}"t": {s["t"]}, "parents": {s["parents"]}, "prefixes": {s["prefixes"]}, '
                       f'"cut_w3": {s["cut_w3"]}, "cut_lb": {s["cut_lb"]}, "survivors": {s["survivors"]}, '
                       f'"distinct": {s["distinct"]}, "proved_unsat": {"true" if s["distinct"] == 0 else "false"}, '
                       f'"seconds": {sec}}}')
        m = self.mitm
        if m["mitm_join"]:
            sec = f"{m['mitm_seconds']:.2f}" if seconds else "0.00"
            out.append(f'{{"dir": "join", "forward": {m["mitm_forward"]}, "backward": {m["mitm_backward"]}, '
                       f'"hash_matches": {m["mitm_hash_matches"]}, "seconds": {sec}}}')
        if self.rc == CIRCUIT:
            if self.depth0:
                out.append('{"found": 0, "circuit": []}')
            else:
                names = ", ".join(f'"{c}"' for c in self.circuit)
                tab = (f', "mitm": [{m["mitm_split"][0]}, {m["mitm_split"][1]}]' if m["mitm_found"] else
                       f', "table": [{self.table_split[0]}, {self.table_split[1]}]' if sum(self.table_split) > 0 else "")
                out.append(f'{{"t": {len(self.circuit)}, "found": {self.n_found or 1}, "circuit": [{names}]{tab}, '
                           f'"seconds": 0.00}}')
        elif self.rc == PROOF and m["mitm_proof"]:
            out.append(f'{{"depth": {depth}, "proved_unsat": true, "mitm": [{m["mitm_split"][0]}, {m["mitm_split"][1]}]}}')
        elif self.rc == PROOF and self.table["table_proof"]:
            out.append(f'{{"depth": {depth}, "proved_unsat": true, "table": {self.table["table_k"]}}}')
        return out

    @property
    def exit_code(self):
        return self.rc
