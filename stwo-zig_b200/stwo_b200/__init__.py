"""Python host binding of libstwo_b200 (the B200 circle-STARK backend).

The API mirrors the reference's wide-Fibonacci proving entry points
(src/examples/wide_fibonacci.zig: prove / provePreparedWithEngine, Statement,
PcsConfig) and the backend-contract operations (src/backend/*.zig). Every call
goes through the C ABI declared in include/stwo_b200.h; there is no CPU
fallback: importing this module without the built library raises.

Device buffers are torch tensors (int32 storage of canonical M31 words, the
values are < 2^31); torch is used for device memory and streams only.
"""
from __future__ import annotations

import ctypes
import threading
import os
from dataclasses import dataclass, field

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libstwo_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"libstwo_b200.so is not built ({LIB_PATH}); run `make -C stwo-zig_b200`")

_lib = ctypes.CDLL(LIB_PATH)

OK = 0
E_INVALID = -1
E_OOM = -2
E_CUDA = -3
E_TIMEOUT = -4
E_CONSTRAINTS = -5
E_BUFFER_TOO_SMALL = -6
E_FALLBACK = -7
E_NO_DEVICE = -8
E_DIVISION_BY_ZERO = -9
E_REJECTED = -10

_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_i32 = ctypes.c_int32
_vp = ctypes.c_void_p


class QM31C(ctypes.Structure):
    _fields_ = [("a", _u32), ("b", _u32), ("c", _u32), ("d", _u32)]


class PcsConfigC(ctypes.Structure):
    _fields_ = [("pow_bits", _u32), ("log_blowup_factor", _u32), ("log_last_layer_degree_bound", _u32),
                ("n_queries", _u32)]


class RequestC(ctypes.Structure):
    _fields_ = [("log_n_rows", _u32), ("sequence_len", _u32), ("config", PcsConfigC), ("trace_host", _vp),
                ("trace_device", _vp), ("trace_kind", _u32), ("has_channel_seed", _u32), ("trace_seed", _u64),
                ("channel_seed", _u64)]


class LogupUseC(ctypes.Structure):
    _fields_ = [("n_words", _u32), ("negate", _u32), ("words", _vp * 8), ("constants", _u32 * 8),
                ("multiplicity", _vp)]


class XorRequestC(ctypes.Structure):
    _fields_ = [("log_n", _u32), ("log_table", _u32), ("config", PcsConfigC), ("seed", _u64),
                ("has_channel_seed", _u32), ("reserved", _u32), ("channel_seed", _u64)]


class ServerConfigC(ctypes.Structure):
    _fields_ = [("slots", _u32), ("profile", _u32), ("memory_budget", _u64), ("flags", _u32)]


class ServerSnapshotC(ctypes.Structure):
    _fields_ = [(n, _u64) for n in ("submitted", "completed", "failed", "rejected", "peak_in_flight",
                                    "peak_workspace_bytes", "budget_bytes")]


class StageTimesC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("upload", "trace", "main_commit", "composition", "composition_commit",
                                              "oods", "quotients", "fri", "pow", "decommit", "total",
                                              "host_encode", "host_gaps")]


class TuneEntryC(ctypes.Structure):
    _fields_ = [("op", _u32), ("log_size", _u32), ("n_cols", _u32), ("variant", _i32), ("ms", ctypes.c_float * 4)]


class RequestStatsC(ctypes.Structure):
    _fields_ = [("accounted_bytes", _u64), ("workspace_bytes", _u64), ("queued_ms", ctypes.c_double),
                ("run_ms", ctypes.c_double), ("slot", _u32), ("stages", StageTimesC)]


_SIGS = {
    "stwo_b200_context_create": [_i32, ctypes.POINTER(_vp)],
    "stwo_b200_context_destroy": [_vp],
    "stwo_b200_prove_wide_fibonacci": [_vp, ctypes.POINTER(RequestC), _vp, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(StageTimesC)],
    "stwo_b200_prove_wide_fibonacci_batch": [_vp, ctypes.POINTER(RequestC), ctypes.c_size_t,
                                             ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_size_t),
                                             ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(_i32), _u32,
                                             ctypes.POINTER(StageTimesC)],
    "stwo_b200_interpolate_columns": [_vp, _u32, _u32, _vp, _u64, _vp],
    "stwo_b200_evaluate_columns": [_vp, _u32, _u32, _vp, _u64, _vp],
    "stwo_b200_interpolate_and_extend": [_vp, _u32, _u32, _u32, _vp, _u64, _vp, _u64, _vp, _u64, _vp],
    "stwo_b200_extend_columns": [_vp, _u32, _u32, _u32, _vp, _u64, _vp, _u64, _vp],
    "stwo_b200_eval_at_point": [_vp, _u32, _u32, _vp, _u64, QM31C, QM31C, _vp, _vp],
    "stwo_b200_eval_at_point_noalloc": [_vp, _u32, _u32, _vp, _u64, QM31C, QM31C, _vp, _vp],
    "stwo_b200_merkle_commit": [_vp, _u32, _u32, _vp, _u64, _vp, _vp, _vp],
    "stwo_b200_merkle_commit_lifted": [_vp, _u32, ctypes.POINTER(_vp), ctypes.POINTER(_u32), _vp, _vp, _vp],
    "stwo_b200_fold_circle_into_line": [_vp, _u32, _vp, _u64, QM31C, _vp, _u64, _i32, _vp],
    "stwo_b200_fold_line": [_vp, _u32, _vp, _u64, QM31C, _vp, _u64, _vp],
    "stwo_b200_accumulate_quotients": [_vp, _u32, _u32, _vp, _vp, QM31C, QM31C, QM31C, QM31C, _vp, _u64, _vp],
    "stwo_b200_wide_fib_trace": [_vp, _u32, _u32, _u32, _u64, _vp, _u64, _vp],
    "stwo_b200_wide_fib_composition": [_vp, _u32, _u32, _vp, _u64, _vp, _u32, _u32, _vp, _u64, _vp],
    "stwo_b200_accumulate": [_vp, _u32, _vp, _u64, _u32, _vp, _u64, QM31C, _vp],
    "stwo_b200_fold_and_commit": [_vp, _i32, _u32, _vp, _u64, QM31C, _vp, _u64, _vp, _vp, _vp],
    "stwo_b200_commit_columns": [_vp, _u32, _u32, _u32, _vp, _u64, _vp, _u64, _vp, _u64, _vp, _vp, _vp],
    "stwo_b200_interpolate_secure_composition": [_vp, _u32, _vp, _u64, _u32, _vp, _u64, _vp],
    "stwo_b200_quadratic_recurrence_trace": [_vp, _u32, _u32, ctypes.POINTER(_u32), _vp, _u64, _vp],
    "stwo_b200_pow_grind": [_vp, ctypes.c_char_p, _u32, ctypes.POINTER(_u64)],
    "stwo_b200_telemetry_snapshot": [ctypes.POINTER(_u64)],
    "stwo_b200_prove_logup_xor": [_vp, ctypes.POINTER(XorRequestC), _vp, ctypes.c_size_t,
                                  ctypes.POINTER(ctypes.c_size_t)],
    "stwo_b200_verify_wide_fibonacci": [ctypes.c_char_p, ctypes.c_size_t, _u32, _u32, _u32, _u64],
    "stwo_b200_verify_logup_xor": [ctypes.c_char_p, ctypes.c_size_t, _u32, _u32, _u32, _u64],
    "stwo_b200_server_create": [_vp, ctypes.POINTER(ServerConfigC), ctypes.POINTER(_vp)],
    "stwo_b200_server_submit": [_vp, ctypes.POINTER(RequestC), ctypes.POINTER(_u64)],
    "stwo_b200_server_submit_xor": [_vp, ctypes.POINTER(XorRequestC), ctypes.POINTER(_u64)],
    "stwo_b200_server_wait": [_vp, _u64, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                              ctypes.POINTER(RequestStatsC)],
    "stwo_b200_server_warmup": [_vp, _u32, _u32, _u32, _u32],
    "stwo_b200_server_snapshot_get": [_vp, ctypes.POINTER(ServerSnapshotC)],
    "stwo_b200_server_destroy": [_vp],
    "stwo_b200_server_set_request_timeout": [_vp, _u32],
    "stwo_b200_arm_allocation_failure_for_testing": [_u32],
    "stwo_b200_arm_quotient_stage_timeout_for_testing": [],
    "stwo_b200_autotune_mode": [_i32],
    "stwo_b200_autotune_wide_fibonacci": [_vp, _u32, _u32, _u32],
    "stwo_b200_autotune_table": [_vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)],
    "stwo_b200_xor_lookup_trace": [_vp, _u32, _u64, _vp, _vp, _vp, _vp],
    "stwo_b200_batch_inverse": [_vp, _u32, _u64, _vp, _u64, _vp, _u64, _vp],
    "stwo_b200_logup_interaction": [_vp, _u32, _u32, ctypes.POINTER(LogupUseC), ctypes.POINTER(QM31C), QM31C,
                                    _u32, _u32, _vp, _u64, ctypes.POINTER(QM31C), _vp],
}
for _name, _args in _SIGS.items():
    _fn = getattr(_lib, _name)
    _fn.argtypes = _args
    _fn.restype = _i32
_lib.stwo_b200_last_error.restype = ctypes.c_char_p
_lib.stwo_b200_status_string.restype = ctypes.c_char_p
_lib.stwo_b200_status_string.argtypes = [_i32]
_lib.stwo_b200_version.restype = ctypes.c_char_p

EXPORTED_SYMBOLS = sorted(list(_SIGS) + ["stwo_b200_last_error", "stwo_b200_status_string", "stwo_b200_version"])


class StwoError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_lib.stwo_b200_status_string(status).decode()} ({status}): {message}")
        self.status = status


def _check(status: int) -> None:
    if status != OK:
        raise StwoError(status, (_lib.stwo_b200_last_error() or b"").decode())


def lib():
    return _lib


def kernel_launches() -> int:
    """Kernels this library has launched in the process (telemetry counter)."""
    v = _u64(0)
    _check(_lib.stwo_b200_telemetry_snapshot(ctypes.byref(v)))
    return v.value


# ---------------------------------------------------------------------------
# Protocol types (src/core/pcs/mod.zig:23-52, src/core/fri/config.zig,
# src/examples/wide_fibonacci/trace.zig:18-21, presets src/prover/native/config.zig:140-160)
# ---------------------------------------------------------------------------
@dataclass
class FriConfig:
    log_blowup_factor: int = 1
    log_last_layer_degree_bound: int = 0
    n_queries: int = 3


@dataclass
class PcsConfig:
    pow_bits: int = 10
    fri_config: FriConfig = field(default_factory=FriConfig)

    @staticmethod
    def preset(name: str) -> "PcsConfig":
        if name == "smoke":
            return PcsConfig(0, FriConfig(1, 0, 3))
        if name == "functional":
            return PcsConfig(10, FriConfig(1, 0, 3))
        if name == "secure":
            return PcsConfig(26, FriConfig(1, 0, 70))
        raise ValueError(name)

    def _c(self) -> PcsConfigC:
        f = self.fri_config
        return PcsConfigC(self.pow_bits, f.log_blowup_factor, f.log_last_layer_degree_bound, f.n_queries)


@dataclass
class Statement:
    log_n_rows: int
    sequence_len: int


def verify_wide_fibonacci(proof: bytes, log_n_rows: int, sequence_len: int, channel_seed: int | None = None) -> bool:
    """Host verification of a wide-Fibonacci proof by the library's C++ verifier (no device use);
    raises StwoError(E_CONSTRAINTS) naming the failed check."""
    _check(_lib.stwo_b200_verify_wide_fibonacci(proof, len(proof), log_n_rows, sequence_len,
                                                int(channel_seed is not None), channel_seed or 0))
    return True


def verify_logup_xor(proof: bytes, log_n: int, log_table: int = 16, channel_seed: int | None = None) -> bool:
    """Host verification of a LogUp XOR-lookup AIR proof (see verify_wide_fibonacci)."""
    _check(_lib.stwo_b200_verify_logup_xor(proof, len(proof), log_n, log_table, int(channel_seed is not None),
                                           channel_seed or 0))
    return True


TRACE_REFERENCE = 0   # (1, row) seeds of the reference's trace generator
TRACE_SEEDED = 1      # seeded uniform col0/col1 in [0, p-1)
TRACE_FIRST_COLUMNS = 2  # the trace argument holds only col0 and col1; the device derives the rest


def _qm(v) -> QM31C:
    return QM31C(*[int(x) for x in v])


def _ptr(t) -> int:
    if t is None:
        return 0
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data  # numpy


def _stream(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return stream if isinstance(stream, int) else stream.cuda_stream


class Context:
    """One device context (point tables, twiddle towers, per-proof workspaces)."""

    def __init__(self, device: int = 0):
        h = _vp()
        _check(_lib.stwo_b200_context_create(device, ctypes.byref(h)))
        self._h = h
        self.device = device
        self._cap = 1 << 21
        self._buffers: list = []  # host output buffers of batch calls, reused across calls
        self._buffers_lock = threading.Lock()

    def _take_buffer(self, nbytes: int):
        import numpy as np
        with self._buffers_lock:
            for i, b in enumerate(self._buffers):
                if b.size >= nbytes:
                    return self._buffers.pop(i)
        return np.empty(nbytes, dtype=np.uint8)

    def _give_buffer(self, buf) -> None:
        with self._buffers_lock:
            self._buffers.append(buf)

    def _with_output(self, call) -> bytes:
        """Runs call(out_ptr, cap, n) with a pooled host buffer of self._cap bytes and returns the
        n bytes written; on E_BUFFER_TOO_SMALL the capacity grows to what was reported and the call
        is repeated once."""
        n = ctypes.c_size_t(0)
        for _ in range(2):
            cap = self._cap
            buf = self._take_buffer(cap)
            try:
                rc = call(buf.ctypes.data, cap, n)
                if rc == OK:
                    return ctypes.string_at(buf.ctypes.data, n.value)
            finally:
                self._give_buffer(buf)
            if rc != E_BUFFER_TOO_SMALL:
                break
            self._cap = max(2 * cap, n.value)
        _check(rc)
        raise StwoError(rc, "output buffer too small")

    def close(self) -> None:
        if self._h:
            _lib.stwo_b200_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- engine level ------------------------------------------------------
    def _request(self, statement: Statement, config: PcsConfig, trace=None, trace_kind=TRACE_REFERENCE,
                 trace_seed=0, channel_seed=None) -> tuple[RequestC, object]:
        req = RequestC()
        req.log_n_rows = statement.log_n_rows
        req.sequence_len = statement.sequence_len
        req.config = config._c()
        keep = None
        if trace is not None:
            if hasattr(trace, "is_cuda") and trace.is_cuda:
                assert trace.is_contiguous()
                req.trace_device = trace.data_ptr()
            else:
                import numpy as np
                keep = trace if (isinstance(trace, np.ndarray) and trace.dtype == np.uint32
                                 and trace.flags.c_contiguous) else np.ascontiguousarray(trace, dtype=np.uint32)
                req.trace_host = keep.ctypes.data
            keep = (keep, trace)
        req.trace_kind = trace_kind
        req.trace_seed = trace_seed
        req.has_channel_seed = int(channel_seed is not None)
        req.channel_seed = channel_seed or 0
        return req, keep

    def prove_wide_fibonacci(self, statement: Statement, config: PcsConfig, trace=None,
                             trace_kind: int = TRACE_REFERENCE, trace_seed: int = 0, channel_seed: int | None = None,
                             with_times: bool = False):
        """Proves the wide-Fibonacci AIR; returns the JSON wire proof bytes (and stage times)."""
        req, keep = self._request(statement, config, trace, trace_kind, trace_seed, channel_seed)
        times = StageTimesC()
        proof = self._with_output(lambda out, cap, n: _lib.stwo_b200_prove_wide_fibonacci(
            self._h, ctypes.byref(req), out, cap, ctypes.byref(n), ctypes.byref(times)))
        del keep
        if with_times:
            return proof, {name: getattr(times, name) for name, _ in StageTimesC._fields_}
        return proof

    def prove_logup_xor(self, log_n: int, config: PcsConfig, seed: int = 0, log_table: int = 16,
                        channel_seed: int | None = None) -> bytes:
        """Proves the LogUp XOR-lookup AIR (2^log_n seeded lookups into the 2^log_table XOR table)."""
        req = XorRequestC(log_n, log_table, config._c(), seed, int(channel_seed is not None), 0, channel_seed or 0)
        return self._with_output(lambda out, cap, n: _lib.stwo_b200_prove_logup_xor(
            self._h, ctypes.byref(req), out, cap, ctypes.byref(n)))

    def prove_wide_fibonacci_batch(self, requests: list[dict], max_in_flight: int = 4, with_times: bool = False,
                                   proof_cap: int = 1 << 21):
        """requests: dicts with statement, config and optional trace / trace_kind / trace_seed / channel_seed."""
        n = len(requests)
        arr = (RequestC * n)()
        keeps = []
        for i, r in enumerate(requests):
            req, keep = self._request(r["statement"], r["config"], r.get("trace"), r.get("trace_kind", TRACE_REFERENCE),
                                      r.get("trace_seed", 0), r.get("channel_seed"))
            arr[i] = req
            keeps.append(keep)
        cap = proof_cap
        # Proof output space: one host buffer of n * cap bytes, taken from a pool kept on the
        # context and reused across calls (neither zero-filled nor page-faulted again per call).
        buf = self._take_buffer(n * cap)
        try:
            base = buf.ctypes.data
            outs = (_vp * n)(*[base + i * cap for i in range(n)])
            caps = (ctypes.c_size_t * n)(*([cap] * n))
            lens = (ctypes.c_size_t * n)()
            statuses = (_i32 * n)()
            times = (StageTimesC * n)()
            _check(_lib.stwo_b200_prove_wide_fibonacci_batch(self._h, arr, n, outs, caps, lens, statuses,
                                                             max_in_flight, times))
            proofs = [ctypes.string_at(base + i * cap, lens[i]) for i in range(n)]
        finally:
            self._give_buffer(buf)
        del keeps
        if with_times:
            return proofs, [{k: getattr(times[i], k) for k, _ in StageTimesC._fields_} for i in range(n)]
        return proofs

    # ---- backend-contract operations (device tensors) ------------------------
    def interpolate(self, cols, log_size: int, n_cols: int, stride: int, stream=None) -> None:
        _check(_lib.stwo_b200_interpolate_columns(self._h, log_size, n_cols, _ptr(cols), stride, _stream(stream)))

    def evaluate(self, cols, log_size: int, n_cols: int, stride: int, stream=None) -> None:
        _check(_lib.stwo_b200_evaluate_columns(self._h, log_size, n_cols, _ptr(cols), stride, _stream(stream)))

    def interpolate_and_extend(self, evals, coeffs, lde, log_size: int, log_blowup: int, n_cols: int,
                               stream=None) -> None:
        _check(_lib.stwo_b200_interpolate_and_extend(self._h, log_size, log_blowup, n_cols, _ptr(evals), 1 << log_size,
                                                     _ptr(coeffs), 1 << log_size, _ptr(lde),
                                                     1 << (log_size + log_blowup), _stream(stream)))

    def extend(self, coeffs, lde, log_size: int, log_blowup: int, n_cols: int, stream=None) -> None:
        _check(_lib.stwo_b200_extend_columns(self._h, log_size, log_blowup, n_cols, _ptr(coeffs), 1 << log_size,
                                             _ptr(lde), 1 << (log_size + log_blowup), _stream(stream)))

    def merkle_commit(self, cols, log_size: int, n_cols: int, layers, stream=None) -> bytes:
        root = ctypes.create_string_buffer(32)
        _check(_lib.stwo_b200_merkle_commit(self._h, log_size, n_cols, _ptr(cols), 1 << log_size, _ptr(layers), root,
                                            _stream(stream)))
        return root.raw

    def merkle_commit_lifted(self, cols: list, layers, stream=None) -> bytes:
        """Lifted Merkle commitment of device columns of mixed power-of-two lengths; returns the root."""
        n = len(cols)
        ptrs = (_vp * max(1, n))(*[_ptr(c) for c in cols])
        logs = (_u32 * max(1, n))(*[int(c.numel()).bit_length() - 1 for c in cols])
        root = ctypes.create_string_buffer(32)
        _check(_lib.stwo_b200_merkle_commit_lifted(self._h, n, ptrs, logs, _ptr(layers), root, _stream(stream)))
        return root.raw

    def fold_and_commit(self, src, dst, src_log: int, alpha, layers=None, circle: bool = False, stream=None):
        """One FRI fold (circle -> line when circle, else line -> half line) and the Merkle tree of the
        folded layer in `layers`; returns its root (None without layers)."""
        root = ctypes.create_string_buffer(32) if layers is not None else None
        _check(_lib.stwo_b200_fold_and_commit(self._h, int(circle), src_log, _ptr(src), 1 << src_log, _qm(alpha),
                                              _ptr(dst), 1 << (src_log - 1),
                                              _ptr(layers) if layers is not None else None, root, _stream(stream)))
        return root.raw if root is not None else None

    def commit_columns(self, evals, coeffs, lde, layers, log_size: int, log_blowup: int, n_cols: int,
                       stream=None) -> bytes:
        """Interpolate, extend and commit n_cols columns; returns the root."""
        root = ctypes.create_string_buffer(32)
        _check(_lib.stwo_b200_commit_columns(self._h, log_size, log_blowup, n_cols, _ptr(evals), 1 << log_size,
                                             _ptr(coeffs), 1 << log_size, _ptr(lde), 1 << (log_size + log_blowup),
                                             _ptr(layers), root, _stream(stream)))
        return root.raw

    def interpolate_secure_composition(self, comp, comp_log: int, log_blowup: int, lde, stream=None) -> None:
        """comp (4 x 2^comp_log evaluations) -> coefficients; lde (8 x 2^(comp_log-1+log_blowup)) the
        extensions of the left then right coefficient halves."""
        _check(_lib.stwo_b200_interpolate_secure_composition(self._h, comp_log, _ptr(comp), 1 << comp_log, log_blowup,
                                                             _ptr(lde), 1 << (comp_log - 1 + log_blowup),
                                                             _stream(stream)))

    def fold_circle_into_line(self, src, dst, src_log: int, alpha, accumulate: bool = False, stream=None) -> None:
        _check(_lib.stwo_b200_fold_circle_into_line(self._h, src_log, _ptr(src), 1 << src_log, _qm(alpha), _ptr(dst),
                                                    1 << (src_log - 1), int(accumulate), _stream(stream)))

    def fold_line(self, src, dst, src_log: int, alpha, stream=None) -> None:
        _check(_lib.stwo_b200_fold_line(self._h, src_log, _ptr(src), 1 << src_log, _qm(alpha), _ptr(dst),
                                        1 << (src_log - 1), _stream(stream)))

    def eval_at_point(self, coeffs, log_size: int, n_cols: int, stride: int, px, py, out, stream=None) -> None:
        _check(_lib.stwo_b200_eval_at_point(self._h, log_size, n_cols, _ptr(coeffs), stride, _qm(px), _qm(py),
                                            _ptr(out), _stream(stream)))

    def eval_at_point_noalloc(self, coeffs, log_size: int, n_cols: int, stride: int, px, py, out,
                              stream=None) -> None:
        """eval_at_point without any device allocation: partial sums go to the library's fixed
        scratch array (shared by all calls on the device; serialize calls that would overlap)."""
        _check(_lib.stwo_b200_eval_at_point_noalloc(self._h, log_size, n_cols, _ptr(coeffs), stride, _qm(px),
                                                    _qm(py), _ptr(out), _stream(stream)))

    def accumulate_quotients(self, log_size: int, col_ptrs, c, px, py, sum_a, sum_b, out, n_cols: int,
                             stream=None) -> None:
        _check(_lib.stwo_b200_accumulate_quotients(self._h, log_size, n_cols, _ptr(col_ptrs), _ptr(c), _qm(px),
                                                   _qm(py), _qm(sum_a), _qm(sum_b), _ptr(out), 1 << log_size,
                                                   _stream(stream)))

    def wide_fib_trace(self, out, log_n_rows: int, sequence_len: int, trace_kind: int = TRACE_REFERENCE,
                       seed: int = 0, stream=None) -> None:
        _check(_lib.stwo_b200_wide_fib_trace(self._h, log_n_rows, sequence_len, trace_kind, seed, _ptr(out),
                                             1 << log_n_rows, _stream(stream)))

    def accumulate(self, dst, dst_log: int, src, src_log: int, coeff=(1, 0, 0, 0), stream=None) -> None:
        """dst (4 x 2^dst_log coordinate words) += coeff * src (4 x 2^src_log), src lifted to dst's size."""
        _check(_lib.stwo_b200_accumulate(self._h, dst_log, _ptr(dst), 1 << dst_log, src_log, _ptr(src), 1 << src_log,
                                         _qm(coeff), _stream(stream)))

    def quadratic_recurrence_trace(self, out, log_n_rows: int, n_cols: int, recipe, stream=None) -> None:
        """n_cols columns of the seven-word quadratic recurrence (recipe) in bit-reversed circle order."""
        r = (_u32 * 7)(*[int(x) for x in recipe])
        _check(_lib.stwo_b200_quadratic_recurrence_trace(self._h, log_n_rows, n_cols, r, _ptr(out), 1 << log_n_rows,
                                                         _stream(stream)))

    def wide_fib_composition(self, eval_cols, log_n_rows: int, sequence_len: int, coeffs, den0: int, den1: int,
                             out, stream=None) -> None:
        _check(_lib.stwo_b200_wide_fib_composition(self._h, log_n_rows, sequence_len, _ptr(eval_cols),
                                                   2 << log_n_rows, _ptr(coeffs), den0, den1, _ptr(out),
                                                   2 << log_n_rows, _stream(stream)))

    def xor_lookup_trace(self, log_n: int, seed: int, main_cols, table, multiplicity, stream=None) -> None:
        """Seeded u8 pairs (a, b), a ^ b, the 2^16-row XOR table and its multiplicities."""
        _check(_lib.stwo_b200_xor_lookup_trace(self._h, log_n, seed, _ptr(main_cols), _ptr(table), _ptr(multiplicity),
                                               _stream(stream)))

    def batch_inverse(self, src, dst, n: int, degree: int = 1, src_stride: int | None = None,
                      dst_stride: int | None = None, stream=None) -> None:
        """Montgomery batch inverse (batchInverse); raises StwoError(E_DIVISION_BY_ZERO) on a zero."""
        _check(_lib.stwo_b200_batch_inverse(self._h, degree, n, _ptr(src), n if src_stride is None else src_stride,
                                            _ptr(dst), n if dst_stride is None else dst_stride, _stream(stream)))

    def logup_interaction(self, log_rows: int, uses: list[dict], alphas, z, out, batch: int = 1, order: int = 1,
                          stream=None) -> tuple:
        """LogUp interaction columns into `out` ((n_cols, 4, 2^log_rows) words); returns the claimed
        sum. uses: dicts with "words" (device columns or int constants), optional "multiplicity"
        (device column) and "negate"."""
        arr = (LogupUseC * len(uses))()
        for u, d in zip(arr, uses):
            u.n_words = len(d["words"])
            u.negate = int(bool(d.get("negate", False)))
            for j, w in enumerate(d["words"][:8]):  # the library rejects more than 8 words
                if isinstance(w, int):
                    u.constants[j] = w
                else:
                    u.words[j] = _ptr(w)
            u.multiplicity = _ptr(d.get("multiplicity"))
        al = (QM31C * max(1, len(alphas)))(*[_qm(a) for a in alphas])
        claimed = QM31C()
        _check(_lib.stwo_b200_logup_interaction(self._h, log_rows, len(uses), arr, al, _qm(z), batch, order,
                                                _ptr(out), 1 << log_rows, ctypes.byref(claimed), _stream(stream)))
        return (claimed.a, claimed.b, claimed.c, claimed.d)

    def autotune_wide_fibonacci(self, log_n_rows: int, sequence_len: int, log_blowup: int = 1) -> None:
        """Tunes the launch variants of one proof shape with the device otherwise idle (one throwaway
        proof without proof of work)."""
        _check(_lib.stwo_b200_autotune_wide_fibonacci(self._h, log_n_rows, sequence_len, log_blowup))

    def pow_grind(self, prefix_digest: bytes, n_bits: int) -> int:
        nonce = _u64(0)
        _check(_lib.stwo_b200_pow_grind(self._h, prefix_digest, n_bits, ctypes.byref(nonce)))
        return nonce.value


class Server:
    """Continuous-batching serving loop on one device (stwo_b200_server_*): `slots` proofs in
    flight, admitted first-in first-out within `memory_budget` bytes of device workspace (0 = 80% of
    free device memory) and the reference's resource profile (0 standard, 1 large, 2 extreme)."""

    def __init__(self, ctx: Context, slots: int = 8, profile: int = 1, memory_budget: int = 0,
                 persistent_workspaces: bool = False, verify: bool = False):
        h = _vp()
        cfg = ServerConfigC(slots, profile, memory_budget, int(persistent_workspaces) | (2 if verify else 0))
        _check(_lib.stwo_b200_server_create(ctx._h, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._ctx = ctx
        self._keep: dict[int, object] = {}

    def submit(self, statement: Statement, config: PcsConfig, trace=None, trace_kind: int = TRACE_REFERENCE,
               trace_seed: int = 0, channel_seed: int | None = None) -> int:
        req, keep = self._ctx._request(statement, config, trace, trace_kind, trace_seed, channel_seed)
        ticket = _u64(0)
        _check(_lib.stwo_b200_server_submit(self._h, ctypes.byref(req), ctypes.byref(ticket)))
        self._keep[ticket.value] = keep
        return ticket.value

    def submit_xor(self, log_n: int, config: PcsConfig, seed: int = 0, log_table: int = 16,
                   channel_seed: int | None = None) -> int:
        req = XorRequestC(log_n, log_table, config._c(), seed, int(channel_seed is not None), 0, channel_seed or 0)
        ticket = _u64(0)
        _check(_lib.stwo_b200_server_submit_xor(self._h, ctypes.byref(req), ctypes.byref(ticket)))
        return ticket.value

    def wait(self, ticket: int) -> tuple[bytes, dict]:
        st = RequestStatsC()
        try:
            proof = self._ctx._with_output(lambda out, cap, n: _lib.stwo_b200_server_wait(
                self._h, ticket, out, cap, ctypes.byref(n), ctypes.byref(st)))
        finally:
            self._keep.pop(ticket, None)
        stats = {name: getattr(st, name) for name, _ in RequestStatsC._fields_ if name != "stages"}
        stats["stages"] = {name: getattr(st.stages, name) for name, _ in StageTimesC._fields_}
        return proof, stats

    def warmup(self, max_log_n_rows: int = 0, max_sequence_len: int = 100, log_blowup: int = 1,
               max_xor_log_n: int = 0) -> None:
        """Sizes every slot for the largest shapes before traffic (call while idle)."""
        _check(_lib.stwo_b200_server_warmup(self._h, max_log_n_rows, max_sequence_len, log_blowup, max_xor_log_n))

    def set_request_timeout(self, timeout_ms: int) -> None:
        """Time limit of every request submitted from now on (0: none); see the C header."""
        _check(_lib.stwo_b200_server_set_request_timeout(self._h, timeout_ms))

    def snapshot(self) -> dict:
        s = ServerSnapshotC()
        _check(_lib.stwo_b200_server_snapshot_get(self._h, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in ServerSnapshotC._fields_}

    def close(self) -> None:
        if self._h:
            _lib.stwo_b200_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def arm_allocation_failure_for_testing(nth: int) -> None:
    """Makes the library's nth device or pinned allocation from now on fail as out of memory
    (0 disarms); a host-side test hook, no GPU fault is involved."""
    _check(_lib.stwo_b200_arm_allocation_failure_for_testing(nth))


def arm_quotient_stage_timeout_for_testing() -> None:
    """Makes the next bulk-staged quotient launch leave its first stage empty: its bounded waits run
    out (about a second), and the proof or op fails with E_CUDA; no GPU fault is involved."""
    _check(_lib.stwo_b200_arm_quotient_stage_timeout_for_testing())


AUTOTUNE_OPS = {0: "interpolate+extend high pass (fused, generic)", 1: "Merkle leaves (5, 6, 4 CTAs/SM)",
                2: "DEEP quotients (6, 3, 9 loads in flight; bulk-staged)"}


def autotune_mode(mode: int) -> None:
    """-1: tune each (op, log_size, n_cols) on its first call (the default); v >= 0: force variant v."""
    _check(_lib.stwo_b200_autotune_mode(mode))


def autotune_table() -> list[dict]:
    """The tuned keys: op, log_size, n_cols, the chosen variant and each variant's measured ms."""
    n = ctypes.c_size_t(0)
    _lib.stwo_b200_autotune_table(None, 0, ctypes.byref(n))
    buf = (TuneEntryC * max(1, n.value))()
    _check(_lib.stwo_b200_autotune_table(buf, n.value, ctypes.byref(n)))
    return [{"op": AUTOTUNE_OPS.get(e.op, e.op), "log_size": e.log_size, "n_cols": e.n_cols, "variant": e.variant,
             "ms": [round(x, 4) for x in e.ms]} for e in buf[:n.value]]
