"""ctypes binding of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker. The product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class PcsConfig(ctypes.Structure):
    _fields_ = [
        ("pow_bits", ctypes.c_uint32),
        ("log_blowup_factor", ctypes.c_uint32),
        ("log_last_layer_degree_bound", ctypes.c_uint32),
        ("n_queries", ctypes.c_uint32),
    ]


# Protocol presets of the reference (src/prover/native/config.zig:140-160).
PRESETS = {
    "smoke": dict(pow_bits=0, log_blowup_factor=1, log_last_layer_degree_bound=0, n_queries=3),
    "functional": dict(pow_bits=10, log_blowup_factor=1, log_last_layer_degree_bound=0, n_queries=3),
    "secure": dict(pow_bits=26, log_blowup_factor=1, log_last_layer_degree_bound=0, n_queries=70),
}


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        _lib.oracle_prove_wide_fib.argtypes = [
            ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(PcsConfig), u32p, ctypes.c_int,
            ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        _lib.oracle_prove_logup_xor.argtypes = [
            ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(PcsConfig), ctypes.c_uint64, ctypes.c_int,
            ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        _lib.oracle_gen_trace.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                          ctypes.c_uint64, u32p]
        _lib.oracle_pow_grind.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_uint64)]
    return _lib


def _u32p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def config(preset: str = "functional", **overrides) -> PcsConfig:
    d = dict(PRESETS[preset])
    d.update(overrides)
    return PcsConfig(**d)


def gen_trace(log_n_rows: int, sequence_len: int, trace_kind: int = 0, seed: int = 0) -> np.ndarray:
    out = np.empty((sequence_len, 1 << log_n_rows), dtype=np.uint32)
    rc = lib().oracle_gen_trace(log_n_rows, sequence_len, trace_kind, seed, _u32p(out))
    assert rc == 0, rc
    return out


def prove_wide_fib(log_n_rows: int, sequence_len: int, cfg: PcsConfig, trace: np.ndarray | None = None,
                   trace_kind: int = 0, trace_seed: int = 0, channel_seed: int | None = None,
                   n_threads: int = 0) -> bytes:
    cap = 1 << 26
    buf = ctypes.create_string_buffer(cap)
    n = ctypes.c_size_t(0)
    tp = None
    if trace is not None:
        trace = np.ascontiguousarray(trace, dtype=np.uint32)
        tp = _u32p(trace)
    rc = lib().oracle_prove_wide_fib(
        log_n_rows, sequence_len, ctypes.byref(cfg), tp, trace_kind, trace_seed,
        int(channel_seed is not None), channel_seed or 0, n_threads, buf, cap, ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(f"oracle prove failed: {rc}")
    return buf.raw[: n.value]


def prove_logup_xor(log_n: int, cfg: PcsConfig, seed: int = 0, log_table: int = 16,
                    channel_seed: int | None = None, n_threads: int = 0) -> bytes:
    """The LogUp XOR-lookup AIR proof of the oracle (oracle.cpp prove_logup_xor)."""
    cap = 1 << 26
    buf = ctypes.create_string_buffer(cap)
    n = ctypes.c_size_t(0)
    rc = lib().oracle_prove_logup_xor(log_n, log_table, ctypes.byref(cfg), seed, int(channel_seed is not None),
                                      channel_seed or 0, n_threads, buf, cap, ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(f"oracle XOR-lookup prove failed: {rc}")
    return buf.raw[: n.value]


def last_pow_seconds() -> float:
    """Wall time of the proof-of-work grind of this thread's last oracle proof."""
    f = lib().oracle_last_pow_seconds
    f.restype = ctypes.c_double
    return f()


def interpolate(values: np.ndarray) -> np.ndarray:
    v = np.array(values, dtype=np.uint32, copy=True)
    log = int(v.size).bit_length() - 1
    assert lib().oracle_interpolate(log, _u32p(v)) == 0
    return v


def evaluate(coeffs: np.ndarray) -> np.ndarray:
    v = np.array(coeffs, dtype=np.uint32, copy=True)
    log = int(v.size).bit_length() - 1
    assert lib().oracle_evaluate(log, _u32p(v)) == 0
    return v


def extend(coeffs: np.ndarray, log_blowup: int = 1) -> np.ndarray:
    c = np.ascontiguousarray(coeffs, dtype=np.uint32)
    log = int(c.size).bit_length() - 1
    out = np.empty(c.size << log_blowup, dtype=np.uint32)
    assert lib().oracle_extend(log, log_blowup, _u32p(c), _u32p(out)) == 0
    return out


def _col_args(cols):
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    logs = np.array([int(c.size).bit_length() - 1 for c in cols], dtype=np.uint32)
    ptrs = (ctypes.POINTER(ctypes.c_uint32) * max(1, len(cols)))(*[_u32p(c) for c in cols])
    return cols, logs, ptrs


def merkle_root(cols) -> bytes:
    cols, logs, ptrs = _col_args(cols)
    out = ctypes.create_string_buffer(32)
    assert lib().oracle_merkle_root(len(cols), _u32p(logs), ptrs, out) == 0
    return out.raw


def merkle_layers(cols) -> list[np.ndarray]:
    """Layers from the leaves (index 0) to the root, each an (n, 32) uint8 array."""
    cols, logs, ptrs = _col_args(cols)
    max_log = int(logs.max()) if len(cols) else 0
    total = (1 << (max_log + 1)) - 1
    out = np.empty(total * 32, dtype=np.uint8)
    assert lib().oracle_merkle_layers(len(cols), _u32p(logs), ptrs, out.ctypes.data_as(ctypes.c_void_p)) == 0
    layers, at = [], 0
    for k in range(max_log, -1, -1):
        n = 1 << k
        layers.append(out[at * 32:(at + n) * 32].reshape(n, 32))
        at += n
    return layers


def fold_circle_into_line(src: np.ndarray, alpha, dst: np.ndarray | None = None) -> np.ndarray:
    """src: (4, 2^k) coordinate columns; returns (4, 2^(k-1)) accumulated into dst (default zero)."""
    src = np.ascontiguousarray(src, dtype=np.uint32)
    k = int(src.shape[1]).bit_length() - 1
    out = np.zeros((4, src.shape[1] // 2), dtype=np.uint32) if dst is None else np.array(dst, dtype=np.uint32)
    a = np.array(alpha, dtype=np.uint32)
    assert lib().oracle_fold_circle_into_line(k, _u32p(src), _u32p(a), _u32p(out)) == 0
    return out


def fold_line(src: np.ndarray, alpha, first_line_log_size: int) -> np.ndarray:
    src = np.ascontiguousarray(src, dtype=np.uint32)
    k = int(src.shape[1]).bit_length() - 1
    out = np.empty((4, src.shape[1] // 2), dtype=np.uint32)
    a = np.array(alpha, dtype=np.uint32)
    assert lib().oracle_fold_line(k, first_line_log_size, _u32p(src), _u32p(a), _u32p(out)) == 0
    return out


def eval_at_point(coeffs: np.ndarray, px, py) -> np.ndarray:
    c = np.ascontiguousarray(coeffs, dtype=np.uint32)
    log = int(c.size).bit_length() - 1
    out = np.empty(4, dtype=np.uint32)
    assert lib().oracle_eval_at_point(log, _u32p(c), _u32p(np.array(px, np.uint32)),
                                      _u32p(np.array(py, np.uint32)), _u32p(out)) == 0
    return out


def blake2s(data: bytes) -> bytes:
    out = ctypes.create_string_buffer(32)
    assert lib().oracle_blake2s(data, len(data), out) == 0
    return out.raw


def pow_grind(digest: bytes, n_bits: int, n_threads: int = 0) -> int:
    nonce = ctypes.c_uint64(0)
    assert lib().oracle_pow_grind(digest, n_bits, n_threads or (os.cpu_count() or 1), ctypes.byref(nonce)) == 0
    return nonce.value


class DivisionByZero(ArithmeticError):
    """The reference's Error.DivisionByZero / error.ZeroDenominator."""


def batch_inverse(values: np.ndarray) -> np.ndarray:
    """values: (n,) M31, or (degree, n) coordinate planes with degree 2 (CM31) or 4 (QM31)."""
    v = np.ascontiguousarray(values, dtype=np.uint32)
    degree, n = (1, v.size) if v.ndim == 1 else (v.shape[0], v.shape[1])
    out = np.empty_like(v)
    r = lib().oracle_batch_inverse(degree, n, _u32p(v), _u32p(out))
    if r == -2:
        raise DivisionByZero("batch_inverse: zero element")
    assert r == 0
    return out


class LogupUse(ctypes.Structure):
    _fields_ = [
        ("n_words", ctypes.c_uint32),
        ("negate", ctypes.c_uint32),
        ("words", ctypes.POINTER(ctypes.c_uint32) * 8),
        ("constants", ctypes.c_uint32 * 8),
        ("multiplicity", ctypes.POINTER(ctypes.c_uint32)),
    ]


def logup_interaction(log_rows: int, uses: list[dict], alphas, z, batch: int = 1, order: int = 1):
    """uses: dicts with "words" (each a uint32 column of 2^log_rows or an int constant), optional
    "multiplicity" (uint32 column) and "negate". Returns (columns (n_cols, 4, rows), claimed (4,))."""
    keep, structs = [], (LogupUse * len(uses))()
    for u, d in zip(structs, uses):
        u.n_words = len(d["words"])
        u.negate = int(bool(d.get("negate", False)))
        for j, w in enumerate(d["words"]):
            if isinstance(w, (int, np.integer)):
                u.constants[j] = int(w)
            else:
                a = np.ascontiguousarray(w, dtype=np.uint32)
                keep.append(a)
                u.words[j] = _u32p(a)
        if d.get("multiplicity") is not None:
            m = np.ascontiguousarray(d["multiplicity"], dtype=np.uint32)
            keep.append(m)
            u.multiplicity = _u32p(m)
    n_cols = (len(uses) + batch - 1) // batch
    rows = 1 << log_rows
    out = np.empty((n_cols, 4, rows), dtype=np.uint32)
    claimed = np.empty(4, dtype=np.uint32)
    al = np.ascontiguousarray(np.array(alphas, dtype=np.uint32).reshape(-1, 4))
    zz = np.array(z, dtype=np.uint32)
    lib().oracle_logup_interaction.argtypes = [
        ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(LogupUse), ctypes.POINTER(ctypes.c_uint32),
        ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
        ctypes.POINTER(ctypes.c_uint32)]
    r = lib().oracle_logup_interaction(log_rows, len(uses), structs, _u32p(al), _u32p(zz), batch, order,
                                       _u32p(out), _u32p(claimed))
    if r == -2:
        raise DivisionByZero("logup_interaction: zero denominator")
    assert r == 0
    return out, claimed


def xor_lookup_trace(log_n: int, seed: int):
    """(main (3, 2^log_n), table (3, 65536), multiplicity (65536,)) of the XOR-lookup trace."""
    main = np.empty((3, 1 << log_n), dtype=np.uint32)
    table = np.empty((3, 65536), dtype=np.uint32)
    mult = np.empty(65536, dtype=np.uint32)
    lib().oracle_xor_lookup_trace.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32),
                                              ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]
    assert lib().oracle_xor_lookup_trace(log_n, seed, _u32p(main), _u32p(table), _u32p(mult)) == 0
    return main, table, mult
