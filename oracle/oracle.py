"""ctypes wrapper of the CPU restatement in ``uc_oracle.c``.

TEST INFRASTRUCTURE ONLY.  This is the checker: tests/, ``__graft_entry__.smoke``
and bench.py's CPU-baseline leg import it to compare against the CUDA path.
The product package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
NONE = 0xFFFFFFFF

_lib = None


def build(force: bool = False) -> str:
    """Compile ``liboracle.so`` from ``uc_oracle.c`` (gcc, -O2)."""
    src = os.path.join(HERE, "uc_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-o", LIB_PATH, src])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        i64p = ctypes.POINTER(ctypes.c_int64)
        L.orc_parse.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int, u32p, ctypes.c_int64, i64p]
        L.orc_parse.restype = ctypes.c_int
        L.orc_lmer_priority.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_uint64]
        L.orc_lmer_priority.restype = ctypes.c_uint32
        L.orc_lmin.argtypes = [u32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, u32p, ctypes.c_uint64, u32p, u32p]
        L.orc_lmin.restype = None
        L.orc_edges.argtypes = [u32p, ctypes.c_int64, ctypes.c_int, u32p, u32p]
        L.orc_edges.restype = ctypes.c_int
        L.orc_contract.argtypes = [u32p, ctypes.c_int64, ctypes.c_int, u32p, u32p, u32p, u32p]
        L.orc_contract.restype = ctypes.c_int64
        L.orc_emit.argtypes = [u32p, ctypes.c_int64, ctypes.c_int, u32p, u32p, u32p, ctypes.c_char_p, ctypes.c_int64]
        L.orc_emit.restype = ctypes.c_int64
        L.orc_compact.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_void_p), i64p, i64p, i64p]
        L.orc_compact.restype = ctypes.c_int
        L.orc_sort_lines.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, i64p]
        L.orc_sort_lines.restype = ctypes.c_int
        L.orc_free.argtypes = [ctypes.c_void_p]
        L.orc_free.restype = None
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


class OracleError(ValueError):
    pass


def comp_words(k: int) -> int:
    return (k + 15) // 16


def parse(text: bytes, k: int) -> np.ndarray:
    """Packed k-mers, shape (n, ceil(k/16)) uint32 in the reference layout."""
    L = lib()
    n = ctypes.c_int64(0)
    st = L.orc_parse(text, len(text), k, None, 0, ctypes.byref(n))
    if st:
        raise OracleError(f"orc_parse status {st}")
    words = np.zeros((max(n.value, 1), comp_words(k)), dtype=np.uint32)
    st = L.orc_parse(text, len(text), k, _p(words), n.value, ctypes.byref(n))
    if st:
        raise OracleError(f"orc_parse status {st}")
    return words[: n.value]


def lmer_priority(lmer: int, l: int, seed: int) -> int:
    return lib().orc_lmer_priority(lmer, l, seed)


def lmin(words: np.ndarray, k: int, l: int, seed: int = 0, table: np.ndarray | None = None):
    words = np.ascontiguousarray(words, dtype=np.uint32)
    n = words.shape[0]
    l1 = np.empty(max(n, 1), np.uint32)
    l2 = np.empty(max(n, 1), np.uint32)
    tp = None if table is None else _p(np.ascontiguousarray(table, dtype=np.uint32))
    lib().orc_lmin(_p(words), n, k, l, tp, seed, _p(l1), _p(l2))
    return l1[:n], l2[:n]


def edges(words: np.ndarray, k: int):
    words = np.ascontiguousarray(words, dtype=np.uint32)
    n = words.shape[0]
    succ = np.empty(max(n, 1), np.uint32)
    pred = np.empty(max(n, 1), np.uint32)
    if lib().orc_edges(_p(words), n, k, _p(succ), _p(pred)):
        raise MemoryError("orc_edges")
    return succ[:n], pred[:n]


def contract(words: np.ndarray, k: int, succ: np.ndarray, pred: np.ndarray):
    words = np.ascontiguousarray(words, dtype=np.uint32)
    n = words.shape[0]
    head = np.empty(max(n, 1), np.uint32)
    rank = np.empty(max(n, 1), np.uint32)
    succ = np.ascontiguousarray(succ, dtype=np.uint32)
    pred = np.ascontiguousarray(pred, dtype=np.uint32)
    cyc = lib().orc_contract(_p(words), n, k, _p(succ), _p(pred), _p(head), _p(rank))
    return head[:n], rank[:n], int(cyc)


def emit(words: np.ndarray, k: int, succ: np.ndarray, head: np.ndarray, rank: np.ndarray) -> bytes:
    words = np.ascontiguousarray(words, dtype=np.uint32)
    n = words.shape[0]
    succ = np.ascontiguousarray(succ, dtype=np.uint32)
    head = np.ascontiguousarray(head, dtype=np.uint32)
    rank = np.ascontiguousarray(rank, dtype=np.uint32)
    L = lib()
    size = L.orc_emit(_p(words), n, k, _p(succ), _p(head), _p(rank), None, 0)
    buf = ctypes.create_string_buffer(max(size, 1))
    L.orc_emit(_p(words), n, k, _p(succ), _p(head), _p(rank), buf, size)
    return buf.raw[:size]


def compact(text: bytes, k: int):
    """Whole path: returns (output bytes, n_kmers, n_cycles)."""
    L = lib()
    out = ctypes.c_void_p()
    olen = ctypes.c_int64(0)
    n = ctypes.c_int64(0)
    cyc = ctypes.c_int64(0)
    st = L.orc_compact(text, len(text), k, ctypes.byref(out), ctypes.byref(olen), ctypes.byref(n), ctypes.byref(cyc))
    if st == 1:
        raise OracleError("malformed k-mer text")
    if st:
        raise MemoryError("orc_compact")
    data = ctypes.string_at(out, olen.value)
    L.orc_free(out)
    return data, n.value, cyc.value


def sorted_lines(data: bytes) -> list[bytes]:
    return sorted(data.split(b"\n")[:-1] if data.endswith(b"\n") else data.split(b"\n"))


def compact_mapped(text_addr: int, size: int, k: int):
    """Whole path over text at a raw address (e.g. a memory-mapped file).
    Returns (ctypes address of the malloc'd output, its length, n, cycles);
    release the output with ``free``."""
    L = lib()
    out = ctypes.c_void_p()
    olen = ctypes.c_int64(0)
    n = ctypes.c_int64(0)
    cyc = ctypes.c_int64(0)
    st = L.orc_compact(ctypes.cast(text_addr, ctypes.c_char_p), size, k, ctypes.byref(out), ctypes.byref(olen),
                       ctypes.byref(n), ctypes.byref(cyc))
    if st == 1:
        raise OracleError("malformed k-mer text")
    if st:
        raise MemoryError("orc_compact")
    return out.value, olen.value, n.value, cyc.value


def free(addr: int) -> None:
    lib().orc_free(addr)


def sort_lines_into(src_addr: int, size: int, dst: np.ndarray) -> int:
    """Copy the '\\n'-terminated lines at src_addr into dst (uint8, >= size
    bytes) in byte order; returns the line count."""
    n = ctypes.c_int64(0)
    st = lib().orc_sort_lines(src_addr, size, dst.ctypes.data, ctypes.byref(n))
    if st == 1:
        raise OracleError("last line has no newline")
    if st:
        raise MemoryError("orc_sort_lines")
    return n.value
