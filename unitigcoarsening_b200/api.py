"""Python binding of libuc.so (the C ABI in include/uc.h).

The functions keep the names of the reference's steps so a caller of the
reference can find each one:

=============================  ==========================================
this module                    reference (euphoricpoptarts/UnitigCoarsening)
=============================  ==========================================
``Compactor.load_kmers``       ``load_kmers`` + ``compact_kmers``  (driver.cpp:257, 227)
``Compactor.find_l_minimizer`` ``get_double_lmin`` (lmin_buckets.h:67)
``Compactor.assemble_pruned_graph``  ``generate_hashmap`` + ``assemble_pruned_graph``
                               (assembler.h:120, 164), bucketed as ``find_l_minimizer``
``Compactor.coarsen_de_bruijn_full_cycle``  ``coarsen_de_bruijn_full_cycle``
                               (coarseners.h:437) -> (head, rank) per k-mer
``Compactor.write_unitigs``    ``write_intra_bucket_outputs`` (compact.h:161)
``Compactor.compact``          ``main`` pipeline on device-resident text (driver.cpp:422)
``Compactor.compact_host``     the same from host memory to host memory
``Compactor.compact_file``     the CLI ``main <k-mer file> k l <output file>``
=============================  ==========================================

Device buffers are torch CUDA tensors; the library runs on torch's current
stream.  There is no CPU fallback: without the CUDA library every call raises.
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libuc.so")
NONE = 0xFFFFFFFF

CONTRACT_POINTER_JUMP = 0
CONTRACT_HEC = 1
STREAM_AUTO, STREAM_ALWAYS, STREAM_NEVER = 0, 1, 2

STATUS = {0: "ok", 1: "invalid input", 2: "out of memory", 3: "HBM budget exceeded",
          4: "device wait timed out", 5: "internal error", 6: "CUDA error", 7: "job not finished"}


class UCError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "n_kmers", "n_copies", "n_cross", "n_tiles", "n_big_tiles",
        "n_segments", "n_unitigs", "n_cycles", "out_bytes", "closed_bytes", "seg_chars")] + \
        [(n, ctypes.c_uint32) for n in ("l_used", "bucket_bits", "tile_capacity", "stitch_rounds", "launches",
                                          "graph_nodes")] + \
        [(n, ctypes.c_float) for n in ("ms_pack", "ms_bucket", "ms_tiles", "ms_stitch", "ms_total",
                                       "ms_tile_warp", "ms_tile_block")]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [("tile_capacity", ctypes.c_uint32), ("tile_threads", ctypes.c_uint32),
                ("bucket_bits", ctypes.c_uint32), ("load_factor_pct", ctypes.c_uint32),
                ("contract_method", ctypes.c_uint32), ("warp_capacity", ctypes.c_uint32),
                ("bucket_fill", ctypes.c_uint32)]


class Faults(ctypes.Structure):
    _fields_ = [("fail_alloc_after", ctypes.c_uint32), ("hec_round_cap", ctypes.c_uint32),
                ("hec_strict", ctypes.c_uint32), ("walk_cap", ctypes.c_uint32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("lanes", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("reserved", ctypes.c_int), ("hbm_budget", ctypes.c_size_t), ("batch_bytes", ctypes.c_size_t),
                ("host_budget", ctypes.c_size_t), ("tuning", Tuning)]


class JobInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("batch", ctypes.c_uint32), ("n_kmers", ctypes.c_uint64),
                ("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double), ("error", ctypes.c_char * 128)]


class ServerTotals(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("jobs_done", "kmers_done", "batches", "batched_jobs", "queued",
                                               "pool_bytes", "pool_peak_bytes")] + \
               [(n, ctypes.c_double) for n in ("p50_ms", "p99_ms", "max_ms", "mean_ms", "wall_s")]


_lib = None


def lib():
    """Load libuc.so; raises if it was not built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with unitigcoarsening_b200.build.build()")
        L = ctypes.CDLL(LIB_PATH)
        vp, sz, i, u64, u32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32
        pu64 = ctypes.POINTER(ctypes.c_uint64)
        sig = {
            "uc_ctx_create": ([i, sz, ctypes.POINTER(vp)], i),
            "uc_ctx_destroy": ([vp], i),
            "uc_ctx_set_stream": ([vp, vp], i),
            "uc_ctx_sync": ([vp], i),
            "uc_ctx_set_tuning": ([vp, ctypes.POINTER(Tuning)], i),
            "uc_ctx_set_sorted_output": ([vp, i], i),
            "uc_ctx_get_tuning": ([vp, ctypes.POINTER(Tuning)], i),
            "uc_ctx_set_faults": ([vp, ctypes.POINTER(Faults)], i),
            "uc_ctx_set_streaming": ([vp, i, u64, u64], i),
            "uc_last_error": ([vp], ctypes.c_char_p),
            "uc_status_str": ([i], ctypes.c_char_p),
            "uc_parse_header": ([vp, vp, sz, pu64, pu64], i),
            "uc_pack": ([vp, vp, sz, i, vp, pu64], i),
            "uc_minimizers": ([vp, vp, u64, i, i, u64, vp, vp, vp], i),
            "uc_find_edges": ([vp, vp, u64, i, i, u64, vp, vp], i),
            "uc_contract": ([vp, vp, vp, vp, u64, i, i, vp, vp, pu64], i),
            "uc_emit": ([vp, vp, vp, vp, vp, u64, i, vp, u64, pu64], i),
            "uc_compact_device": ([vp, vp, sz, i, i, vp, u64, pu64, ctypes.POINTER(Stats)], i),
            "uc_output_bound": ([sz, i], u64),
            "uc_compact_host": ([vp, vp, sz, i, i, vp, sz, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(Stats)], i),
            "uc_compact_host_many": ([vp, i, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_size_t), i, i,
                                      ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_size_t),
                                      ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(Stats)], i),
            "uc_compact_batch": ([vp, i, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_size_t), i, i, vp, u64,
                                  pu64, pu64, ctypes.POINTER(Stats)], i),
            "uc_batch_output_bound": ([i, ctypes.POINTER(ctypes.c_size_t), i], u64),
            "uc_job_submit": ([vp, vp, sz, i, i, ctypes.POINTER(vp)], i),
            "uc_job_poll": ([vp, ctypes.POINTER(ctypes.c_int)], i),
            "uc_job_wait": ([vp], i),
            "uc_job_result": ([vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(Stats)], i),
            "uc_job_release": ([vp], i),
            "uc_free": ([vp], None),
            "uc_compact_file": ([vp, ctypes.c_char_p, i, i, ctypes.c_char_p, ctypes.POINTER(Stats)], i),
            "uc_server_create": ([ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)], i),
            "uc_server_submit": ([vp, vp, sz, i, i, pu64], i),
            "uc_server_poll": ([vp, u64, ctypes.POINTER(ctypes.c_int)], i),
            "uc_server_wait": ([vp, u64, ctypes.c_double, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_size_t),
                                ctypes.POINTER(JobInfo)], i),
            "uc_server_stats": ([vp, ctypes.POINTER(ServerTotals)], i),
            "uc_server_free": ([vp, vp], i),
            "uc_server_destroy": ([vp], i),
            "uc_autotune": ([vp, vp, sz, i, i, i, u32, ctypes.POINTER(Tuning), ctypes.POINTER(ctypes.c_float),
                             ctypes.POINTER(u32)], i),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def key_words(k: int) -> int:
    """64-bit words per packed k-mer."""
    return 1 if k <= 31 else 2


def _ptr(t: torch.Tensor | None):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class Compactor:
    """One library context bound to one GPU (uc_ctx)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("the unitig compactor needs a CUDA device")
        self.device = device
        self._L = lib()
        h = ctypes.c_void_p()
        st = self._L.uc_ctx_create(device, hbm_budget, ctypes.byref(h))
        if st:
            raise UCError(st, "uc_ctx_create failed")
        self._h = h

    # -- plumbing
    def close(self):
        if getattr(self, "_h", None):
            self._L.uc_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _bind_stream(self):
        with torch.cuda.device(self.device):
            s = torch.cuda.current_stream().cuda_stream
        self._L.uc_ctx_set_stream(self._h, ctypes.c_void_p(s))

    def _check(self, st: int):
        if st:
            raise UCError(st, self._L.uc_last_error(self._h).decode())

    def set_tuning(self, **kw):
        t = Tuning()
        self._check(self._L.uc_ctx_get_tuning(self._h, ctypes.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        self._check(self._L.uc_ctx_set_tuning(self._h, ctypes.byref(t)))

    def set_sorted_output(self, on: bool = True):
        """Whole-job calls leave the lines in byte order (deterministic
        output; uc_ctx_set_sorted_output)."""
        self._check(self._L.uc_ctx_set_sorted_output(self._h, 1 if on else 0))

    def set_faults(self, fail_alloc_after: int = 0, hec_round_cap: int = 0, hec_strict: bool = False,
                   walk_cap: int = 0):
        """Failure injection for error-path tests (uc_ctx_set_faults); the
        defaults switch it off.  walk_cap > 0 caps the stitch's line walk, so
        that longer lines take the list-ranking path."""
        f = Faults(int(fail_alloc_after), int(hec_round_cap), 1 if hec_strict else 0, int(walk_cap))
        self._check(self._L.uc_ctx_set_faults(self._h, ctypes.byref(f)))

    def set_streaming(self, mode: int = STREAM_AUTO, chunk_lines: int = 0, group_copies: int = 0):
        """Host jobs beyond the device budget run streamed
        (uc_ctx_set_streaming): STREAM_AUTO, STREAM_ALWAYS or STREAM_NEVER,
        with the chunk and tile-group sizes (0 = defaults)."""
        self._check(self._L.uc_ctx_set_streaming(self._h, int(mode), int(chunk_lines), int(group_copies)))

    def get_tuning(self) -> dict:
        t = Tuning()
        self._check(self._L.uc_ctx_get_tuning(self._h, ctypes.byref(t)))
        return {n: getattr(t, n) for n, _ in Tuning._fields_}

    def _dev(self):
        return torch.device("cuda", self.device)

    # -- phases
    def load_kmers(self, text: torch.Tensor, k: int) -> torch.Tensor:
        """Text (uint8 CUDA tensor) -> packed keys, shape (n, words)."""
        self._bind_stream()
        n = ctypes.c_uint64()
        bn = ctypes.c_uint64()
        self._check(self._L.uc_parse_header(self._h, _ptr(text), text.numel(), ctypes.byref(n), ctypes.byref(bn)))
        keys = torch.empty((max(n.value, 1), key_words(k)), dtype=torch.int64, device=self._dev())
        self._check(self._L.uc_pack(self._h, _ptr(text), text.numel(), k, _ptr(keys), ctypes.byref(n)))
        return keys[: n.value]

    def find_l_minimizer(self, keys: torch.Tensor, k: int, l: int, seed: int = 0,
                         table: torch.Tensor | None = None):
        self._bind_stream()
        n = keys.shape[0]
        l1 = torch.empty(max(n, 1), dtype=torch.int32, device=self._dev())
        l2 = torch.empty_like(l1)
        self._check(self._L.uc_minimizers(self._h, _ptr(keys), n, k, l, seed, _ptr(table), _ptr(l1), _ptr(l2)))
        return l1[:n], l2[:n]

    def assemble_pruned_graph(self, keys: torch.Tensor, k: int, l: int, seed: int = 0):
        """Kept-edge graph by id: (succ, pred) int32 (UC_NONE = -1)."""
        self._bind_stream()
        n = keys.shape[0]
        succ = torch.empty(max(n, 1), dtype=torch.int32, device=self._dev())
        pred = torch.empty_like(succ)
        self._check(self._L.uc_find_edges(self._h, _ptr(keys), n, k, l, seed, _ptr(succ), _ptr(pred)))
        return succ[:n], pred[:n]

    def coarsen_de_bruijn_full_cycle(self, keys, succ, pred, k: int, method: int = CONTRACT_POINTER_JUMP):
        """(head, rank, n_cycles) per k-mer."""
        self._bind_stream()
        n = keys.shape[0]
        head = torch.empty(max(n, 1), dtype=torch.int32, device=self._dev())
        rank = torch.empty_like(head)
        cyc = ctypes.c_uint64()
        self._check(self._L.uc_contract(self._h, _ptr(keys), _ptr(succ), _ptr(pred), n, k, method,
                                        _ptr(head), _ptr(rank), ctypes.byref(cyc)))
        return head[:n], rank[:n], cyc.value

    def write_unitigs(self, keys, succ, head, rank, k: int) -> torch.Tensor:
        """Unitig lines ordered by head id, as a uint8 CUDA tensor."""
        self._bind_stream()
        n = keys.shape[0]
        nb = ctypes.c_uint64()
        self._check(self._L.uc_emit(self._h, _ptr(keys), _ptr(succ), _ptr(head), _ptr(rank), n, k,
                                    None, 0, ctypes.byref(nb)))
        out = torch.empty(max(nb.value, 1), dtype=torch.uint8, device=self._dev())
        self._check(self._L.uc_emit(self._h, _ptr(keys), _ptr(succ), _ptr(head), _ptr(rank), n, k,
                                    _ptr(out), out.numel(), ctypes.byref(nb)))
        return out[: nb.value]

    # -- whole path
    def output_bound(self, text_bytes: int, k: int) -> int:
        return int(self._L.uc_output_bound(text_bytes, k))

    def compact(self, text: torch.Tensor, k: int, l: int, out: torch.Tensor | None = None,
                stats: bool = False):
        """Device-resident text -> unitig lines (uint8 CUDA tensor)."""
        self._bind_stream()
        cap = self.output_bound(text.numel(), k)
        if out is None or out.numel() < cap:
            out = torch.empty(cap, dtype=torch.uint8, device=self._dev())
        nb = ctypes.c_uint64()
        st = Stats()
        self._check(self._L.uc_compact_device(self._h, _ptr(text), text.numel(), k, l, _ptr(out), out.numel(),
                                              ctypes.byref(nb), ctypes.byref(st)))
        res = out[: nb.value]
        return (res, st.as_dict()) if stats else res

    def compact_batch(self, texts, k: int, l: int, out: torch.Tensor | None = None, stats: bool = False):
        """Many device-resident jobs in one pass; returns one uint8 CUDA tensor
        (a view of the shared output buffer) per job."""
        self._bind_stream()
        nj = len(texts)
        ptrs = (ctypes.c_void_p * max(nj, 1))(*[t.data_ptr() for t in texts])
        sizes = (ctypes.c_size_t * max(nj, 1))(*[t.numel() for t in texts])
        cap = int(self._L.uc_batch_output_bound(nj, sizes, k))
        if out is None or out.numel() < cap:
            out = torch.empty(max(cap, 1), dtype=torch.uint8, device=self._dev())
        off = (ctypes.c_uint64 * max(nj, 1))()
        ln = (ctypes.c_uint64 * max(nj, 1))()
        st = Stats()
        self._check(self._L.uc_compact_batch(self._h, nj, ptrs, sizes, k, l, _ptr(out), out.numel(), off, ln,
                                             ctypes.byref(st)))
        res = [out[off[j]: off[j] + ln[j]] for j in range(nj)]
        return (res, st.as_dict()) if stats else res

    def compact_host(self, text, k: int, l: int, out=None, stats: bool = False):
        """Host text (bytes, numpy uint8 or CPU tensor, pinned or not) ->
        host lines.  With ``out`` (a CPU uint8 tensor) the lines land there."""
        if isinstance(text, (bytes, bytearray)):
            src = np.frombuffer(text, dtype=np.uint8)
            tp, tn = src.ctypes.data_as(ctypes.c_void_p), src.nbytes
        elif isinstance(text, np.ndarray):
            tp, tn = text.ctypes.data_as(ctypes.c_void_p), text.nbytes
        else:
            tp, tn = ctypes.c_void_p(text.data_ptr()), text.numel()
        cap = self.output_bound(tn, k)
        if out is None:
            out = torch.empty(cap, dtype=torch.uint8)
        ob = ctypes.c_size_t()
        st = Stats()
        self._check(self._L.uc_compact_host(self._h, tp, tn, k, l, ctypes.c_void_p(out.data_ptr()), out.numel(),
                                            ctypes.byref(ob), ctypes.byref(st)))
        res = out[: ob.value]
        return (res, st.as_dict()) if stats else res

    def autotune(self, text: torch.Tensor, k: int, l: int, reps: int = 3, max_ms: int = 60000,
                 cache: str | None = None) -> dict:
        """Pick the fastest tuning for jobs like ``text`` (device-resident)
        with the library's coordinate-descent tuner (uc_autotune) and leave it
        set on this context.  With ``cache`` (a JSON file) the result is stored
        under this GPU, k and the job's size class, and reused from there on
        later calls without timing anything."""
        key = tuning_key(self.device, k, text.numel())
        if cache:
            got = load_tuning(cache, key)
            if got is not None:
                self.set_tuning(**got)
                return dict(got, cached=True)
        self._bind_stream()
        t = Tuning()
        ms = ctypes.c_float()
        n = ctypes.c_uint32()
        self._check(self._L.uc_autotune(self._h, _ptr(text), text.numel(), k, l, reps, max_ms, ctypes.byref(t),
                                        ctypes.byref(ms), ctypes.byref(n)))
        res = {f: getattr(t, f) for f, _ in Tuning._fields_}
        if cache:
            store_tuning(cache, key, res, ms.value)
        return dict(res, ms=ms.value, trials=n.value, cached=False)

    def compact_host_many(self, texts, k: int, l: int, outs=None, stats: bool = False):
        """A sequence of host jobs with overlapped uploads (uc_compact_host_many):
        each text (bytes, numpy uint8 or CPU tensor; pinned for full link
        speed) goes to the device while the job before it finishes.  ``outs``
        (CPU uint8 tensors, one per job, may repeat) receive the lines;
        returns one view per job."""
        nj = len(texts)
        keep, tp, tn = [], [], []
        for t in texts:
            if isinstance(t, (bytes, bytearray)):
                a = np.frombuffer(t, dtype=np.uint8)
                keep.append(a)
                tp.append(a.ctypes.data)
                tn.append(a.nbytes)
            elif isinstance(t, np.ndarray):
                tp.append(t.ctypes.data)
                tn.append(t.nbytes)
            else:
                tp.append(t.data_ptr())
                tn.append(t.numel())
        if outs is None:
            outs = [torch.empty(self.output_bound(n, k), dtype=torch.uint8) for n in tn]
        ptrs = (ctypes.c_void_p * max(nj, 1))(*tp)
        sizes = (ctypes.c_size_t * max(nj, 1))(*tn)
        optr = (ctypes.c_void_p * max(nj, 1))(*[o.data_ptr() for o in outs])
        ocap = (ctypes.c_size_t * max(nj, 1))(*[o.numel() for o in outs])
        olen = (ctypes.c_size_t * max(nj, 1))()
        st = Stats()
        self._bind_stream()
        self._check(self._L.uc_compact_host_many(self._h, nj, ptrs, sizes, k, l, optr, ocap, olen, ctypes.byref(st)))
        res = [outs[j][: olen[j]] for j in range(nj)]
        return (res, st.as_dict()) if stats else res

    def compact_file(self, in_path: str, k: int, l: int, out_path: str) -> dict:
        st = Stats()
        self._check(self._L.uc_compact_file(self._h, in_path.encode(), k, l, out_path.encode(), ctypes.byref(st)))
        return st.as_dict()


class Server:
    """Serving loop over one GPU (uc_server_*): jobs submitted from host
    memory at any time, admitted by their HBM footprint into one device pool,
    small queued jobs batched into one launch, several lanes overlapping on
    the device.  ``wait`` returns each job's lines and its latency."""

    def __init__(self, device: int = 0, lanes: int = 4, max_batch: int = 64, hbm_budget: int = 0,
                 batch_bytes: int = 0, host_budget: int = 0, tuning: dict | None = None):
        self._L = lib()
        cfg = ServerConfig(device=device, lanes=lanes, max_batch=max_batch, hbm_budget=hbm_budget,
                           batch_bytes=batch_bytes, host_budget=host_budget)
        for k, v in (tuning or {}).items():
            setattr(cfg.tuning, k, int(v))
        h = ctypes.c_void_p()
        st = self._L.uc_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if st:
            raise UCError(st, "uc_server_create failed")
        self._h = h
        self._keep = {}  # ticket -> host text kept alive until its result is taken

    def submit(self, text, k: int, l: int) -> int:
        if isinstance(text, (bytes, bytearray)):
            arr = np.frombuffer(text, dtype=np.uint8)
            ptr, n = arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes
        elif isinstance(text, np.ndarray):
            arr = text
            ptr, n = arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes
        else:
            arr = text
            ptr, n = ctypes.c_void_p(text.data_ptr()), text.numel()
        t = ctypes.c_uint64()
        st = self._L.uc_server_submit(self._h, ptr, n, k, l, ctypes.byref(t))
        if st:
            raise UCError(st, "uc_server_submit failed")
        self._keep[t.value] = arr
        return t.value

    def done(self, ticket: int) -> bool:
        d = ctypes.c_int()
        st = self._L.uc_server_poll(self._h, ticket, ctypes.byref(d))
        if st:
            raise UCError(st, "uc_server_poll failed")
        return bool(d.value)

    def wait(self, ticket: int, timeout: float = 0.0, fetch: bool = True):
        """(lines as bytes, info dict); raises UCError if the job failed.
        fetch=False drops the lines in the server (returns b"")."""
        buf = ctypes.c_void_p()
        n = ctypes.c_size_t()
        info = JobInfo()
        st = self._L.uc_server_wait(self._h, ticket, timeout, ctypes.byref(buf) if fetch else None,
                                    ctypes.byref(n), ctypes.byref(info))
        if st == 4 and info.latency_ms == 0 and not info.error:  # UC_ETIMEOUT: still running
            raise TimeoutError(f"job {ticket} not done within {timeout} s")
        self._keep.pop(ticket, None)
        data = ctypes.string_at(buf, n.value) if buf.value else b""
        if buf.value:
            self._L.uc_server_free(self._h, buf)
        d = {"status": info.status, "batch": info.batch, "n_kmers": info.n_kmers, "queue_ms": info.queue_ms,
             "latency_ms": info.latency_ms, "error": info.error.decode()}
        if st:
            raise UCError(st, d["error"] or "job failed")
        return data, d

    def stats(self) -> dict:
        t = ServerTotals()
        self._L.uc_server_stats(self._h, ctypes.byref(t))
        return {n: getattr(t, n) for n, _ in ServerTotals._fields_}

    def close(self):
        if getattr(self, "_h", None):
            self._L.uc_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tuning_key(device: int, k: int, text_bytes: int) -> str:
    """Cache key of a tuning: GPU name, key width and the job's size class
    (power of two of its text bytes)."""
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    return f"{name}|k{'31' if k <= 31 else '63'}|2^{max(0, int(text_bytes).bit_length() - 1)}"


def load_tuning(path: str, key: str):
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    e = d.get(key)
    return None if e is None else {n: int(e[n]) for n, _ in Tuning._fields_ if n in e}


def store_tuning(path: str, key: str, tuning: dict, ms: float):
    d = {}
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
    d[key] = dict(tuning, ms=round(float(ms), 4))
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def keys_to_words(keys: torch.Tensor, k: int) -> np.ndarray:
    """Packed keys -> the reference's uint32 word layout (n, ceil(k/16))."""
    a = keys.detach().cpu().contiguous().numpy().view(np.uint32).reshape(keys.shape[0], -1)
    return np.ascontiguousarray(a[:, : (k + 15) // 16])


def as_u32(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy().view(np.uint32)
