"""uc_emit_noalloc (line emission with a static scratch array, no device
allocation) against uc_emit on the same keys/head/rank, through the C ABI.

The file name makes pytest collect it last: it must pass both alone in a
fresh process and after every other test has run in the same process."""
import ctypes

import pytest
import torch

from unitigcoarsening_b200 import api, synth

MAX_KMERS = 1 << 20  # UC_EMIT_NOALLOC_MAX_KMERS in include/uc.h


def _noalloc():
    L = ctypes.CDLL(api.LIB_PATH)
    f = L.uc_emit_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [vp, vp, vp, vp, vp, ctypes.c_uint64, ctypes.c_int, vp, ctypes.c_uint64,
                  ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p, ctypes.c_size_t]
    f.restype = ctypes.c_int
    return f


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _call(f, keys, succ, head, rank, k, out):
    nb = ctypes.c_uint64()
    err = ctypes.create_string_buffer(256)
    st = f(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), _ptr(keys), _ptr(succ), _ptr(head),
           _ptr(rank), keys.shape[0], k, _ptr(out), 0 if out is None else out.numel(), ctypes.byref(nb),
           err, len(err))
    return st, nb.value, err.value.decode()


def _graph(comp, text, k, l, limit=None):
    keys = comp.load_kmers(text, k)
    if limit is not None:
        keys = keys[:limit].contiguous()
    succ, pred = comp.assemble_pruned_graph(keys, k, l)
    head, rank, _ = comp.coarsen_de_bruijn_full_cycle(keys, succ, pred, k)
    return keys, succ, head, rank


@pytest.mark.gpu
@pytest.mark.parametrize("k,l,length,limit", [(31, 8, 300_000, None), (63, 10, 200_000, None),
                                              (31, 8, 1_100_000, MAX_KMERS)])
def test_noalloc_emit_matches_emit_twice(comp, k, l, length, limit):
    text = synth.make_text(synth.small_plain(seed=7, length=length), k, device="cuda")
    keys, succ, head, rank = _graph(comp, text, k, l, limit)
    if limit is not None:
        assert keys.shape[0] == limit
    ref = comp.write_unitigs(keys, succ, head, rank, k)
    torch.cuda.synchronize()
    f = _noalloc()
    for _ in range(2):  # the scratch array is reused: the second call must match too
        st, need, msg = _call(f, keys, succ, head, rank, k, None)
        assert st == 0, msg
        assert need == ref.numel()
        out = torch.full((need + 64,), 0x55, dtype=torch.uint8, device="cuda")
        st, nb, msg = _call(f, keys, succ, head, rank, k, out)
        assert st == 0, msg
        assert nb == ref.numel()
        assert torch.equal(out[:nb], ref)
        assert bool((out[nb:] == 0x55).all())


@pytest.mark.gpu
def test_noalloc_emit_takes_no_device_memory(comp):
    """After the first call in this context, a call leaves the device's free
    memory unchanged, and still works while the caller holds all but a
    sliver of it (the position of a process whose own pool owns the GPU)."""
    k = 31
    text = synth.make_text(synth.small_plain(seed=9, length=200_000), k, device="cuda")
    keys, succ, head, rank = _graph(comp, text, k, 8)
    ref = comp.write_unitigs(keys, succ, head, rank, k)
    out = torch.empty(ref.numel() + 64, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    f = _noalloc()
    st, nb, msg = _call(f, keys, succ, head, rank, k, out)  # warm-up: the set-up call
    assert st == 0, msg
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    st, nb, msg = _call(f, keys, succ, head, rank, k, out)
    assert st == 0, msg
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.equal(out[:nb], ref)
    # hold all but 256 MiB of the free memory, then call again
    hold = torch.empty(max(free1 - (256 << 20), 0), dtype=torch.uint8, device="cuda")
    try:
        out.fill_(0)
        st, nb, msg = _call(f, keys, succ, head, rank, k, out)
        assert st == 0, msg
        torch.cuda.synchronize()
        assert torch.equal(out[:nb], ref)
    finally:
        del hold
        torch.cuda.empty_cache()


@pytest.mark.gpu
def test_noalloc_emit_rejects_beyond_maximum(comp):
    # rejected on the host before any device access: the pointers are never read
    keys = torch.zeros((4, 1), dtype=torch.int64, device="cuda")
    ids = torch.zeros(4, dtype=torch.int32, device="cuda")
    f = _noalloc()
    nb = ctypes.c_uint64()
    err = ctypes.create_string_buffer(256)
    st = f(None, _ptr(keys), None, _ptr(ids), _ptr(ids), MAX_KMERS + 1, 31, None, 0, ctypes.byref(nb), err,
           len(err))
    assert st == 1  # UC_EINPUT
    assert "no-allocation maximum" in err.value.decode()
    st, nb2, msg = _call(f, keys[:0], None, ids[:0], ids[:0], 31, None)
    assert st == 0 and nb2 == 0, msg
