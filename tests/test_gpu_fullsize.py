"""Full-size properties of the fused path at the benchmark's sizes, where the
CPU oracle would take too long: the 1 Gbp single job (k=31) and the 200 Mbp
wide-k job (k=63).

- Exactly the input's k-mers are in the output: the order-independent sum of
  a multiplicative hash over every k-mer window of every line equals the same
  sum over the packed input, and the window count equals n.
- Each line holds k + (its k-mers - 1) chars, so the output is k * lines + n
  bytes, and every line has at least k chars.
- Sorted output is deterministic: two runs give equal bytes, in byte order.
- The sorted lines equal, byte for byte, those that the oracle (and for the
  200 Mbp job the reference itself) printed for the same seeded input: line
  count, byte count and sha256 of the lines in byte order, committed in
  tests/golden/checksums_fullsize.json by tests/golden/make_golden.py."""
import hashlib
import json
import os

import pytest
import torch

FULLSIZE = os.path.join(os.path.dirname(__file__), "golden", "checksums_fullsize.json")


def _fullsize_cases():
    if not os.path.exists(FULLSIZE):
        return []
    with open(FULLSIZE) as f:
        return sorted(json.load(f).items())

pytestmark = pytest.mark.gpu

C0 = -7046029254386353131  # 0x9E3779B97F4A7C15 as int64
C1 = -4658895280553007687  # 0xBF58476D1CE4E5B9 as int64


def _input_hash(keys: torch.Tensor):
    h = keys[:, 0] * C0
    if keys.shape[1] > 1:
        h = h + keys[:, 1] * C1
    return int(h.sum().item())


def _output_hash(out: torch.Tensor, k: int, chunk: int = 1 << 27):
    """Hash sum and count of the k-mer windows of all lines (windows that
    contain no line break), in the library's key layout: char x at bits 2x of
    word x // 32."""
    total, count = 0, 0
    n = out.numel()
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        m = c1 - c0  # window starts in [c0, c1)
        seg = out[c0: c1 + k - 1]
        if seg.numel() < k:
            break
        m = min(m, seg.numel() - k + 1)
        codes = ((seg >> 1) ^ (seg >> 2)).to(torch.int64) & 3
        segnl = (seg[: m + k - 1] == 10).to(torch.int32)
        w0 = torch.zeros(m, dtype=torch.int64, device=out.device)
        w1 = torch.zeros(m, dtype=torch.int64, device=out.device)
        bad = torch.zeros(m, dtype=torch.int32, device=out.device)
        for j in range(k):
            if j < 32:
                w0 += codes[j: j + m] << (2 * j)
            else:
                w1 += codes[j: j + m] << (2 * (j - 32))
            bad += segnl[j: j + m]
        ok = bad == 0
        h = w0 * C0 + (w1 * C1 if k > 32 else 0)
        total += int(torch.where(ok, h, torch.zeros_like(h)).sum().item())
        count += int(ok.sum().item())
        del codes, segnl, w0, w1, bad, ok, h
    return total & ((1 << 64) - 1), count


def _lines(out: torch.Tensor):
    ends = torch.nonzero(out == 10).flatten()
    starts = torch.cat([torch.zeros(1, dtype=ends.dtype, device=ends.device), ends[:-1] + 1])
    return starts, ends


@pytest.mark.parametrize("shape", ["scale_plain_1Gbp_k31", "wide_k63_200Mbp"])
def test_fullsize_kmer_multiset_and_lengths(comp, shape):
    from unitigcoarsening_b200 import synth
    if shape == "scale_plain_1Gbp_k31":
        spec, k = synth.scale_plain(), 31
    else:
        spec, k = synth.wide_k(), 63
    text = synth.make_text(spec, k, device="cuda")
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    keys = comp.load_kmers(text, k)
    n = keys.shape[0]
    want = _input_hash(keys) & ((1 << 64) - 1)
    del keys
    torch.cuda.empty_cache()
    out = comp.compact(text, k, 8)
    del text
    torch.cuda.empty_cache()
    got, windows = _output_hash(out, k)
    assert windows == n
    assert got == want
    starts, ends = _lines(out)
    nlines = ends.numel()
    assert out.numel() == k * nlines + n
    assert int((ends - starts).min().item()) >= k
    del out, starts, ends
    torch.cuda.empty_cache()


def test_fullsize_sorted_output_deterministic(comp):
    from unitigcoarsening_b200 import synth
    k = 63
    text = synth.make_text(synth.wide_k(length=50_000_000, seed=13), k, device="cuda")
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    comp.set_sorted_output(True)
    try:
        a = comp.compact(text, k, 8).clone()
        b = comp.compact(text, k, 8)
    finally:
        comp.set_sorted_output(False)
    assert torch.equal(a, b)
    # byte order: each line's first k chars, as big-endian codes, increase
    starts, _ = _lines(a)
    codes = ((a >> 1) ^ (a >> 2)).to(torch.int64) & 3
    # the first k chars as big-endian parts of at most 31 chars (62 bits)
    parts = []
    for p0 in range(0, k, 31):
        v = torch.zeros(starts.numel(), dtype=torch.int64, device=a.device)
        for j in range(p0, min(k, p0 + 31)):
            v = v * 4 + codes[starts + j]
        parts.append(v)
    gt = torch.zeros(starts.numel() - 1, dtype=torch.bool, device=a.device)
    eq = torch.ones_like(gt)
    for v in parts:
        gt |= eq & (v[1:] > v[:-1])
        eq &= v[1:] == v[:-1]
    assert bool(gt.all())


@pytest.mark.parametrize("name,case", _fullsize_cases(), ids=[n for n, _ in _fullsize_cases()])
def test_fullsize_sorted_lines_equal_pinned_checksum(comp, name, case):
    from unitigcoarsening_b200 import synth
    k, l = case["k"], case["l"]
    spec = getattr(synth, case["fn"])(**case["kwargs"])
    text = synth.make_text(spec, k, device="cuda")
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    comp.set_sorted_output(True)
    try:
        out, st = comp.compact(text, k, l, stats=True)
    finally:
        comp.set_sorted_output(False)
    del text
    torch.cuda.synchronize()
    assert st["n_kmers"] == case["n_kmers"]
    assert out.numel() == case["bytes"]
    n_lines = sum(int((out[c0:c0 + (1 << 30)] == 10).sum().item()) for c0 in range(0, out.numel(), 1 << 30))
    assert n_lines == case["n_lines"]
    host = out.cpu()
    del out
    torch.cuda.empty_cache()
    digest = hashlib.sha256(memoryview(host.numpy())).hexdigest()
    assert digest == case["sha256_sorted_lines"], f"{name}: sorted lines differ from {case['printed_by']}"
