"""The streamed path for host jobs larger than the device (uc_ctx_set_streaming):
text in chunks of whole lines (two passes), tiles in groups whose lines return
to host memory group by group, then the stitch.  Forced here with small chunks
and groups, so that every chunk and group boundary is crossed many times, and
compared with the oracle line for line.  The reference handles jobs up to host
memory by moving its 64 minimizer buckets to the device one at a time
(driver.cpp:479-521, README.md:6-7)."""
import os

import pytest

from tests.cases import cyclic_kmers, distinct_path, shuffled, text_of, walk_kmers
from unitigcoarsening_b200 import Compactor, api, synth

pytestmark = pytest.mark.gpu


def _lines(b: bytes):
    return sorted(b.split(b"\n")[:-1])


@pytest.mark.parametrize("k,l,spec,chunk,group", [
    (31, 8, ("small_plain", {"seed": 11, "length": 300_000}), 7_777, 20_000),
    (31, 8, ("scale_plain", {"seed": 12, "length": 400_000}), 50_000, 3_000),
    (63, 10, ("wide_k", {"seed": 13, "length": 300_000}), 9_999, 40_000),
    (47, 9, ("GenomeSpec", {"length": 150_000, "gc": 0.6, "seed": 26, "snp_rate": 0.002, "tandem_frac": 0.05}),
     4_096, 10_000),
])
def test_streamed_matches_oracle(oracle, k, l, spec, chunk, group):
    fn, kw = spec
    text = synth.make_text(getattr(synth, fn)(**kw), k).numpy().tobytes()
    want, n, _ = oracle.compact(text, k)
    with Compactor(0) as c:
        c.set_streaming(api.STREAM_ALWAYS, chunk, group)
        out, st = c.compact_host(text, k, l, stats=True)
        got = out.numpy().tobytes()
        assert st["n_kmers"] == n
        assert _lines(got) == _lines(want)
        # the same context, back to the resident path
        c.set_streaming(api.STREAM_NEVER)
        assert _lines(c.compact_host(text, k, l).numpy().tobytes()) == _lines(want)


def test_streamed_cycles_and_hec(oracle):
    k = 21
    km = cyclic_kmers(500, k, seed=3) + walk_kmers(distinct_path(400, k, seed=5), k)
    text = text_of(shuffled(km, 9))
    want, n, cyc = oracle.compact(text, k)
    assert cyc >= 1
    with Compactor(0) as c:
        c.set_streaming(api.STREAM_ALWAYS, 97, 300)
        for method in (api.CONTRACT_POINTER_JUMP, api.CONTRACT_HEC):
            c.set_tuning(contract_method=method)
            got = c.compact_host(text, k, 6).numpy().tobytes()
            assert _lines(got) == _lines(want)


def test_streamed_when_resident_run_cannot_allocate(oracle):
    """A job whose resident run cannot get its device memory runs streamed
    (the default mode): here the resident run's first allocation fails."""
    text = synth.make_text(synth.small_plain(seed=14, length=200_000), 31).numpy().tobytes()
    want, _, _ = oracle.compact(text, 31)
    with Compactor(0) as c:
        c.set_faults(fail_alloc_after=1)
        got = c.compact_host(text, 31, 8).numpy().tobytes()
        assert _lines(got) == _lines(want)


def test_streamed_rejects_other_layouts():
    with Compactor(0) as c:
        c.set_streaming(api.STREAM_ALWAYS, 100, 1000)
        with pytest.raises(api.UCError) as ei:
            c.compact_host(text_of(["ACGTA", "CGTAC"], crlf=True), 5, 3)
        assert ei.value.status == 1


HUGE = os.environ.get("UC_TEST_HUGE_GBP")


@pytest.mark.skipif(not HUGE, reason="opt-in (UC_TEST_HUGE_GBP=<genome Gbp>): needs ~2.5x the text in host RAM")
def test_streamed_beyond_31_bit_kmer_counts():
    """A job of more than 2^31 k-mers (UC_TEST_HUGE_GBP=2.3 gives ~2.3B), which
    the resident path's 31-bit k-mer ids cannot hold: streamed from host
    memory, checked by size-independent properties (the output's k-mer
    windows are exactly the input's k-mers, as an order-free hash sum and a
    count; every line holds k + its k-mers - 1 chars)."""
    import torch

    from tests.test_gpu_fullsize import C0, _output_hash
    k = 31
    # two genomes of half the length each (one k-mer set of more than 2^31
    # elements is beyond the GPU sort that deduplicates it); a k-mer in both
    # is a repeated input line, which the properties below still hold for
    half = int(float(HUGE) * 1e9) // 2
    parts = []
    for seed in (31, 32):
        with torch.no_grad():
            parts.append(synth.kmer_set(synth.scale_plain(length=half, seed=seed), k, device="cuda").cpu())
        torch.cuda.empty_cache()
    n = sum(p.shape[0] for p in parts)
    # the input's hash in the library's key layout (char x at bits 2x)
    want = 0
    header = f"{n}\n".encode()
    text = torch.empty(len(header) + n * (k + 1), dtype=torch.uint8)
    text[: len(header)] = torch.tensor(list(header), dtype=torch.uint8)
    pos = len(header)
    for km in parts:
        for c0 in range(0, km.shape[0], 1 << 26):
            v = km[c0:c0 + (1 << 26)].cuda()
            lib = torch.zeros_like(v)
            for x in range(k):
                lib |= ((v >> (2 * (k - 1 - x))) & 3) << (2 * x)
            want += int((lib * C0).sum().item())
            lines = synth.kmers_to_lines(v, k).flatten().cpu()
            text[pos: pos + lines.numel()] = lines
            pos += lines.numel()
            del v, lib, lines
    want &= (1 << 64) - 1
    del parts
    torch.cuda.empty_cache()
    with Compactor(0) as c:
        c.set_streaming(api.STREAM_ALWAYS)
        out, st = c.compact_host(text, k, 8, stats=True)
    print(f"streamed job: {n} k-mers, {out.numel()} output bytes, {st['n_cross']} cross k-mers, "
          f"{st['n_tiles']} tiles, device ms {st['ms_total']:.1f}")
    assert st["n_kmers"] == n > (1 << 31)
    del text
    got, windows, lines = 0, 0, 0
    step = 1 << 30
    pos = 0
    while pos < out.numel():  # line-aligned pieces on the GPU
        end = min(out.numel(), pos + step)
        piece = out[pos:end]
        cut = int(torch.nonzero(piece == 10).flatten()[-1].item()) + 1
        d = piece[:cut].cuda()
        h, w = _output_hash(d, k)
        got += h
        windows += w
        lines += int((d == 10).sum().item())
        pos += cut
        del d
    assert windows == n
    assert got & ((1 << 64) - 1) == want
    assert out.numel() == k * lines + n
