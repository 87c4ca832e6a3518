"""GPU parity: every phase of the CUDA path through the C ABI against the CPU
oracle on the same seeded inputs; bit-exact (keys, minimizers, edges, ranks,
bytes, sorted lines)."""
import numpy as np
import pytest
import torch

from tests.cases import MICRO, cyclic_kmers, distinct_path, shuffled, sorted_lines, text_of, walk_kmers

pytestmark = pytest.mark.gpu


def dev(b: bytes) -> torch.Tensor:
    return torch.frombuffer(bytearray(b), dtype=torch.uint8).cuda()


def fused_lines(comp, text: bytes, k: int, l: int):
    out = comp.compact(dev(text), k, l)
    torch.cuda.synchronize()
    return sorted_lines(out.cpu().numpy().tobytes())


@pytest.mark.parametrize("name,k,kmers,expected", MICRO, ids=[m[0] for m in MICRO])
def test_micro_fused(comp, name, k, kmers, expected):
    got = fused_lines(comp, text_of(kmers), k, min(8, k - 1))
    assert got == sorted(x.encode() for x in expected)


def _synth(kind: str):
    from unitigcoarsening_b200 import synth
    if kind == "small_plain":
        return synth.make_text(synth.small_plain(), 31).numpy().tobytes(), 31
    if kind == "wide_k63":
        return synth.make_text(synth.wide_k(length=400_000, seed=11), 63).numpy().tobytes(), 63
    if kind == "k15":
        return synth.make_text(synth.GenomeSpec(length=60_000, gc=0.45, seed=5, snp_rate=0.002), 15).numpy().tobytes(), 15
    if kind == "k47":
        return synth.make_text(synth.GenomeSpec(length=200_000, gc=0.55, seed=6, snp_rate=0.001,
                                                tandem_frac=0.02), 47).numpy().tobytes(), 47
    if kind == "scale_sample":
        return synth.make_text(synth.scale_plain(length=600_000, seed=12), 31).numpy().tobytes(), 31
    if kind == "batched_job":
        return synth.make_text(synth.batched_job(3, scale=0.1), 31).numpy().tobytes(), 31
    raise KeyError(kind)


CONFIGS = ["small_plain", "wide_k63", "k15", "k47", "scale_sample", "batched_job"]


@pytest.fixture(scope="module")
def texts():
    return {c: _synth(c) for c in CONFIGS}


@pytest.mark.parametrize("cfg", CONFIGS)
def test_phases_bit_exact(comp, oracle, texts, cfg):
    text, k = texts[cfg]
    l = min(8, k - 1)
    seed = 0x1234
    words = oracle.parse(text, k)
    keys = comp.load_kmers(dev(text), k)
    from unitigcoarsening_b200 import as_u32, keys_to_words
    assert np.array_equal(keys_to_words(keys, k), words)
    l1, l2 = comp.find_l_minimizer(keys, k, l, seed)
    o1, o2 = oracle.lmin(words, k, l, seed)
    assert np.array_equal(as_u32(l1), o1) and np.array_equal(as_u32(l2), o2)
    succ, pred = comp.assemble_pruned_graph(keys, k, l, seed)
    osucc, opred = oracle.edges(words, k)
    assert np.array_equal(as_u32(succ), osucc)
    assert np.array_equal(as_u32(pred), opred)
    head, rank, cyc = comp.coarsen_de_bruijn_full_cycle(keys, succ, pred, k)
    ohead, orank, ocyc = oracle.contract(words, k, osucc, opred)
    assert np.array_equal(as_u32(head), ohead) and np.array_equal(as_u32(rank), orank)
    assert cyc == ocyc
    lines = comp.write_unitigs(keys, succ, head, rank, k).cpu().numpy().tobytes()
    assert lines == oracle.emit(words, k, osucc, ohead, orank)


@pytest.mark.parametrize("cfg", CONFIGS)
def test_fused_matches_oracle(comp, oracle, texts, cfg):
    text, k = texts[cfg]
    want, n, _ = oracle.compact(text, k)
    got = fused_lines(comp, text, k, min(8, k - 1))
    assert got == sorted_lines(want)


@pytest.mark.parametrize("cap,bits,wcap,lf", [(256, 0, 0, 0), (256, 4, 0, 150), (1024, 12, 0, 0), (2048, 8, 1, 400),
                                              (8192, 9, 1, 0), (4096, 0, 64, 800), (4096, 14, 32, 0),
                                              (4096, 0, 1024, 150), (1024, 0, 512, 300),
                                              (4096, 1, 0, 0)])  # 2 buckets of 300k copies: 16-bit counts wrap
def test_fused_independent_of_tiling(comp, oracle, texts, cap, bits, wcap, lf):
    """Same lines whatever the bucketing, the hash load factor and whichever
    tier (warp tiles, block tiles, oversized tiles in global scratch) works
    each tile."""
    text, k = texts["scale_sample"]
    want, _, _ = oracle.compact(text, k)
    comp.set_tuning(tile_capacity=cap, bucket_bits=bits, warp_capacity=wcap, load_factor_pct=lf)
    try:
        got = fused_lines(comp, text, k, 8)
        keys = comp.load_kmers(dev(text), k)
        succ, pred = comp.assemble_pruned_graph(keys, k, 8)
    finally:
        comp.set_tuning(tile_capacity=0, bucket_bits=0, warp_capacity=0, load_factor_pct=0)
    assert got == sorted_lines(want)
    from unitigcoarsening_b200 import as_u32
    osucc, opred = oracle.edges(oracle.parse(text, k), k)
    assert np.array_equal(as_u32(succ), osucc) and np.array_equal(as_u32(pred), opred)


@pytest.mark.parametrize("l", [3, 8, 12, 16])
@pytest.mark.parametrize("cfg", ["small_plain", "wide_k63"])
def test_fused_independent_of_l(comp, oracle, texts, cfg, l):
    """Any l gives the same lines; a small l gives long runs of k-mers with
    one minimizer, so warp tiles hold segments longer than k + 1 copies,
    whose later chars come partly from their copies and partly from their
    last k-mer."""
    text, k = texts[cfg]
    want, _, _ = oracle.compact(text, k)
    assert fused_lines(comp, text, k, l) == sorted_lines(want)


@pytest.mark.parametrize("k", [31, 63])
def test_cycles_across_tiles(comp, oracle, k):
    km = cyclic_kmers(500, k, seed=k) + walk_kmers(distinct_path(300, k, seed=3 * k), k)
    text = text_of(shuffled(km, 5))
    want, _, ocyc = oracle.compact(text, k)
    assert ocyc == 1
    for cap, bits in [(0, 0), (256, 6)]:
        comp.set_tuning(tile_capacity=cap, bucket_bits=bits)
        try:
            assert fused_lines(comp, text, k, 6) == sorted_lines(want)
        finally:
            comp.set_tuning(tile_capacity=0, bucket_bits=0)


def test_cycle_inside_one_tile(comp, oracle):
    km = cyclic_kmers(60, 21, seed=9)
    text = text_of(shuffled(km, 2))
    want, _, _ = oracle.compact(text, 21)
    comp.set_tuning(bucket_bits=0)
    try:
        assert fused_lines(comp, text, 21, 6) == sorted_lines(want)
    finally:
        comp.set_tuning(bucket_bits=0)


@pytest.mark.parametrize("k", [21, 31, 47, 63])
def test_long_segments_in_one_warp_tile(comp, oracle, k):
    """One bucket per job (bucket_fill 1 and at most 226 k-mers), so a path
    is one segment of one warp tile: its later chars come from its copies
    up to the last k + 1 and from its last k-mer after that.  Paths of 1 to
    220 k-mers, and a tile with two paths and a cycle."""
    def path(n, seed):  # n k-mers
        return walk_kmers(distinct_path(n + k - 1, k, seed=seed), k)
    jobs = [path(n, n + k) for n in (1, 2, k - 1, k, k + 1, k + 2, 2 * k + 5, 220)]
    jobs.append(path(90, 3) + path(60, 4) + cyclic_kmers(max(40, k + 5), k, seed=5))
    comp.set_tuning(bucket_fill=1)
    try:
        for km in jobs:
            text = text_of(shuffled(km, 7))
            want, _, _ = oracle.compact(text, k)
            assert fused_lines(comp, text, k, min(8, k - 1)) == sorted_lines(want)
    finally:
        comp.set_tuning(bucket_fill=0)


def test_general_line_layout(comp, oracle):
    seq = distinct_path(400, 31, seed=1)
    km = shuffled(walk_kmers(seq, 31), 3)
    for text in [text_of(km, extra="\t12"), text_of(km, crlf=True), text_of(km) + b"\n\n"]:
        assert fused_lines(comp, text, 31, 8) == [seq.encode()]
    # non-ACGT bytes pack as A
    t = text_of(["ACGTN" + "A" * 26])
    assert fused_lines(comp, t, 31, 8) == [b"ACGTA" + b"A" * 26]


def test_empty_and_tiny(comp):
    out = comp.compact(dev(b"0\n"), 31, 8)
    assert out.numel() == 0
    assert fused_lines(comp, text_of(["ACGTACGTACGTACGTACGTACGTACGTACG"]), 31, 8) == [
        b"ACGTACGTACGTACGTACGTACGTACGTACG"]


def test_malformed_inputs_raise(comp):
    from unitigcoarsening_b200 import UCError
    with pytest.raises(UCError) as e:
        comp.compact(dev(text_of(["ACG", "AC"])), 3, 2)
    assert e.value.status == 1
    with pytest.raises(UCError) as e:
        comp.compact(dev(text_of(["ACG", "CGT"], header=3)), 3, 2)
    assert e.value.status == 1
    with pytest.raises(UCError):
        comp.compact(dev(text_of(["ACG"])), 3, 3)  # l must be < k


def test_host_path_and_file(comp, oracle, texts, tmp_path):
    text, k = texts["small_plain"]
    want, _, _ = oracle.compact(text, k)
    got = comp.compact_host(text, k, 8)
    assert sorted_lines(got.numpy().tobytes()) == sorted_lines(want)
    inp = tmp_path / "in.txt"
    outp = tmp_path / "out.txt"
    inp.write_bytes(text)
    comp.compact_file(str(inp), k, 8, str(outp))
    comp.compact_file(str(inp), k, 8, str(outp))  # appends like the reference
    data = outp.read_bytes()
    assert len(data) == 2 * len(want)
    assert sorted_lines(data) == sorted(sorted_lines(want) * 2)


@pytest.mark.parametrize("cfg", ["small_plain", "wide_k63", "k47", "k15", "scale_sample"])
def test_sorted_output_is_byte_exact(comp, oracle, texts, cfg):
    """Sorted output: the whole output equals the oracle's lines in byte
    order, byte for byte, on repeated calls and on the host path."""
    text, k = texts[cfg]
    want, _, _ = oracle.compact(text, k)
    expect = b"".join(x + b"\n" for x in sorted_lines(want))
    comp.set_sorted_output(True)
    try:
        a = comp.compact(dev(text), k, min(8, k - 1)).cpu().numpy().tobytes()
        b = comp.compact(dev(text), k, min(8, k - 1)).cpu().numpy().tobytes()
        h = bytes(comp.compact_host(text, k, min(8, k - 1)).numpy())
        # an output buffer that is not 16-byte aligned takes the byte-wise line scan
        buf = torch.empty(comp.output_bound(len(text), k) + 16, dtype=torch.uint8, device="cuda")
        u = comp.compact(dev(text), k, min(8, k - 1), out=buf[3:]).cpu().numpy().tobytes()
    finally:
        comp.set_sorted_output(False)
    assert a == expect
    assert b == expect and h == expect and u == expect


@pytest.mark.parametrize("cfg", ["small_plain", "wide_k63", "k47"])
@pytest.mark.parametrize("shift", [1, 2, 3])
def test_output_buffer_at_any_byte(comp, oracle, texts, cfg, shift):
    """An output buffer that starts at any byte gets the same lines: the
    cross-tile copy stores aligned words in the middle of each segment and
    single bytes at its ends."""
    text, k = texts[cfg]
    want = sorted_lines(oracle.compact(text, k)[0])
    buf = torch.full((comp.output_bound(len(text), k) + 16,), 0x55, dtype=torch.uint8, device="cuda")
    got = comp.compact(dev(text), k, min(8, k - 1), out=buf[shift:])
    nb = got.numel()
    assert sorted_lines(got.cpu().numpy().tobytes()) == want
    assert bool((buf[:shift] == 0x55).all()) and bool((buf[shift + nb:] == 0x55).all())


def test_sorted_output_cli(comp, oracle, texts, tmp_path):
    import subprocess
    from unitigcoarsening_b200 import build as B
    text, k = texts["small_plain"]
    want, _, _ = oracle.compact(text, k)
    inp = tmp_path / "in.txt"
    outp = tmp_path / "out.txt"
    inp.write_bytes(text)
    r = subprocess.run([B.CLI, str(inp), str(k), "8", str(outp), "--sorted"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert outp.read_bytes() == b"".join(x + b"\n" for x in sorted_lines(want))


def test_host_many_overlapped_uploads(comp, oracle, texts):
    """A sequence of host jobs with the next text uploading during the job
    before it: each job's lines equal the oracle's and the job alone,
    including a repeated text and one larger job between smaller ones."""
    seq = [texts["small_plain"], texts["scale_sample"], texts["batched_job"], texts["small_plain"]]
    k = 31
    assert all(kk == k for _, kk in seq)
    want = [sorted_lines(oracle.compact(t, k)[0]) for t, _ in seq]
    outs = [torch.empty(comp.output_bound(len(t), k), dtype=torch.uint8) for t, _ in seq]
    res, st = comp.compact_host_many([t for t, _ in seq], k, 8, outs=outs, stats=True)
    for r, w in zip(res, want):
        assert sorted_lines(bytes(r.numpy())) == w
    assert st["n_kmers"] == sum(int(t[: t.index(b"\n")]) for t, _ in seq)
    # one shared output buffer for every job: each result is read before the next
    one = torch.empty(max(o.numel() for o in outs), dtype=torch.uint8)
    shared = comp.compact_host_many([t for t, _ in seq], k, 8, outs=[one] * len(seq))
    assert sorted_lines(bytes(shared[-1].numpy())) == want[-1]
    # the largest job first and none larger after it, twice in a row on the
    # same context
    order = sorted(range(len(seq)), key=lambda i: -len(seq[i][0]))
    seq2 = [seq[i] for i in order] + [seq[order[0]]]
    want2 = [want[i] for i in order] + [want[order[0]]]
    for _ in range(2):
        outs2 = [torch.empty(comp.output_bound(len(t), k), dtype=torch.uint8) for t, _ in seq2]
        res2 = comp.compact_host_many([t for t, _ in seq2], k, 8, outs=outs2)
        for r, w in zip(res2, want2):
            assert sorted_lines(bytes(r.numpy())) == w


def _golden():
    from tests.test_oracle import _checksum_cases, _golden_cases
    return _golden_cases(), _checksum_cases()


@pytest.mark.parametrize("case", _golden()[0])
def test_fused_matches_reference_fixture(comp, case):
    from tests.test_oracle import load_golden
    text, want, k = load_golden(case)
    assert fused_lines(comp, text, k, 8 if k > 8 else k - 1) == sorted_lines(want)


@pytest.mark.parametrize("name,entry", _golden()[1], ids=[c[0] for c in _golden()[1]])
def test_fused_matches_reference_checksum(comp, name, entry):
    from tests.test_oracle import digest, regen_text
    text = regen_text(entry)
    lines = fused_lines(comp, text, entry["k"], entry["l"])
    assert len(lines) == entry["n_lines"]
    assert digest(lines) == entry["sha256_sorted_lines"]


@pytest.mark.parametrize("cfg", ["small_plain", "wide_k63", "k47"])
def test_hec_contraction_matches_oracle(comp, oracle, texts, cfg):
    """HEC matching rounds (coarsen_HEC + parallel_map_construct) give the
    same (head, rank) as the oracle's path walk."""
    from unitigcoarsening_b200 import CONTRACT_HEC, as_u32
    text, k = texts[cfg]
    words = oracle.parse(text, k)
    keys = comp.load_kmers(dev(text), k)
    succ, pred = comp.assemble_pruned_graph(keys, k, min(8, k - 1))
    head, rank, cyc = comp.coarsen_de_bruijn_full_cycle(keys, succ, pred, k, method=CONTRACT_HEC)
    osucc, opred = oracle.edges(words, k)
    ohead, orank, ocyc = oracle.contract(words, k, osucc, opred)
    assert np.array_equal(as_u32(head), ohead) and np.array_equal(as_u32(rank), orank)
    assert cyc == ocyc


@pytest.mark.parametrize("cfg", ["small_plain", "scale_sample", "wide_k63"])
def test_fused_hec_stitch_matches_oracle(comp, oracle, texts, cfg):
    from unitigcoarsening_b200 import CONTRACT_HEC
    text, k = texts[cfg]
    want, _, _ = oracle.compact(text, k)
    comp.set_tuning(contract_method=CONTRACT_HEC)
    try:
        assert fused_lines(comp, text, k, min(8, k - 1)) == sorted_lines(want)
    finally:
        comp.set_tuning(contract_method=0)


@pytest.mark.parametrize("k", [31, 63])
def test_hec_with_cycles(comp, oracle, k):
    from unitigcoarsening_b200 import CONTRACT_HEC, as_u32
    km = cyclic_kmers(300, k, seed=k + 1) + cyclic_kmers(2, k, seed=k + 2)[:0] + walk_kmers(
        distinct_path(200, k, seed=5 * k), k)
    text = text_of(shuffled(km, 9))
    want, _, ocyc = oracle.compact(text, k)
    comp.set_tuning(contract_method=CONTRACT_HEC, tile_capacity=256, bucket_bits=6)
    try:
        assert fused_lines(comp, text, k, 6) == sorted_lines(want)
    finally:
        comp.set_tuning(contract_method=0, tile_capacity=0, bucket_bits=0)
    words = oracle.parse(text, k)
    keys = comp.load_kmers(dev(text), k)
    succ, pred = comp.assemble_pruned_graph(keys, k, 6)
    head, rank, cyc = comp.coarsen_de_bruijn_full_cycle(keys, succ, pred, k, method=CONTRACT_HEC)
    osucc, opred = oracle.edges(words, k)
    ohead, orank, _ = oracle.contract(words, k, osucc, opred)
    assert np.array_equal(as_u32(head), ohead) and np.array_equal(as_u32(rank), orank)
    assert cyc == ocyc == 1


def test_batch_matches_oracle_and_alone(comp, oracle, texts):
    """Many jobs in one pass: every job's lines equal the oracle's and equal
    the job compacted alone (batched-vs-alone)."""
    from unitigcoarsening_b200 import synth
    jobs = [synth.make_text(synth.batched_job(j, scale=0.02), 31).numpy().tobytes() for j in range(12)]
    jobs += [texts["small_plain"][0], b"0\n", text_of(["ACGTACGTACGTACGTACGTACGTACGTACG"]),
             text_of(cyclic_kmers(80, 31, seed=4))]
    outs = comp.compact_batch([dev(t) for t in jobs], 31, 8)
    torch.cuda.synchronize()
    for t, o in zip(jobs, outs):
        got = sorted_lines(o.cpu().numpy().tobytes())
        want, _, _ = oracle.compact(t, 31)
        assert got == sorted_lines(want)
        assert got == fused_lines(comp, t, 31, 8)


def test_batch_k63_and_mixed_layouts(comp, oracle):
    from unitigcoarsening_b200 import synth
    jobs = [synth.make_text(synth.wide_k(length=30_000 + 7_000 * j, seed=40 + j), 63).numpy().tobytes()
            for j in range(5)]
    outs = comp.compact_batch([dev(t) for t in jobs], 63, 8)
    for t, o in zip(jobs, outs):
        want, _, _ = oracle.compact(t, 63)
        assert sorted_lines(o.cpu().numpy().tobytes()) == sorted_lines(want)
    # a job with CRLF lines sends the batch one job at a time
    seq = distinct_path(300, 31, seed=8)
    mixed = [text_of(walk_kmers(seq, 31), crlf=True), text_of(walk_kmers(distinct_path(200, 31, seed=9), 31))]
    outs = comp.compact_batch([dev(t) for t in mixed], 31, 8)
    for t, o in zip(mixed, outs):
        want, _, _ = oracle.compact(t, 31)
        assert sorted_lines(o.cpu().numpy().tobytes()) == sorted_lines(want)


def test_batch_names_a_malformed_job(comp, texts):
    """A batch with a job whose count line is wrong fails with UC_EINPUT and
    the job's index in the error; without it the same batch succeeds."""
    from unitigcoarsening_b200 import UCError
    good = texts["batched_job"][0]
    head, body = good.split(b"\n", 1)
    bad = str(int(head) - 1).encode() + b"\n" + body
    jobs = [dev(good), dev(good), dev(bad), dev(good)]
    with pytest.raises(UCError) as ei:
        comp.compact_batch(jobs, 31, 8)
    assert ei.value.status == 1 and "job 2" in str(ei.value)
    res = comp.compact_batch([dev(good)] * 3, 31, 8)
    assert len(res) == 3 and res[0].numel() == res[2].numel() > 0


def test_batch_with_tiers_and_hec(comp, oracle):
    from unitigcoarsening_b200 import CONTRACT_HEC, synth
    jobs = [synth.make_text(synth.scale_plain(length=40_000 + 9_000 * j, seed=60 + j), 31).numpy().tobytes()
            for j in range(6)]
    for tune in [dict(warp_capacity=1), dict(tile_capacity=512, warp_capacity=64), dict(contract_method=CONTRACT_HEC)]:
        comp.set_tuning(**tune)
        try:
            outs = comp.compact_batch([dev(t) for t in jobs], 31, 8)
        finally:
            comp.set_tuning(tile_capacity=0, warp_capacity=0, contract_method=0)
        for t, o in zip(jobs, outs):
            want, _, _ = oracle.compact(t, 31)
            assert sorted_lines(o.cpu().numpy().tobytes()) == sorted_lines(want)


@pytest.mark.parametrize("cap", [1, 3])
@pytest.mark.parametrize("cfg", ["small_plain", "wide_k63", "scale_sample"])
def test_walk_cap_sends_long_lines_to_ranking(comp, oracle, texts, cfg, cap):
    """Lines longer than the stitch's line walk take the ranking path
    (pointer jumping from the segment records, one reservation per line, a
    copy per segment) while the walk writes the others: a cap of 1 or 3
    segments splits a small job's lines between the two, and the lines
    equal the oracle's."""
    text, k = texts[cfg]
    want, _, _ = oracle.compact(text, k)
    comp.set_faults(walk_cap=cap)
    try:
        assert fused_lines(comp, text, k, 8) == sorted_lines(want)
    finally:
        comp.set_faults()


def test_walk_cap_with_cycles_and_batches(comp, oracle, texts):
    """The ranking path after a capped walk with cycles in the job, and in a
    batch, where the lines it reserves come in any job order."""
    from unitigcoarsening_b200 import synth
    km = cyclic_kmers(500, 31, seed=2) + walk_kmers(distinct_path(3000, 31, seed=7), 31)
    cyc = text_of(shuffled(km, 5))
    jobs = [synth.make_text(synth.batched_job(j, scale=0.02), 31).numpy().tobytes() for j in range(8)]
    jobs += [cyc, texts["small_plain"][0]]
    comp.set_faults(walk_cap=2)
    try:
        want, _, ocyc = oracle.compact(cyc, 31)
        assert ocyc == 1
        assert fused_lines(comp, cyc, 31, 6) == sorted_lines(want)
        outs = comp.compact_batch([dev(t) for t in jobs], 31, 8)
        torch.cuda.synchronize()
    finally:
        comp.set_faults()
    for t, o in zip(jobs, outs):
        want, _, _ = oracle.compact(t, 31)
        assert sorted_lines(o.cpu().numpy().tobytes()) == sorted_lines(want)
