"""CPU tests: the oracle against hand-worked known answers and the committed
golden vectors (no GPU)."""
import os

import numpy as np
import pytest

from tests.cases import MICRO, distinct_path, shuffled, sorted_lines, text_of, walk_kmers

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name,k,kmers,expected", MICRO, ids=[m[0] for m in MICRO])
def test_micro_known_answers(oracle, name, k, kmers, expected):
    out, n, _ = oracle.compact(text_of(kmers), k)
    assert n == len(kmers)
    assert sorted_lines(out) == sorted(x.encode() for x in expected)


@pytest.mark.parametrize("k", [15, 31, 47, 63])
def test_long_path_each_width(oracle, k):
    seq = distinct_path(3 * k + 40, k, seed=k)
    out, n, cyc = oracle.compact(text_of(shuffled(walk_kmers(seq, k), 7)), k)
    assert sorted_lines(out) == [seq.encode()]
    assert cyc == 0


def test_packing_layout(oracle):
    # char x at bits 2*(x%16) of word x/16; A=0 C=1 G=2 T=3; other bytes -> A
    w = oracle.parse(text_of(["ACGTN" + "A" * 14]), 19)
    assert w.shape == (1, 2)
    assert w[0, 0] == (1 << 2) | (2 << 4) | (3 << 6)
    assert w[0, 1] == 0


def test_extra_columns_and_crlf(oracle):
    km = ["AAC", "ACG", "ACT", "CGT", "CTA"]
    a, _, _ = oracle.compact(text_of(km), 3)
    b, _, _ = oracle.compact(text_of(km, extra="\t17"), 3)
    c, _, _ = oracle.compact(text_of(km, crlf=True), 3)
    assert sorted_lines(a) == sorted_lines(b) == sorted_lines(c)


def test_malformed_inputs(oracle):
    with pytest.raises(oracle.OracleError):
        oracle.compact(text_of(["ACG", "AC"]), 3)          # short line
    with pytest.raises(oracle.OracleError):
        oracle.compact(text_of(["ACG", "CGT"], header=3), 3)  # count mismatch
    with pytest.raises(oracle.OracleError):
        oracle.compact(b"x\nACG\n", 3)                      # no count


def test_empty_input(oracle):
    out, n, _ = oracle.compact(b"0\n", 31)
    assert n == 0 and out == b""


def test_edges_are_exactly_the_unique_overlaps(oracle):
    # brute force the kept-edge rule on a random set and compare
    rng = np.random.default_rng(3)
    k = 7
    km = sorted({"".join("ACGT"[c] for c in rng.integers(0, 4, k)) for _ in range(400)})
    words = oracle.parse(text_of(km), k)
    succ, pred = oracle.edges(words, k)
    pre = {}
    suf = {}
    for i, x in enumerate(km):
        pre.setdefault(x[:-1], []).append(i)
        suf.setdefault(x[1:], []).append(i)
    for u, x in enumerate(km):
        outs = pre.get(x[1:], [])
        if len(outs) == 1 and len(suf[km[outs[0]][:-1]]) == 1:
            assert succ[u] == outs[0]
            assert pred[outs[0]] == u
        else:
            assert succ[u] == oracle.NONE


def _golden_cases():
    return sorted(f[:-len(".in.txt.gz")] for f in os.listdir(GOLDEN) if f.endswith(".in.txt.gz"))


def load_golden(case):
    import gzip
    with open(os.path.join(GOLDEN, case + ".in.txt.gz"), "rb") as f:
        text = gzip.decompress(f.read())
    with open(os.path.join(GOLDEN, case + ".ref.txt.gz"), "rb") as f:
        want = gzip.decompress(f.read())
    import re
    k = int(re.search(r"(?:^|_)k(\d+)", case).group(1))
    return text, want, k


def _checksum_cases():
    import json
    with open(os.path.join(GOLDEN, "checksums.json")) as f:
        return sorted(json.load(f).items())


def digest(lines):
    import hashlib
    h = hashlib.sha256()
    for x in lines:
        h.update(x)
        h.update(b"\n")
    return h.hexdigest()


def regen_text(entry):
    from unitigcoarsening_b200 import synth
    return synth.make_text(getattr(synth, entry["fn"])(**entry["kwargs"]), entry["k"]).numpy().tobytes()


@pytest.mark.parametrize("case", _golden_cases())
def test_oracle_matches_reference_fixture(oracle, case):
    """Golden vectors printed by the reference itself (compiled unmodified)."""
    text, want, k = load_golden(case)
    out, _, _ = oracle.compact(text, k)
    assert sorted_lines(out) == sorted_lines(want)


@pytest.mark.parametrize("name,entry", _checksum_cases(), ids=[c[0] for c in _checksum_cases()])
def test_oracle_matches_reference_checksum(oracle, name, entry):
    text = regen_text(entry)
    assert int(text.split(b"\n", 1)[0]) == entry["n_kmers"]
    out, _, _ = oracle.compact(text, entry["k"])
    lines = sorted_lines(out)
    assert len(lines) == entry["n_lines"] and len(out) == entry["bytes"]
    assert digest(lines) == entry["sha256_sorted_lines"]


REF_BIN = os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "uc_ref_serial")


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference not compiled here")
@pytest.mark.parametrize("seed,k", [(101, 31), (102, 63), (103, 47), (104, 15)])
def test_oracle_matches_live_reference(oracle, tmp_path, seed, k):
    """The reference binary (its own sources against the Kokkos-API shim) on
    fresh seeded inputs, sized above its small-input read overrun."""
    import subprocess
    from unitigcoarsening_b200 import synth
    length = {31: 150_000, 63: 300_000, 47: 200_000, 15: 60_000}[k]
    text = synth.make_text(synth.GenomeSpec(length=length, gc=0.45, seed=seed, snp_rate=0.002,
                                            repeat_frac=0.03, repeat_copies=(2, 8)), k).numpy().tobytes()
    inp, outp = tmp_path / "in.txt", tmp_path / "out.txt"
    inp.write_bytes(text)
    subprocess.run([REF_BIN, str(inp), str(k), "8", str(outp)], check=True, capture_output=True, timeout=300)
    out, _, _ = oracle.compact(text, k)
    assert sorted_lines(outp.read_bytes()) == sorted_lines(out)
