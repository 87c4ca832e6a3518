"""Regenerate the golden vectors in this folder.

Each case is a seeded synthetic k-mer text (the reference's input format) and
the sorted unitig lines the reference itself printed for it: its own
driver.cpp and headers, compiled unmodified against the Kokkos-API shim
(oracle/Makefile, target `ref`, serial build) and run here.  The reference
needs inputs large enough that a 1/64 file chunk holds the header and a line,
a header equal to the line count, no homopolymer k-mer, and k = 15 mod 16.

    python tests/golden/make_golden.py      (needs oracle/_ref/uc_ref_serial)
"""
import gzip
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF = os.path.join(ROOT, "oracle", "_ref", "uc_ref_serial")

# Full fixtures (input and sorted reference lines, gzipped):
# name -> (synth factory, kwargs, k, l)
CASES = {
    "small_plain_k31": ("small_plain", {"length": 20_000, "seed": 21}, 31, 8),
    "scale_like_k31": ("scale_plain", {"length": 30_000, "seed": 22}, 31, 8),
    "batched_job_k31": ("batched_job", {"job": 7, "scale": 0.006}, 31, 6),
    "k15_gc30": ("GenomeSpec", {"length": 30_000, "gc": 0.3, "seed": 24, "snp_rate": 0.003}, 15, 5),
}
# Checksum goldens (the input is regenerated from the seeded spec; the
# reference's sorted lines are pinned by count, bytes and sha256), for sizes
# too large to commit as text.  The reference reads out of bounds on small
# cross-bucket outputs (driver.cpp:632-633), so these stay above that size.
CHECKSUMS = {
    "small_plain_full_k31": ("small_plain", {}, 31, 8),
    "wide_tandem_k63": ("wide_k", {"length": 300_000, "seed": 24}, 63, 8),
    "k47_tandem": ("GenomeSpec", {"length": 120_000, "gc": 0.6, "seed": 26, "snp_rate": 0.002,
                                  "tandem_frac": 0.05}, 47, 9),
    "scale_like_k31": ("scale_plain", {"length": 2_000_000, "seed": 27}, 31, 8),
    "batched_job_k31": ("batched_job", {"job": 11, "scale": 0.3}, 31, 8),
}


def spec_of(fn: str, kw: dict):
    from unitigcoarsening_b200 import synth
    return getattr(synth, fn)(**kw)


def text_of(fn: str, kw: dict, k: int) -> bytes:
    from unitigcoarsening_b200 import synth
    return synth.make_text(spec_of(fn, kw), k).numpy().tobytes()


def digest(lines) -> str:
    import hashlib
    h = hashlib.sha256()
    for x in lines:
        h.update(x)
        h.update(b"\n")
    return h.hexdigest()


def run_reference(text: bytes, k: int, l: int) -> bytes:
    with tempfile.TemporaryDirectory() as td:
        inp, outp = os.path.join(td, "in.txt"), os.path.join(td, "out.txt")
        with open(inp, "wb") as f:
            f.write(text)
        subprocess.run([REF, inp, str(k), str(l), outp], check=True, capture_output=True, timeout=300,
                       env=dict(os.environ, KSHIM_SEED="7"))
        with open(outp, "rb") as f:
            return f.read()


def main():
    import json
    for name, (fn, kw, k, l) in CASES.items():
        text = text_of(fn, kw, k)
        out = run_reference(text, k, l)
        lines = sorted(out.split(b"\n")[:-1])
        with open(os.path.join(HERE, f"{name}.in.txt.gz"), "wb") as f:
            f.write(gzip.compress(text, compresslevel=9, mtime=0))
        with open(os.path.join(HERE, f"{name}.ref.txt.gz"), "wb") as f:
            f.write(gzip.compress(b"".join(x + b"\n" for x in lines), compresslevel=9, mtime=0))
        print(name, "k", k, "l", l, "kmers", text.split(b"\n", 1)[0].decode(), "lines", len(lines))
    sums = {}
    for name, (fn, kw, k, l) in CHECKSUMS.items():
        text = text_of(fn, kw, k)
        out = run_reference(text, k, l)
        lines = sorted(out.split(b"\n")[:-1])
        sums[name] = {"fn": fn, "kwargs": kw, "k": k, "l": l, "n_kmers": int(text.split(b"\n", 1)[0]),
                      "n_lines": len(lines), "bytes": len(out), "sha256_sorted_lines": digest(lines)}
        print(name, sums[name])
    with open(os.path.join(HERE, "checksums.json"), "w") as f:
        json.dump(sums, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
