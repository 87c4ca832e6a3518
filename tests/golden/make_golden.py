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

# name -> (genome spec factory, k, l)
CASES = {
    "small_plain_k31": (lambda s: s.small_plain(length=20_000, seed=21), 31, 8),
    "scale_like_k31": (lambda s: s.scale_plain(length=30_000, seed=22), 31, 8),
    "batched_job_k31": (lambda s: s.batched_job(7, scale=0.006), 31, 6),
    "wide_tandem_k63": (lambda s: s.wide_k(length=20_000, seed=23), 63, 8),
    "k15_gc30": (lambda s: s.GenomeSpec(length=8_000, gc=0.3, seed=24, snp_rate=0.003), 15, 5),
    "k47_tandem": (lambda s: s.GenomeSpec(length=15_000, gc=0.6, seed=25, snp_rate=0.002, tandem_frac=0.05), 47, 9),
}


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
    from unitigcoarsening_b200 import synth
    for name, (mk, k, l) in CASES.items():
        text = synth.make_text(mk(synth), k).numpy().tobytes()
        out = run_reference(text, k, l)
        lines = sorted(out.split(b"\n")[:-1])
        with open(os.path.join(HERE, f"{name}.in.txt.gz"), "wb") as f:
            f.write(gzip.compress(text, compresslevel=9, mtime=0))
        with open(os.path.join(HERE, f"{name}.ref.txt.gz"), "wb") as f:
            f.write(gzip.compress(b"".join(x + b"\n" for x in lines), compresslevel=9, mtime=0))
        print(name, "k", k, "l", l, "kmers", text.split(b"\n", 1)[0].decode(), "lines", len(lines))


if __name__ == "__main__":
    main()
