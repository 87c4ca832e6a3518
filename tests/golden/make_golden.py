"""Regenerate the golden vectors in this folder.

Each case is a seeded synthetic k-mer text (the reference's input format) and
the sorted unitig lines the reference itself printed for it: its own
driver.cpp and headers, compiled unmodified against the Kokkos-API shim
(oracle/Makefile, target `ref`, serial build) and run here.  The reference
needs inputs large enough that a 1/64 file chunk holds the header and a line,
a header equal to the line count, no homopolymer k-mer, and k = 15 mod 16.

    python tests/golden/make_golden.py      (needs oracle/_ref/uc_ref_serial)

Full-size checksums (checksums_fullsize.json) of the benchmark's own single-job
inputs, which are far too large to commit or to sort as Python objects:

    python tests/golden/make_golden.py --fullsize NAME --workdir DIR [--reference]

writes the input text to DIR, runs the oracle (oracle/liboracle.so, itself
pinned to the reference by the fixtures above) and, with --reference, the
reference's OpenMP build (oracle/_ref/uc_ref_large) on it, sorts each output's
lines with the oracle's C helper and records count, bytes and sha256 with the
name of every program that printed them.  Both must agree when both run.
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


# Full-size single-job shapes: name -> (synth factory, kwargs, k, l)
FULLSIZE = {
    "scale_plain_1Gbp_k31": ("scale_plain", {}, 31, 8),
    "wide_k63_200Mbp": ("wide_k", {}, 63, 8),
}
REF_OMP = os.path.join(ROOT, "oracle", "_ref", "uc_ref_large")


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


def write_text(fn: str, kw: dict, k: int, path: str, chunk: int = 1 << 24) -> int:
    """The seeded input written to path in the reference format, streamed in
    chunks of k-mers (the whole text is never held); returns n."""
    from unitigcoarsening_b200 import synth
    km = synth.kmer_set(spec_of(fn, kw), k)
    n = km.shape[0]
    with open(path, "wb") as f:
        f.write(f"{n}\n".encode())
        for c0 in range(0, n, chunk):
            synth.kmers_to_lines(km[c0:c0 + chunk], k).numpy().tofile(f)
    del km
    return n


def sorted_digest(addr: int, size: int):
    """(lines, sha256 of the lines in byte order) of the output at addr."""
    import hashlib

    import numpy as np

    from oracle import oracle as O
    dst = np.empty(max(size, 1), dtype=np.uint8)
    nl = O.sort_lines_into(addr, size, dst)
    h = hashlib.sha256(memoryview(dst)[:size]).hexdigest()
    del dst
    return nl, h


def _sorted_copy(addr: int, size: int) -> bytes:
    import numpy as np

    from oracle import oracle as O
    dst = np.empty(max(size, 1), dtype=np.uint8)
    O.sort_lines_into(addr, size, dst)
    return dst[:size].tobytes()


def _kmers_of(lines, k: int):
    out = []
    for x in lines:
        out += [x[i:i + k] for i in range(len(x) - k + 1)]
    return sorted(out)


def cycle_only_difference(a: bytes, b: bytes, k: int, cycles: int):
    """Compare two outputs line by line (both sorted).  The reference leaves
    the member order of an isolated cycle unspecified (coarseners.h:191-230),
    so outputs may differ in cycle lines only.  Returns the differing lines
    of each side when they are at most `cycles` lines each and hold the same
    k-mers as a set (each a rotation of the same cycle); None otherwise."""
    la = a.split(b"\n")[:-1]
    lb = b.split(b"\n")[:-1]
    i = j = 0
    da, db = [], []
    while i < len(la) or j < len(lb):
        if j >= len(lb) or (i < len(la) and la[i] < lb[j]):
            da.append(la[i]); i += 1
        elif i >= len(la) or lb[j] < la[i]:
            db.append(lb[j]); j += 1
        else:
            i += 1; j += 1
        if len(da) > cycles or len(db) > cycles:
            return None
    # a cycle of m k-mers spells k + m - 1 chars starting anywhere on it: its
    # k-mer set (the windows of the circular string) is the same
    if len(da) != len(db):
        return None
    if set(_kmers_of(da, k)) != set(_kmers_of(db, k)):
        return None
    return da, db


def fullsize(name: str, workdir: str, with_reference: bool) -> None:
    import json
    import time

    import numpy as np

    from oracle import oracle as O
    fn, kw, k, l = FULLSIZE[name]
    os.makedirs(workdir, exist_ok=True)
    path = os.path.join(workdir, f"{name}.txt")
    t0 = time.time()
    if not os.path.exists(path):
        write_text(fn, kw, k, path + ".part")
        os.replace(path + ".part", path)
    print(name, "text", os.path.getsize(path), "bytes", f"{time.time() - t0:.0f} s", flush=True)
    results = {}
    t0 = time.time()
    text = np.memmap(path, dtype=np.uint8, mode="r")
    out, size, n, cyc = O.compact_mapped(text.ctypes.data, text.size, k)
    del text
    try:
        nl, h = sorted_digest(out, size)
    finally:
        O.free(out)
    results["oracle"] = {"n_kmers": n, "n_lines": nl, "bytes": size, "sha256_sorted_lines": h, "cycles": cyc}
    print(name, "oracle", results["oracle"], f"{time.time() - t0:.0f} s", flush=True)
    if with_reference:
        outp = os.path.join(workdir, f"{name}.ref.out")
        if os.path.exists(outp):
            os.remove(outp)  # the reference appends
        t0 = time.time()
        env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()), OMP_PROC_BIND="spread", KSHIM_SEED="7")
        r = subprocess.run([REF_OMP, path, str(k), str(l), outp], check=True, capture_output=True, env=env)
        ref = np.memmap(outp, dtype=np.uint8, mode="r")
        nl, h = sorted_digest(ref.ctypes.data, ref.size)
        results["reference"] = {"n_kmers": n, "n_lines": nl, "bytes": int(ref.size), "sha256_sorted_lines": h}
        tot = [x for x in r.stdout.decode().splitlines() if "Total time" in x]
        print(name, "reference", results["reference"], f"{time.time() - t0:.0f} s", tot, flush=True)
        a, b = results["oracle"], results["reference"]
        if any(a[x] != b[x] for x in ("n_lines", "bytes", "sha256_sorted_lines")):
            # allowed only in the lines of isolated cycles, whose order the
            # reference leaves unspecified
            rb = _sorted_copy(ref.ctypes.data, ref.size)
            del ref
            text = np.memmap(path, dtype=np.uint8, mode="r")
            out, size, _, _ = O.compact_mapped(text.ctypes.data, text.size, k)
            del text
            try:
                ob = _sorted_copy(out, size)
            finally:
                O.free(out)
            d = cycle_only_difference(ob, rb, k, results["oracle"]["cycles"])
            if d is None:
                raise SystemExit(f"{name}: oracle and reference disagree beyond cycle lines: {a} vs {b}")
            results["reference"]["differs_only_in_cycle_lines"] = len(d[0])
            print(name, "reference differs from the oracle only in", len(d[0]), "cycle line(s):",
                  [x[:80] for x in d[0]], [x[:80] for x in d[1]], flush=True)
        else:
            del ref
        os.remove(outp)
    dst = os.path.join(HERE, "checksums_fullsize.json")
    sums = {}
    if os.path.exists(dst):
        with open(dst) as f:
            sums = json.load(f)
    o = results["oracle"]
    sums[name] = {"fn": fn, "kwargs": kw, "k": k, "l": l, "n_kmers": o["n_kmers"], "n_lines": o["n_lines"],
                  "bytes": o["bytes"], "sha256_sorted_lines": o["sha256_sorted_lines"], "cycles": o["cycles"],
                  "printed_by": sorted(results)}
    if "reference" in results:
        sums[name]["reference"] = results["reference"]
    with open(dst, "w") as f:
        json.dump(sums, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--fullsize", choices=sorted(FULLSIZE))
    ap.add_argument("--workdir", default=os.path.join(ROOT, "_data"))
    ap.add_argument("--reference", action="store_true")
    a = ap.parse_args()
    if a.fullsize:
        fullsize(a.fullsize, a.workdir, a.reference)
    else:
        main()
