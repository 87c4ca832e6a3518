"""Known-answer cases and text helpers shared by the CPU and GPU tests.

The expected lines of the micro cases are worked out by hand from the
reference's rules: a forward (k-1)-overlap edge u->v is kept iff v is u's only
successor and u is v's only predecessor (assembler.h:120-197); each maximal
path is written as its first k-mer followed by the last char of every later
k-mer (compact.h:192-206).  Cycles (no reference order exists, its
transpose_and_sort leaves them unordered) start at the smallest packed k-mer.
"""
from __future__ import annotations

import random


def text_of(kmers, extra: str = "", crlf: bool = False, header=None) -> bytes:
    nl = "\r\n" if crlf else "\n"
    h = len(kmers) if header is None else header
    return (f"{h}{nl}" + "".join(f"{x}{extra}{nl}" for x in kmers)).encode()


def walk_kmers(seq: str, k: int):
    return [seq[i:i + k] for i in range(len(seq) - k + 1)]


# (name, k, kmers, expected sorted lines)
MICRO = [
    ("single_path", 5, walk_kmers("ACGGTCATTGCAGTCCA", 5), ["ACGGTCATTGCAGTCCA"]),
    # AAC has two successors (ACG, ACT): both of its out-edges drop
    ("branch_out", 3, ["AAC", "ACG", "ACT", "CGT", "CTA"], ["AAC", "ACGT", "ACTA"]),
    # CGA has two predecessors: both in-edges drop
    ("branch_in", 3, ["ACG", "TCG", "CGA"], ["ACG", "CGA", "TCG"]),
    # ACG->CGA->GAC->ACG is a cycle; smallest packed key is CGA (1 + 2*4 = 9)
    ("cycle3", 3, ["GAC", "ACG", "CGA"], ["CGACG"]),
    # a homopolymer's only edge is a self-loop (the reference spins on it)
    ("self_loop", 3, ["AAA"], ["AAA"]),
    # duplicate prefix "CG" shared by CGA and CGT, and a chain TAC->ACG
    ("shared_prefix", 3, ["TAC", "ACG", "CGA", "CGT"], ["CGA", "CGT", "TACG"]),
    ("one_kmer", 31, ["ACGTACGTACGTACGTACGTACGTACGTACG"], ["ACGTACGTACGTACGTACGTACGTACGTACG"]),
]


def random_seq(n: int, seed: int) -> str:
    r = random.Random(seed)
    return "".join(r.choice("ACGT") for _ in range(n))


def distinct_path(length: int, k: int, seed: int) -> str:
    """A random sequence whose k-mers and (k-1)-mers are all distinct, so the
    whole sequence is one unitig."""
    s = seed
    while True:
        q = random_seq(length, s)
        km = walk_kmers(q, k)
        km1 = walk_kmers(q, k - 1)
        if len(set(km)) == len(km) and len(set(km1)) == len(km1):
            return q
        s += 1000


def shuffled(kmers, seed: int):
    x = list(kmers)
    random.Random(seed).shuffle(x)
    return x


def sorted_lines(data: bytes):
    s = data.split(b"\n")
    if s and s[-1] == b"":
        s = s[:-1]
    return sorted(s)


def cyclic_kmers(length: int, k: int, seed: int):
    """All k-mers of a random circular sequence with distinct (k-1)-mers: one
    isolated cycle of `length` k-mers."""
    s = seed
    while True:
        q = random_seq(length, s)
        ext = q + q[: k - 1]
        km = [ext[i:i + k] for i in range(length)]
        km1 = [ext[i:i + k - 1] for i in range(length)]
        if len(set(km)) == length and len(set(km1)) == length:
            return km
        s += 7919
