"""Seeded synthetic k-mer inputs in the reference's text format.

The reference names no dataset; its README says the input comes from a k-mer
counter (KMC) dumped as text with a count header (README.md:3-4,
driver.cpp:251-256).  These generators build genomes with the shapes the
workloads call for (i.i.d. bases at a GC content, SNP bubbles, repeat families,
tandem repeats), extract every k-mer of both haplotypes, keep the
lexicographically smaller of each k-mer and its reverse complement, drop
duplicates, shuffle, and format one k-mer per line under a count line.

Randomness is counter based (splitmix64 of (seed, stream, index)) and all
arithmetic is int64 torch, so the same call gives the same bytes on the CPU
and on a GPU.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import torch

M64 = (1 << 64) - 1
_LUT = torch.tensor([ord("A"), ord("C"), ord("G"), ord("T")], dtype=torch.uint8)


def _i64(v: int) -> int:
    v &= M64
    return v - (1 << 64) if v >= (1 << 63) else v


def _srl(x: torch.Tensor, s: int) -> torch.Tensor:
    """Logical right shift of int64 viewed as uint64."""
    return (x >> s) & ((1 << (64 - s)) - 1)


def _mix(z: torch.Tensor) -> torch.Tensor:
    z = (z ^ _srl(z, 30)) * _i64(0xBF58476D1CE4E5B9)
    z = (z ^ _srl(z, 27)) * _i64(0x94D049BB133111EB)
    return z ^ _srl(z, 31)


def rand_u64(seed: int, stream: int, idx: torch.Tensor) -> torch.Tensor:
    """splitmix64 output for counter idx of (seed, stream), as int64 bits."""
    base = _i64((seed * 0x9E3779B97F4A7C15 + stream * 0xD1B54A32D192ED03 + 0x632BE59BD9B4E019))
    z = idx.to(torch.int64) * _i64(0x9E3779B97F4A7C15) + base
    return _mix(z)


def rand_unit(seed: int, stream: int, idx: torch.Tensor) -> torch.Tensor:
    """Uniform float64 in [0, 1)."""
    return _srl(rand_u64(seed, stream, idx), 11).to(torch.float64) * (1.0 / (1 << 53))


def rand_int(seed: int, stream: int, idx: torch.Tensor, lo: int, hi: int) -> torch.Tensor:
    """Uniform integers in [lo, hi]."""
    u = rand_unit(seed, stream, idx)
    return (lo + torch.floor(u * (hi - lo + 1))).to(torch.int64).clamp_(lo, hi)


class _Stream:
    """Sequential scalar draws for the host-side layout decisions."""

    def __init__(self, seed: int, stream: int):
        self.seed, self.stream, self.i = seed, stream, 0

    def _next(self) -> int:
        t = torch.tensor([self.i], dtype=torch.int64)
        self.i += 1
        return int(rand_u64(self.seed, self.stream, t)[0]) & M64

    def unit(self) -> float:
        return (self._next() >> 11) * (1.0 / (1 << 53))

    def randint(self, lo: int, hi: int) -> int:
        return min(hi, lo + int(self.unit() * (hi - lo + 1)))


_CHUNK = 1 << 26  # elements per pass of the per-position draws (bounds peak memory)


def random_bases(n: int, gc: float, seed: int, stream: int, device, offset: int = 0) -> torch.Tensor:
    """i.i.d. bases (0..3 = A,C,G,T) with P(C)=P(G)=gc/2.  Each base depends
    only on its own counter, so the draws run in chunks of _CHUNK positions."""
    out = torch.empty(n, dtype=torch.uint8, device=device)
    for c0 in range(0, n, _CHUNK):
        c1 = min(n, c0 + _CHUNK)
        idx = torch.arange(offset + c0, offset + c1, device=device, dtype=torch.int64)
        u = rand_unit(seed, stream, idx)
        gc_side = u < gc
        v = torch.where(gc_side, u / max(gc, 1e-300), (u - gc) / max(1.0 - gc, 1e-300))
        hi_half = v >= 0.5
        # GC side: C (1) / G (2); AT side: A (0) / T (3)
        b = torch.where(gc_side, torch.where(hi_half, 2, 1), torch.where(hi_half, 3, 0))
        out[c0:c1] = b.to(torch.uint8)
    return out


def _mutate(seq: torch.Tensor, rate: float, seed: int, stream: int, offset: int = 0) -> torch.Tensor:
    """Point mutations: each base changes with probability rate to a different base."""
    idx = torch.arange(offset, offset + seq.numel(), device=seq.device, dtype=torch.int64)
    hit = rand_unit(seed, stream, idx) < rate
    shift = rand_int(seed, stream + 1, idx, 1, 3).to(torch.uint8)
    out = seq.clone().view(-1)
    out[hit.view(-1)] = (out.view(-1)[hit.view(-1)] + shift.view(-1)[hit.view(-1)]) % 4
    return out.view(seq.shape)


@dataclass
class GenomeSpec:
    length: int
    gc: float = 0.5
    seed: int = 1
    snp_count: int | None = None      # exact number of SNP positions (second allele)
    snp_rate: float = 0.0             # else a rate
    repeat_frac: float = 0.0          # repeat families (interspersed)
    repeat_len: tuple = (300, 6000)
    repeat_copies: tuple = (2, 50)
    repeat_mut: tuple = (0.01, 0.03)
    tandem_frac: float = 0.0          # tandem repeats
    tandem_unit: tuple = (2, 200)
    tandem_copies: tuple = (5, 100)
    extra: dict = field(default_factory=dict)


def make_genome(spec: GenomeSpec, device="cpu"):
    """Returns (haplotype-1 bases, SNP positions, SNP alt bases)."""
    L = spec.length
    g = random_bases(L, spec.gc, spec.seed, 1, device)
    rng = _Stream(spec.seed, 2)
    if spec.repeat_frac > 0:
        target = int(spec.repeat_frac * L)
        placed, fam = 0, 0
        while placed < target:
            flen = rng.randint(*spec.repeat_len)
            if flen >= L:
                break
            copies = rng.randint(*spec.repeat_copies)
            mut = spec.repeat_mut[0] + rng.unit() * (spec.repeat_mut[1] - spec.repeat_mut[0])
            unit = random_bases(flen, spec.gc, spec.seed, 1000 + 7 * fam, device)
            pos = [rng.randint(0, L - flen) for _ in range(copies)]
            reps = unit.unsqueeze(0).expand(copies, flen)
            reps = _mutate(reps.contiguous(), mut, spec.seed, 1003 + 7 * fam)
            for c, p in enumerate(pos):
                g[p:p + flen] = reps[c]
            placed += copies * flen
            fam += 1
    if spec.tandem_frac > 0:
        target = int(spec.tandem_frac * L)
        placed, t = 0, 0
        while placed < target:
            ulen = rng.randint(*spec.tandem_unit)
            copies = rng.randint(*spec.tandem_copies)
            tot = ulen * copies
            if tot >= L:
                t += 1
                continue
            unit = random_bases(ulen, spec.gc, spec.seed, 500000 + 3 * t, device)
            # homopolymer units make a k-mer whose only edge is a self-loop
            if ulen == 1 or bool((unit == unit[0]).all()):
                unit[-1] = (unit[0] + 1) % 4
            p = rng.randint(0, L - tot)
            g[p:p + tot] = unit.repeat(copies)
            placed += tot
            t += 1
    if spec.snp_count is not None:
        m = spec.snp_count
        idx = torch.arange(m, device=device, dtype=torch.int64)
        pos = rand_int(spec.seed, 3, idx, 0, L - 1)
    elif spec.snp_rate > 0:
        hits = []
        for c0 in range(0, L, _CHUNK):
            idx = torch.arange(c0, min(L, c0 + _CHUNK), device=device, dtype=torch.int64)
            hits.append(torch.nonzero(rand_unit(spec.seed, 3, idx) < spec.snp_rate).flatten() + c0)
        pos = torch.cat(hits)
    else:
        pos = torch.zeros(0, dtype=torch.int64, device=device)
    pos = torch.unique(pos)
    alt = ((g[pos].to(torch.int64) + rand_int(spec.seed, 4, pos, 1, 3)) % 4).to(torch.uint8)
    return g, pos, alt


def _windows_be(codes: torch.Tensor, starts: torch.Tensor, k: int, rc: bool):
    """Big-endian packed k-mer values (first char in the top bits) of the
    windows codes[s : s+k], or of their reverse complements.  k <= 31 -> one
    int64 tensor; k <= 63 -> (hi: chars 0..31 with the sign bit flipped so
    signed order is unsigned order, lo: chars 32..k-1)."""
    def part(j0, j1):
        v = torch.zeros(starts.numel(), dtype=torch.int64, device=codes.device)
        for j in range(j0, j1):
            if rc:
                c = 3 - codes[starts + (k - 1 - j)].to(torch.int64)
            else:
                c = codes[starts + j].to(torch.int64)
            v = (v << 2) | c
        return v
    if k <= 31:
        return part(0, k)
    hi = part(0, 32) ^ (-(1 << 63))
    lo = part(32, k)
    return hi, lo


def canonical_kmers(g: torch.Tensor, pos: torch.Tensor, alt: torch.Tensor, k: int, chunk: int = 1 << 26):
    """Distinct canonical k-mers of both haplotypes, sorted (lexicographic)."""
    L = g.numel()
    dev = g.device
    parts = []

    def add(codes, starts):
        for s in range(0, starts.numel(), chunk):
            st = starts[s:s + chunk]
            f = _windows_be(codes, st, k, False)
            r = _windows_be(codes, st, k, True)
            if k <= 31:
                parts.append(torch.minimum(f, r))
            else:
                use_f = (f[0] < r[0]) | ((f[0] == r[0]) & (f[1] <= r[1]))
                parts.append(torch.stack([torch.where(use_f, f[0], r[0]), torch.where(use_f, f[1], r[1])], 1))

    if L >= k:
        add(g, torch.arange(0, L - k + 1, device=dev, dtype=torch.int64))
    if pos.numel() > 0 and L >= k:
        g2 = g.clone()
        g2[pos] = alt
        off = torch.arange(-(k - 1), 1, device=dev, dtype=torch.int64)
        st = (pos.unsqueeze(1) + off.unsqueeze(0)).flatten()
        st = torch.unique(st[(st >= 0) & (st <= L - k)])
        add(g2, st)
    if k <= 31:
        allv = torch.cat(parts) if parts else torch.zeros(0, dtype=torch.int64, device=dev)
        return torch.unique(allv)
    allv = torch.cat(parts, 0) if parts else torch.zeros((0, 2), dtype=torch.int64, device=dev)
    return _unique_rows(allv)


def _unique_rows(a: torch.Tensor) -> torch.Tensor:
    o = torch.argsort(a[:, 1], stable=True)
    a = a[o]
    o = torch.argsort(a[:, 0], stable=True)
    a = a[o]
    if a.shape[0] == 0:
        return a
    keep = torch.ones(a.shape[0], dtype=torch.bool, device=a.device)
    keep[1:] = (a[1:, 0] != a[:-1, 0]) | (a[1:, 1] != a[:-1, 1])
    return a[keep]


def drop_homopolymers(kmers: torch.Tensor, k: int) -> torch.Tensor:
    """Remove A^k and C^k (the only canonical homopolymers): the reference
    spins forever on a k-mer whose only kept edge is a self-loop."""
    if k <= 31:
        cpoly = 0
        for _ in range(k):
            cpoly = (cpoly << 2) | 1
        return kmers[(kmers != 0) & (kmers != cpoly)]
    c_hi = 0
    for _ in range(32):
        c_hi = (c_hi << 2) | 1
    c_lo = 0
    for _ in range(k - 32):
        c_lo = (c_lo << 2) | 1
    a_row = (kmers[:, 0] == (-(1 << 63))) & (kmers[:, 1] == 0)
    c_row = (kmers[:, 0] == (_i64(c_hi) ^ (-(1 << 63)))) & (kmers[:, 1] == c_lo)
    return kmers[~(a_row | c_row)]


def shuffle(kmers: torch.Tensor, seed: int) -> torch.Tensor:
    if kmers.dim() == 1:
        key = _mix(kmers ^ _i64(seed * 0xA24BAED4963EE407 + 1))
    else:
        key = _mix(_mix(kmers[:, 0] ^ _i64(seed * 0xA24BAED4963EE407 + 1)) ^ kmers[:, 1])
    return kmers[torch.argsort(key)]


def kmers_to_lines(kmers: torch.Tensor, k: int) -> torch.Tensor:
    """uint8 (n, k+1): k chars then '\\n'."""
    n = kmers.shape[0]
    out = torch.empty((n, k + 1), dtype=torch.uint8, device=kmers.device)
    lut = _LUT.to(kmers.device)
    if k <= 31:
        for j in range(k):
            out[:, j] = lut[_srl(kmers, 2 * (k - 1 - j)) & 3]
    else:
        hi = kmers[:, 0] ^ (-(1 << 63))
        lo = kmers[:, 1]
        for j in range(32):
            out[:, j] = lut[_srl(hi, 2 * (31 - j)) & 3]
        for j in range(32, k):
            out[:, j] = lut[_srl(lo, 2 * (k - 1 - j)) & 3]
    out[:, k] = ord("\n")
    return out


def format_text(kmers: torch.Tensor, k: int) -> torch.Tensor:
    """The whole file as a flat uint8 tensor on kmers.device."""
    header = torch.tensor(list(f"{kmers.shape[0]}\n".encode()), dtype=torch.uint8, device=kmers.device)
    return torch.cat([header, kmers_to_lines(kmers, k).flatten()])


def kmer_set(spec: GenomeSpec, k: int, device="cpu") -> torch.Tensor:
    g, pos, alt = make_genome(spec, device)
    km = canonical_kmers(g, pos, alt, k)
    km = drop_homopolymers(km, k)
    return shuffle(km, spec.seed)


def make_text(spec: GenomeSpec, k: int, device="cpu") -> torch.Tensor:
    return format_text(kmer_set(spec, k, device), k)


# ----------------------------------------------------------------- workloads

def small_plain(seed: int = 1, length: int = 1_000_000) -> GenomeSpec:
    """1 Mbp i.i.d. uniform genome with 200 SNP bubbles (k=31, ~1M k-mers)."""
    return GenomeSpec(length=length, gc=0.5, seed=seed, snp_count=200)


def scale_plain(length: int = 1_000_000_000, seed: int = 2) -> GenomeSpec:
    """41% GC genome with 5% repeat families (300 bp-6 kb, 2-50 copies,
    1-3% mutations per copy) and 0.1% SNPs (k=31; ~1B k-mers at 1 Gbp)."""
    return GenomeSpec(length=length, gc=0.41, seed=seed, snp_rate=0.001, repeat_frac=0.05)


def wide_k(length: int = 200_000_000, seed: int = 3) -> GenomeSpec:
    """50% GC genome with 3% tandem repeats (unit 2-200 bp, 5-100 copies) and
    0.05% SNPs (k=63; ~200M k-mers at 200 Mbp)."""
    return GenomeSpec(length=length, gc=0.5, seed=seed, snp_rate=0.0005, tandem_frac=0.03)


def batched_job(job: int, seed: int = 4, scale: float = 1.0) -> GenomeSpec:
    """One job of the many-small-jobs workload: log-normal length (median
    3 Mbp, clamped to 0.5-8 Mbp), GC uniform in [0.3, 0.7], 0.2% SNPs."""
    r = _Stream(seed * 1_000_003 + job, 9)
    u1, u2 = max(r.unit(), 1e-12), r.unit()
    z = math.sqrt(-2 * math.log(u1)) * math.cos(2 * math.pi * u2)
    length = int(min(8e6, max(5e5, 3e6 * math.exp(0.6 * z))) * scale)
    gc = 0.3 + 0.4 * r.unit()
    return GenomeSpec(length=max(length, 1000), gc=gc, seed=seed * 7919 + job, snp_rate=0.002)


def served_job(job: int, seed: int = 5, scale: float = 1.0):
    """One request of the serving workload: k-mer count log-uniform in
    [10k, 50M] (genome length ~ count), k = 31 (p=0.7) or 63 (p=0.3)."""
    r = _Stream(seed * 1_000_003 + job, 11)
    n = math.exp(math.log(1e4) + r.unit() * (math.log(5e7) - math.log(1e4)))
    k = 31 if r.unit() < 0.7 else 63
    gc = 0.3 + 0.4 * r.unit()
    return GenomeSpec(length=max(int(n * scale), 2000), gc=gc, seed=seed * 7919 + job, snp_rate=0.001), k
