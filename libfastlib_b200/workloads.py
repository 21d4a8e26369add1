"""Seeded synthetic inputs for the benchmark workloads.

Raw-WAH workload: bitvectors of 2^28 bits made of alternating 0/1 runs (a
0-run first) whose lengths are geometric — 1-runs with mean 8 bits, 0-runs
with mean 8(1-d)/d for set-bit density d — built the way the reference's
appendFill (src/bitvector.h:800) builds them: whole 31-bit groups become
literal words, runs of two or more all-0 / all-1 groups become fill words,
a single all-0 / all-1 group stays a literal, and the trailing bits form the
active word.
"""
from __future__ import annotations

import numpy as np

ALLONES = 0x7FFFFFFF


def geometric_runs(seed: int, nbits: int, density: float, mean1: float = 8.0) -> np.ndarray:
    """Alternating run lengths (0-run first) summing to nbits; PCG64 stream
    per seed, so the inputs are the same on every platform."""
    rng = np.random.Generator(np.random.PCG64(seed))
    mean0 = max(mean1 * (1.0 - density) / density, 1.0)
    parts = []
    total = 0
    chunk = max(1024, int(nbits / (mean0 + mean1)) + 1024)
    while total < nbits:
        inter = np.empty(2 * chunk, dtype=np.int64)
        inter[0::2] = rng.geometric(1.0 / mean0, size=chunk)
        inter[1::2] = rng.geometric(1.0 / mean1, size=chunk)
        cs = np.cumsum(inter)
        need = nbits - total
        cut = int(np.searchsorted(cs, need, side="left"))
        if cut < len(inter):
            inter = inter[: cut + 1]
            inter[-1] -= int(cs[cut]) - need
            parts.append(inter)
            total = nbits
        else:
            parts.append(inter)
            total += int(cs[-1])
    return np.concatenate(parts).astype(np.uint64)


def groups_from_runs(runs: np.ndarray, device: str = "cpu"):
    """Dense 31-bit group literals (first row = bit 30) and the trailing
    (active) bits of the bit sequence described by alternating runs."""
    import torch
    r = torch.as_tensor(np.asarray(runs, dtype=np.int64), device=device)
    nbits = int(r.sum().item())
    ends = torch.cumsum(r, 0)
    starts = ends - r
    ones = torch.arange(len(r), device=device) % 2 == 1
    delta = torch.zeros(nbits + 1, dtype=torch.int32, device=device)
    s1, e1 = starts[ones], ends[ones]
    delta.index_add_(0, s1, torch.ones_like(s1, dtype=torch.int32))
    delta.index_add_(0, e1, -torch.ones_like(e1, dtype=torch.int32))
    bits = torch.cumsum(delta[:nbits], 0, dtype=torch.int32)
    G = nbits // 31
    anb = nbits - 31 * G
    w = torch.pow(2, torch.arange(30, -1, -1, device=device, dtype=torch.int64))
    groups = (bits[: 31 * G].view(G, 31).to(torch.int64) * w).sum(1).to(torch.int64)
    aval = 0
    for k in range(anb):
        aval = (aval << 1) | int(bits[31 * G + k].item())
    return groups.cpu().numpy().astype(np.uint32), anb, aval


def canonical_wah(groups: np.ndarray, anb: int = 0, aval: int = 0) -> np.ndarray:
    """Serialized WAH of dense group literals in appendFill's form."""
    g = np.asarray(groups, dtype=np.uint32)
    if len(g) == 0:
        body = np.zeros(0, np.uint32)
    else:
        cls = np.where(g == 0, 0, np.where(g == ALLONES, 1, 2)).astype(np.int8)
        # a new run starts where the class changes or at every mixed group
        head = np.ones(len(g), dtype=bool)
        head[1:] = (cls[1:] != cls[:-1]) | (cls[1:] == 2)
        hidx = np.flatnonzero(head)
        lens = np.diff(np.append(hidx, len(g)))
        hc = cls[hidx]
        body = g[hidx].copy()
        fill = (hc != 2) & (lens >= 2)
        body[fill] = np.where(hc[fill] == 1, 0xC0000000, 0x80000000).astype(np.uint32) | lens[fill].astype(np.uint32)
    tail = [aval & ((1 << anb) - 1), anb] if anb > 0 else [0]
    return np.concatenate([body, np.asarray(tail, dtype=np.uint32)])


def raw_wah_operand(seed: int, nbits: int, density: float, device: str = "cpu") -> np.ndarray:
    groups, anb, aval = groups_from_runs(geometric_runs(seed, nbits, density), device)
    return canonical_wah(groups, anb, aval)


# ---------------------------------------------------------------- range workloads
# Columns are generated on the device with a seeded torch generator, so a
# workload is the same on every run of the same GPU model.

def _gen(seed: int, device: str):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return g


def zipf_column(seed: int, n: int, s: float, ranks: int, device: str = "cuda"):
    """Ranks 1..`ranks` drawn with P(k) ~ k^-s (inverse CDF), as float64."""
    import torch
    g = _gen(seed, device)
    k = torch.arange(1, ranks + 1, device=device, dtype=torch.float64)
    cdf = torch.cumsum(k.pow(-s), 0)
    cdf /= cdf[-1].clone()
    u = torch.rand(n, generator=g, device=device, dtype=torch.float64)
    return (torch.searchsorted(cdf, u).clamp_(max=ranks - 1) + 1).to(torch.float64)


def mixture_column(seed: int, n: int, device: str = "cuda"):
    """float32: with probability 0.7 Normal(0, 1), else a Zipf(1.2) rank over
    10^5 values (the binned range workload's column)."""
    import torch
    g = _gen(seed, device)
    norm = torch.randn(n, generator=g, device=device, dtype=torch.float32)
    pick = torch.rand(n, generator=g, device=device) < 0.7
    z = zipf_column(seed + 1, n, 1.2, 100_000, device).to(torch.float32)
    return torch.where(pick, norm, z)


def uniform_int_column(seed: int, n: int, card: int, device: str = "cuda", dtype=None):
    import torch
    g = _gen(seed, device)
    t = torch.randint(0, card, (n,), generator=g, device=device, dtype=torch.int64)
    return t.to(dtype or torch.int32)


def normal_column(seed: int, n: int, device: str = "cuda"):
    import torch
    return torch.randn(n, generator=_gen(seed, device), device=device, dtype=torch.float32)


def bin_edge_term(rng, keys: np.ndarray, nobs: int, span: int):
    """A range over `span` consecutive bins whose two ends fall inside the
    first and last bin (so both edge bins need row checks): (lo, hi) for
    lo <= x < hi."""
    span = max(1, min(span, nobs - 2))
    b = int(rng.integers(1, max(2, nobs - span)))
    e = min(b + span - 1, nobs - 1)
    mn, mx = keys[:nobs], keys[nobs:]
    lo = mn[b] + rng.random() * (mx[b] - mn[b])
    hi = mn[e] + rng.random() * (mx[e] - mn[e])
    if hi <= lo:
        hi = np.nextafter(lo, np.inf)
    return float(lo), float(hi)


def binned_range_queries(seed: int, keys: np.ndarray, nobs: int, nq: int = 1000, max_span: int = 500):
    """The binned range workload's queries: bin span uniform in [1, max_span],
    start bin uniform, both ends jittered inside their edge bins."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [bin_edge_term(rng, keys, nobs, int(rng.integers(1, max_span + 1))) for _ in range(nq)]


def conjunctive_queries(seed: int, columns, nq: int, max_terms: int = 4):
    """WHERE clauses of 1..max_terms distinct columns, each a range of uneven
    span.  columns: list of dicts {kind: 'relic'|'bin', card | (keys, nobs)};
    returns [[(column, lo, hi), ...], ...] for lo <= x < hi."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(nq):
        k = int(rng.integers(1, max_terms + 1))
        cols = rng.choice(len(columns), size=min(k, len(columns)), replace=False)
        q = []
        for c in cols:
            col = columns[int(c)]
            if col["kind"] == "relic":
                card = col["card"]
                span = int(rng.integers(1, max(2, card // 2 + 1)))
                lo = int(rng.integers(0, max(1, card - span + 1)))
                q.append((int(c), float(lo), float(lo + span)))
            else:
                span = int(rng.integers(1, col.get("max_span", 256) + 1))
                q.append((int(c),) + bin_edge_term(rng, col["keys"], col["nobs"], span))
        out.append(q)
    return out
