"""A CPU model of the two-pass group-space engine (libfastlib_b200/csrc/
wah_gop.cuh: k_gop, k_gpack) checked against the oracle: the word range of
each 512-group tile from the group-tile index, word placement by start
markers and a running maximum, the dense result patterns, the run heads
(with the group before the tile), the per-segment totals that give each
tile its output offset and the next head after it, and the words and bpos
entries written from them.  It mirrors the kernels' index arithmetic at tile
granularity (not their lanes), so a change to that arithmetic can be tried
here before it runs on a GPU."""
import numpy as np
import pytest

import oracle
from oracle import wahgen as G

ALL, H0, H1, MAXC = 0x7FFFFFFF, 0x80000000, 0xC0000000, 0x3FFFFFFF
DT = GT = 512           # group-tile index stride = groups per tile
NCH = GT // 128         # chunks of 128 groups per tile
GWS = (GT + 4 + 31) // 32 * 32  # staged words per operand
SEG = 256               # tiles per segment
NONE = 0xFFFFFFFF


def wgroups(w):
    return np.where(w > ALL, w & MAXC, 1).astype(np.int64)


def wpattern(w):
    return np.where(w > ALL, np.where(w >= H1, ALL, 0), w).astype(np.int64)


def gtile(w, groups):
    """k_gtile: (word covering group k*DT, its first group), k = 0..ceil(G/DT)."""
    starts = np.concatenate([[0], np.cumsum(wgroups(w))])
    nt = (groups + DT - 1) // DT
    out = []
    for k in range(nt + 1):
        g = k * DT
        if g >= groups:
            out.append((len(w), groups))
        else:
            i = int(np.searchsorted(starts, g, side="right") - 1)
            out.append((i, int(starts[i])))
    return out


def tile_patterns(w, gt, g0, g1):
    """gop_range + gop_mark + gop_chunk: the pattern of every group of the
    tile, and of the group before it."""
    n, ng = len(w), g1 - g0
    wi0, s0 = gt[g0 // DT]
    wi1, s1 = gt[(g1 + DT - 1) // DT]
    wend = wi1 + 1 if (wi1 < n and s1 < g1) else wi1
    nw = wend - wi0
    assert 0 < nw <= GT and wend <= n
    prev = None
    if g0 > 0:
        prev = int(wpattern(np.array([w[wi0 if s0 < g0 else wi0 - 1]]))[0])
    ws = w[wi0:wend]
    if s0 == g0 and nw == ng:                       # pure: one word per group
        pat = np.zeros(GT, np.int64)
        pat[:nw] = wpattern(ws)
        return pat, prev
    c = wgroups(ws)
    p = s0 + np.concatenate([[0], np.cumsum(c)[:-1]])
    keep = (p < g1) & (p + c > g0)
    mk = np.zeros(GT, np.int64)
    mk[np.maximum(p[keep], g0) - g0] = np.nonzero(keep)[0] + 1
    idx = np.maximum.accumulate(mk)                # >= 1 inside the tile
    return wpattern(ws[np.maximum(idx, 1) - 1]), prev


def apply(op, a, b):
    return [a & b, a | b, a ^ b, a & ~b & ALL][op]


def cls(v):
    return np.where(v == 0, 0, np.where(v == ALL, 1, 2))


def gpack_lanes(head, g0, cnt, nxt):
    """k_gpack's lane arithmetic for one tile: head[i] is True for the run
    heads among the tile's GT groups (lane l of chunk j holds groups
    128 j + 4 l .. + 3).  Chunks are taken last to first; a lane's first
    output index is the heads of the chunks before (the tile's count minus
    the chunks already taken) plus those of the lanes before it (from the
    bits of each lane's 0..4 count), and the head after its last one is the
    first head of the nearest higher lane holding one, else the first head
    after the chunk.  Returns {group: (output index within the tile, next
    head)}."""
    hm = [0] * 32
    for i in range(GT):
        if head[i]:
            j, rem = divmod(i, 128)
            hm[rem // 4] |= 1 << (4 * j + rem % 4)
    out = {}
    later, rest = nxt, cnt
    for j in range(NCH - 1, -1, -1):
        m = [(hm[l] >> (4 * j)) & 15 for l in range(32)]
        hl = sum(1 << l for l in range(32) if m[l])
        if hl == 0:
            continue
        nh = [bin(x).count("1") for x in m]
        ballots = [sum(1 << l for l in range(32) if nh[l] & bit) for bit in (1, 2, 4)]
        rest -= sum(bin(b).count("1") << k for k, b in enumerate(ballots))
        assert rest >= 0
        mine = [g0 + 128 * j + 4 * l + ((m[l] & -m[l]).bit_length() - 1) if m[l] else NONE for l in range(32)]
        for l in range(32):
            lt = (1 << l) - 1
            o = rest + sum(bin(b & lt).count("1") << k for k, b in enumerate(ballots))
            above = hl & ~((2 << l) - 1) & 0xFFFFFFFF
            after = mine[(above & -above).bit_length() - 1] if above else later
            for e in range(4):
                if (m[l] >> e) & 1:
                    more = m[l] >> (e + 1)
                    g = g0 + 128 * j + 4 * l + e
                    nx = g + ((more & -more).bit_length()) if more else after
                    out[g] = (o, nx)
                    o += 1
        later = mine[(hl & -hl).bit_length() - 1]
    return out


def two_pass(op, wa, wb, groups):
    """Words and bpos of the engine's result (whole words only)."""
    wa, wb = np.asarray(wa, np.int64), np.asarray(wb, np.int64)
    ga, gb = gtile(wa, groups), gtile(wb, groups)
    T = (groups + GT - 1) // GT
    R = np.zeros(T * GT, np.int64)
    tiles = []                                     # (heads, first, popc)
    for t in range(T):
        g0 = t * GT
        g1 = min(g0 + GT, groups)
        ng = g1 - g0
        pa, xp = tile_patterns(wa, ga, g0, g1)
        pb, yp = tile_patterns(wb, gb, g0, g1)
        r = apply(op, pa, pb)
        R[g0:g0 + GT] = r
        c = cls(r[:ng])
        before = np.concatenate([[cls(np.array([apply(op, xp, yp)]))[0] if g0 else -1], c[:-1]])
        head = (c == 2) | (c != before)
        if g0 == 0:
            head[0] = True
        pos = np.nonzero(head)[0]
        tiles.append((len(pos), g0 + int(pos[0]) if len(pos) else NONE,
                      int(sum(bin(int(v)).count("1") for v in r[:ng]))))
    nseg = (T + SEG - 1) // SEG
    segs = [[0, 0] for _ in range(nseg)]           # heads, NONE - first (0: none)
    for t, (h, f, _) in enumerate(tiles):
        segs[t // SEG][0] += h
        if f != NONE:
            segs[t // SEG][1] = max(segs[t // SEG][1], NONE - f)
    n = sum(h for h, _, _ in tiles)
    out = np.zeros(n, np.int64)
    bpos = {(n + 31) // 32: groups}
    for t, (cnt, _, _) in enumerate(tiles):
        sg = t // SEG
        off = sum(s[0] for s in segs[:sg]) + sum(x[0] for x in tiles[sg * SEG:t])
        if cnt == 0:
            continue
        nxt = NONE
        for i in range(t + 1, min(T, (sg + 1) * SEG)):
            if tiles[i][1] != NONE:
                nxt = tiles[i][1]
                break
        if nxt == NONE:
            for i in range(sg + 1, nseg):
                if segs[i][1]:
                    nxt = NONE - segs[i][1]
                    break
        if nxt == NONE:
            nxt = groups
        g0 = t * GT
        g1 = min(g0 + GT, groups)
        r = R[g0:g1]
        c = cls(r)
        prevc = cls(np.array([R[g0 - 1]]))[0] if g0 else -1
        before = np.concatenate([[prevc], c[:-1]])
        head = (c == 2) | (c != before)
        if g0 == 0:
            head[0] = True
        pos = np.nonzero(head)[0]
        lanes = gpack_lanes(np.concatenate([head, np.zeros(GT - len(head), bool)]), g0, cnt, nxt)
        assert sorted(lanes) == [g0 + int(p) for p in pos]
        for k, p in enumerate(pos):
            nx = g0 + pos[k + 1] if k + 1 < len(pos) else nxt
            assert lanes[g0 + int(p)] == (k, nx), (t, p)
            length = nx - (g0 + p)
            if c[p] == 2:
                wd = r[p]
            elif length >= 2:
                wd = (H1 if c[p] else H0) | length
            else:
                wd = ALL if c[p] else 0
            o = off + k
            out[o] = wd
            if o % 32 == 0:
                bpos[o // 32] = g0 + p
    return out, bpos, sum(x[2] for x in tiles)


def _dense_words(rng, ngroups):
    words, g = [], 0
    while g < ngroups:
        left = ngroups - g
        if rng.random() < 0.3:
            c = int(min(left, rng.integers(1, 3000)))
            words.append(G.fill(int(rng.integers(0, 2)), c))
            g += c
            continue
        k = int(min(left, rng.integers(1, 2500)))
        lit = rng.integers(1, ALL, size=k, dtype=np.int64)
        r = rng.random(k)
        lit[r < 0.02] = 0
        lit[(r >= 0.02) & (r < 0.04)] = ALL
        out = [int(x) for x in lit]
        for i in np.nonzero(r > 0.995)[0]:
            out[i] = G.fill(int(rng.integers(0, 2)), 1)
        words.extend(out)
        g += k
    return words


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_model_equals_oracle(seed):
    rng = np.random.default_rng(seed)
    checked = 0
    for trial in range(6):
        ng = int(rng.integers(1, 5)) * 1024 + int(rng.integers(0, 1024)) if trial % 3 else int(rng.integers(1, 900))
        wa, wb = _dense_words(rng, ng), _dense_words(rng, ng)
        if len(wa) + len(wb) <= ng:      # not the canonical-result path
            continue
        anb = int(rng.integers(0, 31))
        a = G.serialize(wa, anb, int(rng.integers(0, 1 << 31)))
        b = G.serialize(wb, anb, int(rng.integers(0, 1 << 31)))
        if oracle.is_degenerate(a) or oracle.is_degenerate(b):
            continue
        for op in range(4):
            ref, _ = oracle.binop(op, a, b, inplace=False)
            body = ref[:-1] if ref[-1] == 0 else ref[:-2]
            words, bpos, _ = two_pass(op, wa, wb, ng)
            assert np.array_equal(words, body.astype(np.int64)), (seed, trial, op)
            starts = np.concatenate([[0], np.cumsum(wgroups(words))])
            for k, g in bpos.items():
                assert g == (starts[32 * k] if 32 * k < len(words) else ng), (seed, trial, op, k)
            checked += 1
    assert checked > 0


def test_segments_span_many_tiles():
    """More than one segment of tiles, and a long 0-fill that leaves tiles
    without heads, so offsets and next heads cross segments."""
    ng = (SEG + 40) * GT
    wa = [G.fill(0, ng // 2)] + [0x1234567] * 5 + [G.fill(0, ng - ng // 2 - 5)]
    wb = [0x2AAAAAAA] * ng
    a, b = G.serialize(wa, 3, 5), G.serialize(wb, 3, 2)
    for op in (1, 2):
        ref, _ = oracle.binop(op, a, b, inplace=False)
        body = ref[:-1] if ref[-1] == 0 else ref[:-2]
        words, _, _ = two_pass(op, wa, wb, ng)
        assert np.array_equal(words, body.astype(np.int64)), op


def stage_copies(wi0, nw, n):
    """gop_stage's copies for words [wi0, wi0 + nw) of an n-word array:
    (shared index, global word, words) per copy."""
    a0, end = wi0 & ~3, wi0 + nw
    nfull = min((end - a0 + 3) // 4, (n - a0) // 4)
    copies = [(4 * c, a0 + 4 * c, 4) for c in range(nfull)]
    copies += [(i - a0, i, 1) for i in range(a0 + 4 * nfull, end)]
    return a0, copies


def test_stage_arithmetic():
    """16-byte copies start on 16-byte boundaries on both sides, no copy
    reads past the array, every word of the tile lands at ws[k + (wi0 & 3)]
    and the staging buffer (GWS words) is never overrun."""
    rng = np.random.default_rng(3)
    cases = [(w, nw, n) for n in (1, 2, 3, 4, 5, 7, 8, 512, 513, 515, 1024, 1025, 1027, 5000)
             for w in range(0, min(n, 9)) for nw in (1, 2, 3, 4, 5, n - w) if 0 < nw <= min(GT, n - w)]
    for _ in range(3000):
        n = int(rng.integers(1, 40000))
        w = int(rng.integers(0, n))
        cases.append((w, int(rng.integers(1, min(GT, n - w) + 1)), n))
    for wi0, nw, n in cases:
        a0, copies = stage_copies(wi0, nw, n)
        ws = {}
        for si, gi, k in copies:
            if k == 4:
                assert si % 4 == 0 and gi % 4 == 0
            assert gi + k <= n and si + k <= GWS, (wi0, nw, n)
            for e in range(k):
                ws[si + e] = gi + e
        for kk in range(nw):
            assert ws[kk + (wi0 & 3)] == wi0 + kk, (wi0, nw, n, kk)
