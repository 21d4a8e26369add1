"""A CPU model of the single-pass group-space engine (libfastlib_b200/csrc/
wah_fuse.cuh: k_gfuse) checked against the oracle.  It follows the kernel
thread by thread: the word slots loaded from the 16-byte boundary below each
tile's first word, the clipped word lengths and their packed (16-bit halves)
block scan, the painting of patterns into the transposed group arrays, the
group phase's heads and popcount with the group before each thread, the
{heads, last head, ones} scan and look-back, and the write phase in which
the next head writes a uniform run's word (deferred across tiles) and the
last tile the final run.  Every shared-memory and global index is asserted
in range, so a change to that arithmetic can be tried here before it runs
on a GPU.  A second model follows the write phase of the warp-tile engine
(wah_gone.cuh: k_gone) lane by lane and chunk by chunk."""
import numpy as np
import pytest

import oracle
from oracle import wahgen as G

ALL, H0, H1, MAXC = 0x7FFFFFFF, 0x80000000, 0xC0000000, 0x3FFFFFFF
DT = 512
FWPT, FGPT = 8, 8
C_ZERO, C_ONE, C_MIXED = 0, 1, 2


def shape(FT):
    """FCfg<FT>: warps for FT + 3 word slots, FT / 8 group-phase threads."""
    warps = (FT + 3 + FWPT * 32 - 1) // (FWPT * 32)
    return warps * 32, FT // FGPT, FT // FGPT


def wgroups(w):
    return (w & MAXC) if w > ALL else 1


def wpattern(w):
    return (ALL if w >= H1 else 0) if w > ALL else w


def cls_of(v):
    return C_ZERO if v == 0 else (C_ONE if v == ALL else C_MIXED)


def op2(op, a, b):
    return [a & b, a | b, a ^ b, a & ~b & ALL][op]


def fidx(q, FT):
    assert 0 <= q < FT
    return (q % FGPT) * (FT // FGPT) + q // FGPT


def gtile(w, groups):
    starts = np.concatenate([[0], np.cumsum([wgroups(int(x)) for x in w])]).astype(np.int64)
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


def fuse_range(gt, n, g0, g1, FT):
    wi0, s0 = gt[g0 // DT]
    wi1, s1 = gt[(g1 + DT - 1) // DT]
    wend = wi1 + 1 if (wi1 < n and s1 < g1) else wi1
    nw = wend - wi0
    assert wi0 < n and wend <= n and wend > wi0 and nw <= FT and s0 <= g0 and not (g0 > 0 and s0 == g0 and wi0 == 0)
    return wi0, s0, nw


def fuse_len(w, k, wi0, nw, s0, g0, g1, FT):
    if k < wi0 or k - wi0 >= nw:
        return 0
    c = wgroups(w)
    if k == wi0:
        c = min(s0 + c, g1) - g0
    return min(c, FT)


def run_word(c, ln):
    return ((H1 if c else H0) | ln) if ln >= 2 else (ALL if c else 0)


def model(op, xw, yw, groups, FT=2048):
    """The words k_gfuse<OP, FT> writes, and the popcount of m_vec."""
    FTHREADS, FGTHREADS, FROWS = shape(FT)
    xw = [int(v) for v in xw]
    yw = [int(v) for v in yw]
    nx, ny = len(xw), len(yw)
    gx, gy = gtile(xw, groups), gtile(yw, groups)
    ntiles = (groups + FT - 1) // FT
    cap = nx + ny
    out = [None] * cap
    recs = []  # inclusive prefix per tile (the look-back result)
    for t in range(ntiles):
        g0 = t * FT
        g1 = min(g0 + FT, groups)
        ng = g1 - g0
        xi0, xs0, xn = fuse_range(gx, nx, g0, g1, FT)
        yi0, ys0, yn = fuse_range(gy, ny, g0, g1, FT)
        pat = [[None] * FT, [None] * FT]
        run = 0
        for tid in range(FTHREADS):
            kx = (xi0 & ~3) + tid * FWPT
            ky = (yi0 & ~3) + tid * FWPT
            for j in range(FWPT):
                wxv = xw[kx + j] if kx + j < xi0 + xn else 0
                wyv = yw[ky + j] if ky + j < yi0 + yn else 0
                packed = fuse_len(wxv, kx + j, xi0, xn, xs0, g0, g1, FT) | (fuse_len(wyv, ky + j, yi0, yn, ys0, g0, g1, FT) << 16)
                ex = run
                run += packed
                assert (run & 0xFFFF) <= 2 * FT and (run >> 16) <= 2 * FT
                for o, (w, ln, q) in enumerate(((wxv, packed & 0xFFFF, ex & 0xFFFF), (wyv, packed >> 16, ex >> 16))):
                    if ln and q < ng:
                        for e in range(min(ln, ng - q)):
                            pat[o][fidx(q + e, FT)] = wpattern(w)
        for q in range(ng):
            assert pat[0][fidx(q, FT)] is not None and pat[1][fidx(q, FT)] is not None, (t, q)
        thr = []
        for tid in range(FGTHREADS):
            q0 = tid * FGPT
            if tid > 0:
                pr = op2(op, pat[0][fidx(q0 - 1, FT)] or 0, pat[1][fidx(q0 - 1, FT)] or 0)
            elif g0 > 0:
                pr = op2(op, wpattern(xw[xi0 if xs0 < g0 else xi0 - 1]), wpattern(yw[yi0 if ys0 < g0 else yi0 - 1]))
            else:
                pr = 0
            pc = cls_of(pr)
            hm, ones, lasth, r = 0, 0, 0, []
            for e in range(FGPT):
                q = q0 + e
                inr = q < ng
                rv = op2(op, pat[0][fidx(q, FT)] if inr else 0, pat[1][fidx(q, FT)] if inr else 0)
                r.append(rv)
                c = cls_of(rv)
                if inr:
                    if g0 + q == 0 or c == C_MIXED or c != pc:
                        hm |= 1 << e
                        lasth = ((g0 + q + 1) << 2) | c
                    ones += bin(rv).count("1")
                pc = c
            thr.append((hm, ones, lasth, r))
        exs = []
        acc = (0, 0, 0)
        for hm, ones, lasth, r in thr:
            exs.append(acc)
            acc = (acc[0] + bin(hm).count("1"), max(acc[1], lasth), acc[2] + ones)
        tot = acc
        pre = recs[-1] if recs else (0, 0, 0)
        recs.append((pre[0] + tot[0], max(pre[1], tot[1]), pre[2] + tot[2]))
        assert pre[0] + tot[0] <= cap
        obase, oal = pre[0], pre[0] & ~3
        last_tile = t == ntiles - 1
        sout = [None] * (FT + 4)
        deferred = {}

        def emit(idx, wd):
            if idx >= obase:
                assert 0 <= idx - oal < FT + 4
                sout[idx - oal] = wd
            else:
                assert idx == obase - 1
                deferred[idx] = wd

        for tid, (hm, ones, lasth, r) in enumerate(thr):
            if not (hm or (last_tile and tid == 0 and tot[0] == 0)):
                continue
            o = obase + exs[tid][0]
            prevh = max(pre[1], exs[tid][1])
            for e in range(FGPT):
                if (hm >> e) & 1:
                    q = g0 + tid * FGPT + e
                    if prevh and (prevh & 3) != C_MIXED:
                        emit(o - 1, run_word(prevh & 3, q - ((prevh >> 2) - 1)))
                    c = cls_of(r[e])
                    if c == C_MIXED:
                        emit(o, r[e])
                    prevh = ((q + 1) << 2) | c
                    o += 1
            if last_tile and exs[tid][0] + bin(hm).count("1") == tot[0] and prevh and (prevh & 3) != C_MIXED:
                emit(o - 1, run_word(prevh & 3, groups - ((prevh >> 2) - 1)))
        cnt = tot[0] - (1 if (not last_tile and tot[0] and (tot[1] & 3) != C_MIXED) else 0)
        for i in range(cnt):
            assert sout[obase + i - oal] is not None, (t, i)
            out[obase + i] = sout[obase + i - oal]
        for k, v in deferred.items():
            out[k] = v
    n = recs[-1][0]
    assert all(v is not None for v in out[:n])
    return np.array(out[:n], dtype=np.uint32), recs[-1][2]


def _split(ser):
    w = np.asarray(ser, dtype=np.uint32)
    if 0 < w[-1] < 31:
        return w[:-2]
    return w[:-1]


def _expect(op, a, b):
    """The oracle's result bits in canonical words (the form compress()
    leaves on the dense paths: no count-1 fill)."""
    ref, _ = oracle.binop(op, a, b, inplace=True)
    g = []
    for w in _split(ref):
        w = int(w)
        if w > ALL:
            g.extend([ALL if w >= H1 else 0] * (w & MAXC))
        else:
            g.append(w)
    return G.canonicalize(g), g


@pytest.mark.parametrize("FT", [1024, 2048, 4096])
@pytest.mark.parametrize("seed", range(6))
def test_model_equals_oracle(seed, FT):
    rng = np.random.default_rng(100 + seed)
    styles = ["dense", "mixed", "short", "sparse", "canon"]
    ng = int(rng.integers(1, 3 * FT + 700)) if seed else 5 * FT
    wa = G.random_words(rng, ng, styles[seed % 5])
    wb = G.random_words(rng, ng, styles[(seed + 2) % 5])
    if seed == 3:
        wa = [G.fill(1, ng)]  # one fill over every tile
    a, b = G.serialize(wa), G.serialize(wb)
    for op in range(4):
        want, groups = _expect(op, a, b)
        got, ones = model(op, wa, wb, ng, FT)
        assert np.array_equal(got, np.asarray(want, np.uint32)), (seed, op)
        assert ones == sum(bin(v).count("1") for v in groups)


def test_model_geometric_runs():
    """The raw-WAH workload's form (appendFill of geometric runs) at 2^17 bits."""
    for d in (0.1, 0.5):
        a = oracle.build_runs(G.geometric_runs(5, 1 << 17, d))
        b = oracle.build_runs(G.geometric_runs(6, 1 << 17, d))
        ba, bb = _split(a), _split(b)
        groups = sum(wgroups(int(w)) for w in ba)
        for op in range(4):
            want, _ = _expect(op, a, b)
            got, _ = model(op, ba, bb, groups)
            assert np.array_equal(got, np.asarray(want, np.uint32)), (d, op)


def model_warp_tiles(op, groups_a, groups_b, GT=512):
    """The words k_gone<OP> (libfastlib_b200/csrc/wah_gone.cuh) writes, from
    the operands' group patterns (its expansion is the two-pass engine's,
    checked on the GPU): per tile of GT groups the lane heads of chunks of
    128 groups (lane l holding groups 4 l .. 4 l + 3), the look-back prefix
    {heads, last head}, then the write phase in lane and chunk order with
    every index asserted in range."""
    G_ = len(groups_a)
    r = [op2(op, int(a), int(b)) for a, b in zip(groups_a, groups_b)]
    ntiles = (G_ + GT - 1) // GT
    tiles = []
    for t in range(ntiles):
        g0, g1 = t * GT, min(t * GT + GT, G_)
        heads, lasth = 0, 0
        for q in range(g0, g1):
            c = cls_of(r[q])
            if q == 0 or c == C_MIXED or c != cls_of(r[q - 1]):
                heads += 1
                lasth = ((q + 1) << 2) | c
        tiles.append((heads, lasth))
    n = sum(h for h, _ in tiles)
    out = [None] * n
    pre_h, pre_l = 0, 0
    for t in range(ntiles):
        g0 = t * GT
        heads, lasth = tiles[t]
        acc, carry = pre_h, pre_l
        for j in range(GT // 128):
            lane_m = []
            for lane in range(32):
                q0 = g0 + 128 * j + 4 * lane
                m = 0
                for e in range(4):
                    q = q0 + e
                    if q < min(g0 + GT, G_):
                        c = cls_of(r[q])
                        pc = cls_of(r[q - 1]) if q > 0 else None
                        if q == 0 or c == C_MIXED or c != pc:
                            m |= 1 << e
                lane_m.append(m)
            mine = []
            for lane, m in enumerate(lane_m):
                v = 0
                for e in range(4):
                    if (m >> e) & 1:
                        q = g0 + 128 * j + 4 * lane + e
                        v = ((q + 1) << 2) | cls_of(r[q])
                mine.append(v)
            sums = np.cumsum([bin(m).count("1") for m in lane_m]).tolist()
            for lane, m in enumerate(lane_m):
                prevh = max([carry] + mine[:lane])
                o = acc + sums[lane] - bin(m).count("1")
                for e in range(4):
                    if not (m >> e) & 1:
                        continue
                    q = g0 + 128 * j + 4 * lane + e
                    if prevh and (prevh & 3) != C_MIXED:
                        assert 1 <= o <= n
                        out[o - 1] = run_word(prevh & 3, q - ((prevh >> 2) - 1))
                    c = cls_of(r[q])
                    if c == C_MIXED:
                        assert 0 <= o < n
                        out[o] = r[q]
                    prevh = ((q + 1) << 2) | c
                    o += 1
            acc += sums[-1]
            carry = max([carry] + mine)
        if t == ntiles - 1 and carry and (carry & 3) != C_MIXED:
            assert 1 <= acc <= n
            out[acc - 1] = run_word(carry & 3, G_ - ((carry >> 2) - 1))
        pre_h, pre_l = pre_h + heads, max(pre_l, lasth)
    assert all(v is not None for v in out)
    return np.array(out, dtype=np.uint32)


@pytest.mark.parametrize("seed", range(5))
def test_warp_tile_model_equals_oracle(seed):
    rng = np.random.default_rng(300 + seed)
    styles = ["dense", "mixed", "short", "sparse", "canon"]
    ng = int(rng.integers(1, 3 * 1024 + 700)) if seed else 4 * 1024
    wa = G.random_words(rng, ng, styles[seed % 5])
    wb = G.random_words(rng, ng, styles[(seed + 1) % 5])
    if seed == 3:
        wa = [G.fill(1, ng)]  # one run over every tile
    a, b = G.serialize(wa), G.serialize(wb)
    _, ga = _expect(0, a, a)
    _, gb = _expect(0, b, b)
    for op in range(4):
        want, _ = _expect(op, a, b)
        got = model_warp_tiles(op, ga, gb)
        assert np.array_equal(got, np.asarray(want, np.uint32)), (seed, op)
