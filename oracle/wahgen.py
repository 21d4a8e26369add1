"""Seeded generators of serialized WAH bitvectors and requests for the oracle
driver — TEST INFRASTRUCTURE ONLY.

A serialized bitvector is the reference's write(array_t&) layout
(bitvector.cpp:2283-2313): the whole words of m_vec, then the active word's
value if it holds any bits, then the active word's bit count.

The word generator deliberately produces forms the reference itself can hold
(count-1 fills, lone 0/all-ones literals, adjacent same-valued fills,
uncompressed runs of literals) so the emission rules are exercised beyond
canonical inputs.
"""
import struct
import subprocess
import numpy as np

ALLONES = 0x7FFFFFFF
HEADER0 = 0x80000000
HEADER1 = 0xC0000000


def fill(v, n):
    return (HEADER1 if v else HEADER0) | n


def groups_of(words):
    g = 0
    for w in words:
        g += (w & 0x3FFFFFFF) if w & 0x80000000 else 1
    return g


def serialize(words, anb=0, aval=0):
    out = list(words)
    if anb > 0:
        out.append(aval & ((1 << anb) - 1))
    out.append(anb)
    return out


def random_words(rng, ngroups, style):
    """Returns a list of WAH words covering exactly ngroups 31-bit groups."""
    words = []
    g = 0
    while g < ngroups:
        left = ngroups - g
        r = rng.random()
        if style == "dense":
            k = rng.integers(0, 4)
            w = [0, ALLONES, int(rng.integers(0, ALLONES + 1)), int(rng.integers(0, ALLONES + 1))][k]
            words.append(w)
            g += 1
            continue
        if style == "sparse":
            pf = 0.55
        elif style == "canon":
            pf = 0.45
        else:
            pf = 0.4
        if r < pf and left >= 1:
            maxc = left if style != "short" else min(left, 4)
            if style == "canon":
                if left < 2:
                    words.append(int(rng.integers(1, ALLONES)))
                    g += 1
                    continue
                c = int(rng.integers(2, min(maxc, 60) + 1))
            else:
                c = int(rng.integers(1, min(maxc, 40) + 1))
            v = int(rng.integers(0, 2))
            words.append(fill(v, c))
            g += c
        else:
            k = rng.random()
            if style == "canon" or k < 0.6:
                w = int(rng.integers(1, ALLONES))
            elif k < 0.8:
                w = 0
            else:
                w = ALLONES
            words.append(w)
            g += 1
    if style == "canon":
        words = canonicalize(words)
    return words


def canonicalize(words):
    """Merge runs like compress() and turn count-1 fills into literals."""
    out = []
    for w in words:
        if w & 0x80000000:
            v, c = (w >> 30) & 1, w & 0x3FFFFFFF
        elif w == 0:
            v, c = 0, 1
        elif w == ALLONES:
            v, c = 1, 1
        else:
            out.append(w)
            continue
        if out and out[-1] & 0x80000000 and ((out[-1] >> 30) & 1) == v:
            out[-1] += c
        elif out and out[-1] == (ALLONES if v else 0):
            out[-1] = fill(v, c + 1)
        elif c >= 2:
            out.append(fill(v, c))
        else:
            out.append(ALLONES if v else 0)
    return out


def random_pair(rng, equal=True):
    """Two serialized operands for a binary operator."""
    styles = ["mixed", "short", "dense", "sparse", "canon"]
    ng = int(rng.choice([1, 2, 3, 5, 8, 20, 60, 200]))
    anb = int(rng.integers(0, 31)) if rng.random() < 0.7 else 0
    sa = styles[int(rng.integers(0, len(styles)))]
    sb = styles[int(rng.integers(0, len(styles)))]
    wa = random_words(rng, ng, sa) if rng.random() > 0.03 else []
    ngb = ng if equal else max(0, ng + int(rng.integers(-3, 4)))
    anb_b = anb if equal else int(rng.integers(0, 31))
    if not wa:
        ng = 0
        ngb = 0 if equal else ngb
    wb = random_words(rng, ngb, sb) if ngb else []
    if rng.random() < 0.05 and wa:
        wa = [fill(int(rng.integers(0, 2)), ng)] if ng > 1 else wa
    if rng.random() < 0.05 and wb:
        wb = [fill(int(rng.integers(0, 2)), ngb)] if ngb > 1 else wb
    a = serialize(wa, anb, int(rng.integers(0, 1 << 31)))
    b = serialize(wb, anb_b, int(rng.integers(0, 1 << 31)))
    return a, b


def geometric_runs(seed, nbits, density, mean1=8.0):
    """Alternating 0/1 run lengths (0-run first) summing to nbits: 1-runs
    are Geometric with mean mean1 (>= 1), 0-runs Geometric with mean
    mean1*(1-d)/d, so a fraction d of the bits are 1.  numpy's PCG64 stream
    per seed keeps the fixtures platform independent."""
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
    runs = np.concatenate(parts)
    if len(parts) > 1:
        # chunks keep the 0/1 alternation because each holds an even count
        pass
    return runs.astype(np.uint64)


# ------------------------------------------------------------- driver I/O
def _u32(v):
    return struct.pack("<I", v & 0xFFFFFFFF)


def _vec(words):
    return _u32(len(words)) + np.asarray(words, dtype=np.uint32).tobytes()


def req_binop(op, inplace, compress, a, b):
    return _u32(1) + _u32(op) + _u32(inplace) + _u32(compress) + _vec(a) + _vec(b)


def req_unary(kind, a):
    return _u32(kind) + _vec(a)


def req_runs(runs):
    runs = np.asarray(runs, dtype=np.uint64)
    return _u32(4) + struct.pack("<Q", len(runs)) + runs.tobytes()


def req_relic(vals, queries):
    vals = np.asarray(vals, dtype=np.uint32)
    q = np.asarray(queries, dtype=np.float64).reshape(-1, 2)
    return (_u32(5) + _u32(len(vals)) + vals.tobytes() + _u32(len(q)) + q.tobytes())


class Reader:
    def __init__(self, data):
        self.d = data
        self.p = 0

    def u32(self):
        v = struct.unpack_from("<I", self.d, self.p)[0]
        self.p += 4
        return v

    def vec(self, dtype=np.uint32, size=4):
        n = self.u32()
        v = np.frombuffer(self.d, dtype=dtype, count=n, offset=self.p).copy()
        self.p += n * size
        return v

    def bv(self):
        st = self.u32()
        cnt = self.u32()
        w = self.vec()
        return st, cnt, w


def run_refdrv(refdrv, reqs, tmpdir):
    import os
    fi = os.path.join(tmpdir, "req.bin")
    fo = os.path.join(tmpdir, "rep.bin")
    with open(fi, "wb") as f:
        f.write(b"".join(reqs))
    subprocess.run([refdrv, fi, fo], check=True)
    with open(fo, "rb") as f:
        return Reader(f.read())
