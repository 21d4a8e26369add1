"""GPU parity of the WAH operators through the C ABI (libwahgpu.so):
word-for-word against the reference's golden outputs and against the oracle
at the full 2^28-bit size of the raw-WAH workload."""
import numpy as np
import pytest

import oracle
from oracle import wahgen as G
from conftest import load_golden, unpack

pytestmark = pytest.mark.gpu


def _bin(ctx, op, a, b, inplace):
    import libfastlib_b200 as L
    A, B = ctx.bitvector(a), ctx.bitvector(b)
    r = A._binop(op, B, inplace)
    return r.write(), r.cnt()


def test_random_golden(gpu_ctx):
    import libfastlib_b200 as L
    g = load_golden("binop_random.npz")
    ndeg = 0
    for i in range(len(g["op"])):
        if g["status"][i] != 0:
            continue
        a, b = unpack(g, "a", i), unpack(g, "b", i)
        op, ip = int(g["op"][i]), int(g["inplace"][i])
        if oracle.is_degenerate(a) or oracle.is_degenerate(b):
            with pytest.raises(L.WahError) as e:
                _bin(gpu_ctx, op, a, b, ip)
            assert e.value.code == -9
            ndeg += 1
            continue
        w, c = _bin(gpu_ctx, op, a, b, ip)
        assert c == int(g["cnt"][i]), (i, op, ip)
        assert np.array_equal(w, unpack(g, "res", i)), (i, op, ip, [hex(x) for x in a], [hex(x) for x in b])
    assert ndeg > 0


def test_geometric_golden(gpu_ctx):
    g = load_golden("binop_geom.npz")
    for k, (di, op, ip) in enumerate(g["case"]):
        a, b = unpack(g, "operands", 2 * di), unpack(g, "operands", 2 * di + 1)
        w, c = _bin(gpu_ctx, int(op), a, b, int(ip))
        assert c == int(g["cnt"][k]), (di, op, ip)
        assert np.array_equal(w, unpack(g, "res", k)), (di, op, ip)


@pytest.mark.parametrize("density", [1e-4, 1e-3, 1e-2, 0.1, 0.5])
def test_full_size_against_oracle(gpu_ctx, density):
    """2^28-bit operands (the raw-WAH workload) — every op, both forms."""
    _full_size(gpu_ctx, density)


@pytest.mark.parametrize("tile", [1024, 4096])
@pytest.mark.parametrize("density", [0.1, 0.5])
def test_full_size_dense_tiles(gpu_ctx, density, tile):
    """The dense-path kernel with other tile sizes gives the same words."""
    with _tile(gpu_ctx, tile):
        _full_size(gpu_ctx, density)


class _tile:
    """The pipelined group-space kernel (WAHGPU_TUNE_DENSE_ENGINE = 1) at a
    given tile size."""

    def __init__(self, ctx, tile):
        self.ctx, self.tile = ctx, tile

    def __enter__(self):
        import libfastlib_b200 as L
        self.old = self.ctx.get_tuning(L.TUNE_DENSE_TILE)
        self.old_engine = self.ctx.get_tuning(L.TUNE_DENSE_ENGINE)
        self.ctx.set_tuning(L.TUNE_DENSE_TILE, self.tile)
        self.ctx.set_tuning(L.TUNE_DENSE_ENGINE, 1)

    def __exit__(self, *exc):
        import libfastlib_b200 as L
        self.ctx.set_tuning(L.TUNE_DENSE_TILE, self.old)
        self.ctx.set_tuning(L.TUNE_DENSE_ENGINE, self.old_engine)


def _full_size(gpu_ctx, density):
    nbits = 1 << 28
    a = oracle.build_runs(G.geometric_runs(11, nbits, density))
    b = oracle.build_runs(G.geometric_runs(12, nbits, density))
    A, B = gpu_ctx.bitvector(a), gpu_ctx.bitvector(b)
    assert A.size() == nbits and B.size() == nbits
    for op in range(4):
        for ip in (0, 1):
            ref, rc = oracle.binop(op, a, b, inplace=bool(ip))
            r = A._binop(op, B, bool(ip))
            w = r.write()
            assert r.cnt() == rc, (op, ip)
            assert np.array_equal(w, ref), (op, ip)


class _engine:
    """A given engine for canonical-result operators
    (WAHGPU_TUNE_DENSE_ENGINE: 3 two-pass, the default; 4 single-pass CTA
    tiles; 5 single-pass warp tiles) and tile size
    (WAHGPU_TUNE_DENSE_TILE, used by engine 4)."""

    def __init__(self, ctx, engine, tile=2048):
        self.ctx, self.engine, self.tile = ctx, engine, tile

    def __enter__(self):
        import libfastlib_b200 as L
        self.old = (self.ctx.get_tuning(L.TUNE_DENSE_ENGINE), self.ctx.get_tuning(L.TUNE_DENSE_TILE))
        self.ctx.set_tuning(L.TUNE_DENSE_ENGINE, self.engine)
        self.ctx.set_tuning(L.TUNE_DENSE_TILE, self.tile)

    def __exit__(self, *exc):
        import libfastlib_b200 as L
        self.ctx.set_tuning(L.TUNE_DENSE_ENGINE, self.old[0])
        self.ctx.set_tuning(L.TUNE_DENSE_TILE, self.old[1])


ENGINES = [(3, 2048), (4, 1024), (4, 2048), (4, 4096), (5, 2048)]


@pytest.mark.parametrize("engine,tile", ENGINES)
@pytest.mark.parametrize("density", [0.1, 0.5])
def test_full_size_group_space_engines(gpu_ctx, density, engine, tile):
    """The two-pass and the single-pass group-space engines (every tile
    size of the CTA-tile one) give the same words at full size."""
    with _engine(gpu_ctx, engine, tile):
        _full_size(gpu_ctx, density)


@pytest.mark.parametrize("engine,tile", ENGINES)
def test_many_tiles_fuzz_engines(gpu_ctx, engine, tile):
    with _engine(gpu_ctx, engine, tile):
        _fuzz(gpu_ctx)


@pytest.mark.parametrize("tile", [1024, 2048, 4096])
def test_many_tiles_fuzz(gpu_ctx, tile):
    """Operands of ~10^5 words of mixed forms so results span many tiles and
    the look-back carries runs, heads and step states across tile edges."""
    with _tile(gpu_ctx, tile):
        _fuzz(gpu_ctx)


def _fuzz(gpu_ctx):
    rng = np.random.default_rng(5)
    for trial in range(12):
        ng = int(rng.integers(20000, 200000))
        style_a = ["mixed", "short", "sparse", "canon", "dense"][trial % 5]
        style_b = ["canon", "sparse", "mixed", "short", "mixed"][trial % 5]
        wa = G.random_words(rng, ng, style_a)
        wb = G.random_words(rng, ng, style_b)
        anb = int(rng.integers(0, 31))
        a = G.serialize(wa, anb, int(rng.integers(0, 1 << 31)))
        b = G.serialize(wb, anb, int(rng.integers(0, 1 << 31)))
        if oracle.is_degenerate(a) or oracle.is_degenerate(b):
            continue
        for op in range(4):
            ip = int(rng.integers(0, 2))
            ref, rc = oracle.binop(op, a, b, inplace=bool(ip))
            w, c = _bin(gpu_ctx, op, a, b, ip)
            assert c == rc and np.array_equal(w, ref), (trial, op, ip)


def test_unary_golden(gpu_ctx):
    g = load_golden("unary.npz")
    for i in range(len(g["src_off"]) - 1):
        src = unpack(g, "src", i)
        A = gpu_ctx.bitvector(src)
        assert np.array_equal(A.rids(), unpack(g, "rids", i)), i
        A.compress()
        assert np.array_equal(A.write(), unpack(g, "compress", i)), i
        assert A.cnt() == int(g["compress_cnt"][i])
        B = gpu_ctx.bitvector(src)
        B.decompress()
        ref = unpack(g, "decompress", i)
        got = B.write()
        # decompress() of an all-zero vector is collapsed again by the cnt()
        # the fixture took after write(); compare bits through compress()
        assert np.array_equal(got, ref) or np.array_equal(oracle.compress(got)[0], oracle.compress(ref)[0]), i
        C = gpu_ctx.bitvector(src)
        C.flip()
        assert np.array_equal(C.write(), oracle.compress(unpack(g, "flip", i))[0]), i


def test_rids_large(gpu_ctx):
    nbits = 1 << 24
    a = oracle.build_runs(G.geometric_runs(3, nbits, 0.3, mean1=200.0))
    A = gpu_ctx.bitvector(a)
    assert np.array_equal(A.rids(), oracle.rids(a))


def test_many_one_fills_per_tile(gpu_ctx):
    """Row ids and decompress of words that are all 1-fills (more per 4096-word
    tile than the kernels' shared fill list holds)."""
    words = [0xC0000002] * 9000 + [0x12345, 0x80000003] * 500
    a = G.serialize(words, 5, 0b10110)
    A = gpu_ctx.bitvector(a)
    assert np.array_equal(A.rids(), oracle.rids(a))
    B = gpu_ctx.bitvector(a)
    B.decompress()
    assert np.array_equal(B.write(), oracle.decompress(a))


def _dense_words(rng, ngroups):
    """Literal stretches (mostly mixed, some 0/ALLONES literals and count-1
    fills) between fills of up to a few thousand groups, so tiles are pure,
    impure, all-mixed, or covered by fills that cross tile edges."""
    words, g = [], 0
    while g < ngroups:
        left = ngroups - g
        if rng.random() < 0.3:
            c = int(min(left, rng.integers(1, 6000)))
            words.append(G.fill(int(rng.integers(0, 2)), c))
            g += c
            continue
        k = int(min(left, rng.integers(1, 5000)))
        lit = rng.integers(1, G.ALLONES, size=k, dtype=np.int64)
        r = rng.random(k)
        lit[r < 0.02] = 0
        lit[(r >= 0.02) & (r < 0.04)] = G.ALLONES
        out = [int(x) for x in lit]
        for i in np.nonzero(r > 0.995)[0]:
            out[i] = G.fill(int(rng.integers(0, 2)), 1)
        words.extend(out)
        g += k
    return words


@pytest.mark.parametrize("tile", [1024, 2048, 4096])
def test_dense_path_fuzz(gpu_ctx, tile):
    """Operands dense enough for the _d2 path, sizes that leave partial last
    tiles, fills longer than a tile, count-1 fill words among literals."""
    rng = np.random.default_rng(77)
    with _tile(gpu_ctx, tile):
        for trial in range(10):
            ng = int(rng.integers(1, 12)) * tile + int(rng.integers(0, tile))
            wa, wb = _dense_words(rng, ng), _dense_words(rng, ng)
            anb = int(rng.integers(0, 31))
            a = G.serialize(wa, anb, int(rng.integers(0, 1 << 31)))
            b = G.serialize(wb, anb, int(rng.integers(0, 1 << 31)))
            if oracle.is_degenerate(a) or oracle.is_degenerate(b):
                continue
            for op in range(4):
                for ip in (0, 1):
                    ref, rc = oracle.binop(op, a, b, inplace=bool(ip))
                    w, c = _bin(gpu_ctx, op, a, b, ip)
                    assert c == rc and np.array_equal(w, ref), (trial, op, ip)


@pytest.mark.parametrize("engine", [1, 3, 4, 5])
def test_group_space_engines_fuzz(gpu_ctx, engine):
    """The group-space engines (1 pipelined, 3 two-pass, 4 and 5 single
    pass): dense operands
    with fills longer than a tile, pure and impure tiles, count-1
    fill words among literals, partial last tiles."""
    import libfastlib_b200 as L
    rng = np.random.default_rng(78 + engine)
    gpu_ctx.set_tuning(L.TUNE_DENSE_ENGINE, engine)
    try:
        for trial in range(12):
            ng = int(rng.integers(1, 12)) * 4096 + int(rng.integers(0, 4096)) if trial % 3 else int(rng.integers(1, 5000))
            wa, wb = _dense_words(rng, ng), _dense_words(rng, ng)
            anb = int(rng.integers(0, 31))
            a = G.serialize(wa, anb, int(rng.integers(0, 1 << 31)))
            b = G.serialize(wb, anb, int(rng.integers(0, 1 << 31)))
            if oracle.is_degenerate(a) or oracle.is_degenerate(b):
                continue
            for op in range(4):
                for ip in (0, 1):
                    ref, rc = oracle.binop(op, a, b, inplace=bool(ip))
                    w, c = _bin(gpu_ctx, op, a, b, ip)
                    assert c == rc and np.array_equal(w, ref), (trial, op, ip)
    finally:
        gpu_ctx.set_tuning(L.TUNE_DENSE_ENGINE, 0)


@pytest.mark.parametrize("engine", [1, 3])
@pytest.mark.parametrize("density", [0.1, 0.5])
def test_group_space_engines_full_size(gpu_ctx, density, engine):
    """Both group-space engines give the reference's words at 2^28 bits."""
    import libfastlib_b200 as L
    gpu_ctx.set_tuning(L.TUNE_DENSE_ENGINE, engine)
    try:
        _full_size(gpu_ctx, density)
    finally:
        gpu_ctx.set_tuning(L.TUNE_DENSE_ENGINE, 0)


def test_dense_small_sizes(gpu_ctx):
    """1 to 3 tiles and tiny vectors: grids smaller than the SM count, a
    control warp that meets the end at once."""
    rng = np.random.default_rng(9)
    for ng in (2, 3, 31, 127, 128, 129, 1023, 1024, 1025, 2047, 2049, 3000):
        wa, wb = _dense_words(rng, ng), _dense_words(rng, ng)
        a = G.serialize(wa, 7, 0x55)
        b = G.serialize(wb, 7, 0x2A)
        if oracle.is_degenerate(a) or oracle.is_degenerate(b):
            continue
        for op in range(4):
            ref, rc = oracle.binop(op, a, b, inplace=False)
            w, c = _bin(gpu_ctx, op, a, b, 0)
            assert c == rc and np.array_equal(w, ref), (ng, op)


@pytest.mark.parametrize("density", [0.1, 0.5])
def test_word_space_engine_same_words(gpu_ctx, density):
    """Canonical-result operators through the word-space merge
    (WAHGPU_TUNE_DENSE_ENGINE = 2) give the same words."""
    import libfastlib_b200 as L
    gpu_ctx.set_tuning(L.TUNE_DENSE_ENGINE, 2)
    try:
        _full_size(gpu_ctx, density)
    finally:
        gpu_ctx.set_tuning(L.TUNE_DENSE_ENGINE, 0)


def test_unequal_sizes_golden(gpu_ctx):
    """Operands of different sizes against the reference's own answers."""
    g = load_golden("binop_unequal.npz")
    for i in range(len(g["op"])):
        a, b = unpack(g, "a", i), unpack(g, "b", i)
        w, c = _bin(gpu_ctx, int(g["op"][i]), a, b, int(g["inplace"][i]))
        assert c == int(g["cnt"][i]) and np.array_equal(w, unpack(g, "res", i)), i


def test_unequal_sizes(gpu_ctx):
    """Operands of different sizes: the shorter one is padded with 0 bits
    (adjustSize) and the operator runs in the OP= form, as the reference
    does; tails that end in a literal 0, a 0-fill, a 1-fill or active bits
    exercise the merges of the padding."""
    rng = np.random.default_rng(405)
    styles = ["mixed", "short", "sparse", "canon", "dense"]
    checked = 0
    for trial in range(60):
        ga = int(rng.integers(1, 3000))
        gb = int(rng.integers(1, 3000))
        wa = G.random_words(rng, ga, styles[trial % 5])
        wb = G.random_words(rng, gb, styles[(trial + 2) % 5])
        if trial % 6 == 1:
            wa = list(wa[:-1]) + [0]               # ends in a literal 0
        if trial % 6 == 2:
            wb = list(wb) + [G.fill(0, 5)]         # ends in a 0-fill
        if trial % 6 == 3:
            wa = list(wa) + [G.fill(1, 3)]         # ends in a 1-fill
        a = G.serialize(wa, int(rng.integers(0, 31)), int(rng.integers(0, 1 << 31)))
        b = G.serialize(wb, int(rng.integers(0, 31)), int(rng.integers(0, 1 << 31)))
        if oracle.is_degenerate(a) or oracle.is_degenerate(b):
            continue
        for op in range(4):
            for ip in (0, 1):
                ref, rc = oracle.binop(op, a, b, inplace=bool(ip))
                w, c = _bin(gpu_ctx, op, a, b, ip)
                assert c == rc and np.array_equal(w, ref), (trial, op, ip, len(a), len(b))
                checked += 1
    assert checked > 300


@pytest.mark.parametrize("tile", [16, 32, 64])
def test_merge_tile_sizes(gpu_ctx, tile):
    """The word-space merge at every tile size (WAHGPU_TUNE_MERGE_TILE):
    the many-tile fuzz, the sparse full-size pairs and unary copies."""
    import libfastlib_b200 as L
    gpu_ctx.set_tuning(L.TUNE_MERGE_TILE, tile)
    try:
        _fuzz(gpu_ctx)
        for density in (1e-4, 1e-2):
            _full_size(gpu_ctx, density)
        rng = np.random.default_rng(90 + tile)
        for style in ("sparse", "mixed"):
            src = G.serialize(G.random_words(rng, 60000, style))
            A = gpu_ctx.bitvector(src)
            A.compress()
            ref, cnt = oracle.compress(src)
            assert np.array_equal(A.write(), ref) and A.cnt() == cnt, style
            B = gpu_ctx.bitvector(src)
            B.flip()  # results are held in compress()ed form
            assert np.array_equal(B.write(), oracle.compress(oracle.flip(src))[0]), style
    finally:
        gpu_ctx.set_tuning(L.TUNE_MERGE_TILE, 0)
