"""CPU replays of the index arithmetic of two kernels, run before their GPU use.

cost.cu (cost volume): every (x, d) of a row is written exactly once with the
matching cost (popcount of the census XOR, 64 where x - d < 0, 0 in the pads),
every census load stays inside the planes' guard words and is 16-byte aligned,
and every shared-memory tile index stays inside the launch's allocation.

census.cu (staging): the asynchronously staged rows of an interior tile are
16-byte aligned, read only inside the image row, fit the shared memory the
launch reserves, and every window tap lands on the pixel the clamped staging
puts there.

wta.cu (row loop): the lane form chosen per pair (16 or 8 disparities a lane),
every 16-byte store into the per-warp sums rows aligned and inside the
dynamic shared memory, for odd widths too; the padded right-view key indices
inside their array and the atomics' bank conflicts bounded.

The constants mirror the kernels' (cost.cu: kBlockPx, kTileRows, kMaxTileBytes;
kernels.cuh: kCensusGuardWords, kWtaThreads, kWtaSumsPerWarp)."""
import random

K_BLOCK_PX, K_WARPS, K_TILE_ROWS, K_MAX_TILE_BYTES = 128, 8, 132, 56 * 1024
K_GUARD_WORDS = 352
K_WTA_THREADS, K_WTA_SUMS_PER_WARP = 256, 1024


def _tile_stride(dv):
    return (dv // 16) | 1


def _blocks_per_pass(dv):
    chunks = dv // 16
    best, best_num, best_den = 1, 0, 1
    for nb in range(1, K_WARPS + 1):
        if nb * K_TILE_ROWS * _tile_stride(dv) * 16 > K_MAX_TILE_BYTES:
            break
        items = nb * chunks
        den = K_WARPS * ((items + K_WARPS - 1) // K_WARPS)
        if items * best_den > best_num * den:
            best, best_num, best_den = nb, items, den
    return best


def _tile_units(dv):
    return _blocks_per_pass(dv) * K_TILE_ROWS * _tile_stride(dv)


def _replay_cost_row(W, H, D, y, dp_max, cl, cr):
    dv = (D + 15) // 16 * 16
    chunks, ts, nb = dv // 16, _tile_stride(dv), _blocks_per_pass(dv)
    units = max(_tile_units(v) for v in range(16, (dp_max + 15) // 16 * 16 + 1, 16))
    assert units * 16 <= K_MAX_TILE_BYTES                     # the launch's smem bound
    row0 = y * W
    out = {}
    xb = -(row0 & 3)
    while xb < W:
        tile = {}
        for it in range(nb * chunks):
            blk, ch = divmod(it, chunks)
            for lane in range(32):
                x4 = xb + blk * K_BLOCK_PX + 4 * lane
                if x4 >= W:
                    continue
                a = row0 + x4
                assert a % 4 == 0 and a >= 0
                base = a - 16 * ch - 16                  # 20 right words, 5 aligned vectors
                assert base % 4 == 0
                assert -K_GUARD_WORDS <= base and base + 19 < H * W + K_GUARD_WORDS
                assert a + 3 < H * W + K_GUARD_WORDS
                n0, dmax = x4 - 16 * ch, D - 16 * ch
                check = not (n0 >= 15 and dmax >= 16)
                for i in range(4):
                    v = []
                    for e in range(16):
                        c = bin(cl[a + i] ^ cr[base + i - e + 16]).count("1")
                        if check:
                            c = 0 if e >= dmax else (64 if e > n0 + i else c)
                        v.append(c)
                    idx = (blk * K_TILE_ROWS + lane) * ts + ch + i * 33 * ts
                    assert 0 <= idx < units and idx not in tile
                    tile[idx] = v
        p0, p1 = max(xb, 0) - xb, min(nb * K_BLOCK_PX, W - xb)
        for q in range((p1 - p0) * chunks):
            pq, c = divmod(q, chunks)
            pp = pq + p0
            row = (pp >> 7) * K_TILE_ROWS + (pp & 3) * 33 + ((pp & 127) >> 2)
            x, cc = divmod((xb + p0) * dv + 16 * q, dv)
            assert cc == 16 * c and x == xb + pp and 0 <= x < W
            for e in range(16):
                assert (x, 16 * c + e) not in out
                out[(x, 16 * c + e)] = tile[row * ts + c][e]
        xb += nb * K_BLOCK_PX
    assert len(out) == W * dv
    for x in range(W):
        for d in range(dv):
            want = 0 if d >= D else (64 if x < d else bin(cl[row0 + x] ^ cr[row0 + x - d]).count("1"))
            assert out[(x, d)] == want, (W, D, y, x, d)


def test_cost_kernel_mapping_covers_rows_in_bounds():
    rng = random.Random(7)
    for (W, H, D, dp_max) in [(1, 2, 1, 8), (5, 3, 16, 16), (37, 3, 64, 256), (130, 2, 80, 80),
                              (129, 2, 256, 256), (300, 2, 144, 144), (77, 3, 40, 256), (261, 2, 48, 64),
                              (97, 2, 33, 40), (200, 2, 192, 192)]:
        cl = {i: rng.getrandbits(24) for i in range(-K_GUARD_WORDS, H * W + K_GUARD_WORDS)}
        cr = {i: rng.getrandbits(24) for i in range(-K_GUARD_WORDS, H * W + K_GUARD_WORDS)}
        for y in range(H):
            _replay_cost_row(W, H, D, y, dp_max, cl, cr)


def test_cost_kernel_passes_fill_the_warps():
    # The pass sizes chosen for the disparity counts of the benchmark mix leave no
    # warp idle at the pass barrier, within four CTAs' worth of tile an SM.
    for D in (64, 128, 192, 256):
        dv = (D + 15) // 16 * 16
        assert (_blocks_per_pass(dv) * (dv // 16)) % K_WARPS == 0, D
    for dv in range(16, 257, 16):
        assert _tile_units(dv) * 16 <= K_MAX_TILE_BYTES


FORM_BYTES16, FORM_BYTES8, FORM_WIDE = 0, 1, 2


def _wta_k(form):
    return 16 if form == FORM_BYTES16 else 8


def _wta_seg(dv, form):
    chunks, cap = dv // _wta_k(form), 16 if form == FORM_BYTES16 else 8
    seg = 1
    while seg < chunks and seg < cap:
        seg <<= 1
    return seg


def _wta_form(dv, wide):
    if wide:
        return FORM_WIDE
    c16, s16 = dv // 16, _wta_seg(dv, FORM_BYTES16)
    c8, s8 = dv // 8, _wta_seg(dv, FORM_BYTES8)
    slots16, slots8 = s16 * -(-c16 // s16), s8 * -(-c8 // s8)
    return FORM_BYTES8 if c8 * slots16 > c16 * slots8 else FORM_BYTES16


def _right_key_words(w):
    return w + ((w + 15) >> 4) * 4


def _right_key_pad(seg, form):
    return 0 if form != FORM_BYTES16 else 2 if seg >= 16 else 4 if seg == 8 else 0


def _right_key_index(a, pad):
    return a + (a >> 4) * pad


def _wta_sums_base(w):
    return ((_right_key_words(w) + 2 * w + 3) & ~3) * 4           # bytes


def _wta_smem_bytes(max_width):
    return _wta_sums_base(max_width) + (K_WTA_THREADS // 32) * K_WTA_SUMS_PER_WARP * 2


def test_wta_forms_keep_lanes_busy():
    # 16 disparities a lane unless 8 fills more lane-rounds: D = 144..192 (Dv / 16 = 9..12).
    forms = {d: _wta_form((d + 15) // 16 * 16, False) for d in range(1, 257)}
    assert {d for d, f in forms.items() if f == FORM_BYTES8} == set(range(129, 193))
    assert forms[64] == forms[128] == forms[256] == FORM_BYTES16 and forms[192] == FORM_BYTES8
    # The largest launch fits the 227 KB a CTA may hold.
    assert _wta_smem_bytes(16384) <= 227 * 1024


def test_wta_sums_rows_aligned_and_in_bounds():
    for D in range(1, 257):
        dv = (D + 15) // 16 * 16
        for form in {_wta_form(dv, False), FORM_WIDE}:
            k, seg = _wta_k(form), _wta_seg(dv, form)
            chunks = dv // k
            rounds = (chunks + seg - 1) // seg
            assert (32 // seg) * k * seg * rounds <= K_WTA_SUMS_PER_WARP
            for W in (1, 2, 3, 5, 7, 33, 1241, 1242, 16383, 16384):
                base = _wta_sums_base(W)
                assert base % 16 == 0
                for warp in range(K_WTA_THREADS // 32):
                    for lane in range(32):
                        sub, c = divmod(lane, seg)
                        row = base + (warp * K_WTA_SUMS_PER_WARP + sub * k * seg * rounds) * 2
                        for r in range(rounds):
                            for q in range(k // 8):
                                off = row + 2 * (k * (r * seg + c) + 8 * q)
                                assert off % 16 == 0 and off + 16 <= _wta_smem_bytes(W)
                        assert row + 2 * D <= _wta_smem_bytes(W)   # the S(bd +- 1) reads


def test_wta_right_keys_in_bounds_and_spread_over_banks():
    # Every right-view column 0..W-1 maps inside the padded array, below the
    # per-pixel arrays; one atomicMin instruction (fixed key index j) of a warp
    # meets at most 2 lanes on a bank (the byte form at 8 and 16 lanes a pixel: 1).
    for W in (1, 15, 16, 17, 1242, 16384):
        for form in (FORM_BYTES16, FORM_BYTES8, FORM_WIDE):
            for seg in (1, 2, 4, 8, 16):
                pad = _right_key_pad(seg, form)
                assert _right_key_index(W - 1, pad) < _right_key_words(W)
    for D in (64, 128, 192, 256, 48, 96, 200):
        dv = (D + 15) // 16 * 16
        form = _wta_form(dv, False)
        k, seg = _wta_k(form), _wta_seg(dv, form)
        pad = _right_key_pad(seg, form)
        worst = 0
        for xb in range(256, 256 + 64):
            for j in range(k):
                banks = {}
                for lane in range(32):
                    s, c = divmod(lane, seg)
                    if k * c >= D:
                        continue
                    b = _right_key_index(xb + s - k * c - j, pad) % 32
                    banks[b] = banks.get(b, 0) + 1
                worst = max(worst, max(banks.values()))
        assert worst <= 2, (D, worst)
        if form == FORM_BYTES16 and seg >= 8 and D % 128 == 0:
            assert worst == 1, (D, worst)


K_CENSUS_TILE = 32


def _census_lead(rx):
    return (16 - (rx & 15)) & 15


def _census_row_bytes(rx):
    return (_census_lead(rx) + K_CENSUS_TILE + 2 * rx + 15) & ~15


def _census_smem(max_rx, max_ry):
    w = max([K_CENSUS_TILE + 2 * max_rx] + [_census_row_bytes(r) for r in range(max_rx + 1)])
    return w * (K_CENSUS_TILE + 2 * max_ry)


def test_census_async_staging_geometry():
    import numpy as np
    rng = np.random.default_rng(3)
    for rx in range(0, 32):
        lead, rw = _census_lead(rx), _census_row_bytes(rx)
        assert rw % 16 == 0 and lead + K_CENSUS_TILE + 2 * rx <= rw
        for ry in (0, 1, 3, 7, 31):
            assert rw * (K_CENSUS_TILE + 2 * ry) <= _census_smem(rx, ry) <= 48 * 1024
        for W, H in ((97, 70), (1242, 375), (160, 120), (2048, 99)):
            img = rng.integers(0, 256, (H, W), dtype=np.uint8)
            ry = min(rx, 5)
            sh = K_CENSUS_TILE + 2 * ry
            for bx in range(0, W, 32):
                for by in range(0, H, 32):
                    x0 = bx - rx - lead
                    interior = x0 >= 0 and x0 + rw <= W and by - ry >= 0 and by + K_CENSUS_TILE + ry <= H
                    if not interior:
                        continue
                    assert x0 % 16 == 0                       # 16-byte aligned source (pitch, base aligned)
                    staged = img[by - ry:by - ry + sh, x0:x0 + rw]  # the copies: inside rows, inside the image
                    sw = K_CENSUS_TILE + 2 * rx
                    ys = np.clip(np.arange(by - ry, by - ry + sh), 0, H - 1)
                    xs = np.clip(np.arange(bx - rx, bx - rx + sw), 0, W - 1)
                    clamped = img[np.ix_(ys, xs)]
                    # window tap (tx + dx, ty + dy) of both stagings
                    assert np.array_equal(staged[:, lead:lead + sw], clamped)

