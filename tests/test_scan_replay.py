"""CPU replay of the across-lanes scan form of the path aggregation
(vx-rs_b200/csrc/aggregate_scan.cu), run before its GPU use and kept as a check
of its arithmetic.

The kernel evaluates each pixel of a scanline as an exact-integer (min, +)
prefix scan over d: lanes of K disparities compose their maps
f_d(x) = min(a_d, x + b_d) serially, the segment scans the lanes' compositions
(Kogge-Stone over a power-of-two segment), each lane applies the incoming value;
a pixel whose ushort arithmetic could leave [0, 65535] is recomputed in the
shader's serial order. This replay follows the same steps with numpy on the same
lane geometry (K = 8 disparities a lane) and must reproduce the oracle's
per-path costs L_r bit for bit (vx-vision/shaders/SGMStereo.metal:120-172),
including a scene and penalties under which the shader's ushort values wrap."""
import numpy as np
import pytest

import oracle
import vx_sgm

INF = 1 << 30


def _geometry(dv):
    k = 8
    lanes = dv // k
    seg = 1
    while seg < lanes:
        seg <<= 1
    return k, lanes, seg


def _costs(cl, cr, nd):
    h, w = cl.shape
    dv = (nd + 15) // 16 * 16
    C = np.zeros((h, w, dv), np.int64)
    for d in range(nd):
        c = np.full((h, w), 64, np.int64)
        if d < w:
            c[:, d:] = np.bitwise_count(cl[:, d:] ^ cr[:, :w - d]).astype(np.int64)
        C[:, :, d] = c
    return C


def _serial(L, m, C, D, P1, P2):
    y = np.empty_like(L)
    prev = 0
    for d in range(len(L)):
        if d < D:
            q1 = 0xFFFF if d == 0 else (prev + P1) & 0xFFFF
            q2 = 0xFFFF if d == D - 1 else (int(L[d + 1]) + P1) & 0xFFFF
            q3 = (m + P2) & 0xFFFF
            prev = (int(C[d]) + min(int(L[d]), q1, q2, q3) - m) & 0xFFFF
        y[d] = prev
    return y


def _scan_pixel(L, m, pmx, C, D, P1, P2, stats):
    """One pixel step as the kernel computes it: returns (new state, min, max)."""
    dv = len(C)
    k, lanes, seg = _geometry(dv)
    d = np.arange(dv)
    nb = np.append(L[1:], 0)
    o3 = m + P2
    o2 = np.where(d == D - 1, 0xFFFF, nb + P1)
    A = np.minimum(np.minimum(L, o2), o3)
    real = d < D
    a = np.where(real, C - m + A, INF)
    b = np.where(real, C - m + P1, 0)
    # each lane composes its K maps; lanes past `lanes` (pads only) are identities
    AL = np.full(seg, INF, np.int64)
    BL = np.zeros(seg, np.int64)
    for li in range(lanes):
        al, bl = a[li * k], b[li * k]
        for j in range(1, k):
            al = min(a[li * k + j], al + b[li * k + j])
            bl += b[li * k + j]
        AL[li], BL[li] = al, bl
    o = 1
    while o < seg:                                  # Kogge-Stone, all lanes at once
        Ap, Bp = AL.copy(), BL.copy()
        for li in range(o, seg):
            AL[li] = min(Ap[li], Ap[li - o] + Bp[li])
            BL[li] = Bp[li] + Bp[li - o]
        o <<= 1
    y = np.empty(dv, np.int64)
    for li in range(lanes):
        X = INF if li == 0 else AL[li - 1]
        for j in range(k):
            X = min(X + b[li * k + j], a[li * k + j])
            y[li * k + j] = X
    mn, mx = int(y.min()), int(y.max())
    if not (pmx + P1 <= 0xFFFF and o3 <= 0xFFFF and mn >= 0 and mx + P1 <= 0xFFFF):
        stats["serial"] += 1
        y = _serial(L, m, C, D, P1, P2)
        mn, mx = int(y[:D].min()), int(y[:D].max())
    stats["pixels"] += 1
    return y, mn, mx


def _replay_path(C, D, P1, P2, dx, dy, stats):
    h, w, dv = C.shape
    out = np.zeros((h, w, D), np.int64)
    starts = []
    if dy == 0:
        starts = [((0 if dx > 0 else w - 1), y) for y in range(h)]
    else:
        y0 = 0 if dy > 0 else h - 1
        starts = [(x, y0) for x in range(w)]
        if dx != 0:   # diagonals entering through the side column
            xs = 0 if dx > 0 else w - 1
            starts += [(xs, y) for y in (range(1, h) if dy > 0 else range(h - 1))]
    for (x, y) in starts:
        L = np.zeros(dv, np.int64)
        m = pmx = 0
        while 0 <= x < w and 0 <= y < h:
            L, m, pmx = _scan_pixel(L, m, pmx, C[y, x], D, P1, P2, stats)
            out[y, x] = L[:D]
            x += dx
            y += dy
    return out


@pytest.mark.parametrize("nd,p1,p2,w,h", [
    (64, 10, 120, 37, 9), (100, 10, 120, 41, 7), (192, 10, 120, 29, 6), (256, 7, 90, 23, 5),
    (7, 10, 120, 19, 8), (48, 60000, 60000, 21, 7), (128, 15, 300, 25, 6), (96, 10, 5000, 27, 6),
])
def test_scan_form_reproduces_the_path_costs(nd, p1, p2, w, h):
    L, R, _ = vx_sgm.synth_pair(0, w, h, 0, max(1, min(nd - 2, w - 2)), nd * 31 + w)
    cl, cr = oracle.census(L, 2, 2), oracle.census(R, 2, 2)
    C = _costs(cl, cr, nd)
    stats = {"pixels": 0, "serial": 0}
    wraps = 0
    for k in (0, 1, 4, 7):
        dx, dy = oracle.path_dir(k)
        want = oracle.path_costs(cl, cr, nd, p1, p2, dx, dy).astype(np.int64)
        got = _replay_path(C, nd, p1, p2, dx, dy, stats)
        bad = np.argwhere(got != want)
        assert bad.size == 0, f"path ({dx},{dy}) differs at {bad[:3]}"
        wraps += _oracle_wrap_steps(cl, cr, nd, p1, p2, dx, dy)
    # every pixel whose ushort arithmetic wrapped went through the serial fallback
    assert stats["serial"] >= wraps


def _oracle_wrap_steps(cl, cr, nd, p1, p2, dx, dy):
    import ctypes
    h, w = cl.shape
    st = oracle.OracleStats()
    r = oracle.lib().oracle_path(ctypes.c_void_p(cl.ctypes.data), ctypes.c_void_p(cr.ctypes.data), w, h, nd,
                                 int(p1), int(p2), dx, dy, None, None, ctypes.byref(st), 0)
    assert r == 0
    return int(st.wrap_steps)


def test_wrapping_pixels_take_the_serial_order():
    """A scene and penalties under which the shader's values wrap (P1 = 0: the
    in-place o1 term pulls values below the previous minimum): the replay meets
    those pixels, recomputes them serially and still equals the oracle."""
    nd, p1, p2, w, h = 64, 0, 2000, 48, 10
    L, R, _ = vx_sgm.synth_pair(2, w, h, 0, 40, 5)
    cl, cr = oracle.census(L, 2, 2), oracle.census(R, 2, 2)
    C = _costs(cl, cr, nd)
    stats = {"pixels": 0, "serial": 0}
    wraps = 0
    for k in range(8):
        dx, dy = oracle.path_dir(k)
        want = oracle.path_costs(cl, cr, nd, p1, p2, dx, dy).astype(np.int64)
        assert np.array_equal(_replay_path(C, nd, p1, p2, dx, dy, stats), want), (dx, dy)
        wraps += _oracle_wrap_steps(cl, cr, nd, p1, p2, dx, dy)
    assert wraps > 0 and stats["serial"] >= wraps


def test_geometry_covers_every_disparity_count():
    for D in range(1, 257):
        dv = (D + 15) // 16 * 16
        k, lanes, seg = _geometry(dv)
        assert lanes * k == dv and lanes <= seg <= 32 and 32 % seg == 0
        assert (seg & (seg - 1)) == 0 and 32 // seg >= 1
