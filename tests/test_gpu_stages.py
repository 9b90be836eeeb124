"""Per-operator parity on the GPU: every C-ABI operator of libisa.so against
the FP64 oracle on the same seeded inputs (oracle/isa_oracle.c, pinned to the
reference kernels by tests/test_oracle_golden.py).

Tolerances (stated per test): the GPU computes in FP32 (FP64 where the
reference's FP32 arithmetic is ill-conditioned: LK 2x2 solve, window sums,
kernel parameters, shift solve), so continuous outputs are compared at FP32
rounding level relative to their magnitude; discrete outputs (integer argmin,
outlier status) must be identical except at ties within a stated margin."""
import ctypes

import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P

import golden_cases

pytestmark = pytest.mark.gpu

L = None


def lib():
    global L
    if L is None:
        L = isa.lib()
    return L


_alive = []


@pytest.fixture(autouse=True)
def _release_buffers():
    yield
    _alive.clear()


def dev(a, dtype=None):
    """Device copy of a host array. The tensor is kept alive until the test
    ends: a pointer handed to the C ABI must outlive the asynchronous launch
    (a temporary would go back to torch's allocator and be reused)."""
    import torch
    a = np.array(a, copy=True)
    if dtype is not None:
        a = a.astype(dtype)
    if a.dtype == np.uint16:
        t = torch.from_numpy(a.view(np.int16)).cuda()
    else:
        t = torch.from_numpy(a).cuda()
    _alive.append(t)
    return t


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def ok(rc):
    isa.check(rc)


S0 = ctypes.c_void_p(None)
sz = ctypes.c_size_t


def f3(v):
    return (ctypes.c_float * 3)(*[float(x) for x in v])


def i4(v):
    return (ctypes.c_int * 4)(*[int(x) for x in v])


def close(got, want, atol, rtol=0.0, what=""):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    assert got.shape == want.shape, what
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want), err_msg=what)
    fin = np.isfinite(want)
    err = np.abs(got[fin] - want[fin])
    lim = atol + rtol * np.abs(want[fin])
    bad = err > lim
    assert not bad.any(), f"{what}: {bad.sum()} of {bad.size} beyond tolerance, worst {err.max():.3e}"


@pytest.fixture(scope="module")
def rng():
    return np.random.default_rng(1234)


@pytest.mark.parametrize("cfa", [(0, 1, 1, 2), (2, 1, 1, 0), (1, 0, 2, 1), (1, 2, 0, 1)])
def test_debayer_full(cuda, oracle, rng, cfa):
    raw = golden_cases._raw(rng, 96, 64)
    black, scale, div = (512.0, 500.0, 520.0), np.float32([1.0, 1 / 1.5, 0.5]), np.float32([15871.0, 15871.0 / 1.5, 15871.0 / 2])
    want = oracle.debayer_full(raw, cfa, black, scale, div)
    out = dev(np.zeros((64, 96, 3), np.float32))
    ok(lib().isa_debayer_full(isa.vp(dev(raw)), sz(192), 96, 64, i4(cfa), f3(black), f3(scale), f3(div), isa.vp(out), sz(96 * 12), S0))
    close(host(out), want, atol=2e-6, rtol=2e-6, what="debayer")  # values ~1, FP32 rounding


def test_gamma(cuda, oracle, rng):
    rgb = rng.uniform(-0.1, 1.1, (40, 48, 3)).astype(np.float32)
    rgb[3, 4, 1] = np.nan
    want = oracle.gamma_srgb(rgb.astype(np.float64))
    t = dev(rgb)
    ok(lib().isa_gamma_srgb(isa.vp(t), sz(48 * 12), 48, 40, S0))
    close(host(t), want, atol=1e-6, what="gamma")


@pytest.mark.parametrize("high_pass", [0, 1])
def test_bw_image(cuda, oracle, small_burst, high_pass):
    import pipeline as PL
    b = small_burst
    p = P.MergeParams()
    want = PL.bw_image(oracle, b, 1, 0.5, bool(high_pass), p)
    m = isa.Merger(b.width, b.height, b.n)
    out = dev(np.zeros((b.height, b.width), np.float32))
    info = isa.make_info(b)
    ok(lib().isa_bw_image(m.ctx, isa.vp(dev(b.raw[1])), sz(b.width * 2), b.width, b.height, ctypes.byref(info), ctypes.c_float(0.5),
                          high_pass, isa.vp(out), sz(b.width * 4), S0))
    # FP32 demosaic + the library's FFT high-pass against FP64 numpy FFT
    close(host(out), want, atol=2e-5 if high_pass else 2e-6, what="bw")
    m.close()


@pytest.mark.parametrize("W,H,params", [
    (188, 250, {}),                                   # rows of 94 = 2 * 47, columns 2 * 5^3 (the 6016 x 4000 factors)
    (134, 106, {}),                                   # rows of 67 (prime), columns 2 * 53 (prime)
    (240, 162, {"high_pass": 0.05}),                 # radix 3 in both directions, a wider high-pass band
    (160, 96, {"high_pass": 0.02, "clear_axis": 2}),  # axis clearing: every column through the column pass
])
def test_bw_image_fft_sizes(cuda, oracle, W, H, params):
    """The full-frame high-pass (PreAlignment.FourierFilter) through the hand-written FFT at frame sizes whose
    row and column lengths take every kind of stage (radix 8, 4, 2, 5, 3 and the paired prime stage), and with
    filter parameters that send every column through the column pass, against numpy's FP64 FFT."""
    import pipeline as PL
    from imagestackalignator_b200 import synthetic
    b = synthetic.make_burst(W, H, 2, seed=W + H, max_shift=2, max_rot_deg=0.1)
    p = P.MergeParams()
    p.levels = P.default_levels(1)  # the context is only needed for the transforms' tables and spectrum
    for k, v in params.items():
        setattr(p, k, v)
    want = PL.bw_image(oracle, b, 1, 0.5, True, p)
    m = isa.Merger(W, H, 2, p)
    out = dev(np.zeros((H, W), np.float32))
    info = isa.make_info(b)
    ok(lib().isa_bw_image(m.ctx, isa.vp(dev(b.raw[1])), sz(W * 2), W, H, ctypes.byref(info), ctypes.c_float(0.5), 1, isa.vp(out), sz(W * 4), S0))
    close(host(out), want, atol=2e-5, what=f"bw {W}x{H}")
    m.close()


def test_gauss_resize(cuda, oracle, rng):
    img = rng.uniform(0, 1, (50, 70)).astype(np.float32)
    for sigma in (0.5, 1.0, 2.5):
        want = oracle.gauss_filter(img.astype(np.float64), oracle.gauss_taps(sigma))
        a, o, t = dev(img), dev(np.zeros_like(img)), dev(np.zeros_like(img))
        ok(lib().isa_gauss_filter(isa.vp(a), sz(280), isa.vp(o), sz(280), isa.vp(t), sz(280), 70, 50, 1, ctypes.c_float(sigma), S0))
        close(host(o), want, atol=1e-6, what=f"gauss {sigma}")
    for L_ in (2, 4, 8):
        want = oracle.resize_box(img.astype(np.float64), L_)
        o = dev(np.zeros((50 // L_, 70 // L_), np.float32))
        ok(lib().isa_resize_box(isa.vp(dev(img)), sz(280), 70, 50, L_, isa.vp(o), sz((70 // L_) * 4), S0))
        close(host(o), want, atol=1e-6, what=f"resize {L_}")


@pytest.mark.parametrize("S", [2, 4])
def test_track_level_argmin_exact(cuda, oracle, rng, S):
    """Integer tile shifts: the first-minimum index of every tile's L2 map must
    equal the oracle's, except where the oracle's best and second-best scores
    are within a relative margin of 1e-5 (a tie at FP32 resolution)."""
    W, H, T = 648, 392, 32
    ref = golden_cases._img(rng, W, H)
    npairs = 3
    frames = [ref] + [np.roll(ref, (k, -2 * k), axis=(0, 1)) + rng.normal(0, 0.01, (H, W)) for k in range(1, npairs + 1)]
    tcx, tcy = (W - 2 * S) // T, (H - 2 * S) // T
    pre = rng.uniform(-2.5, 2.5, (npairs, tcy, tcx, 2))
    D = 2 * S + 1
    ftab = [dev(f.astype(np.float32)) for f in frames]
    import torch
    ptrs = torch.tensor([t.data_ptr() for t in ftab], dtype=torch.int64, device="cuda")
    pairs = (isa.IsaTrackPair * npairs)()
    base = [((0.5, -0.25), 0.001), ((1.5, 0.75), -0.002), ((-1.0, 2.0), 0.0), ((0.0, 0.0), 0.0)]
    for k in range(npairs):
        pairs[k].reference, pairs[k].to_track, pairs[k].grid = 0, k + 1, k
        pairs[k].base_shift_ref[0], pairs[k].base_shift_ref[1] = base[0][0]
        pairs[k].rotation_ref = base[0][1]
        pairs[k].base_shift_trk[0], pairs[k].base_shift_trk[1] = base[k + 1][0]
        pairs[k].rotation_trk = base[k + 1][1]
    pd = dev(np.frombuffer(bytes(pairs), np.uint8))
    grids = dev(pre.astype(np.float32))
    scores = dev(np.zeros((npairs, tcy * tcx, D * D), np.float32))
    amin = dev(np.zeros((npairs, tcy * tcx), np.int32))
    ok(lib().isa_track_level(isa.vp(ptrs), sz(W * 4), W, H, T, S, tcx, tcy, isa.vp(pd), npairs, isa.vp(grids), sz(tcx * 8),
                             sz(tcx * tcy * 8), ctypes.c_float(1.0), isa.vp(scores), isa.vp(amin), S0))
    g, sc, am = host(grids), host(scores), host(amin)
    ties = 0
    for k in range(npairs):
        want_g, want_sc = oracle.track_pair(frames[k + 1].astype(np.float32), frames[0].astype(np.float32), T, S, tcx, tcy, pre[k].astype(np.float32),
                                            base[0][0], base[0][1], base[k + 1][0], base[k + 1][1], 1.0, want_scores=True)
        close(sc[k], want_sc, atol=1e-4, rtol=2e-5, what="L2 maps")
        srt = np.sort(want_sc, axis=1)
        tie = (srt[:, 1] - srt[:, 0]) <= 1e-5 * np.maximum(srt[:, 0], 1e-12)
        want_am = np.argmin(want_sc, axis=1)
        assert ((am[k] == want_am) | tie).all(), "integer tile shift differs outside a tie"
        ties += int(tie.sum())
        same = am[k] == want_am
        close(g[k].reshape(-1, 2)[same], want_g.reshape(-1, 2)[same], atol=2e-4, what="sub-pixel shifts")
    assert ties <= 2


def test_upsample(cuda, oracle, rng):
    grid = rng.uniform(-3, 3, (6, 9, 2)).astype(np.float32)
    want = oracle.upsample_shifts(grid.astype(np.float64), 4, 2, 17, 12, 32, 32)
    out = dev(np.zeros((12, 17, 2), np.float32))
    ok(lib().isa_upsample_shifts(isa.vp(dev(grid)), sz(9 * 8), sz(6 * 9 * 8), isa.vp(out), sz(17 * 8), sz(12 * 17 * 8), 1, 4, 2, 9, 6, 17, 12,
                                 32, 32, S0))
    close(host(out), want, atol=2e-6, what="upsample")


@pytest.mark.parametrize("strategy,n,ref", [(P.FULL, 6, 0), (P.FULL, 20, 0), (P.FULL, 50, 0), (P.ONLY_ON_REFERENCE, 5, 2),
                                            (P.ON_REFERENCE_BLOCK, 9, 6), (P.BLOCKS, 7, 0)])
def test_solve_shifts(cuda, oracle, rng, strategy, n, ref):
    A = P.shift_matrix(n, ref, strategy, 3)
    m = A.shape[0]
    tcx, tcy = 7, 5
    truth = rng.uniform(-4, 4, (tcx * tcy, n - 1, 2))
    meas = (np.einsum("mk,tkc->tmc", A, truth) + rng.normal(0, 0.05, (tcx * tcy, m, 2))).astype(np.float32)
    meas[::2, rng.integers(0, m), :] += 6.0
    meas[1::3, rng.integers(0, m), 1] -= 9.0
    want_meas, want_x, want_st = oracle.solve_shifts(A, meas.astype(np.float64))
    grids = dev(np.ascontiguousarray(meas.transpose(1, 0, 2).reshape(m, tcy, tcx, 2)))
    x = dev(np.zeros((tcx * tcy, n - 1, 2), np.float32))
    st = dev(np.zeros(tcx * tcy, np.int32))
    mg = isa.Merger(512, 512, max(n, 2))
    ok(lib().isa_solve_shifts(mg.ctx, n, ref, strategy, 3, isa.vp(grids), sz(tcx * 8), sz(tcx * tcy * 8), tcx, tcy, isa.vp(x), isa.vp(st), S0))
    np.testing.assert_array_equal(host(st), want_st)
    close(host(x), want_x, atol=2e-5, what="one-to-one shifts")
    close(host(grids).reshape(m, -1, 2).transpose(1, 0, 2), want_meas, atol=5e-5, what="pair shifts")
    # getOptimalShifts
    for trk in (0, n - 1, n // 2):
        out = dev(np.zeros((tcy, tcx, 2), np.float32))
        ok(lib().isa_optimal_shifts(isa.vp(x), n, tcx, tcy, ref, trk, isa.vp(out), sz(tcx * 8), S0))
        close(host(out), oracle.optimal_shifts(host(x).astype(np.float64), tcx, tcy, ref, trk), atol=1e-5, what="optimal")
    mg.close()


def test_flow_warp_derivatives(cuda, oracle, rng):
    W, H = 160, 120
    tiles = rng.uniform(-3, 3, (4, 5, 2)).astype(np.float32)
    want_flow = oracle.flow_from_tiles(tiles.astype(np.float64), W, H, np.float32([1.25, -0.5]), float(np.float32(0.004)), 32)
    flow = dev(np.zeros((H, W, 2), np.float32))
    ok(lib().isa_flow_from_tiles(isa.vp(dev(tiles)), sz(5 * 8), 5, 4, W, H, (ctypes.c_float * 2)(1.25, -0.5), ctypes.c_float(0.004),
                                 isa.vp(flow), sz(W * 8), S0))
    fl = host(flow)
    close(fl, want_flow, atol=2e-5, what="flow from tiles")
    src, tgt = golden_cases._img(rng, W, H).astype(np.float32), golden_cases._img(rng, W, H).astype(np.float32)
    out = dev(np.zeros((H, W), np.float32))
    ok(lib().isa_warp(isa.vp(dev(src)), sz(W * 4), W, H, isa.vp(flow), sz(W * 8), isa.vp(out), sz(W * 4), S0))
    warped = host(out)
    close(warped, oracle.warp(src.astype(np.float64), fl.astype(np.float64)), atol=2e-6, what="warp")
    ix, iy, it = (dev(np.zeros((H, W), np.float32)) for _ in range(3))
    ok(lib().isa_derivatives(isa.vp(dev(warped)), isa.vp(dev(tgt)), sz(W * 4), W, H, isa.vp(ix), isa.vp(iy), isa.vp(it), sz(W * 4), S0))
    wx, wy, wt = oracle.derivatives(warped.astype(np.float64), tgt.astype(np.float64))
    close(host(ix), wx, atol=1e-6, what="Ix")
    close(host(iy), wy, atol=1e-6, what="Iy")
    close(host(it), wt, atol=1e-6, what="It")
    dx, dy = dev(np.zeros((H, W), np.float32)), dev(np.zeros((H, W), np.float32))
    ok(lib().isa_derivatives2(isa.vp(dev(src)), sz(W * 4), W, H, isa.vp(dx), isa.vp(dy), sz(W * 4), S0))
    ex, ey = oracle.derivatives2(src.astype(np.float64))
    close(host(dx), ex, atol=1e-6, what="dx")
    close(host(dy), ey, atol=1e-6, what="dy")
    # lucasKanadeOptim on the same derivative images
    f2 = dev(fl)
    ok(lib().isa_lucas_kanade(isa.vp(f2), sz(W * 8), isa.vp(ix), isa.vp(iy), isa.vp(it), sz(W * 4), W, H, ctypes.c_float(0.01), 11, S0))
    want = oracle.lucas_kanade(fl.astype(np.float64), host(ix).astype(np.float64), host(iy).astype(np.float64), host(it).astype(np.float64), 5,
                               float(np.float32(0.01)))
    close(host(f2), want, atol=1e-4, rtol=1e-5, what="LK update")


def test_lk_iteration_fused(cuda, oracle, rng):
    """The fused iteration (warp + derivatives + windowed LK) equals the
    oracle's three separate steps."""
    W, H = 200, 136
    ref = golden_cases._img(rng, W, H)
    src = np.roll(ref, (1, 2), axis=(0, 1)) + rng.normal(0, 0.002, (H, W))
    flow0 = (rng.uniform(-0.5, 0.5, (H, W, 2)) + np.array([1.7, 0.8])).astype(np.float32)
    a, b = dev(flow0), dev(np.zeros_like(flow0))
    ok(lib().isa_lk_iteration(isa.vp(a), isa.vp(b), sz(W * 8), isa.vp(dev(src.astype(np.float32))), isa.vp(dev(ref.astype(np.float32))),
                              sz(W * 4), W, H, ctypes.c_float(0.01), 11, S0))
    s64, r64 = src.astype(np.float32).astype(np.float64), ref.astype(np.float32).astype(np.float64)
    warped = oracle.warp(s64, flow0.astype(np.float64))
    ix, iy, it = oracle.derivatives(warped, r64)
    want = oracle.lucas_kanade(flow0.astype(np.float64), ix, iy, it, 5, float(np.float32(0.01)))
    got = host(b)
    err = np.abs(got - want).max(axis=2)
    # FP32 derivatives vs FP64: ill-conditioned windows amplify them; bound the tail
    assert np.percentile(err, 99.9) < 1e-4
    assert err.max() < 5e-3


def test_subsample_robustness_erode(cuda, oracle, rng):
    W, H = 192, 128
    raw = golden_cases._raw(rng, W, H)
    raw2 = np.roll(raw, (2, -4), axis=(0, 1))
    h1 = oracle.debayer_subsample(raw, (0, 1, 1, 2), 16383.0)
    h2 = oracle.debayer_subsample(raw2, (0, 1, 1, 2), 16383.0)
    o1 = dev(np.zeros((H // 2, W // 2, 3), np.float32))
    ok(lib().isa_debayer_subsample(isa.vp(dev(raw)), sz(W * 2), W, H, i4((0, 1, 1, 2)), ctypes.c_float(16383.0), isa.vp(o1), sz(W // 2 * 12), S0))
    close(host(o1), h1, atol=1e-7, what="subsample")
    o2 = dev(np.zeros((H // 2, W // 2, 3), np.float32))
    ok(lib().isa_debayer_subsample(isa.vp(dev(raw2)), sz(W * 2), W, H, i4((0, 1, 1, 2)), ctypes.c_float(16383.0), isa.vp(o2), sz(W // 2 * 12), S0))
    fl = rng.uniform(-3, 3, (H, W, 2)).astype(np.float32)
    alpha, beta = float(np.float32(4e-4)), float(np.float32(2e-6))
    for thr in (1e5, 5e-3):
        want = oracle.robustness_mask(host(o1).astype(np.float64), host(o2).astype(np.float64), fl.astype(np.float64), alpha, beta, thr,
                                      np.ones((H // 2, W // 2, 4)))
        mask = dev(np.ones((H // 2, W // 2, 4), np.float32))
        ok(lib().isa_robustness_mask(isa.vp(o1), isa.vp(o2), sz(W // 2 * 12), isa.vp(mask), sz(W // 2 * 16), W // 2, H // 2, isa.vp(dev(fl)),
                                     sz(W * 8), W, H, ctypes.c_float(alpha), ctypes.c_float(beta), ctypes.c_float(thr), ctypes.c_float(1.5),
                                     ctypes.c_float(0.12), S0))
        got = host(mask)
        err = np.abs(got - want)[..., :3]
        # a pixel whose shift round(flow/2) flips at .5 reads another neighbourhood: allow none here (flow is generic)
        assert err.max() < 2e-5, err.max()
        eroded = dev(np.zeros_like(got))
        ok(lib().isa_erode(isa.vp(mask), sz(W // 2 * 16), isa.vp(eroded), sz(W // 2 * 16), W // 2, H // 2, 5, S0))
        close(host(eroded), oracle.erode(got.astype(np.float64), 5), atol=0, what="erode")
        fused = dev(np.zeros_like(got))
        ok(lib().isa_robustness_erode(isa.vp(o1), isa.vp(o2), sz(W // 2 * 12), W // 2, H // 2, isa.vp(dev(fl)), sz(W * 8), W, H,
                                      ctypes.c_float(alpha), ctypes.c_float(beta), ctypes.c_float(thr), ctypes.c_float(1.5),
                                      ctypes.c_float(0.12), 5, isa.vp(fused), sz(W // 2 * 16), S0))
        close(host(fused), host(eroded), atol=0, what="fused mask+erode")


def test_kernel_params(cuda, oracle, rng):
    W, H = 128, 96
    img = (golden_cases._img(rng, W, H) * 0.3).astype(np.float32)
    st = dev(np.zeros((H, W, 3), np.float32))
    ok(lib().isa_structure_tensor(isa.vp(dev(img)), sz(W * 4), W, H, isa.vp(st), sz(W * 12), S0))
    dx, dy = oracle.derivatives2(img.astype(np.float64))
    want_st = oracle.structure_tensor(dx, dy)
    close(host(st), want_st, atol=1e-9, rtol=1e-5, what="structure tensor")
    g = host(st).astype(np.float64)
    kp = dev(np.zeros((H, W, 4), np.float32))
    p = P.MergeParams()
    ok(lib().isa_kernel_param(isa.vp(st), sz(W * 12), W, H, isa.vp(kp), sz(W * 16), 4, ctypes.c_float(p.dth), ctypes.c_float(p.dtr),
                              ctypes.c_float(p.k_detail), ctypes.c_float(p.k_denoise), ctypes.c_float(p.k_stretch), ctypes.c_float(p.k_shrink), S0))
    want = oracle.kernel_param(g, p)
    got = host(kp)
    close(got[..., :3], want, atol=0, rtol=2e-6, what="kernel params (FP64 from the same tensor)")
    assert (got[..., 3] == 0).all()


@pytest.mark.parametrize("mode", ["plain", "super", "full2x", "x1.5", "x3"])
def test_accumulate(cuda, oracle, rng, mode):
    W, H = 96, 64
    raw = golden_cases._raw(rng, W, H)
    kp = oracle.kernel_param(oracle.structure_tensor(*oracle.derivatives2(golden_cases._img(rng, W, H) * 0.3)), P.MergeParams())
    kp[3, 5] = np.nan
    fl = rng.uniform(-2.5, 2.5, (H, W, 2))
    mk = rng.uniform(0, 1, (H // 2, W // 2, 4))
    mk[2, 3, 1] = np.nan
    white, black = (15871.0, 15000.0, 14000.0), (512.0, 520.0, 500.0)
    if mode == "plain":
        s, org, crop, Wo, Ho = 1.0, (0, 0), (0, 0, W - 1, H - 1), W, H
    elif mode == "super":
        s, org, crop, Wo, Ho = 2.0, (W // 2, H // 2), (W // 4, H // 4, W // 2 - 1 + W // 4, H // 2 - 1 + H // 4), W, H
    else:
        s = {"full2x": 2.0, "x1.5": 1.5, "x3": 3.0}[mode]
        org, crop, Wo, Ho = (0, 0), (0, 0, W - 1, H - 1), int(round(W * s)), int(round(H * s))
    kp32, fl32, mk32 = kp.astype(np.float32), fl.astype(np.float32), mk.astype(np.float32)
    acc0 = rng.uniform(0, 1, (Ho, Wo, 3))
    w0 = rng.uniform(0, 1, (Ho, Wo, 3))
    want_a, want_w = acc0.copy(), w0.copy()
    oracle.accumulate(raw, (0, 1, 1, 2), want_a, want_w, mk32.astype(np.float64), kp32.astype(np.float64), fl32.astype(np.float64), white, black,
                      s, org, crop)
    a, w = dev(acc0.astype(np.float32)), dev(w0.astype(np.float32))
    kp4 = np.concatenate([kp32, np.zeros((H, W, 1), np.float32)], axis=2)
    ok(lib().isa_accumulate(isa.vp(dev(raw)), sz(W * 2), W, H, i4((0, 1, 1, 2)), isa.vp(a), isa.vp(w), sz(Wo * 12), Wo, Ho, isa.vp(dev(mk32)),
                            sz(W // 2 * 16), isa.vp(dev(kp4)), sz(W * 16), 4, isa.vp(dev(fl32)), sz(W * 8), f3(white), f3(black),
                            ctypes.c_float(s), org[0], org[1], i4(crop), S0))
    # output pixels whose round(s * flow) is within 1e-4 of .5 may take the
    # other integer shift in FP32 (a tie); everywhere else the 25-tap sums
    # (values ~1..10) agree at FP32 rounding level
    tie = rounding_ties(fl32.astype(np.float64), s, org, Wo, Ho)
    assert tie.mean() < 2e-3
    ga, gw = host(a), host(w)
    close(ga[~tie], want_a[~tie], atol=2e-5, rtol=2e-6, what="acc")
    close(gw[~tie], want_w[~tie], atol=2e-5, rtol=2e-6, what="wsum")


def rounding_ties(flow, s, org, Wo, Ho, margin=1e-4):
    """Output pixels whose shift round(s * flow(p)) sits within `margin` of a
    half-integer (flow sampled bilinearly with mirror addressing at the
    pixel's input position, as DeBayerKernels.cu:398-404 does)."""
    H, W, _ = flow.shape

    def axis(n_out, o, n_in):
        xb = (np.arange(n_out) + 0.5 + o) / s - 0.5
        f = np.floor(xb)
        i = f.astype(np.int64)
        a = xb - f
        m = lambda k: np.where(k < 0, -k - 1, np.where(k >= n_in, 2 * n_in - 1 - k, k))
        return m(i), m(i + 1), a

    x0, x1, ax = axis(Wo, org[0], W)
    y0, y1, ay = axis(Ho, org[1], H)
    A, B = ax[None, :, None], ay[:, None, None]
    f = (1 - A) * (1 - B) * flow[y0][:, x0] + A * (1 - B) * flow[y0][:, x1] + (1 - A) * B * flow[y1][:, x0] + A * B * flow[y1][:, x1]
    v = s * f
    return (np.abs(v - np.floor(v) - 0.5) < margin).any(axis=2)


def test_apply_weighting(cuda, oracle, rng):
    W, H = 64, 40
    acc = rng.uniform(0, 3, (H, W, 3)).astype(np.float32)
    ws = rng.uniform(0, 3, (H, W, 3)).astype(np.float32)
    ws[0, 0] = 0
    acc[0, 0] = 0
    dec = rng.uniform(0, 1, (H, W, 3)).astype(np.float32)
    for thr in (0.0, 1.0):
        want = oracle.apply_weighting(dec.astype(np.float64), acc.astype(np.float64), ws.astype(np.float64), thr)
        img = dev(dec)
        ok(lib().isa_apply_weighting(isa.vp(img), isa.vp(dev(acc)), isa.vp(dev(ws)), sz(W * 12), W, H, ctypes.c_float(thr), S0))
        close(host(img), want, atol=1e-6, rtol=1e-6, what=f"apply weighting {thr}")
