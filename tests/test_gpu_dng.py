"""DNG pixel data on the GPU (isa_dng_decode) against the restated reference
reader (oracle/raw.py over orc_dng_decode), bit-exact: lossless-JPEG tiles
with every predictor and one or two interleaved components, strips,
restart markers, tiles that overhang the frame, linearisation and black-
level deltas, a sample above the bit depth (the reference stops), and
uncompressed 16-bit and packed strips. Predictor-1 frames without restarts
go through the parallel decoder (isa_dng_decode_path() == 1), the rest
through the per-part reader; random entropy data (0xFF runs, empty code
entries, data that ends early) and the hand-back to the per-part reader
are checked on both."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa

import raw as R

pytestmark = pytest.mark.gpu


def run(file, W, H, offs, cnts, **kw):
    import torch
    out = isa.dng_decode(file, W, H, offs, cnts, **kw)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint16)


@pytest.mark.parametrize("psv", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("clrs", [1, 2])
def test_lj92_tiles(cuda, psv, clrs):
    rng = np.random.default_rng(psv * 10 + clrs)
    H, W = 100, 160
    img = np.clip(rng.normal(3000, 500, (H, W)), 0, 16383).astype(np.uint16)
    f, offs, cnts = R.dng_tiles(img, 64, 48, clrs=clrs, bits=14, psv=psv)
    kw = dict(tiled=True, tile_w=64, tile_h=48)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0 and np.array_equal(want, img)
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)
    assert isa.dng_decode_path() == (1 if psv == 1 else 0)


def _data_start(part):
    """Offset of the entropy data in a lossless-JPEG part (after the SOS segment)."""
    p = bytes(bytearray(part))
    pos = 2
    while True:
        tag = p[pos] << 8 | p[pos + 1]
        pos += 2 + (p[pos + 2] << 8 | p[pos + 3])
        if tag == 0xFFDA:
            return pos


def _random_entropy(f, offs, cnts, seed, ff, nbytes=None, ff_run=0):
    """The same headers with random entropy bytes (a fraction `ff` of them 0xFF, optionally one long 0xFF run)."""
    r = np.random.default_rng(seed)
    parts, no, nc, pos = [f[:offs[0]]], [], [], offs[0]
    for o, c in zip(offs, cnts):
        p = f[o:o + c]
        h = _data_start(p)
        n = nbytes if nbytes is not None else c - h
        d = r.integers(0, 256, n).astype(np.uint8)
        d[r.random(n) < ff] = 0xFF
        if ff_run:
            d[n // 2:n // 2 + ff_run] = 0xFF
        q = np.concatenate([p[:h], d])
        no.append(pos); nc.append(len(q)); parts.append(q); pos += len(q)
    return np.concatenate(parts), no, nc


@pytest.mark.parametrize("seed", range(8))
def test_lj92_random_entropy_data(cuda, seed):
    """16-bit frames (every decoded value is in range) whose entropy bytes are random: 0xFF
    runs for the byte skipping, empty code-book entries that stop a part, data that ends early."""
    rng = np.random.default_rng(100 + seed)
    H, W = 120, 200
    img = rng.integers(0, 32768, (H, W)).astype(np.uint16)  # differences stay inside categories 0..15
    clrs = 1 + seed % 2
    f, offs, cnts = R.dng_tiles(img, 64, 40, clrs=clrs, bits=16, psv=1)
    nbytes = [None, None, None, 50, None, 7, None, None][seed]
    f, offs, cnts = _random_entropy(f, offs, cnts, seed, ff=[0.02, 0.3, 0.6, 0.0, 0.1, 0.0, 0.45, 0.05][seed], nbytes=nbytes)
    kw = dict(tiled=True, tile_w=64, tile_h=40, large=seed % 3 != 0)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)
    assert isa.dng_decode_path() == 1


def test_lj92_long_ff_run_goes_to_the_per_part_reader(cuda):
    """A run of more than 64 0xFF bytes is handed back to the per-part reader: same result."""
    rng = np.random.default_rng(7)
    H, W = 80, 128
    img = rng.integers(0, 32768, (H, W)).astype(np.uint16)  # differences stay inside categories 0..15
    f, offs, cnts = R.dng_tiles(img, 64, 40, clrs=2, bits=16, psv=1)
    f, offs, cnts = _random_entropy(f, offs, cnts, 3, ff=0.05, ff_run=101)
    kw = dict(tiled=True, tile_w=64, tile_h=40)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)
    assert isa.dng_decode_path() == 0


def test_lj92_strips_restart_lin_black(cuda):
    rng = np.random.default_rng(3)
    H, W = 90, 128
    img = np.clip(rng.normal(2000, 400, (H, W)), 0, 4095).astype(np.uint16)
    parts, offs, cnts, pos = [np.zeros(16, np.uint8)], [], [], 16
    rps = 30
    for s in range(0, H, rps):
        t = R.lj92_encode(img[s:s + rps], clrs=2, bits=12, psv=1, restart=64 * 10)
        offs.append(pos); cnts.append(len(t)); parts.append(t); pos += len(t)
    f = np.concatenate(parts)
    lin = (np.arange(4096) * 3 // 2).astype(np.uint16)
    bh = rng.integers(0, 40, W).astype(np.uint16)
    bv = rng.integers(0, 40, H).astype(np.uint16)
    kw = dict(tiled=False, rows_per_strip=rps, linearization=lin, black_h=bh, black_v=bv)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)


def test_lj92_overhanging_tiles_and_large_frame(cuda):
    rng = np.random.default_rng(4)
    H, W = 600, 1000                  # tiles of 256 overhang both edges
    img = np.clip(rng.normal(8000, 900, (H, W)), 0, 16383).astype(np.uint16)
    f, offs, cnts = R.dng_tiles(img, 256, 256, clrs=2, bits=14, psv=1)
    kw = dict(tiled=True, tile_w=256, tile_h=256)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0 and np.array_equal(want, img)
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)
    assert isa.dng_decode_path() == 1


def test_lj92_sample_above_bit_depth_is_an_error(cuda):
    img = np.full((16, 32), 5000, np.uint16)
    f, offs, cnts = R.dng_tiles(img, 32, 16, clrs=1, bits=14, psv=1)
    # declare 12 bits in the frame header (SOF3 precision byte follows the 4-byte marker/length after SOI)
    g = f.copy()
    sof = 32 + 2
    assert g[sof] == 0xFF and g[sof + 1] == 0xC3
    g[sof + 4] = 12
    st, _ = R.dng_decode(g, 32, 16, offs, cnts, tiled=True, tile_w=32, tile_h=16)
    assert st == -1
    with pytest.raises(isa.IsaError):
        run(g, 32, 16, offs, cnts, tiled=True, tile_w=32, tile_h=16)


@pytest.mark.parametrize("depth", [16, 14, 12, 10])
def test_uncompressed_strips(cuda, depth):
    rng = np.random.default_rng(depth)
    H, W, rps = 77, 150, 20
    img = rng.integers(0, 1 << depth, (H, W)).astype(np.uint16)
    parts, offs, cnts, pos = [np.full(40, 7, np.uint8)], [], [], 40
    for s in range(0, H, rps):
        blk = img[s:s + rps]
        b = blk.astype("<u2").tobytes() if depth == 16 else R.pack(blk, depth).tobytes()
        b = np.frombuffer(b, np.uint8)
        offs.append(pos); cnts.append(len(b)); parts.append(b); pos += len(b)
    f = np.concatenate(parts)
    kw = dict(compression=1, tiled=False, rows_per_strip=rps, bit_depth=depth)
    st, want = R.dng_decode(f, W, H, offs, cnts, **kw)
    assert st == 0 and np.array_equal(want, img)
    assert np.array_equal(run(f, W, H, offs, cnts, **kw), want)


def test_dng_file_to_tiff_chain(cuda, tmp_path):
    """The reference's flow from DNG tags and pixel data to the 16-bit TIFF:
    levels and geometry of DNGFile.SetMembers (isa_dng_levels, with an active
    area and black-level deltas), tiles decoded with the placed deltas
    (isa_dng_decode), the burst merged with those levels, the colour spec from
    the tags (isa_dng_color_spec), SaveAs16BitTiff with the DNG crop."""
    import torch
    from imagestackalignator_b200 import params as P, synthetic
    import post as PO
    import rawmeta as RM
    b = synthetic.make_burst(512, 384, 3, seed=21, max_shift=3, max_rot_deg=0.0)
    W, H = b.width, b.height
    aa = [2, 4, H - 2, W - 4]
    rng = np.random.default_rng(8)
    dv = rng.integers(0, 6, aa[2] - aa[0]).astype(float)
    dh = rng.integers(0, 4, aa[3] - aa[1]).astype(float)
    cm1 = [0.9, -0.2, -0.1, -0.4, 1.2, 0.2, -0.05, 0.2, 0.6]
    c2p, cw, xy = isa.dng_color_spec(color_matrix1=cm1, illuminant1=21, as_shot_neutral=[0.5, 1.0, 0.7])
    tags = dict(width=W, height=H, cfa_pattern=list(b.cfa), white_level=16383.0, camera_white=cw, black_level=[512, 512, 512, 512],
                active_area=aa, black_delta_v=dv, black_delta_h=dh, noise_profile=[b.noise_a, b.noise_b])
    lv = isa.dng_levels(**tags)
    want = RM.dng_levels(**tags)
    assert np.array_equal(lv["black_h"], want["black_h"]) and np.array_equal(lv["white"], want["white"])
    assert lv["cfa"] == list(b.cfa)           # even active-area origin: the CFA stays
    frames = []
    for f in range(b.n):
        file, offs, cnts = R.dng_tiles(b.raw[f], 128, 128, clrs=2, bits=14, psv=1)
        kw = dict(tiled=True, tile_w=128, tile_h=128, black_h=lv["black_h"], black_v=lv["black_v"])
        st, ref = R.dng_decode(file, W, H, offs, cnts, **kw)
        assert st == 0
        got = isa.dng_decode(file, W, H, offs, cnts, **kw)
        torch.cuda.synchronize()
        assert np.array_equal(got.cpu().numpy().view(np.uint16), ref)
        frames.append(got)
    raw = torch.stack(frames)
    m = isa.Merger(W, H, b.n, P.MergeParams())
    merged = m.merge(raw, lv["info"])
    torch.cuda.synchronize()
    assert np.isfinite(merged.cpu().numpy()).all()
    t1, t2 = isa.color_twists(c2p)
    lx = np.float32(np.round(np.arange(256) / 255.0, 9))
    x, y, w, h = lv["crop"]
    crop = (x, y, min(w, W - x), min(h, H - y))
    pp, keep = isa.post_params(crop, np.float32(cw), t1, t2, lx, lx, 0.0)
    path = tmp_path / "dng.tif"
    isa.save_as_16bit_tiff(merged, pp, str(path))
    tags_out, img = PO.parse_tiff16(path.read_bytes())
    assert img.shape == (crop[3], crop[2], 3)
    wantimg = PO.postprocess(merged.cpu().numpy(), crop, np.float32(cw), t1, t2, lx, lx, 0.0)
    d = np.abs(img.astype(np.int64) - wantimg.astype(np.int64))
    assert d.max() <= 1 and (d > 0).sum() <= max(3, 2e-3 * d.size)
    assert img.std() > 100


def test_dng_files_to_tiff(cuda, tmp_path):
    """A burst of DNG files through the C ABI alone: isa_dng_open, isa_dng_color_spec,
    isa_dng_levels, isa_dng_decode (the parallel decoder), the merge with the file's
    levels and SaveAs16BitTiff with the file's crop and colour spec."""
    import torch
    from imagestackalignator_b200 import params as P, synthetic
    import post as PO
    b = synthetic.make_burst(512, 384, 3, seed=31, max_shift=3, max_rot_deg=0.0)
    W, H = b.width, b.height
    color = dict(color_matrix1=[0.9, -0.2, -0.1, -0.4, 1.2, 0.2, -0.05, 0.2, 0.6], illuminant1=21, as_shot_neutral=[0.52, 1.0, 0.71])
    dh = [1, 0, 2, 0] * ((W - 8) // 4)
    dv = [0, 1] * ((H - 4) // 2)
    frames, lv, c2p, cw = [], None, None, None
    for f in range(b.n):
        file, offs, cnts = synthetic.dng_file(b.raw[f], cfa=tuple(b.cfa), tile=128, active_area=[2, 4, H - 2, W - 4], deltas=(dh, dv),
                                              noise=[b.noise_a, b.noise_b], color=color, big_endian=f == 1)
        d = isa.dng_open(file)
        assert (d["width"], d["height"]) == (W, H)
        c2p, cw, xy = isa.dng_color_spec(**d["color"])
        lv = isa.dng_levels(camera_white=cw, **d["levels"])
        got = isa.dng_decode(file, W, H, black_h=lv["black_h"], black_v=lv["black_v"], **d["layout"])
        torch.cuda.synchronize()
        assert isa.dng_decode_path() == 1
        st, want = R.dng_decode(file, W, H, offs, cnts, tiled=True, tile_w=128, tile_h=128, black_h=lv["black_h"], black_v=lv["black_v"])
        assert st == 0 and np.array_equal(got.cpu().numpy().view(np.uint16), want)
        frames.append(got)
    assert lv["cfa"] == list(b.cfa) and lv["noise"] == (np.float32(b.noise_a), np.float32(b.noise_b))
    merged = isa.Merger(W, H, b.n, P.MergeParams()).merge(torch.stack(frames), lv["info"])
    torch.cuda.synchronize()
    t1, t2 = isa.color_twists(c2p)
    lx = np.float32(np.round(np.arange(256) / 255.0, 9))
    x, y, w, h = lv["crop"]
    crop = (x, y, min(w, W - x), min(h, H - y))
    pp, keep = isa.post_params(crop, np.float32(cw), t1, t2, lx, lx, 0.0)
    path = tmp_path / "burst.tif"
    isa.save_as_16bit_tiff(merged, pp, str(path))
    tags, img = PO.parse_tiff16(path.read_bytes())
    want = PO.postprocess(merged.cpu().numpy(), crop, np.float32(cw), t1, t2, lx, lx, 0.0)
    d = np.abs(img.astype(np.int64) - want.astype(np.int64))
    assert d.max() <= 1 and (d > 0).sum() <= max(3, 2e-3 * d.size)
    assert img.std() > 100


def test_begin_finish_over_many_frames(cuda):
    """isa_dng_decode_begin for every frame, then isa_dng_decode_finish for every frame:
    each output equals isa_dng_decode's, for frames of the parallel decoder, a frame it
    hands back (a long 0xFF run) and a frame of the per-part reader (predictor 2)."""
    import torch
    rng = np.random.default_rng(17)
    H, W = 80, 128
    cases = []
    for kind in ("parallel", "handback", "psv2", "parallel"):
        img = rng.integers(0, 32768, (H, W)).astype(np.uint16)
        f, offs, cnts = R.dng_tiles(img, 64, 40, clrs=2, bits=16, psv=2 if kind == "psv2" else 1)
        if kind == "handback":
            f, offs, cnts = _random_entropy(f, offs, cnts, 9, ff=0.05, ff_run=101)
        cases.append((kind, f, offs, cnts))
    kw = dict(tiled=True, tile_w=64, tile_h=40)
    want = [run(f, W, H, o, c, **kw) for _, f, o, c in cases]
    jobs = []
    for kind, f, o, c in cases:
        dev = torch.from_numpy(f).cuda()
        scratch = torch.empty(isa.dng_decode_scratch(f, W, H, o, c, **kw), dtype=torch.uint8, device="cuda")
        out = torch.full((H, W), -1, dtype=torch.int16, device="cuda")
        isa.dng_decode(f, W, H, o, c, file_dev=dev, scratch=scratch, out=out, phase="begin", **kw)
        jobs.append((f, o, c, dev, scratch, out))
    paths = []
    for f, o, c, dev, scratch, out in jobs:
        isa.dng_decode(f, W, H, o, c, file_dev=dev, scratch=scratch, out=out, phase="finish", **kw)
        paths.append(isa.dng_decode_path())
    torch.cuda.synchronize()
    assert paths == [1, 0, 0, 1]
    for (f, o, c, dev, scratch, out), w in zip(jobs, want):
        assert np.array_equal(out.cpu().numpy().view(np.uint16), w)
