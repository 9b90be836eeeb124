"""isa_postprocess and isa_save_as_16bit_tiff on the GPU against the FP32
restatement (oracle/post.py), through the C ABI.

Tolerance: the kernel rounds every operation on its own exactly as the
restatement does, except the gamma: CUDA's powf (and the contraction of the
gamma's multiply-subtract into one FMA, as in the reference's own kernel)
may differ from the C library's powf by an ulp, which can move a converted
value by one code. So at most 1 code (16-bit or 8-bit) of difference, on at
most 2e-3 of the values (or 3 values in a tiny crop); everything else
bit-exact."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa, params as P, synthetic

import post as PO

pytestmark = pytest.mark.gpu


def lut_levels():
    return np.float32(np.round(np.arange(256) / 255.0, 9))


def tone(x):
    x = np.asarray(x, np.float64)
    return np.float32(np.clip(x + 0.12 * np.sin(2 * np.pi * x) / (2 * np.pi) + 0.02 * x * (1 - x), 0, 1))


def close(got, want):
    d = np.abs(got.astype(np.int64) - want.astype(np.int64))
    assert d.max() <= 1, d.max()
    assert (d > 0).sum() <= max(3, 2e-3 * d.size), (d > 0).sum()


def make_image(h, w, seed):
    rng = np.random.default_rng(seed)
    img = (rng.random((h, w, 3)) * 1.4 - 0.1).astype(np.float32)
    flat = img.reshape(-1)
    idx = rng.choice(flat.size, 40, replace=False)
    flat[idx[:10]] = np.nan
    flat[idx[10:20]] = np.inf
    flat[idx[20:30]] = -np.inf
    flat[idx[30:]] = -0.0
    return img


CAM = np.array([[0.62, 0.24, 0.10], [0.27, 0.69, 0.04], [0.03, 0.12, 0.68]])


@pytest.mark.parametrize("fmt", [isa.POST_RGB16, isa.POST_BGRA8])
@pytest.mark.parametrize("case", ["uniform", "irregular", "exposure", "crop"])
def test_postprocess_matches_oracle(cuda, fmt, case):
    import torch
    h, w = 257, 389
    img = make_image(h, w, 11)
    lx = lut_levels()
    if case == "irregular":
        lx = np.float32(np.sort(np.concatenate([[0.0, 1.0], np.random.default_rng(5).random(60)])))
    ly = tone(lx)
    crop = (0, 0, w, h) if case != "crop" else (7, 3, 301, 250)
    exposure = 0.7 if case == "exposure" else 0.0
    wb = [1.0, 0.9, 1.15]
    t1, t2 = isa.color_twists(CAM)
    pp, keep = isa.post_params(crop, wb, t1, t2, lx, ly, exposure)
    dev = torch.from_numpy(img).cuda()
    got = isa.postprocess(dev, pp, fmt)
    torch.cuda.synchronize()
    got = got.cpu().numpy()
    if fmt == isa.POST_RGB16:
        got = got.view(np.uint16)
    want = PO.postprocess(img, crop, wb, t1, t2, lx, ly, exposure, fmt=fmt)
    assert got.shape == want.shape
    close(got, want)
    if fmt == isa.POST_BGRA8:
        assert np.all(got[..., 3] == 255)


def test_merge_then_save_tiff(cuda, tmp_path):
    """A merged burst through SaveAs16BitTiff: the file is the restatement's bytes
    for the GPU-converted image, and that image is within tolerance of the oracle."""
    import torch
    b = synthetic.make_burst(512, 384, 3, seed=9, max_shift=3, max_rot_deg=0.0)
    m = isa.Merger(b.width, b.height, b.n, P.MergeParams())
    raw = torch.from_numpy(np.ascontiguousarray(b.raw).view(np.int16)).cuda()
    merged = m.merge(raw, isa.make_info(b))
    torch.cuda.synchronize()
    t1, t2 = isa.color_twists(CAM)
    lx = lut_levels()
    ly = tone(lx)
    crop = (2, 2, b.width - 4, b.height - 4)
    pp, keep = isa.post_params(crop, [1, 1, 1], t1, t2, lx, ly, 0.3)
    path = tmp_path / "merged.tif"
    isa.save_as_16bit_tiff(merged, pp, str(path))
    buf = path.read_bytes()
    tags, img = PO.parse_tiff16(buf)
    assert img.shape == (crop[3], crop[2], 3)
    gpu = isa.postprocess(merged, pp, isa.POST_RGB16)
    torch.cuda.synchronize()
    gpu = gpu.cpu().numpy().view(np.uint16)
    assert buf == PO.tiff16_bytes(gpu)
    close(gpu, PO.postprocess(merged.cpu().numpy(), crop, [1, 1, 1], t1, t2, lx, ly, 0.3))
    assert img.std() > 100  # a real picture, not a constant


def test_postprocess_large_crop_edges(cuda):
    """Crop sizes that are not multiples of the 64 x 4 thread block, at the far corner."""
    import torch
    h, w = 131, 200
    img = make_image(h, w, 3)
    lx = lut_levels()
    t1, t2 = isa.color_twists(np.eye(3) * 0.8)
    for crop in [(w - 1, h - 1, 1, 1), (w - 65, h - 5, 65, 5), (0, 0, 63, 131)]:
        pp, keep = isa.post_params(crop, [1, 1, 1], t1, t2, lx, lx, 0.0)
        got = isa.postprocess(torch.from_numpy(img).cuda(), pp, isa.POST_RGB16)
        torch.cuda.synchronize()
        close(got.cpu().numpy().view(np.uint16), PO.postprocess(img, crop, [1, 1, 1], t1, t2, lx, lx, 0.0))


def test_pef_file_to_tiff_chain(cuda, tmp_path):
    """The reference's flow from PEF pixel data to the 16-bit TIFF: frames
    decoded from the compressed stream layout (isa_pef_decode), merged, the
    colour spec of PEFFile.SetMembers from the white balance
    (isa_pef_color_spec), its camera white and twists into SaveAs16BitTiff."""
    import torch
    from imagestackalignator_b200 import synthetic as S
    import raw as R
    import colorspec as CS
    b = synthetic.make_burst(512, 384, 3, seed=12, max_shift=3, max_rot_deg=0.0)
    code, lens = S.pef_code_book()
    table = isa.pef_huff_table(S.pef_maker_note(code, lens))
    frames = []
    for f in range(b.n):
        stream = S.pef_stream(b.raw[f], code, lens)
        out = isa.pef_decode(torch.from_numpy(stream).cuda(), table, b.width, b.height)
        frames.append(out)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint16), R.decode(stream, R.huff_table(S.pef_maker_note(code, lens)), b.width, b.height))
    raw = torch.stack(frames)
    assert np.array_equal(raw.cpu().numpy().view(np.uint16), b.raw)
    m = isa.Merger(b.width, b.height, b.n, P.MergeParams())
    merged = m.merge(raw, isa.make_info(b))
    torch.cuda.synchronize()
    wb = np.float32([1.9, 1.0, 1.6])
    c2p, cw, xy = isa.pef_color_spec(wb)
    want_spec = CS.pef_color_spec(wb)
    assert np.array_equal(c2p, want_spec[0]) and np.array_equal(cw, want_spec[1])
    t1, t2 = isa.color_twists(c2p)
    lx = lut_levels()
    crop = (2, 2, b.width - 4, b.height - 4)   # the PEF crop (PEFFile.cs:266-270)
    pp, keep = isa.post_params(crop, np.float32(cw), t1, t2, lx, tone(lx), 0.0)
    path = tmp_path / "burst.tif"
    isa.save_as_16bit_tiff(merged, pp, str(path))
    tags, img = PO.parse_tiff16(path.read_bytes())
    close(img, PO.postprocess(merged.cpu().numpy(), crop, np.float32(cw), t1, t2, lx, tone(lx), 0.0))


def test_pef_files_to_tiff(cuda, tmp_path):
    """A burst of PEF files through the C ABI alone: isa_pef_open (IFD 0 strip, Exif CFA
    pattern, Pentax maker note), isa_pef_huff_table, isa_pef_levels, isa_pef_decode of the
    strip, the merge with those levels, the PEF colour spec and SaveAs16BitTiff."""
    import torch
    b = synthetic.make_burst(512, 384, 3, seed=14, max_shift=3, max_rot_deg=0.0)
    frames = []
    for f in range(b.n):
        file, offs, cnts = synthetic.pef_file(b.raw[f], cfa=tuple(b.cfa), big_endian=f == 2, note=["AOC", "PENTAX", "AOC"][f],
                                              black=(512, 512, 512, 512), white_point=(15000, 8192, 8192, 12000), scaling=8192,
                                              white_level=16383)
        d = isa.pef_open(file)
        assert d["compressed"] and (d["width"], d["height"]) == (b.width, b.height) and d["cfa"] == list(b.cfa)
        table = isa.pef_huff_table(d["huffman_table"], big_endian=d["huffman_big_endian"])
        o, n = d["strip_offsets"][0], d["strip_sizes"][0]
        strip = torch.from_numpy(np.ascontiguousarray(file[o:o + n])).cuda()
        out = isa.pef_decode(strip, table, b.width, b.height)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint16), b.raw[f])
        frames.append(out)
    black, white, wb = isa.pef_levels(d["cfa"], d["black_point"], d["white_level"], d["white_point"], d["scaling"], d["bit_depth"])
    info = isa.make_info(b)
    for c in range(3):
        info.black[c] = float(black[c])
        info.white[c] = float(white[c])
    c2p, cw, xy = isa.pef_color_spec(wb)
    for c in range(3):
        info.camera_white[c] = float(cw[c])
    merged = isa.Merger(b.width, b.height, b.n, P.MergeParams()).merge(torch.stack(frames), info)
    torch.cuda.synchronize()
    t1, t2 = isa.color_twists(c2p)
    lx = lut_levels()
    crop = (2, 2, b.width - 4, b.height - 4)
    pp, keep = isa.post_params(crop, np.float32(cw), t1, t2, lx, tone(lx), 0.0)
    path = tmp_path / "pef_burst.tif"
    isa.save_as_16bit_tiff(merged, pp, str(path))
    tags, img = PO.parse_tiff16(path.read_bytes())
    close(img, PO.postprocess(merged.cpu().numpy(), crop, np.float32(cw), t1, t2, lx, tone(lx), 0.0))
    assert img.std() > 100
