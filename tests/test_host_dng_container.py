"""The DNG container reader (isa_dng_open / isa_dng_file_info, host code of
libisa.so) without a GPU: files written by synthetic.dng_file in both byte
orders, with the raw image in a SubIFD or in IFD 0, read back tag by tag;
the raw-IFD rule of DNGFile.SetMembers; the parsed tags through
isa_dng_color_spec and isa_dng_levels against the restatements in
oracle/colorspec.py and oracle/rawmeta.py; files the reference cannot read."""
import struct

import numpy as np
import pytest

from imagestackalignator_b200 import isa, synthetic as S

import colorspec as CS
import rawmeta as RM

COLOR = dict(color_matrix1=[0.9, -0.2, -0.1, -0.4, 1.2, 0.2, -0.05, 0.2, 0.6], color_matrix2=[1.1, -0.3, 0.0, -0.3, 1.3, 0.1, 0.0, 0.1, 0.8],
             illuminant1=17, illuminant2=21, forward_matrix1=[0.6, 0.3, 0.1, 0.25, 0.7, 0.05, 0.0, 0.1, 0.7],
             camera_calibration1=[1.02, 0, 0, 0, 1.0, 0, 0, 0, 0.98], analog_balance=[1.0, 1.0, 1.0], as_shot_neutral=[0.45, 1.0, 0.62])


def _img(h=96, w=160, seed=0):
    return np.random.default_rng(seed).integers(512, 16000, (h, w)).astype(np.uint16)


def _rat(v, den=1000):
    return round(v * den) / den


@pytest.mark.parametrize("big", [False, True])
@pytest.mark.parametrize("sub", [True, False])
def test_tags_read_back(big, sub):
    img = _img()
    aa = [2, 4, 94, 156]
    dh, dv = [1, 2] * 76, [0, 3] * 46
    noise = [2e-5, 1e-7, 3e-5, 2e-7, 4e-5, 3e-7]
    f, offs, cnts = S.dng_file(img, cfa=(1, 0, 2, 1), big_endian=big, raw_in_subifd=sub, active_area=aa, crop=[3.5, 2, 140, 80],
                               deltas=(dh, dv), noise=noise, plane_color=[0, 1, 2], iso=400, color=COLOR, extra_chain_ifd=True,
                               linearization=np.arange(0, 32768, 2))
    d = isa.dng_open(f)
    assert (d["width"], d["height"]) == (160, 96)
    L = d["layout"]
    assert L["tiled"] and (L["tile_w"], L["tile_h"]) == (128, 128) and L["offsets"] == offs and L["counts"] == cnts
    assert L["compression"] == 7 and L["bit_depth"] == 16 and L["large"] and L["linearization"] == list(range(0, 32768, 2))
    G = d["levels"]
    assert G["cfa_pattern"] == [1, 0, 2, 1] and G["cfa_repeat"] == (2, 2) and G["white_level"] == 16383 and G["black_level"] == [512.0]
    assert G["active_area"] == aa and G["plane_color"] == [0, 1, 2] and G["iso"] == 400
    assert G["default_crop_origin"] == [3.5, 2.0] and G["default_crop_size"] == [140.0, 80.0]
    assert G["noise_profile"] == noise and G["black_delta_h"] == [float(v) for v in dh] and G["black_delta_v"] == [float(v) for v in dv]
    C = d["color"]
    for k in ("color_matrix1", "color_matrix2", "forward_matrix1", "camera_calibration1", "analog_balance", "as_shot_neutral"):
        assert C[k] == [_rat(v, 10000) for v in COLOR[k]], k
    assert C["camera_calibration2"] == C["camera_calibration1"]   # the reference reads CameraCalibration1 for both
    assert (C["illuminant1"], C["illuminant2"]) == (17, 21) and C["forward_matrix2"] is None and C["as_shot_white_xy"] is None


def test_parsed_tags_through_levels_and_color_spec():
    img = _img(seed=1)
    f, offs, cnts = S.dng_file(img, active_area=[1, 3, 95, 157], crop=[2, 2, 120, 60], deltas=([2] * 154, [1] * 94),
                               noise=[2e-5, 1e-7], black=(510, 512, 514, 516), iso=800, color=COLOR)
    d = isa.dng_open(f)
    got = isa.dng_color_spec(**d["color"])
    want = CS.dng_color_spec(**d["color"])
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g).reshape(-1), np.asarray(w).reshape(-1))
    lv = isa.dng_levels(camera_white=got[1], **d["levels"])
    ref = RM.dng_levels(camera_white=want[1], **d["levels"])
    for k in ("black", "white", "camera_white", "white_balance", "color_twist", "black_h", "black_v"):
        assert np.array_equal(lv[k], ref[k]), k
    assert lv["cfa"] == ref["cfa"] and lv["crop"] == ref["crop"] and lv["noise"] == ref["noise"]
    assert lv["cfa"] == [2, 1, 1, 0]   # odd ActiveArea origin in both axes shifts RGGB


def test_dng_version_decides_the_large_category():
    img = _img(32, 32)
    assert isa.dng_open(S.dng_file(img, tile=32, version=(1, 1, 0, 0))[0])["layout"]["large"] is False
    assert isa.dng_open(S.dng_file(img, tile=32, version=(1, 2, 0, 0))[0])["layout"]["large"] is True
    assert isa.dng_open(S.dng_file(img, tile=32, version=None)[0])["layout"]["large"] is True


def test_raw_ifd_is_the_last_chain_ifds_cfa_subifd():
    """No CFA IFD in the chain: each chain IFD's first CFA SubIFD replaces the previous one (DNGFile.cs:639-660)."""
    out = bytearray(b"II" + struct.pack("<HI", 42, 0))

    def cfa_ifd(width):
        return [(256, 4, [width]), (257, 4, [8]), (258, 3, [16]), (259, 3, [7]), (262, 3, [32803]), (273, 4, [8]), (279, 4, [4]),
                (33421, 3, [2, 2]), (33422, 1, [0, 1, 1, 2]), (50717, 4, [4095])]
    at = {}
    for name, w in (("a1", 32), ("a2", 40), ("b1", 64)):
        at[name] = len(out)
        out += S._ifd_bytes(cfa_ifd(w), len(out), False, 0)
    at["ifd1"] = len(out)
    out += S._ifd_bytes([(254, 4, [1]), (330, 4, [at["b1"]])], len(out), False, 0)
    at["ifd0"] = len(out)
    out += S._ifd_bytes([(254, 4, [1]), (330, 4, [at["a1"], at["a2"]])], len(out), False, at["ifd1"])
    struct.pack_into("<I", out, 4, at["ifd0"])
    assert isa.dng_open(bytes(out))["width"] == 64


@pytest.mark.parametrize("damage", ["order", "magic", "truncated", "loop", "no_white", "no_cfa"])
def test_unreadable_files(damage):
    img = _img(32, 32)
    f, offs, cnts = S.dng_file(img, tile=32)
    b = bytearray(f.tobytes())
    if damage == "order":
        b[0:2] = b"IM"
    elif damage == "magic":
        b[2:4] = struct.pack("<H", 43)
    elif damage == "truncated":
        ifd0 = struct.unpack_from("<I", b, 4)[0]
        b = b[:ifd0 + 20]
    elif damage == "loop":
        ifd0 = struct.unpack_from("<I", b, 4)[0]
        n = struct.unpack_from("<H", b, ifd0)[0]
        struct.pack_into("<I", b, ifd0 + 2 + 12 * n, ifd0)
    elif damage == "no_white":
        i = bytes(b).find(struct.pack("<HH", 50717, 4))
        struct.pack_into("<H", b, i, 50718)   # a tag the reader does not know
    elif damage == "no_cfa":
        i = bytes(b).find(struct.pack("<HHI", 262, 3, 1) + struct.pack("<H", 32803))
        struct.pack_into("<H", b, i + 8, 32804)
    with pytest.raises(isa.IsaError) as e:
        isa.dng_open(bytes(b))
    assert e.value.code == isa.ISA_EINVAL


def test_out_of_range_tag_values_are_refused():
    """Tag values that do not fit the integer they stand for (a rational width of
    2^32 - 1, a negative strip offset) are ISA_EINVAL, not a wrapped number."""
    def cfa_file(width_entry, offsets_entry):
        out = bytearray(b"II" + struct.pack("<HI", 42, 0))
        ifd = [width_entry, (257, 4, [8]), (258, 3, [16]), (259, 3, [7]), (262, 3, [32803]), offsets_entry, (279, 4, [4]),
               (33421, 3, [2, 2]), (33422, 1, [0, 1, 1, 2]), (50717, 4, [4095])]
        at = len(out)
        out += S._ifd_bytes(ifd, at, False, 0)
        struct.pack_into("<I", out, 4, at)
        return bytes(out)
    assert isa.dng_open(cfa_file((256, 4, [32]), (273, 4, [8])))["width"] == 32
    for bad in (cfa_file((256, 5, [(2 ** 32 - 1, 1)]), (273, 4, [8])), cfa_file((256, 4, [32]), (273, 10, [(-8, 1)]))):
        with pytest.raises(isa.IsaError) as e:
            isa.dng_open(bad)
        assert e.value.code == isa.ISA_EINVAL


@pytest.mark.parametrize("note", ["AOC", "PENTAX"])
@pytest.mark.parametrize("big", [False, True])
def test_roll_angle_from_private_data(note, big):
    """The Pentax maker note copied into DNGPrivateData behind the "Adobe\\0MakN" header
    (offsets from the original file for "AOC", from the note for "PENTAX"): LevelInfo's roll angle."""
    img = _img(32, 32)
    assert isa.dng_open(S.dng_file(img, tile=32, big_endian=big, private_note=note, roll_byte=-9)[0])["roll_angle"] == 4.5
    assert isa.dng_open(S.dng_file(img, tile=32, big_endian=big)[0])["roll_angle"] is None
