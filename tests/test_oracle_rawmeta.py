"""Raw-file metadata without a GPU: isa_dng_levels, isa_noise_model,
isa_crop_window and isa_profile_color_spec (host code of libisa.so) against
the restatement in oracle/rawmeta.py and oracle/colorspec.py, field for
field and bit for bit, plus the reference's throwing cases."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa

import colorspec as CS
import rawmeta as RM

CFAS = [[0, 1, 1, 2], [1, 0, 2, 1], [2, 1, 1, 0], [1, 2, 0, 1]]


def same(got, want):
    for k in ("cfa", "crop", "color_twist_identity"):
        assert got[k] == want[k] or list(got[k]) == list(want[k]), k
    for k in ("black", "white", "camera_white", "white_balance", "color_twist", "black_h", "black_v"):
        assert np.array_equal(got[k], want[k]), (k, got[k], want[k])
    assert got["noise"][0] == want["noise"][0] and got["noise"][1] == want["noise"][1]


def random_tags(rng):
    W = int(rng.integers(24, 200))
    H = int(rng.integers(24, 160))
    t = dict(width=W, height=H, cfa_pattern=CFAS[rng.integers(4)], white_level=float(rng.choice([4095, 16383, 65535])),
             camera_white=list(rng.random(3) * 0.7 + 0.3))
    if rng.random() < 0.5:
        t["plane_color"] = list(rng.permutation(3))
    nb = int(rng.choice([0, 1, 3, 4]))
    if nb:
        t["black_level"] = list(rng.integers(0, 1024, nb) + rng.random(nb) * (rng.random() < 0.3))
    aa = None
    if rng.random() < 0.6:
        top, left = int(rng.integers(0, 9)), int(rng.integers(0, 9))
        aa = [top, left, H - int(rng.integers(0, 7)), W - int(rng.integers(0, 7))]
        t["active_area"] = aa
    if rng.random() < 0.4:
        t["default_crop_origin"] = [float(rng.integers(0, 12)) + 0.5 * (rng.random() < 0.5), 3.0]
        t["default_crop_size"] = [float(rng.integers(10, min(W, H))), 9.0]
    r = rng.random()
    if r < 0.3:
        t["noise_profile"] = list(rng.random(2) * 1e-4)
    elif r < 0.6:
        t["noise_profile"] = list(rng.random(6) * 1e-4)
    if rng.random() < 0.5:
        top, left, bottom, right = aa if aa else (0, 0, H, W)
        t["black_delta_v"] = list(rng.integers(0, 40, bottom - top) + rng.random(bottom - top))
        if rng.random() < 0.7:
            t["black_delta_h"] = list(rng.integers(0, 30, right - left).astype(float))
    if rng.random() < 0.5:
        isos = sorted(rng.choice([100, 200, 400, 800, 1600, 3200, 6400], int(rng.integers(1, 5)), replace=False).tolist())
        alpha = list(rng.random(len(isos)) * 1e-4 * (rng.random() < 0.8))
        beta = list(rng.random(len(isos)) * 1e-6)
        t["profile_noise"] = (isos, alpha, beta)
        t["iso"] = int(rng.integers(50, 8000))
    return t


@pytest.mark.parametrize("seed", range(40))
def test_dng_levels_match_oracle(seed):
    t = random_tags(np.random.default_rng(seed))
    same(isa.dng_levels(**t), RM.dng_levels(**t))


def test_dng_levels_reference_cases():
    base = dict(width=64, height=48, cfa_pattern=[0, 1, 1, 2], white_level=16383, camera_white=[0.5, 1.0, 0.8])
    # four black values per CFA position: green = max of the two greens
    r = isa.dng_levels(**base, black_level=[512, 520, 530, 540])
    assert list(r["black"]) == [512, 530, 540] and list(r["white"]) == [16383 - 512, 16383 - 530, 16383 - 540]
    # three per plane follow CFAPlaneColor
    r = isa.dng_levels(**base, black_level=[10, 20, 30], plane_color=[2, 1, 0])
    assert list(r["black"]) == [30, 20, 10] and not r["color_twist_identity"]
    assert np.array_equal(r["color_twist"][:, :3], np.array([[0, 0, 1], [0, 1, 0], [1, 0, 0]], np.float32))
    # an odd active-area origin shifts the CFA: rows for the top, columns for the left
    assert isa.dng_levels(**base, active_area=[1, 0, 48, 64])["cfa"] == [1, 2, 0, 1]
    assert isa.dng_levels(**base, active_area=[0, 1, 48, 64])["cfa"] == [1, 0, 2, 1]
    assert isa.dng_levels(**base, active_area=[1, 1, 48, 64])["cfa"] == [2, 1, 1, 0]
    # the crop starts two pixels in; its size is cut against the uncorrected origin, so without
    # any crop tag the window reaches the right and bottom edges; DefaultCrop's entry 0 serves both axes
    assert isa.dng_levels(**base)["crop"] == (2, 2, 62, 46)
    assert isa.dng_levels(**base, default_crop_origin=[4, 7], default_crop_size=[30, 20])["crop"] == (4, 4, 30, 30)
    # the white level loses the largest black delta sum
    r = isa.dng_levels(**base, black_delta_v=[0] * 47 + [9], black_delta_h=[3] + [0] * 63)
    assert list(r["white"]) == [16383 - 12] * 3 and r["black_v"][47] == 9 and r["black_h"][0] == 3
    # noise: the green plane's pair of a per-plane profile, overridden by a camera profile with alpha != 0
    r = isa.dng_levels(**base, noise_profile=[1, 2, 3, 4, 5, 6], plane_color=[1, 0, 2])
    assert r["noise"] == (np.float32(1), np.float32(2))
    r = isa.dng_levels(**base, noise_profile=[1e-5, 2e-7], iso=300, profile_noise=([200, 400], [2e-5, 4e-5], [1e-7, 3e-7]))
    assert r["noise"] == (np.float32(3e-5), np.float32(2e-7))
    r = isa.dng_levels(**base, noise_profile=[1e-5, 2e-7], iso=300, profile_noise=([200, 400], [0.0, 0.0], [1e-7, 3e-7]))
    assert r["noise"] == (np.float32(1e-5), np.float32(2e-7))


@pytest.mark.parametrize("bad", [
    dict(cfa_repeat=(2, 4)),
    dict(plane_color=[0, 1, 3]),
    dict(plane_color=[0, 1]),
    dict(cfa_pattern=[1, 1, 1, 2], black_level=[1, 2, 3, 4]),
    dict(black_delta_v=[1] * 47),
    dict(active_area=[2, 2, 40, 60], black_delta_h=[1] * 60),
    dict(noise_profile=[1.0]),
])
def test_dng_levels_rejects_what_the_reference_throws_on(bad):
    base = dict(width=64, height=48, cfa_pattern=[0, 1, 1, 2], white_level=16383, camera_white=[0.5, 1.0, 0.8])
    base.update(bad)
    with pytest.raises(isa.IsaError) as e:
        isa.dng_levels(**base)
    assert e.value.code == isa.ISA_EINVAL
    with pytest.raises(RM.ReferenceThrows):
        RM.dng_levels(**base)


@pytest.mark.parametrize("iso", [50, 100, 150, 199, 200, 333, 800, 1000, 6400, 12800])
def test_noise_model_matches_oracle(iso):
    prof = ([100, 200, 800, 6400], [1e-5, 2e-5, 7e-5, 3e-4], [1e-7, 3e-7, 2e-6, 9e-6])
    assert isa.noise_model(iso, *prof) == RM.noise_model(iso, *prof)
    assert isa.noise_model(iso, [], [], []) == (0.0, 0.0)


@pytest.mark.parametrize("args", [(0, 0, 100, 80, 100, 80), (5, 1, 90, 79, 100, 80), (3, 3, 10, 10, 100, 80), (-4, 6, 120, 40, 100, 80)])
def test_crop_window_matches_oracle(args):
    assert isa.crop_window(*args) == RM.crop_window(*args)


@pytest.mark.parametrize("seed", range(6))
def test_profile_color_spec_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    cm1 = np.eye(3) * 0.8 + rng.random((3, 3)) * 0.2
    cm2 = None if seed % 3 == 0 else np.eye(3) * 0.7 + rng.random((3, 3)) * 0.3
    il1, il2 = [(17, 21), (21, 17), (23, 23), (1, 0), (3, 10), (0, 0)][seed]
    wb = np.float32(rng.random(3) * 1.5 + 0.6)
    got = isa.profile_color_spec(wb, cm1, cm2, il1, il2)
    neutral = [float(np.float32(1.0) / w) for w in wb]
    want = CS.dng_color_spec(color_matrix1=cm1.reshape(-1), color_matrix2=None if cm2 is None else cm2.reshape(-1), illuminant1=il1,
                             illuminant2=il2, as_shot_neutral=neutral)
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g).reshape(-1), np.asarray(w).reshape(-1))


def test_profile_color_spec_identity_is_the_pef_spec():
    wb = np.float32([1.9, 1.0, 1.6])
    got = isa.profile_color_spec(wb, np.eye(3), np.eye(3), 23, 23)
    for g, w in zip(got, isa.pef_color_spec(wb)):
        assert np.array_equal(g, w)
