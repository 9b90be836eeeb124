"""The DNG colour specification without a GPU: libisa.so's host
implementation (isa_dng_color_spec, isa_pef_color_spec) against the
restatement in oracle/colorspec.py, bit for bit in FP64, and properties of
the result (the white point maps to the PCS white, temperatures of the
daylight locus, interpolation endpoints)."""
import numpy as np
import pytest

from imagestackalignator_b200 import isa

import colorspec as CS

# camera matrices of plausible shape (XYZ -> camera, rows summing near 1)
CM_A = [1.1, -0.3, -0.05, -0.5, 1.4, 0.1, -0.1, 0.25, 0.6]
CM_D65 = [0.95, -0.25, -0.1, -0.45, 1.3, 0.15, -0.08, 0.2, 0.7]
FM1 = [0.7, 0.15, 0.1, 0.28, 0.68, 0.04, 0.02, 0.1, 0.7]
FM2 = [0.68, 0.18, 0.1, 0.27, 0.7, 0.03, 0.01, 0.09, 0.72]


CASES = {
    "one_matrix_neutral": dict(color_matrix1=CM_D65, illuminant1=21, as_shot_neutral=[0.5, 1.0, 0.7]),
    "two_matrices_neutral": dict(color_matrix1=CM_A, color_matrix2=CM_D65, illuminant1=17, illuminant2=21,
                                 as_shot_neutral=[0.45, 1.0, 0.62]),
    "two_matrices_swapped": dict(color_matrix1=CM_D65, color_matrix2=CM_A, illuminant1=21, illuminant2=17,
                                 as_shot_neutral=[0.45, 1.0, 0.62]),
    "as_shot_xy": dict(color_matrix1=CM_A, color_matrix2=CM_D65, illuminant1=17, illuminant2=21, as_shot_white_xy=[0.3127, 0.329]),
    "forward_matrices": dict(color_matrix1=CM_A, color_matrix2=CM_D65, illuminant1=17, illuminant2=21, forward_matrix1=FM1,
                             forward_matrix2=FM2, as_shot_neutral=[0.5, 1.0, 0.66]),
    "calibration_balance": dict(color_matrix1=CM_A, color_matrix2=CM_D65, illuminant1=17, illuminant2=21,
                                camera_calibration1=[1.02, 0, 0, 0, 1, 0, 0, 0, 0.97], camera_calibration2=[1.02, 0, 0, 0, 1, 0, 0, 0, 0.97],
                                analog_balance=[1.0, 1.0, 1.05], as_shot_neutral=[0.6, 1.0, 0.5]),
    "unknown_illuminant": dict(color_matrix1=CM_A, color_matrix2=CM_D65, illuminant1=0, illuminant2=21, as_shot_neutral=[0.5, 1.0, 0.7]),
}


@pytest.mark.parametrize("name", list(CASES))
def test_dng_color_spec_matches_oracle(name):
    kw = CASES[name]
    got = isa.dng_color_spec(**kw)
    want = CS.dng_color_spec(**kw)
    for g, w in zip(got, want):
        assert np.array_equal(g, w), (name, g, w)


@pytest.mark.parametrize("wb", [[2.0, 1.0, 1.5], [1.8, 1.0, 2.3], [1.0, 1.0, 1.0], [0.39, 0.78, 1.56]])
def test_pef_color_spec_matches_oracle(wb):
    got = isa.pef_color_spec(wb)
    want = CS.pef_color_spec(wb)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    c2p, cw, xy = got
    # the camera white (the neutral) maps to the D50 PCS white up to the white scale
    pcs = c2p @ cw
    d50 = np.array(CS.xy_to_xyz(CS.D50))
    assert np.allclose(pcs / pcs[1], d50 / d50[1], atol=1e-9)


def test_temperature_of_daylight_locus():
    # CIE daylight chromaticities near 5000 K and 6500 K
    assert abs(CS.temperature_of((0.3457, 0.3585)) - 5000) < 60
    assert abs(CS.temperature_of((0.3127, 0.3290)) - 6500) < 60


def test_interpolation_endpoints():
    """A white far below the first illuminant's temperature uses colour matrix 1 alone."""
    kw = dict(color_matrix1=CM_A, color_matrix2=CM_D65, illuminant1=17, illuminant2=21)
    warm = CS.dng_color_spec(**kw, as_shot_white_xy=[0.5, 0.41])
    only1 = CS.dng_color_spec(color_matrix1=CM_A, illuminant1=17, as_shot_white_xy=[0.5, 0.41])
    assert np.array_equal(warm[0], only1[0])


def test_color_spec_arguments():
    with pytest.raises(isa.IsaError):
        isa.dng_color_spec(color_matrix1=CM_A)          # no as-shot white
    with pytest.raises(isa.IsaError):
        isa.pef_color_spec([1.0, 0.0, 1.0])
    with pytest.raises(isa.IsaError):
        isa.dng_color_spec(color_matrix1=[0] * 9, as_shot_neutral=[1, 1, 1])  # singular
