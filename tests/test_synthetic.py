"""The burst generator's independently moving object (the large-burst
workload with local motion): a rigid disc of the requested area fraction
whose centre steps object_step px per frame, reflected inside the frame."""
import numpy as np

from imagestackalignator_b200 import synthetic


def test_moving_object_area_and_path():
    b = synthetic.make_burst(320, 240, 12, seed=9, max_shift=4, moving_object=0.05, object_step=(2.0, 40.0))
    ref = synthetic.make_burst(320, 240, 12, seed=9, max_shift=4)
    assert b.object_path.shape == (12, 2)
    steps = np.linalg.norm(np.diff(b.object_path, axis=0), axis=1)
    assert (steps <= 40.0 + 1e-9).all()
    rad = np.sqrt(0.05 * 320 * 240 / np.pi)
    assert (b.object_path[:, 0] >= rad).all() and (b.object_path[:, 0] <= 320 - rad).all()
    assert (b.object_path[:, 1] >= rad).all() and (b.object_path[:, 1] <= 240 - rad).all()
    # the object replaces the background inside its disc only (same noise realisation outside)
    for f in (0, 5, 11):
        yy, xx = np.mgrid[0:240, 0:320]
        disc = (xx - b.object_path[f, 0]) ** 2 + (yy - b.object_path[f, 1]) ** 2 <= rad * rad
        assert (b.raw[f][~disc] == ref.raw[f][~disc]).all()
        assert abs(disc.mean() - 0.05) < 0.005
        assert (b.raw[f][disc] != ref.raw[f][disc]).mean() > 0.5
