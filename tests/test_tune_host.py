"""Host logic of the autotuner (imagestackalignator_b200/tune.py): burst
classes and the conservative choice (the library's own shape unless another
is at least MARGIN faster). The timings themselves run on a GPU
(tests/test_gpu_tuning.py)."""
from imagestackalignator_b200 import tune


def test_classes_group_by_scale_aspect_and_area():
    assert tune.burst_class(4000, 3000, 2.0) == "s2-4:3-12MP"
    assert tune.burst_class(4240, 2832, 1.0) == "s1-3:2-12MP"
    assert tune.burst_class(2048, 1536, 2.0) == tune.burst_class(2064, 1552, 2.0)
    assert tune.burst_class(2048, 1536, 2.0) != tune.burst_class(2048, 1536, 1.0)


def test_pick_keeps_the_default_within_the_margin():
    times = {0: 10.0, 32: 9.8, 64: 9.9}
    assert tune._pick((0, 32, 64), times.__getitem__) == 0
    times[64] = 9.0
    assert tune._pick((0, 32, 64), times.__getitem__) == 64
