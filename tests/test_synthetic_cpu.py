"""The slice-by-slice stack generator: a z-window regenerated on its own
(noise with a reflected halo, smoothed, cropped) equals the same slices of
the whole stack generated at once, at the stack's ends and in its middle.
Both arms of the benchmark rely on this to filter the same input."""

import importlib.util
import os

import numpy as np
import pytest

from oracle import restate as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _synthetic():
    spec = importlib.util.spec_from_file_location(
        "cimx_test_synthetic", os.path.join(ROOT, "cucim_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("z0,z1", [(0, 5), (9, 17), (26, 30), (0, 30)])
def test_window_equals_whole_stack(z0, z1):
    S = _synthetic()
    shape = (30, 17, 23)
    noise = S.stack_noise(range(shape[0]), shape[1:], threads=2)
    sm = R.gaussian_filter(noise, S.STACK_SIGMA, mode="reflect", truncate=S.STACK_TRUNCATE)
    whole = S.stack_shot(sm, range(shape[0]), threads=2)
    win = S.stack_window(z0, z1, shape, R.gaussian_filter, threads=3)
    assert win.dtype == np.uint16 and win.shape == (z1 - z0,) + shape[1:]
    np.testing.assert_array_equal(win, whole[z0:z1])


def test_stack_value_range():
    S = _synthetic()
    w = S.stack_window(0, 4, (64, 128, 128), R.gaussian_filter)
    # the mapped mean sits at the middle of [0, 65535]
    assert 30000 < w.mean() < 35500
    assert w.min() < 20000 and w.max() > 45000
