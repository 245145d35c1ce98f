"""Host-side parts of the autotuner's reference interface
(GPUSimulators/Autotuner.py:226-287): the benchmark case and the sanity check."""

import numpy as np

from finitevolumegpu_b200.Autotuner import Autotuner, size_class


def test_gen_test_data_is_the_cosine_bump():
    h, hu, hv, dx, dy, dt = Autotuner.gen_test_data(128, 96, 9.81)
    assert h.shape == hu.shape == hv.shape == (96, 128)
    assert h.dtype == np.float32 and hu.dtype == np.float32
    assert dx == 100.0 / 128 and dy == 100.0 / 96
    # depth 0.5 outside the bump, up to 0.6 at its centre; momentum 0 .. 0.1
    assert abs(float(h.min()) - 0.5) < 1e-6 and abs(float(h.max()) - 0.6) < 1e-3
    assert np.array_equal(hu, hv) and float(hu.min()) >= 0.0 and float(hu.max()) <= 0.1 + 1e-6
    assert np.allclose(h - 0.5, hu, atol=1e-6)
    assert abs(dt - 0.7 * min(dx, dy) / (0.1 * np.sqrt(2.0) + np.sqrt(9.81 * 0.6))) < 1e-12
    # the bump (radius width / 5 = 20) is centred: symmetric under both flips
    assert np.allclose(h, h[:, ::-1]) and np.allclose(h, h[::-1, :])


def test_sanity_check():
    a = np.array([0.4, 0.5, 0.6], dtype=np.float32)
    assert Autotuner.sanity_check(a, 0.3, 0.7)
    assert not Autotuner.sanity_check(a, 0.45, 0.7)
    assert not Autotuner.sanity_check(a, 0.3, 0.55)
    assert not Autotuner.sanity_check(np.array([0.4, np.nan], dtype=np.float32), 0.3, 0.7)


def test_size_classes():
    assert size_class(4096, 4096) == "4^12"
    assert size_class(256, 256) == "4^8"
    assert size_class(4096, 1024) == size_class(2048, 2048) == "4^11"
