"""Binary output (hr_write_npy): files numpy reads back bit for bit."""
import numpy as np
import pytest

import highreg


@pytest.mark.parametrize("shape", [(7,), (3, 5), (2, 3, 4), (0,), (1, 1, 1, 1)])
def test_write_npy_round_trip(tmp_path, shape):
    a = np.random.default_rng(1).standard_normal(shape)
    f = tmp_path / "a.npy"
    highreg.write_npy(f, a)
    b = np.load(f)
    assert b.dtype == np.float64 and b.shape == a.shape
    assert np.array_equal(a, b)
    # the header is padded so the data starts on a 64-byte boundary
    raw = f.read_bytes()
    assert raw[:6] == b"\x93NUMPY" and (10 + int.from_bytes(raw[8:10], "little")) % 64 == 0


def test_write_npy_solution_layout(tmp_path):
    """The two-surface solution as (n, 3) velocities per surface (the vel1 / vel2 files)."""
    x = np.arange(30, dtype=np.float64)
    highreg.write_npy(tmp_path / "vel1.npy", x[:18].reshape(6, 3))
    assert np.array_equal(np.load(tmp_path / "vel1.npy"), x[:18].reshape(6, 3))


def test_write_npy_rejects_bad_path(tmp_path):
    with pytest.raises(highreg.HrError):
        highreg.write_npy(tmp_path / "missing_dir" / "a.npy", np.zeros(3))
