"""Device-side ballot sampler: valid permutations, determinism, Mallows concentration."""
import numpy as np
import pytest
import torch

from scalingelections_b200.ballots import mallows_ballots_device

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("C", [1, 2, 7, 128, 1000, 4097])
def test_device_ballots_are_permutations(C):
    b = mallows_ballots_device(300, C, 0.8, seed=C).cpu().numpy()
    assert b.shape == (300, C)
    assert (np.sort(b, axis=1) == np.arange(C)).all()


def test_device_ballots_deterministic():
    a = mallows_ballots_device(50, 333, 0.5, seed=9)
    b = mallows_ballots_device(50, 333, 0.5, seed=9)
    c = mallows_ballots_device(50, 333, 0.5, seed=10)
    assert torch.equal(a, b) and not torch.equal(a, c)


def test_device_mallows_concentration():
    ref = np.arange(40, dtype=np.int32)

    def mean_disp(phi):
        b = mallows_ballots_device(2000, 40, phi, seed=3, reference=ref).cpu().numpy()
        pos = np.argsort(b, axis=1)
        return np.abs(pos - ref).mean()

    tight, mid, loose = mean_disp(0.2), mean_disp(0.8), mean_disp(1.0)
    assert tight < mid < loose
    # Uniform permutations of 40 items: E|pos - i| = (n^2 - 1) / (3n) = 13.3.
    assert abs(loose - (40 * 40 - 1) / (3 * 40)) < 0.5


@pytest.mark.parametrize("C,high", [(1, None), (300, None), (1000, 7), (4096, 65535)])
def test_random_preferences_device_bit_exact(C, high):
    """The device's random benchmark matrix equals its host restatement bit for bit, and its
    values cover [0, high)."""
    from scalingelections_b200.ballots import random_matrix_host, random_preferences_device

    d = random_preferences_device(C, seed=42, high=high)
    got = d.view(torch.int32).cpu().numpy().view(np.uint32)
    assert np.array_equal(got, random_matrix_host(C, 42, high))
    hi = high or C
    assert got.max() < hi and (C < 64 or got.max() == hi - 1)
    if C >= 1000:
        assert abs(got.mean() - (hi - 1) / 2) < 0.01 * hi
    assert not np.array_equal(random_preferences_device(C, seed=43, high=high).view(torch.int32).cpu().numpy(),
                              got.view(np.int32)) or C == 1
