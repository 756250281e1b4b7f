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
