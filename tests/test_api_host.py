"""Host-side behaviour of the reference-compatible API that needs no GPU: argument checks,
error messages (scaling_elections.cu:868-871, 900), ballot preparation."""
import numpy as np
import pytest

from scalingelections_b200 import api


def test_dimension_and_shape_errors():
    with pytest.raises(RuntimeError, match="Number of dimensions must be two"):
        api.compute_strongest_paths(np.zeros(4, np.uint32), allow_gpu=True, tile_size=32)
    with pytest.raises(RuntimeError, match="Preferences matrix must be square"):
        api.compute_strongest_paths(np.zeros((3, 4), np.uint32), allow_gpu=True, tile_size=32)


def test_cpu_path_is_not_provided():
    with pytest.raises(RuntimeError, match="GPU only"):
        api.compute_strongest_paths(np.zeros((4, 4), np.uint32))


@pytest.mark.parametrize("tile", [0, 3, 64, 128])
def test_unsupported_tile_sizes(tile):
    with pytest.raises(RuntimeError, match="Unsupported tile size"):
        api.compute_strongest_paths(np.zeros((4, 4), np.uint32), allow_gpu=True, tile_size=tile)


def test_ballots_csr_and_candidate_count():
    b = api.Ballots.from_rankings([np.array([2, 0]), np.array([1]), np.array([4, 3, 2, 1, 0])])
    assert b.num_candidates == 5 and b.num_voters == 3
    assert list(b.offsets) == [0, 2, 3, 8]
    dense = api.Ballots.from_rankings(np.array([[1, 0, 2], [2, 1, 0]]))
    assert dense.num_candidates == 3 and list(dense.offsets) == [0, 3, 6]
    assert api.Ballots.from_rankings([]).num_candidates == 1


def test_empty_ballot_raises_like_the_reference():
    with pytest.raises(ValueError, match="zero-size array"):
        api.Ballots.from_rankings([np.array([0, 1]), np.array([], dtype=np.int64)])


def test_negative_ids_rejected():
    with pytest.raises(ValueError):
        api.Ballots.from_rankings([np.array([0, -1])])


def test_dropin_module_surface():
    import importlib
    import sys

    from conftest import ROOT

    sys.path.insert(0, str(ROOT / "scalingelections_b200" / "dropin"))
    try:
        sys.modules.pop("scaling_elections", None)
        m = importlib.import_module("scaling_elections")
        for name in ("compute_strongest_paths", "log_gpus"):
            assert callable(getattr(m, name))
        assert m.compute_strongest_paths is api.compute_strongest_paths
    finally:
        sys.path.pop(0)
        sys.modules.pop("scaling_elections", None)
