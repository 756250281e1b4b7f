"""Ranking parity (get_winner_and_ranking, scaling_elections.py:274-296) and the whole
pipeline on the participation-paradox known answer."""
import numpy as np
import pytest
import torch

from conftest import ballots_of, golden_names, load_golden
from scalingelections_b200 import _lib, api

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_names())
def test_golden_ranking(name):
    case = load_golden(name)
    if "strongest" not in case:
        pytest.skip("hash-only fixture")
    S = case["strongest"]
    winner, ranking = api.get_winner_and_ranking(list(range(S.shape[0])), S)
    assert winner == int(case["winner"])
    assert ranking == list(case["ranking"])


def test_ties_keep_index_order(orc):
    rng = np.random.default_rng(0)
    for C in (3, 31, 32, 33, 1000, 1025, 3000):
        S = rng.integers(0, 3, size=(C, C)).astype(np.uint32)  # many equal pairs -> ties
        wins_ref, rank_ref = orc.wins_and_ranking(S)
        w, r = api.rank_device(api._to_device_u32(S, "cuda"))
        assert np.array_equal(w.cpu().numpy(), wins_ref)
        assert np.array_equal(r.cpu().numpy(), rank_ref)


@pytest.mark.parametrize("C", [1, 2, 63, 64, 65, 128, 129, 2048, 2049, 4100, 6000, 8128, 8192, 8193])
def test_wins_and_places_across_tile_and_strip_edges(orc, C):
    """Sizes on each side of the 64-cell tile pairs and of the 128-candidate / 2048-entry strips
    of the place count, and of the wins count's blocked pair order (tile grids that are a
    multiple of 16 tiles from 128 tiles: C = 8192, not 8128 or 8193); with ties (values in
    [0, 3)) and without (values up to 2^32 - 1)."""
    rng = np.random.default_rng(C + 5)
    for hi in (3, 2**32 - 1):
        S = rng.integers(0, hi, size=(C, C), dtype=np.uint64).astype(np.uint32)
        wins_ref, rank_ref = orc.wins_and_ranking(S)
        w, r = api.rank_device(api._to_device_u32(S, "cuda"))
        assert np.array_equal(w.cpu().numpy(), wins_ref), (C, hi)
        assert np.array_equal(r.cpu().numpy(), rank_ref), (C, hi)


def key_matrix(key):
    """S[i][j] = 1 where key[i] > key[j], built on the GPU: wins[i] = #{j : key[j] < key[i]},
    known without an O(C^2) count, so sizes of tens of thousands stay cheap to check."""
    k = torch.from_numpy(key.astype(np.int64)).cuda()
    return (k[:, None] > k[None, :]).to(torch.int32).view(torch.uint32)


def key_wins_and_ranking(key):
    wins = np.searchsorted(np.sort(key), key, side="left").astype(np.int32)
    return wins, np.argsort(-wins, kind="stable").astype(np.int32)


def test_key_matrix_closed_form(orc):
    """The closed form above equals the oracle's count where the oracle is quick."""
    rng = np.random.default_rng(3)
    for C, distinct in ((1, 1), (7, 2), (300, 3), (300, 300), (1000, 40)):
        key = rng.integers(0, distinct, size=C)
        S = api._to_host_u32(key_matrix(key))
        wins_ref, rank_ref = orc.wins_and_ranking(S)
        wins, ranking = key_wins_and_ranking(key)
        assert np.array_equal(wins, wins_ref) and np.array_equal(ranking, rank_ref)


@pytest.mark.parametrize("C", [4095, 4096, 4097, 16384, 49152, 49153])
def test_places_on_both_sides_of_the_histogram_limit(C):
    """Up to 49152 candidates the places come from per-CTA histograms of the wins, above from
    the strip count: both give the stable order, with every candidate tied, a few distinct wins,
    many ties and none."""
    rng = np.random.default_rng(C)
    for distinct in (1, 3, C // 7 + 1, C):
        key = rng.permutation(C) if distinct == C else rng.integers(0, distinct, size=C)
        S = key_matrix(key)
        w, r = api.rank_device(S)
        del S
        wins, ranking = key_wins_and_ranking(key)
        assert np.array_equal(w.cpu().numpy(), wins), (C, distinct)
        assert np.array_equal(r.cpu().numpy(), ranking), (C, distinct)
    torch.cuda.empty_cache()


def test_wins_buffer_off_a_16_byte_boundary(orc):
    """A wins buffer 4 bytes past a 16-byte boundary: the place histogram reads the wins one at
    a time instead of four; same wins and ranking."""
    C = 3000
    S = np.random.default_rng(11).integers(0, 4, size=(C, C)).astype(np.uint32)
    wins_ref, rank_ref = orc.wins_and_ranking(S)
    d = api._to_device_u32(S, "cuda")
    buf = torch.zeros(C + 4, dtype=torch.int32, device="cuda")
    ranking = torch.empty(C, dtype=torch.int32, device="cuda")
    _lib.check(_lib.lib().se_rank(d.data_ptr(), C, C, buf.data_ptr() + 4, ranking.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert np.array_equal(buf[1:C + 1].cpu().numpy(), wins_ref)
    assert np.array_equal(ranking.cpu().numpy(), rank_ref)


@pytest.mark.parametrize("C", [64, 200])
def test_strided_and_unaligned_rows(orc, C):
    """Row strides that are not a multiple of 4 cells, and a first cell off a 16-byte boundary,
    take the scalar-load path of the wins count; same results."""
    rng = np.random.default_rng(C)
    S = rng.integers(0, 50, size=(C, C)).astype(np.uint32)
    wins_ref, rank_ref = orc.wins_and_ranking(S)
    big = torch.zeros((C, C + 3), dtype=torch.int32, device="cuda")
    big[:, 1:C + 1] = torch.from_numpy(S.view(np.int32)).cuda()
    for view in (big[:, 1:C + 1], big[:, :C + 3][:, 1:C + 1].contiguous()):
        w, r = api.rank_device(view.view(torch.uint32))
        assert np.array_equal(w.cpu().numpy(), wins_ref)
        assert np.array_equal(r.cpu().numpy(), rank_ref)


def test_candidate_labels():
    S = np.array([[0, 2, 2], [1, 0, 1], [1, 2, 0]], np.uint32)
    assert api.get_winner_and_ranking(["a", "b", "c"], S) == ("a", ["a", "c", "b"])


def test_paradox_pipeline():
    names = ["Python", "Rust", "Go", "Java"]
    before = api.schulze(ballots_of(load_golden("paradox_before")))
    after = api.schulze(ballots_of(load_golden("paradox_after")))
    assert (names[before.winner], names[after.winner]) == ("Java", "Python")


@pytest.mark.parametrize("name", ["uniform_c128_v2000", "mallows_c300_v500_phi08", "incomplete_c40_v151"])
def test_pipeline_matches_reference(name):
    case = load_golden(name)
    r = api.schulze(ballots_of(case), return_paths=True)
    assert r.winner == int(case["winner"])
    assert list(r.ranking) == list(case["ranking"])
    assert np.array_equal(r.strongest_paths, case["strongest"])


def test_dropin_reference_calls():
    """The calls scaling_elections.py makes (py:425-430) on the reference's default size."""
    case = load_golden("uniform_c128_v2000")
    P = case["preferences"]
    for tma in (False, True):
        out = api.compute_strongest_paths(P, allow_gpu=True, allow_tma=tma, tile_size=32)
        assert out.dtype == np.uint32 and out.flags.c_contiguous
        assert np.array_equal(out, case["strongest"])
    out = api.compute_strongest_paths(P.astype(np.int64), allow_gpu=True, tile_size=16)
    assert np.array_equal(out, case["strongest"])
    api.log_gpus()
