"""GPU parity of the cell search with the reference: bit-exact pairs and cell order."""
import numpy as np
import pytest
import torch

from oracle import neighbors as on

pytestmark = pytest.mark.gpu


def test_cell_linked_pairs_match_reference_fixtures(gpu, golden):
    from tensorsph_b200.neighbor_search import brute_force_pairs, cell_linked_pairs, cell_order
    g = golden("pairs")
    for k in range(int(g["count"])):
        pos = torch.from_numpy(g[f"c{k}_pos"]).to(gpu)
        cutoff = float(g[f"c{k}_cutoff"])
        pairs = cell_linked_pairs(pos, cutoff).cpu().numpy()
        assert np.array_equal(pairs, g[f"c{k}_pairs"]), k
        order = cell_order(pos, cutoff).cpu().numpy()
        assert np.array_equal(order, g[f"c{k}_order"]), k
        if pos.shape[0] <= 2000:
            assert np.array_equal(brute_force_pairs(pos, cutoff).cpu().numpy(), g[f"c{k}_pairs"])


def test_periodic_pairs_match_reference_fixtures(gpu, golden):
    from tensorsph_b200.threed import periodic_pairs
    g = golden("periodic")
    for k in range(int(g["count"])):
        pos = torch.from_numpy(g[f"c{k}_pos"]).to(gpu)
        pairs = periodic_pairs(pos, float(g[f"c{k}_box"]), float(g[f"c{k}_cutoff"]))
        assert np.array_equal(pairs.cpu().numpy(), g[f"c{k}_pairs"]), k


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_random_clouds_match_oracle(gpu, dim, dtype):
    from tensorsph_b200.neighbor_search import cell_linked_pairs
    rng = np.random.default_rng(100 + dim)
    pos = (rng.random((3000, dim)) * 3.0 - 1.0).astype(dtype)
    pos[5] = pos[4]
    for cutoff in (0.05, 0.17):
        expect = on.cell_linked_pairs(pos, cutoff)
        got = cell_linked_pairs(torch.from_numpy(pos).to(gpu), cutoff).cpu().numpy()
        assert np.array_equal(got, expect)


def test_edge_cases_and_errors(gpu):
    from tensorsph_b200.neighbor_search import cell_linked_pairs
    assert cell_linked_pairs(torch.empty((0, 2), dtype=torch.float64, device=gpu), 1.0).shape == (0, 2)
    assert cell_linked_pairs(torch.zeros((1, 2), device=gpu), 1.0).shape == (0, 2)
    two = torch.tensor([[0.0, 0.0], [1.0, 0.0]], dtype=torch.float64, device=gpu)
    assert cell_linked_pairs(two, 1.0).tolist() == [[0, 1]]  # exactly at the cutoff
    clustered = torch.full((30, 2), 2.5, dtype=torch.float64, device=gpu)
    clustered[0] = torch.tensor([-4.0, 7.0], dtype=torch.float64)
    assert cell_linked_pairs(clustered, 0.2).shape[0] == 29 * 28 // 2
    with pytest.raises(ValueError):
        cell_linked_pairs(torch.tensor([[float("nan"), 0.0], [0.0, 0.0]], device=gpu), 1.0)
    with pytest.raises(ValueError):
        cell_linked_pairs(torch.zeros((2, 2), device=gpu), 0.0)
    with pytest.raises(TypeError):
        cell_linked_pairs(torch.ones((2, 2), dtype=torch.int64, device=gpu), 1.0)
    # CPU input: result comes back on the CPU
    cpu = torch.rand((50, 2), dtype=torch.float64)
    out = cell_linked_pairs(cpu, 0.3)
    assert out.device.type == "cpu"
    assert np.array_equal(out.numpy(), on.cell_linked_pairs(cpu.numpy(), 0.3))


def test_dense_cluster_long_rows(gpu):
    """Rows longer than the warp and block sort tiers (9,000 particles in one cell)."""
    from tensorsph_b200.neighbor_search import cell_linked_pairs
    rng = np.random.default_rng(9)
    m = 9000
    pos = np.concatenate((rng.random((m, 2)) * 0.01, 1.0 + rng.random((200, 2)) * 5.0))
    got = cell_linked_pairs(torch.from_numpy(pos).to(gpu), 0.02)
    i, j = got[:, 0].cpu().numpy(), got[:, 1].cpu().numpy()
    key = i * pos.shape[0] + j
    assert np.all(np.diff(key) > 0)
    assert ((i < m) & (j < m)).sum() == m * (m - 1) // 2


def test_sparse_grid_path(gpu):
    """Widely spread cloud: the cell grid exceeds the dense-table limit."""
    from tensorsph_b200.neighbor_search import cell_linked_pairs
    rng = np.random.default_rng(4)
    pos = rng.random((400, 3)) * 2000.0
    pos[1:40] = pos[0] + rng.random((39, 3)) * 0.5
    expect = on.cell_linked_pairs(pos, 0.3)
    got = cell_linked_pairs(torch.from_numpy(pos).to(gpu), 0.3).cpu().numpy()
    assert np.array_equal(got, expect)


def test_pair_cache_semantics(gpu):
    from tensorsph_b200.neighbor_search import PairListCache
    rng = np.random.default_rng(3)
    pos = torch.from_numpy(rng.random((500, 2))).to(gpu)
    cache = PairListCache(0.1, 0.02, fluid_count=400)
    ref = on.PairListCache(0.1, 0.02, fluid_count=400)
    for shift in (0.0, 0.006, 0.02):
        p, rebuilt = cache.get(pos + shift)
        q, rebuilt_ref = ref.get(pos.cpu().numpy() + shift)
        assert rebuilt == rebuilt_ref
        assert np.array_equal(p.cpu().numpy(), q)
    assert (cache.rebuilds, cache.reuses, cache.pruned) == (ref.rebuilds, ref.reuses, ref.pruned)
    assert cache.displacement(pos) == pytest.approx(ref.displacement(pos.cpu().numpy()), rel=1e-12)
