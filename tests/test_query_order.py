"""The query order (gq_query_order / Scene.order, and the `sort` flag of every query):
points along a Hilbert curve on a grid over twice the scene's box (1024 cells per axis in
3D, 32768 in 2D).  On a block of 16^D cells aligned to 16 the curve visits every cell
once, one after another, and steps between face-adjacent cells only; a Morton curve
jumps between quadrants inside such a block."""
import numpy as np
import pytest
import torch

from gquery_b200.scene import Scene

pytestmark = pytest.mark.gpu


def _square_scene(dim):
    """The boundary of [-1, 1]^dim: root box [-1, 1]^dim, key grid over [-2, 2]^dim."""
    if dim == 3:
        v = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float32)
        f = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                      [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]], np.int32)
    else:
        v = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], np.float32)
        f = np.array([[0, 1], [1, 2], [2, 3], [3, 0]], np.int32)
    return Scene(v, f, dim, device=0)


@pytest.mark.parametrize("dim", [2, 3])
def test_order_walks_an_aligned_block_cell_by_cell(dim):
    cells_per_axis = 1024 if dim == 3 else 32768
    scale = cells_per_axis / 4.0  # cells per unit over [-2, 2]
    base = cells_per_axis // 2  # a multiple of 16
    a = np.arange(base, base + 16)
    cells = np.stack(np.meshgrid(*([a] * dim), indexing="ij"), -1).reshape(-1, dim)
    rng = np.random.default_rng(5)
    cells = cells[rng.permutation(len(cells))]
    pts = (-2.0 + (cells + 0.5) / scale).astype(np.float32)  # cell centres, exact in FP32
    s = _square_scene(dim)
    perm = s.order(torch.as_tensor(pts).cuda()).cpu().numpy()
    assert np.array_equal(np.sort(perm), np.arange(len(cells)))
    walk = cells[perm]
    steps = np.abs(np.diff(walk, axis=0)).sum(axis=1)
    assert np.all(steps == 1), np.unique(steps, return_counts=True)


def test_sorted_and_unsorted_queries_give_the_same_answers():
    s = _square_scene(3)
    q = torch.as_tensor(np.random.default_rng(6).uniform(-2, 2, (20000, 3)).astype(np.float32)).cuda()
    a = s.closest_point(q, variant="exact", sort=True)
    b = s.closest_point(q, variant="exact", sort=False)
    for k in ("valid", "d", "prim_id", "p"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
