"""The oracle's own seeded R-MAT generator (used by the CPU legs that must not
load the product library) builds exactly the library's graph: the same edge
count, inverse-row offsets, in-degrees, in-neighbour order and out-degrees,
for several scales, edge factors, seeds and quadrant probabilities."""
import numpy as np
import pytest


@pytest.mark.parametrize("scale,ef,seed,abc", [(10, 16, 1, (0.57, 0.19, 0.19)), (13, 8, 27491095, (0.57, 0.19, 0.19)),
                                               (16, 16, 27491095, (0.57, 0.19, 0.19)),
                                               (12, 32, 7, (0.45, 0.15, 0.15)), (11, 4, 3, (0.25, 0.25, 0.25))])
def test_oracle_rmat_equals_library_graph(ag, oracle, scale, ef, seed, abc):
    o = oracle.rmat_inverse(scale, ef, seed, *abc)
    g = ag.Graph.rmat(scale, ef, a=abc[0], b=abc[1], c=abc[2], seed=seed, flags=ag.AG_BUILD_DEDUPE)
    n = g.num_vertices
    assert o["num_edges"] == g.num_edges
    assert np.array_equal(o["in_idx"][:n], g.in_edges_idx()[:n])
    assert int(o["in_idx"][n]) == g.num_edges
    assert np.array_equal(o["in_deg"], g.in_degree())
    assert np.array_equal(o["in_nb"], g.in_neighbours())
    assert np.array_equal(o["out_deg"], g.out_degree())
