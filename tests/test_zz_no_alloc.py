"""The PageRank entry point that allocates nothing (gpr_pagerank_noalloc).

Callers whose device memory is owned by their own allocator, or that may not
take the synchronisation a cudaMalloc / cudaFree can cause, need a solver that
allocates no memory.  gpr_pagerank_noalloc keeps its scratch in a fixed device
array inside the library; this test calls it through the C ABI on device
arrays, twice in a row (the second call reuses the array the first one left
behind), and checks each result against the existing entry point
(gpr_graph_create + gpr_pagerank) within the tolerance the other PageRank
tests use: 1e-6 absolute per vertex and the same sweep count within one.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ABS_TOL = 1e-6


def test_noalloc_matches_existing_entry_point_twice(G, O):
    torch = pytest.importorskip("torch")
    rp, col, od = O.rmat_graph(15, 16, seed=21)
    m, nnz = len(rp) - 1, len(col)
    with G.Graph(rp, col, od) as g:
        ref, st_ref = g.pagerank(tol=1e-6, max_iter=100)
    d_rp = torch.from_numpy(rp).cuda()
    d_col = torch.from_numpy(col).cuda()
    d_od = torch.from_numpy(od).cuda()
    for call in range(2):
        d_s = torch.full((m,), float(np.float32(1.0) / np.float32(m)), dtype=torch.float32,
                         device="cuda")
        st = G.pagerank_noalloc(m, nnz, d_rp, d_col, d_od, d_s, tol=1e-6, max_iter=100)
        s = d_s.cpu().numpy()
        assert abs(st.iterations - st_ref.iterations) <= 1, (call, st.iterations, st_ref.iterations)
        assert np.abs(s - ref).max() <= ABS_TOL, call


def test_noalloc_rejects_sizes_beyond_its_scratch(G):
    limit = G.pagerank_noalloc_max_vertices()
    assert limit == 1 << 20
    with pytest.raises(G.GprError) as e:
        G.pagerank_noalloc(limit + 1, 0, 1, 1, 1, 1)
    assert e.value.status == G.GPR_EINVAL and "limit" in str(e.value)
