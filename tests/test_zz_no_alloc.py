"""The PageRank entry point that allocates nothing (gpr_pagerank_noalloc).

Callers whose device memory is owned by their own allocator, or that may not
take the synchronisation a cudaMalloc / cudaFree can cause, need a solver that
allocates no memory.  gpr_pagerank_noalloc keeps its scratch in a fixed device
array inside the library; this test calls it through the C ABI on device
arrays, twice in a row (the second call reuses the array the first one left
behind), and checks each result against the existing entry point
(gpr_graph_create + gpr_pagerank) within the tolerance the other PageRank
tests use: 1e-6 absolute per vertex and the same sweep count within one.
Its sweep sums each row in CSR order with the reference's float operations,
so its scores are also compared bit for bit with the oracle's restatement of
the reference's OpenMP solver (src/pr/omp_base.cc:9-49).  Malformed CSR input
is rejected with GPR_EINVAL.  This file is collected last so that a run
stopping at the first failure has already run every other test.
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


def test_noalloc_is_bit_identical_to_the_oracle(G, O):
    torch = pytest.importorskip("torch")
    rp, col, od = O.rmat_graph(14, 16, seed=5)
    m, nnz = len(rp) - 1, len(col)
    d_rp, d_col, d_od = (torch.from_numpy(a).cuda() for a in (rp, col, od))
    for tol, max_iter in ((1e-4, 100), (0.0, 7)):
        d_s = torch.full((m,), float(np.float32(1.0) / np.float32(m)), dtype=torch.float32,
                         device="cuda")
        st = G.pagerank_noalloc(m, nnz, d_rp, d_col, d_od, d_s, tol=tol, max_iter=max_iter)
        ref, n_ref, _ = O.pr_plain_f32(rp, col, od, tol=tol, max_iter=max_iter)
        assert abs(st.iterations - n_ref) <= 1, (st.iterations, n_ref)
        if st.iterations != n_ref:  # residual within rounding of tol: same sweeps as the GPU
            ref, _, _ = O.pr_plain_f32(rp, col, od, tol=0.0, max_iter=st.iterations)
        assert np.array_equal(d_s.cpu().numpy(), ref), (tol, max_iter)


@pytest.mark.parametrize("case", ["column_out_of_range", "last_offset", "decreasing",
                                  "negative_degree", "edges_without_vertices"])
@pytest.mark.parametrize("max_iter", [30, 0])
def test_noalloc_rejects_malformed_csr(G, case, max_iter):
    torch = pytest.importorskip("torch")
    rp = np.array([0, 2, 3, 5], dtype=np.int32)
    col = np.array([1, 2, 0, 0, 1], dtype=np.int32)
    od = np.array([2, 2, 1], dtype=np.int32)
    m, nnz = 3, 5
    if case == "column_out_of_range":
        col[3] = 3
    elif case == "last_offset":
        rp[3] = 4
    elif case == "decreasing":
        rp[1], rp[2] = 3, 2
    elif case == "negative_degree":
        od[1] = -1
    else:
        m = 0
    d = [torch.from_numpy(a).cuda() for a in (rp, col, od)]
    d_s = torch.full((3,), 1.0 / 3, dtype=torch.float32, device="cuda")
    with pytest.raises(G.GprError) as e:
        G.pagerank_noalloc(m, nnz, d[0], d[1], d[2], d_s, tol=1e-4, max_iter=max_iter)
    assert e.value.status == G.GPR_EINVAL


def test_noalloc_rejects_sizes_beyond_its_scratch(G):
    limit = G.pagerank_noalloc_max_vertices()
    assert limit == 1 << 20
    with pytest.raises(G.GprError) as e:
        G.pagerank_noalloc(limit + 1, 0, 1, 1, 1, 1)
    assert e.value.status == G.GPR_EINVAL and "limit" in str(e.value)
