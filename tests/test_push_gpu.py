"""Push-style PageRank (atomic scatter over a source-sorted edge list) on the
GPU, held to the plain path's bar against the reference's pull recurrence
(1e-6 per vertex plus the reference's own float error on hub rows, sweeps
within one).  Atomic adds make the last bits vary between runs."""
import numpy as np
import pytest

from graphs import degree_ladder, erdos_renyi, star

pytestmark = pytest.mark.gpu


def check(O, rp, col, od, s, it, tol, max_iter):
    ref, ref_it, _ = O.pr_plain_f32(rp, col, od, tol=tol, max_iter=max_iter)
    assert abs(it - ref_it) <= 1
    s64, _, _ = O.pr_f64(rp, col, od, tol=0.0, max_iter=it)
    assert np.all(np.abs(s - ref) <= 1e-6 + np.abs(ref - s64))


@pytest.mark.parametrize("maker", ["rmat", "er", "star", "ladder"])
def test_push_matches_reference(G, O, maker):
    rp, col, od = {"rmat": lambda: O.rmat_graph(15, 16, seed=3),
                   "er": lambda: erdos_renyi(20000, 8, seed=4),
                   "star": star, "ladder": degree_ladder}[maker]()
    # On the hub graphs the L1 residual's float rounding floor is about
    # m * ulp(score) ~ 1e-7; the tolerance sits well above it (as for the
    # pull solver's hub tests), where the arithmetic, not the rounding
    # noise of the atomic sums, decides the sweep count.
    tol = 1e-5 if maker in ("star", "ladder") else 1e-6
    with G.Graph(rp, col, od, push=True) as g:
        s, st = g.pagerank_push(tol=tol, max_iter=100)
        s2, st2 = g.pagerank_push(tol=tol, max_iter=100)
    check(O, rp, col, od, s, st.iterations, tol, 100)
    assert abs(st2.iterations - st.iterations) <= 1
    assert np.abs(s - s2).max() <= 1e-6


def test_push_caps_and_small_graphs(G, O):
    rp, col, od = O.rmat_graph(10, 8, seed=2)  # m < the shared-memory prefix
    with G.Graph(rp, col, od, push=True) as g:
        s, st = g.pagerank_push(tol=0.0, max_iter=5)
        assert st.iterations == 5
        check(O, rp, col, od, s, 5, 0.0, 5)
        s, st = g.pagerank_push(tol=1e-6, max_iter=0)
        assert st.iterations == 0
        assert np.all(s == np.float32(1.0) / np.float32(len(rp) - 1))


def test_push_needs_the_csr(G, O):
    rp, col, od = O.rmat_graph(8, 8, seed=1)
    with G.Graph(rp, col, od) as g:
        with pytest.raises(G.GprError) as e:
            g.pagerank_push()
        assert e.value.status == G.GPR_EUNSUPPORTED


def test_push_barrier_timeout(G, O):
    rp, col, od = O.rmat_graph(10, 8, seed=2)
    with G.Graph(rp, col, od, push=True) as g:
        o = G.options(tol=1e-6, max_iter=10, timeout_s=0.5)
        o.reserved[0] = 1
        with pytest.raises(G.GprError) as e:
            g.pagerank_push(opts=o)
        assert e.value.status == G.GPR_ETIMEOUT
        s, st = g.pagerank_push(tol=1e-6, max_iter=10)
        assert st.iterations > 0
