"""Loaders with the CSR built on the GPU, checked against the reference
loader's own output (golden fixtures made by the reference, tests/golden)."""
import itertools
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLD = os.path.join(ROOT, "tests", "golden")
FILES = [n + e for n in ("graph_small", "graph_dups", "graph_simple")
         for e in (".mtx", ".gr", ".graph")]


def multiset_equal(rp, c, w, w_ref):
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    return np.array_equal(w[np.lexsort((w, c, rows))], w_ref[np.lexsort((w_ref, c, rows))])


@pytest.mark.parametrize("name", FILES)
def test_read_graph_gpu_matches_reference_loader(G, name):
    path = os.path.join(GOLD, name)
    gold = np.load(os.path.join(GOLD, "loader.npz"))
    for fl in itertools.product([False, True], repeat=5):
        key = name + ":" + "".join(str(int(x)) for x in fl)
        A, W = G.read_graph_gpu(path, *fl)
        rp, col, deg, w = A.rowptr.to_numpy(), A.col.to_numpy(), A.third.to_numpy(), W.to_numpy()
        A.close()
        W.close()
        assert np.array_equal(rp, gold[key + ":rowptr"]), key
        assert np.array_equal(col, gold[key + ":col"]), key
        assert np.array_equal(deg, np.diff(rp)), key
        sym, trans, srt, sl, rd = fl
        if not srt:
            assert np.array_equal(w, gold[key + ":weight"]), key
        elif not rd:
            assert multiset_equal(rp, col, w, gold[key + ":weight"]), key


@pytest.mark.parametrize("name", FILES)
@pytest.mark.parametrize("symmetrize", [False, True])
def test_read_graph_pr_one_parse_matches_two_reads(G, name, symmetrize):
    gold = np.load(os.path.join(GOLD, "loader.npz"))
    out, inn = G.read_graph_pr(os.path.join(GOLD, name), symmetrize)
    s = str(int(symmetrize))
    ko, ki = name + f":{s}0011", name + f":{s}1011"
    assert np.array_equal(out.rowptr.to_numpy(), gold[ko + ":rowptr"])
    assert np.array_equal(out.col.to_numpy(), gold[ko + ":col"])
    assert np.array_equal(out.third.to_numpy(), np.diff(gold[ko + ":rowptr"]))
    assert np.array_equal(inn.rowptr.to_numpy(), gold[ki + ":rowptr"])
    assert np.array_equal(inn.col.to_numpy(), gold[ki + ":col"])
    out.close()
    inn.close()


def test_csr_from_edges_rejects_out_of_range(G):
    with pytest.raises(G.GprError) as e:
        G.csr_from_edges(4, np.array([0, 4], np.int32), np.array([1, 2], np.int32))
    assert e.value.status == G.GPR_EINVAL


def test_csr_from_edges_large_random(G, O):
    # a million pushes with many repeats and self-loops, every flag
    rng = np.random.default_rng(3)
    m = 5000
    row = rng.integers(0, m, 1_000_000).astype(np.int32)
    col = rng.integers(0, m, 1_000_000).astype(np.int32)
    col[::97] = row[::97]
    wt = rng.random(1_000_000).astype(np.float32)
    for srt, sl, rd in itertools.product([False, True], repeat=3):
        A = G.csr_from_edges(m, row, col, wt, srt, sl, rd)
        rp, c, w = O.csr_from_pushes(m, row, col, wt, srt, sl, rd)
        assert np.array_equal(A.rowptr.to_numpy(), rp)
        assert np.array_equal(A.col.to_numpy(), c)
        assert np.array_equal(A.third.to_numpy(), w)  # both stable
        A.close()
