"""Small seeded graphs for the tests (numpy only; no GPU, no oracle)."""
import numpy as np


def in_csr(m, src, dst, dedup=True, drop_self=True):
    """Pull CSR of edges src->dst: row = dst, columns ascending (when dedup)
    or in edge order; returns (rowptr, col, outdeg)."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    if drop_self:
        keep = src != dst
        src, dst = src[keep], dst[keep]
    if dedup:
        key = np.unique(dst * m + src)
        dst, src = key // m, key % m
    else:
        order = np.argsort(dst, kind="stable")
        src, dst = src[order], dst[order]
    rowptr = np.zeros(m + 1, dtype=np.int32)
    np.cumsum(np.bincount(dst, minlength=m), out=rowptr[1:])
    outdeg = np.bincount(src, minlength=m).astype(np.int32)
    return rowptr, src.astype(np.int32), outdeg


def erdos_renyi(m, avg_deg, seed):
    rng = np.random.default_rng(seed)
    ne = int(m * avg_deg)
    return in_csr(m, rng.integers(0, m, ne), rng.integers(0, m, ne))


def star(m=100000, seed=0):
    """Every vertex points at vertex 0 (in-degree m-1, many chunks); vertex 0
    points at 1; plus a sprinkle of random edges."""
    rng = np.random.default_rng(seed)
    src = np.concatenate([np.arange(1, m), [0], rng.integers(0, m, m)])
    dst = np.concatenate([np.zeros(m - 1, dtype=np.int64), [1], rng.integers(0, m, m)])
    return in_csr(m, src, dst)


def degree_ladder(seed=0):
    """Rows whose in-degrees sit on and around the bin edges (0, 1, 63, 64,
    65, 127, 128, 129, 2047, 2048, 2049, 5000): exercises every bin."""
    rng = np.random.default_rng(seed)
    degs = [0, 1, 2, 3, 31, 32, 33, 63, 64, 65, 127, 128, 129, 2047, 2048, 2049, 4096, 5000]
    m = 6000
    src, dst = [], []
    for v, d in enumerate(degs):
        s = rng.choice(m, size=d, replace=False)
        s = s[s != v][: max(d - 1, 0)] if d > 0 else s
        src.append(s)
        dst.append(np.full(len(s), v))
    src.append(rng.integers(0, m, 4 * m))
    dst.append(rng.integers(len(degs), m, 4 * m))
    return in_csr(m, np.concatenate(src), np.concatenate(dst))


def zoo(kind, seed):
    """One small graph of a given shape for property tests: 'er' uniform,
    'power' power-law sources and targets, 'chain' a directed path plus a
    few back edges, 'islands' disconnected pieces with isolated vertices,
    'sink' many vertices without out-edges."""
    rng = np.random.default_rng(seed)
    m = int(rng.integers(300, 30000))
    if kind == "er":
        return erdos_renyi(m, float(rng.uniform(1, 12)), seed)
    if kind == "power":
        w = 1.0 / np.arange(1, m + 1) ** rng.uniform(0.6, 1.1)
        p = w / w.sum()
        ne = int(m * rng.uniform(4, 16))
        return in_csr(m, rng.choice(m, ne, p=p), rng.permutation(m)[rng.choice(m, ne, p=p)])
    if kind == "chain":
        src = np.concatenate([np.arange(m - 1), rng.integers(0, m, m // 10)])
        dst = np.concatenate([np.arange(1, m), rng.integers(0, m, m // 10)])
        return in_csr(m, src, dst)
    if kind == "islands":
        k = int(rng.integers(2, 8))
        cuts = np.sort(rng.choice(np.arange(1, m), k - 1, replace=False))
        bounds = np.concatenate([[0], cuts, [m]])
        src, dst = [], []
        for a, b in zip(bounds[:-1], bounds[1:]):
            if b - a > 3:
                n = (b - a) * 4
                src.append(rng.integers(a, b - 2, n))   # the last two of each piece isolated
                dst.append(rng.integers(a, b - 2, n))
        return in_csr(m, np.concatenate(src), np.concatenate(dst))
    if kind == "sink":
        ne = m * 6
        src = rng.integers(0, m // 3, ne)               # two thirds have no out-edges
        return in_csr(m, src, rng.integers(0, m, ne))
    raise ValueError(kind)
