"""Generates the golden fixtures in this directory from the reference itself.

Run where the reference tree is present and oracle/_ref is built
(`make -C oracle`):

    python tests/golden/make_golden.py

Outputs (committed, so machines without the reference tree keep the pin):

* graph_{small,dups,simple}.{mtx,gr,graph} -- seeded synthetic graphs written
  by this script (not reference data): duplicate edges, self-loops and
  negative .mtx weights exercise every loader flag; graph_simple has none;
* loader.npz -- the reference loader's CSR (include/graph_io.h:280 read_graph)
  for every file above under every flag combination the reference's drivers
  use, plus the reference's own datasets test_pr.mtx, chesapeake.mtx, 4.mtx
  and 4.graph as read by the PR driver (src/pr/main.cc:23-24);
* pr.npz -- the reference's OpenMP PRSolver (src/pr/omp_base.cc) scores and
  printed sweep counts on those graphs and on a seeded RMAT scale-10 graph,
  at its compiled-in constants (1e-3 / 30) and at 1e-4 / 100;
* spmv.npz -- the reference's OpenMP SpmvSolver (src/spmv/omp_base.cc) on the
  same CSRs with seeded x and y;
* symgs.npz -- the reference's OpenMP SymGSSolver (src/symgs/omp_base.cc), one
  multicolour sweep with a first-fit colouring, on the synthetic .mtx files
  read as its driver reads them (src/symgs/main.cc:17: symmetrized, sorted,
  self-loops kept, repeats removed) and on a 27-point stencil, seeded x and b.

`python tests/golden/make_golden.py symgs` regenerates symgs.npz alone.
"""
import itertools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

REF_DATA = os.path.join(O.reference_root(), "datasets")
FLAGS = list(itertools.product([False, True], repeat=5))  # sym, trans, sorted, selfloops, dups


def write_files(name, m, src, dst, wt):
    """Writes one edge list in the three formats the loaders read (1-based)."""
    with open(os.path.join(HERE, name + ".mtx"), "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n% synthetic, seeded\n")
        f.write(f"{m} {m} {len(src)}\n")
        for s, d, w in zip(src, dst, wt):
            f.write(f"{s + 1} {d + 1} {w:.6g}\n")
    with open(os.path.join(HERE, name + ".gr"), "w") as f:
        f.write("c synthetic, seeded\n")
        f.write(f"p sp {m} {len(src)}\n")
        for s, d in zip(src, dst):
            f.write(f"a {s + 1} {d + 1} 1\n")
    rows = [[] for _ in range(m)]
    for s, d in zip(src, dst):
        rows[s].append(d + 1)
    with open(os.path.join(HERE, name + ".graph"), "w") as f:
        f.write(f"{m} {len(src)}\n")
        for r in rows:
            f.write(" ".join(str(x) for x in r) + "\n")


def synthetic():
    rng = np.random.default_rng(2024)
    out = {}
    m = 40
    src = rng.integers(0, m, 260)
    dst = rng.integers(0, m, 260)
    wt = np.round(rng.normal(0, 2, 260), 3)
    out["graph_small"] = (m, src, dst, wt)
    m = 12
    base_s = rng.integers(0, m, 30)
    base_d = rng.integers(0, m, 30)
    src = np.concatenate([base_s, base_s[:10], np.arange(4)])  # duplicates, self-loops
    dst = np.concatenate([base_d, base_d[:10], np.arange(4)])
    wt = np.round(rng.normal(0, 1, len(src)), 3)
    out["graph_dups"] = (m, src, dst, wt)
    m = 60
    pairs = np.unique(rng.integers(0, m, (400, 2)), axis=0)
    pairs = pairs[pairs[:, 0] != pairs[:, 1]]
    rng.shuffle(pairs)
    out["graph_simple"] = (m, pairs[:, 0], pairs[:, 1], np.ones(len(pairs)))
    return out


def symgs_golden():
    out = {}
    cases = {}
    for name in ("graph_small.mtx", "graph_dups.mtx", "graph_simple.mtx"):
        rp, col, _, wt, _ = O.ref_read_graph(os.path.join(HERE, name), True, False, True, False,
                                             True)
        cases[name] = (rp, col, wt)
    cases["stencil27_n9"] = O.stencil27(9)
    for name, (rp, col, wt) in cases.items():
        m = len(rp) - 1
        idx, co = O.greedy_coloring(rp, col)
        x = O.uniform_f32(m, 13)
        b = O.uniform_f32(m, 14)
        xr, _ = O.ref_symgs_solver(rp, col, wt, idx, co, x, b)
        for k, v in (("Ap", rp), ("Aj", col), ("Ax", wt), ("indices", idx),
                     ("color_offsets", co), ("x0", x), ("b", b), ("x", xr)):
            out[f"{name}:{k}"] = v
    np.savez_compressed(os.path.join(HERE, "symgs.npz"), **out)
    print(f"wrote {len(out)} symgs arrays")


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref is not built (needs the reference tree)")
    if sys.argv[1:] == ["symgs"]:
        symgs_golden()
        return
    if not O.ref_available():
        sys.exit("oracle/_ref is not built (needs the reference tree)")
    loader, pr, spmv = {}, {}, {}
    files = []
    for name, (m, s, d, w) in synthetic().items():
        write_files(name, m, s, d, w)
        files += [os.path.join(HERE, name + ext) for ext in (".mtx", ".gr", ".graph")]
    for path in files:
        base = os.path.basename(path)
        for fl in FLAGS:
            rp, col, deg, wt, _ = O.ref_read_graph(path, *fl)
            key = base + ":" + "".join(str(int(x)) for x in fl)
            loader[key + ":rowptr"] = rp
            loader[key + ":col"] = col
            loader[key + ":weight"] = wt
    pr_graphs = {}
    # datasets/4.gr is left out: its arcs are 0-based ("a 0 13 92") while gr2csr
    # subtracts one (include/graph_io.h:157-158), so the reference loader
    # indexes vertex -1 and corrupts its heap on that file.
    for ds in ("test_pr.mtx", "chesapeake.mtx", "4.mtx", "4.graph"):
        p = os.path.join(REF_DATA, ds)
        orp, ocol, odeg, _, _ = O.ref_read_graph(p, False, False, False)
        irp, icol, _, _, _ = O.ref_read_graph(p, False, True, False)
        loader[f"ref:{ds}:out_rowptr"], loader[f"ref:{ds}:out_col"] = orp, ocol
        loader[f"ref:{ds}:in_rowptr"], loader[f"ref:{ds}:in_col"] = irp, icol
        pr_graphs[ds] = (irp, icol, odeg, orp, ocol)
    for name in ("graph_small.mtx", "graph_dups.mtx", "graph_simple.mtx"):
        p = os.path.join(HERE, name)
        orp, ocol, odeg, _, _ = O.ref_read_graph(p, False, False, False)
        irp, icol, _, _, _ = O.ref_read_graph(p, False, True, False)
        pr_graphs[name] = (irp, icol, odeg, orp, ocol)
    rp, col, od = O.rmat_graph(10, 16, seed=1)
    pr_graphs["rmat10"] = (rp, col, od, None, None)
    for gname, (irp, icol, odeg, orp, ocol) in pr_graphs.items():
        pr[f"{gname}:in_rowptr"], pr[f"{gname}:in_col"], pr[f"{gname}:outdeg"] = irp, icol, odeg
        for tol, mi in ((1e-3, 30), (1e-4, 100)):
            s, printed, _ = O.ref_pr_solver(irp, icol, odeg, tol=tol, max_iter=mi)
            pr[f"{gname}:{tol:g}:{mi}:scores"] = s
            pr[f"{gname}:{tol:g}:{mi}:printed_iterations"] = np.array([printed])
        m = len(irp) - 1
        x = O.uniform_f32(m, 5)
        y = O.uniform_f32(m, 6)
        vals = (1.0 - 2.0 * O.uniform_f32(len(icol), 7)).astype(np.float32)
        yr, _ = O.ref_spmv_solver(irp, icol, vals, x, y)
        spmv[f"{gname}:Ap"], spmv[f"{gname}:Aj"], spmv[f"{gname}:Ax"] = irp, icol, vals
        spmv[f"{gname}:x"], spmv[f"{gname}:y0"], spmv[f"{gname}:y"] = x, y, yr
    np.savez_compressed(os.path.join(HERE, "loader.npz"), **loader)
    np.savez_compressed(os.path.join(HERE, "pr.npz"), **pr)
    np.savez_compressed(os.path.join(HERE, "spmv.npz"), **spmv)
    print(f"wrote {len(loader)} loader, {len(pr)} pr, {len(spmv)} spmv arrays")
    symgs_golden()


if __name__ == "__main__":
    main()
