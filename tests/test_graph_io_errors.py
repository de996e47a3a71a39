"""Malformed graph files (host only, no GPU).

The C entry gpr_read_graph returns a status and keeps the caller's process
alive; the C++ read_graph drop-in keeps the reference's behaviour on a bad
file (include/graph_io.h:280-295): a message, then exit.  Both report the
same reason, and gpr_parse_edges refuses the same files."""
import os
import subprocess

import pytest

from conftest import ROOT

MTX = "%%MatrixMarket matrix coordinate pattern general\n"

# file name -> (contents, reason in the message)
CASES = {
    "empty.mtx": ("", "empty file"),
    "header_only.mtx": (MTX, "missing size line"),
    "negative_m.mtx": (MTX + "-4 4 3\n1 2\n", "bad size line"),
    "short.mtx": (MTX + "4 4 5\n1 2\n2 3\n", "fewer entries than announced"),
    "out_of_range.mtx": (MTX + "4 4 2\n1 2\n1 9\n", "index out of range"),
    "zero_index.mtx": (MTX + "4 4 1\n0 2\n", "index out of range"),
    "short.gr": ("p sp 4 5\na 1 2 1\n", "fewer arcs than announced"),
    "negative_m.gr": ("p sp -4 1\na 1 2 1\n", "bad problem line"),
    "out_of_range.gr": ("p sp 4 1\na 1 7 1\n", "index out of range"),
    "empty.graph": ("", "empty file"),
    "negative_m.graph": ("-3 2\n", "bad size line"),
    "out_of_range.graph": ("3 2\n9\n\n\n", "index out of range"),
    "edges.txt": ("1 2\n", "unrecognizable input file format"),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_c_entry_returns_einval(G, tmp_path, name):
    text, why = CASES[name]
    p = tmp_path / name
    p.write_text(text)
    with pytest.raises(G.GprError) as e:
        G.read_graph(str(p))
    assert e.value.status == G.GPR_EINVAL
    assert why in str(e.value)
    if not name.endswith(".txt"):
        with pytest.raises(G.GprError):
            G.parse_edges(str(p))


def test_c_entry_missing_file_and_good_file_after_errors(G, tmp_path):
    with pytest.raises(G.GprError) as e:
        G.read_graph(str(tmp_path / "absent.mtx"))
    assert e.value.status == G.GPR_EINVAL and "cannot open" in str(e.value)
    # an edge count below the announced one in .graph is the reference's
    # behaviour (lines past the last vertex are not read), not an error
    p = tmp_path / "ok.graph"
    p.write_text("3 2\n2 3\n\n\n")
    m, nnz, rp, col, deg, wt = G.read_graph(str(p))
    assert (m, nnz) == (3, 2) and list(rp) == [0, 2, 2, 2] and list(col) == [1, 2]
    assert list(deg) == [2, 0, 0]


@pytest.fixture(scope="module")
def dropin_reader(G, tmp_path_factory):
    """A program that calls the C++ read_graph drop-in the way the
    reference's drivers do (src/pr/main.cc:23)."""
    d = tmp_path_factory.mktemp("reader")
    src = d / "reader.cc"
    src.write_text(
        '#include <stdio.h>\n#include "gardenia_graph_io.h"\n'
        "int main(int argc, char *argv[]) {\n"
        "  int m, n, nnz, *rp = nullptr, *col = nullptr, *deg = nullptr;\n"
        "  WeightT *w = nullptr;\n"
        "  read_graph(argc, argv, m, n, nnz, rp, col, deg, w, false, false, false, true, true);\n"
        '  printf("read %d %d\\n", m, nnz);\n  return 0;\n}\n')
    exe = d / "reader"
    lib_dir = os.path.dirname(G.LIB_PATH)
    p = subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", str(src), "-o", str(exe),
                        "-I", os.path.join(ROOT, "include"), G.LIB_PATH,
                        "-Wl,--allow-shlib-undefined", f"-Wl,-rpath,{lib_dir}"],
                       capture_output=True, text=True)
    if p.returncode != 0:
        pytest.skip("cannot link a host program against libgpr here: " + p.stderr[-300:])
    return str(exe)


@pytest.mark.parametrize("name", ["negative_m.mtx", "short.gr", "out_of_range.graph"])
def test_cpp_dropin_prints_and_exits(dropin_reader, tmp_path, name):
    text, why = CASES[name]
    p = tmp_path / name
    p.write_text(text)
    r = subprocess.run([dropin_reader, str(p)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert f"read_graph: {p}: {why}" in r.stderr
    assert "read " not in r.stdout


def test_cpp_dropin_unknown_format_exits_zero(dropin_reader, tmp_path):
    p = tmp_path / "edges.txt"
    p.write_text("1 2\n")
    r = subprocess.run([dropin_reader, str(p)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "Unrecognizable input file format" in r.stdout
    assert "read " not in r.stdout


def test_cpp_dropin_reads_a_good_file(dropin_reader):
    r = subprocess.run([dropin_reader, os.path.join(ROOT, "tests", "golden", "graph_small.mtx")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "read " in r.stdout
