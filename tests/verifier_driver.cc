// Test driver for the restated verifiers exported by libgpr (PRVerifier,
// SpmvVerifier, SymGSVerifier; src/pr/verifier.cc:10-69,
// src/spmv/verifier.cc:24-62, src/symgs/verifier.cc:64-88).  It reads the
// arrays a test wrote into a directory as raw little-endian files and calls
// one verifier, whose verdict line goes to stdout.
//
//   verifier_driver pr    DIR   # in_rowptr in_col out_rowptr out_col outdeg scores (+ target)
//   verifier_driver spmv  DIR   # Ap Aj Ax x y test_y
//   verifier_driver symgs DIR   # Ap Aj Ax indices color_offsets test_x x b
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "gardenia_pr.h"
#include "gardenia_spmv.h"
#include "gardenia_symgs.h"

template <typename T>
static std::vector<T> load(const std::string &dir, const char *name) {
  const std::string path = dir + "/" + name + ".bin";
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path.c_str());
    exit(2);
  }
  fseek(f, 0, SEEK_END);
  const long bytes = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<T> v(bytes / sizeof(T));
  if (!v.empty() && fread(v.data(), sizeof(T), v.size(), f) != v.size()) exit(2);
  fclose(f);
  return v;
}

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  const std::string kind = argv[1], dir = argv[2];
  if (kind == "pr") {
    auto irp = load<int>(dir, "in_rowptr"), icol = load<int>(dir, "in_col");
    auto orp = load<int>(dir, "out_rowptr"), ocol = load<int>(dir, "out_col");
    auto deg = load<int>(dir, "outdeg");
    auto s = load<float>(dir, "scores");
    auto target = load<double>(dir, "target");
    PRVerifier((int)irp.size() - 1, irp.data(), icol.data(), orp.data(), ocol.data(), deg.data(),
               s.data(), target[0]);
  } else if (kind == "spmv") {
    auto Ap = load<int>(dir, "Ap"), Aj = load<int>(dir, "Aj");
    auto Ax = load<float>(dir, "Ax"), x = load<float>(dir, "x"), y = load<float>(dir, "y");
    auto ty = load<float>(dir, "test_y");
    SpmvVerifier((int)Ap.size() - 1, (int)Aj.size(), Ap.data(), Aj.data(), Ax.data(), x.data(),
                 y.data(), ty.data());
  } else if (kind == "symgs") {
    auto Ap = load<int>(dir, "Ap"), Aj = load<int>(dir, "Aj"), idx = load<int>(dir, "indices");
    auto co = load<int>(dir, "color_offsets");
    auto Ax = load<float>(dir, "Ax"), tx = load<float>(dir, "test_x");
    auto x = load<float>(dir, "x"), b = load<float>(dir, "b");
    SymGSVerifier((int)Ap.size() - 1, Ap.data(), Aj.data(), idx.data(), Ax.data(), tx.data(),
                  x.data(), b.data(), co);
  } else {
    return 2;
  }
  return 0;
}
