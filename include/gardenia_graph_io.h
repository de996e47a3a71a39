/*
 * gardenia_graph_io.h -- CSR loaders with the reference's interface and
 * flag semantics (include/graph_io.h:21-295).
 *
 * read_graph(argc, argv, ...) reads argv[1], picking the parser by file
 * name (".mtx", then ".graph", then ".gr", as graph_io.h:282-288 does), and
 * returns malloc'd row_offsets / column_indices / degree / weight arrays
 * owned by the caller (free()).  Flags, exactly as the reference applies
 * them (graph_io.h:21-130):
 *   is_symmetrize      add the reverse of every edge (and, as in the
 *                      reference, stop transposing once set)
 *   is_transpose       store edge (u,v) in row v (in-CSR)
 *   sorted             sort each row by column (std::sort on column)
 *   remove_selfloops   drop (v,v)
 *   remove_redundents  drop a column equal to the previous kept one in the
 *                      row (all duplicates only when sorted)
 * .mtx weights are made non-negative; .gr/.graph weights are 1; indices in
 * every format are 1-based on disk.  degree[v] = row length.
 */
#ifndef GARDENIA_GRAPH_IO_H_
#define GARDENIA_GRAPH_IO_H_

typedef float WeightT; /* include/graph_io.h:13 */

void read_graph(int argc, char *argv[], int &m, int &n, int &nnz,
                int *&row_offsets, int *&column_indices, int *&degree,
                WeightT *&weight, bool is_symmetrize = false,
                bool is_transpose = false, bool sorted = true,
                bool remove_selfloops = true, bool remove_redundents = true);

#endif
