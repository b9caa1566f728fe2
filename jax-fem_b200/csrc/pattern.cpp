// Block-CSR sparsity pattern and cell->block scatter map (host, one-off setup).
//
// Replaces the duplicated COO pattern I, J of Problem.__post_init__
// (problem.py:86-107, num_cells*576 int64 pairs) and PETSc's
// setPreallocationCOO (solver.py:469-475).  The pattern is the node
// adjacency graph (one vec x vec block per pair of nodes sharing a cell);
// the scatter map gives, for every cell and local node pair (a, b), the
// index of block (cells[c,a], cells[c,b]) so assembly adds straight into the
// values array.  Columns are sorted within each block row.  Any number of
// nodes per cell (nen): HEX8 and the other element types of basis.py:19-114
// share this code.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "host_error.h"
#include <climits>

namespace {

struct Adjacency {
  std::vector<int64_t> start;  // node -> first incident cell slot
  std::vector<int32_t> cells;  // incident cells
};

int build_adjacency(const int32_t* cells, int64_t C, int nen, int64_t N, Adjacency* adj) {
  adj->start.assign(size_t(N) + 1, 0);
  for (int64_t i = 0; i < C * nen; ++i) {
    const int32_t n = cells[i];
    if (n < 0 || n >= N) {
      fem::set_error("fem_bsr_pattern: cell %lld references node %d outside [0, %lld)",
                     (long long)(i / nen), n, (long long)N);
      return FEM_ERR_ARG;
    }
    adj->start[size_t(n) + 1]++;
  }
  for (int64_t n = 0; n < N; ++n) adj->start[n + 1] += adj->start[n];
  adj->cells.resize(size_t(C) * nen);
  std::vector<int64_t> fill(adj->start.begin(), adj->start.end() - 1);
  for (int64_t c = 0; c < C; ++c)
    for (int a = 0; a < nen; ++a) {
      const int32_t n = cells[c * nen + a];
      // a cell listing the same node twice is adjacent once
      bool dup = false;
      for (int b = 0; b < a; ++b) dup |= (cells[c * nen + b] == n);
      if (!dup) adj->cells[fill[n]++] = int32_t(c);
    }
  // shrink ranges to the filled part (duplicates leave holes at the end)
  return FEM_OK;
}

// Sorted unique neighbours of node n.
void neighbours(const int32_t* cells, int nen, const Adjacency& adj, const std::vector<int64_t>& fill_end,
                int64_t n, std::vector<int32_t>* out) {
  out->clear();
  for (int64_t k = adj.start[n]; k < fill_end[n]; ++k) {
    const int32_t c = adj.cells[k];
    for (int b = 0; b < nen; ++b) out->push_back(cells[int64_t(c) * nen + b]);
  }
  std::sort(out->begin(), out->end());
  out->erase(std::unique(out->begin(), out->end()), out->end());
}

}  // namespace

extern "C" int fem_bsr_pattern_nen(const int32_t* h_cells, int64_t num_cells, int nen, int64_t num_nodes,
                                   int32_t* h_row_ptr, int64_t* h_nnzb, int32_t* h_col_idx,
                                   int64_t col_capacity, int32_t* h_scatter, int32_t* h_diag) {
  FEM_CHECK_ARG(num_cells >= 0 && num_nodes >= 0, "negative sizes");
  FEM_CHECK_ARG(nen >= 1 && nen <= 256, "nodes per cell %d outside [1, 256]", nen);
  FEM_CHECK_ARG(num_cells == 0 || h_cells != nullptr, "cells is NULL");
  FEM_CHECK_ARG(h_row_ptr != nullptr && h_nnzb != nullptr, "row_ptr/nnzb is NULL");
  Adjacency adj;
  int rc = build_adjacency(h_cells, num_cells, nen, num_nodes, &adj);
  if (rc != FEM_OK) return rc;
  // end of the filled range of each node
  std::vector<int64_t> fill_end(size_t(num_nodes), 0);
  {
    std::vector<int64_t> fill(adj.start.begin(), adj.start.end() - 1);
    for (int64_t c = 0; c < num_cells; ++c)
      for (int a = 0; a < nen; ++a) {
        const int32_t n = h_cells[c * nen + a];
        bool dup = false;
        for (int b = 0; b < a; ++b) dup |= (h_cells[c * nen + b] == n);
        if (!dup) fill[n]++;
      }
    for (int64_t n = 0; n < num_nodes; ++n) fill_end[n] = fill[n];
  }
  std::vector<int32_t> nb;
  int64_t nnzb = 0;
  h_row_ptr[0] = 0;
  for (int64_t n = 0; n < num_nodes; ++n) {
    neighbours(h_cells, nen, adj, fill_end, n, &nb);
    if (nb.empty()) nb.push_back(int32_t(n));  // isolated node keeps its diagonal block
    if (h_col_idx != nullptr) {
      if (nnzb + int64_t(nb.size()) > col_capacity) {
        fem::set_error("fem_bsr_pattern: col capacity %lld too small", (long long)col_capacity);
        return FEM_ERR_CAPACITY;
      }
      std::copy(nb.begin(), nb.end(), h_col_idx + nnzb);
      if (h_diag != nullptr) {
        auto it = std::lower_bound(nb.begin(), nb.end(), int32_t(n));
        h_diag[n] = int32_t(nnzb + (it - nb.begin()));
      }
    }
    nnzb += int64_t(nb.size());
    if (nnzb > INT32_MAX) {
      fem::set_error("fem_bsr_pattern: %lld blocks exceed int32 indexing", (long long)nnzb);
      return FEM_ERR_CAPACITY;
    }
    h_row_ptr[n + 1] = int32_t(nnzb);
  }
  *h_nnzb = nnzb;
  if (h_col_idx != nullptr && h_scatter != nullptr) {
    const int64_t nn = int64_t(nen) * nen;
    for (int64_t c = 0; c < num_cells; ++c)
      for (int a = 0; a < nen; ++a) {
        const int32_t na = h_cells[c * nen + a];
        const int32_t* b0 = h_col_idx + h_row_ptr[na];
        const int32_t* b1 = h_col_idx + h_row_ptr[na + 1];
        for (int b = 0; b < nen; ++b) {
          const int32_t nbn = h_cells[c * nen + b];
          const int32_t* it = std::lower_bound(b0, b1, nbn);
          h_scatter[c * nn + a * nen + b] = int32_t(it - h_col_idx);
        }
      }
  }
  return FEM_OK;
}

extern "C" int fem_bsr_pattern(const int32_t* h_cells, int64_t num_cells, int64_t num_nodes,
                               int32_t* h_row_ptr, int64_t* h_nnzb, int32_t* h_col_idx,
                               int64_t col_capacity, int32_t* h_scatter, int32_t* h_diag) {
  return fem_bsr_pattern_nen(h_cells, num_cells, 8, num_nodes, h_row_ptr, h_nnzb, h_col_idx, col_capacity,
                             h_scatter, h_diag);
}

// Block transpose map of a block-CSR pattern: h_tmap[k] = index of block
// (j, i) for block k = (i, j).  Used by assembly to write the lower block
// triangle from the upper one.  Fails if the pattern is not structurally
// symmetric or a row's columns are not sorted.
extern "C" int fem_bsr_transpose_map(const int32_t* h_row_ptr, const int32_t* h_col_idx, int64_t n_brows,
                                     int32_t* h_tmap) {
  if (h_row_ptr == nullptr || h_col_idx == nullptr || h_tmap == nullptr || n_brows < 0) {
    fem::set_error("fem_bsr_transpose_map: NULL pointer or negative size");
    return FEM_ERR_ARG;
  }
  for (int64_t i = 0; i < n_brows; ++i) {
    for (int32_t k = h_row_ptr[i]; k < h_row_ptr[i + 1]; ++k) {
      const int32_t j = h_col_idx[k];
      if (j < 0 || j >= n_brows || (k > h_row_ptr[i] && h_col_idx[k - 1] >= j)) {
        fem::set_error("fem_bsr_transpose_map: row %lld: columns not sorted or out of range", (long long)i);
        return FEM_ERR_ARG;
      }
      const int32_t* b = h_col_idx + h_row_ptr[j];
      const int32_t* e = h_col_idx + h_row_ptr[j + 1];
      const int32_t* f = std::lower_bound(b, e, int32_t(i));
      if (f == e || *f != int32_t(i)) {
        fem::set_error("fem_bsr_transpose_map: block (%lld, %d) has no transpose partner", (long long)i, j);
        return FEM_ERR_ARG;
      }
      h_tmap[k] = int32_t(f - h_col_idx);
    }
  }
  return FEM_OK;
}
