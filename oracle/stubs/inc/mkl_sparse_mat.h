/* Oracle build stub for the reference's MKL matrix facade, reduced to the
 * read-only accessors that its reordering sources (RCM, BFS, union-find)
 * call: sizes, index base and shared row/column index arrays. */
#pragma once
#include <memory>
#include <vector>
#include "mkl_types.h"
namespace mkl_wrapper {
class mkl_sparse_mat {
public:
  mkl_sparse_mat(MKL_INT rows, MKL_INT cols, std::shared_ptr<MKL_INT[]> ai,
                 std::shared_ptr<MKL_INT[]> aj, int base)
      : _rows(rows), _cols(cols), _ai(std::move(ai)), _aj(std::move(aj)),
        _base(base) {}
  MKL_INT rows() const { return _rows; }
  MKL_INT cols() const { return _cols; }
  MKL_INT nnz() const { return _ai[_rows] - _ai[0]; }
  int mkl_base() const { return _base; }
  std::shared_ptr<const MKL_INT[]> get_ai() const { return _ai; }
  std::shared_ptr<const MKL_INT[]> get_aj() const { return _aj; }
  void get_adjacency_graph(std::vector<MKL_INT> &, std::vector<MKL_INT> &) const {}

private:
  MKL_INT _rows, _cols;
  std::shared_ptr<MKL_INT[]> _ai, _aj;
  int _base;
};
} // namespace mkl_wrapper
