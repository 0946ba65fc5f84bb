/* Oracle build stub for the absent fast_matrix_market library.
 * The reference's utils.h names these types in a reader template that the
 * oracle never instantiates; Matrix Market files are parsed by the oracle's
 * own reader instead.  Only declarations needed to compile are provided. */
#pragma once
#include <algorithm>
#include <cmath>
#include <istream>
#include <numeric>
namespace fast_matrix_market {
struct read_options {};
struct matrix_market_header {
  long long nrows = 0;
  long long ncols = 0;
};
template <typename IVEC, typename VVEC>
void read_matrix_market_triplet(std::istream &, matrix_market_header &, IVEC &,
                                IVEC &, VVEC &, const read_options &) {}
} // namespace fast_matrix_market
