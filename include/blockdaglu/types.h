// Matrix type of the blockdaglu::Solver drop-in.
//
// Same definition as the reference's blockdaglu::CooMatrix
// (blockdaglu/include/blockdaglu/types.h:10): a vector of (row, col, value)
// triplets, so callers that build or receive that type compile unchanged.
#pragma once

#include <tuple>
#include <vector>

namespace blockdaglu {

using CooMatrix = std::vector<std::tuple<int, int, double>>;

}  // namespace blockdaglu
