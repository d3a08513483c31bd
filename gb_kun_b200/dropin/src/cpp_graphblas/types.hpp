// The reference's src/cpp_graphblas/types.hpp, which its algorithms/cc/cc.hpp
// includes directly: the operator, monoid and semiring vocabulary.
#pragma once

#include "lablas/types.hpp"
