// Umbrella header of the lablas:: API on B200 -- the drop-in for the
// reference's src/gb_kun.h: the same class, function and macro names, with
// every vector and matrix held in GPU memory and every operation running as
// sm_100a kernels through the gbk C ABI (libgbk.so).  Link with -lgbk.
#pragma once

#include <iostream>
#include <string>
#include <vector>

#include "lablas/types.hpp"
#include "lablas/core.hpp"
#include "lablas/descriptor.hpp"
#include "lablas/vector.hpp"
#include "lablas/matrix.hpp"
#include "lablas/operations.hpp"
#include "lablas/cblas_wrappers.hpp"
#include "lablas/stats.hpp"
