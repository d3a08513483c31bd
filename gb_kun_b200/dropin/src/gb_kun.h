// Drop-in replacement for the reference's src/gb_kun.h.
//
// Put this directory where the reference's src/ directory was (the
// reference's own algorithms/ directory stays beside it, unchanged: its files
// include "../../src/gb_kun.h").  Everything the reference's header made
// visible to its callers comes from here: the lablas:: API (vectors and
// matrices in GPU memory, every operation a sm_100a kernel through
// libgbk.so), the GrB_* wrappers and LAGraph_Graph, the backend CSR view the
// sequential checkers read, the SAVE_STATS / SAVE_TEPS statistics macros and
// the standard-library names the reference's header brings into the global
// namespace (its src/gb_kun.h:1-40 includes these headers and declares
// `using namespace std`).
#pragma once

#include <algorithm>
#include <cassert>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <list>
#include <map>
#include <queue>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "lablas/gb_kun.h"
#include "lablas/stats.hpp"

using namespace std;
