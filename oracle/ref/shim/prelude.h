// Included ahead of every reference source in the oracle build: the
// reference predates g++ 13, whose headers no longer pull <limits> in
// transitively (Limiter.cpp:174 uses std::numeric_limits).
#pragma once
#include <limits>
#include <cmath>
#include <algorithm>
