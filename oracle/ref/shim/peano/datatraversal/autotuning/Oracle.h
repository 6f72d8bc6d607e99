// stand-in for the grain-size oracle: every loop runs serially
#pragma once
#include "peano/datatraversal/autotuning/MethodTrace.h"
namespace peano { namespace datatraversal { namespace autotuning {
struct GrainSize { int getGrainSize() const { return 0; } void parallelSectionHasTerminated() {} };
struct Oracle {
  static Oracle& getInstance() { static Oracle o; return o; }
  GrainSize parallelise(int, MethodTrace) { return GrainSize(); }
};
}}}
