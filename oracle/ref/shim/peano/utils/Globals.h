#pragma once
#include "tarch/Assertions.h"
#define DIMENSIONS_TIMES_TWO (2 * DIMENSIONS)
