#include "harness.h"
