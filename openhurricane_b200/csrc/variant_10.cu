// Cell-group kernel variant for mechanisms whose N = nsp + 1 equations fit 10 (cell group of 32 lanes).
#include "launch.cuh"
#include "variants.h"

HC_DEFINE_VARIANT(10, 10, 32)
