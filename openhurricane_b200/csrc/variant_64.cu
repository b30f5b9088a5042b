// Cell-group kernel variant for mechanisms whose N = nsp + 1 equations fit 64 (cell group of 64 lanes).
#include "launch.cuh"
#include "variants.h"

HC_DEFINE_VARIANT(64, 64, 64)
