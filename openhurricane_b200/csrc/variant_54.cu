// Cell-group kernel variant for mechanisms whose N = nsp + 1 equations fit 54 (cell group of 64 lanes).
#include "launch.cuh"
#include "variants.h"

HC_DEFINE_VARIANT(54, 54, 64)
