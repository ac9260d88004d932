// Silo family: silo, slow_silo.
#include "cc_launch.cuh"
GCC_FAMILY(silo, S_SILO, S_SLOW_SILO, -1, -1)
