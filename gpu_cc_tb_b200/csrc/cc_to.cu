// Timestamp-ordering family: to, slow_to.
#include "cc_launch.cuh"
GCC_FAMILY(to, S_TO, S_SLOW_TO, -1, -1)
