// Deterministic ordered family: gacco, gputx.
#include "cc_launch.cuh"
GCC_FAMILY(ordered, S_GACCO, S_GPUTX, -1, -1)
