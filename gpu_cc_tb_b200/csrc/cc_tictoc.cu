// TicToc family: tictoc, slow_tictoc.
#include "cc_launch.cuh"
GCC_FAMILY(tictoc, S_TICTOC, S_SLOW_TICTOC, -1, -1)
