// MVCC family: mvcc, slow_mvcc.
#include "cc_launch.cuh"
GCC_FAMILY(mvcc, S_MVCC, S_SLOW_MVCC, -1, -1)
