// Variable-length transactions (up to 64 requests) under the latch ("slow_")
// variants: slow_tpl_nw, slow_tpl_wd, slow_to, slow_silo, slow_tictoc,
// slow_mvcc at G in {4, 8, 16, 32} (a translation unit of its own so that it
// compiles beside cc_var.cu).
#include "cc_launch.cuh"

namespace gcc {

cudaError_t launch_var_slow(int s, int G, int grid, int block, const KParams &p, cudaStream_t st) {
    switch (s) {
        case S_SLOW_TPL_NW: return launch_var_one<S_SLOW_TPL_NW>(G, grid, block, p, st);
        case S_SLOW_TPL_WD: return launch_var_one<S_SLOW_TPL_WD>(G, grid, block, p, st);
        case S_SLOW_TO: return launch_var_one<S_SLOW_TO>(G, grid, block, p, st);
        case S_SLOW_SILO: return launch_var_one<S_SLOW_SILO>(G, grid, block, p, st);
        case S_SLOW_TICTOC: return launch_var_one<S_SLOW_TICTOC>(G, grid, block, p, st);
        case S_SLOW_MVCC: return launch_var_one<S_SLOW_MVCC>(G, grid, block, p, st);
        default: return cudaErrorInvalidValue;
    }
}

int occupancy_var_slow(int s, int G, int block) {
    switch (s) {
        case S_SLOW_TPL_NW: return occupancy_var_one<S_SLOW_TPL_NW>(G, block);
        case S_SLOW_TPL_WD: return occupancy_var_one<S_SLOW_TPL_WD>(G, block);
        case S_SLOW_TO: return occupancy_var_one<S_SLOW_TO>(G, block);
        case S_SLOW_SILO: return occupancy_var_one<S_SLOW_SILO>(G, block);
        case S_SLOW_TICTOC: return occupancy_var_one<S_SLOW_TICTOC>(G, block);
        case S_SLOW_MVCC: return occupancy_var_one<S_SLOW_MVCC>(G, block);
        default: return -1;
    }
}

}  // namespace gcc
