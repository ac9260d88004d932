// Variable-length transactions (up to 64 requests) for the batched-queue
// executor: tpl_nw, tpl_wd, to, silo, tictoc, mvcc at G in {4, 8, 16, 32};
// the latch variants are in cc_var_slow.cu.
#include "cc_launch.cuh"

namespace gcc {

cudaError_t launch_var(int s, int G, int grid, int block, const KParams &p, cudaStream_t st) {
    switch (s) {
        case S_TPL_NW: return launch_var_one<S_TPL_NW>(G, grid, block, p, st);
        case S_TPL_WD: return launch_var_one<S_TPL_WD>(G, grid, block, p, st);
        case S_TO: return launch_var_one<S_TO>(G, grid, block, p, st);
        case S_SILO: return launch_var_one<S_SILO>(G, grid, block, p, st);
        case S_TICTOC: return launch_var_one<S_TICTOC>(G, grid, block, p, st);
        case S_MVCC: return launch_var_one<S_MVCC>(G, grid, block, p, st);
        default: return launch_var_slow(s, G, grid, block, p, st);
    }
}

int occupancy_var(int s, int G, int block) {
    switch (s) {
        case S_TPL_NW: return occupancy_var_one<S_TPL_NW>(G, block);
        case S_TPL_WD: return occupancy_var_one<S_TPL_WD>(G, block);
        case S_TO: return occupancy_var_one<S_TO>(G, block);
        case S_SILO: return occupancy_var_one<S_SILO>(G, block);
        case S_TICTOC: return occupancy_var_one<S_TICTOC>(G, block);
        case S_MVCC: return occupancy_var_one<S_MVCC>(G, block);
        default: return occupancy_var_slow(s, G, block);
    }
}

}  // namespace gcc
