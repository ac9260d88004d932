// cc_launch.cuh -- per-scheme launch / occupancy helpers over the group size
// G = 2^warp_density. Each scheme family is instantiated in its own
// translation unit so the six G variants of every scheme compile in parallel.
#pragma once
#include "cc_kernel.cuh"

namespace gcc {

template <int SCH>
cudaError_t launch_one(int G, int grid, int block, const KParams &p, cudaStream_t st) {
    switch (G) {
        case 1: ycsb_kernel<SCH, 1><<<grid, block, 0, st>>>(p); break;
        case 2: ycsb_kernel<SCH, 2><<<grid, block, 0, st>>>(p); break;
        case 4: ycsb_kernel<SCH, 4><<<grid, block, 0, st>>>(p); break;
        case 8: ycsb_kernel<SCH, 8><<<grid, block, 0, st>>>(p); break;
        case 16: ycsb_kernel<SCH, 16><<<grid, block, 0, st>>>(p); break;
        case 32: ycsb_kernel<SCH, 32><<<grid, block, 0, st>>>(p); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int SCH>
int occupancy_one(int G, int block) {
    int n = 0;
    cudaError_t e = cudaErrorInvalidValue;
    switch (G) {
        case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 1>, block, 0); break;
        case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 2>, block, 0); break;
        case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 4>, block, 0); break;
        case 8: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 8>, block, 0); break;
        case 16: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 16>, block, 0); break;
        case 32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 32>, block, 0); break;
        default: break;
    }
    return e == cudaSuccess ? n : -1;
}

// Variable-length transactions (up to 64 requests): G in {4, 8, 16, 32}.
template <int SCH>
cudaError_t launch_var_one(int G, int grid, int block, const KParams &p, cudaStream_t st) {
    switch (G) {
        case 4: ycsb_kernel<SCH, 4, kMaxVarOps><<<grid, block, 0, st>>>(p); break;
        case 8: ycsb_kernel<SCH, 8, kMaxVarOps><<<grid, block, 0, st>>>(p); break;
        case 16: ycsb_kernel<SCH, 16, kMaxVarOps><<<grid, block, 0, st>>>(p); break;
        case 32: ycsb_kernel<SCH, 32, kMaxVarOps><<<grid, block, 0, st>>>(p); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
template <int SCH>
int occupancy_var_one(int G, int block) {
    int n = 0;
    cudaError_t e = cudaErrorInvalidValue;
    switch (G) {
        case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 4, kMaxVarOps>, block, 0); break;
        case 8: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 8, kMaxVarOps>, block, 0); break;
        case 16: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 16, kMaxVarOps>, block, 0); break;
        case 32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ycsb_kernel<SCH, 32, kMaxVarOps>, block, 0); break;
        default: break;
    }
    return e == cudaSuccess ? n : -1;
}
cudaError_t launch_var(int s, int G, int grid, int block, const KParams &p, cudaStream_t st);
int occupancy_var(int s, int G, int block);
cudaError_t launch_var_slow(int s, int G, int grid, int block, const KParams &p, cudaStream_t st);
int occupancy_var_slow(int s, int G, int block);

// Declared per family; defined in cc_<family>.cu.
cudaError_t launch_family_tpl(int s, int G, int grid, int block, const KParams &p, cudaStream_t st);
cudaError_t launch_family_to(int s, int G, int grid, int block, const KParams &p, cudaStream_t st);
cudaError_t launch_family_mvcc(int s, int G, int grid, int block, const KParams &p, cudaStream_t st);
cudaError_t launch_family_silo(int s, int G, int grid, int block, const KParams &p, cudaStream_t st);
cudaError_t launch_family_tictoc(int s, int G, int grid, int block, const KParams &p, cudaStream_t st);
cudaError_t launch_family_ordered(int s, int G, int grid, int block, const KParams &p, cudaStream_t st);
int occupancy_family_tpl(int s, int G, int block);
int occupancy_family_to(int s, int G, int block);
int occupancy_family_mvcc(int s, int G, int block);
int occupancy_family_silo(int s, int G, int block);
int occupancy_family_tictoc(int s, int G, int block);
int occupancy_family_ordered(int s, int G, int block);

}  // namespace gcc

#define GCC_FAMILY(NAME, S1, S2, S3, S4)                                                       \
    namespace gcc {                                                                            \
    cudaError_t launch_family_##NAME(int s, int G, int grid, int block, const KParams &p,      \
                                     cudaStream_t st) {                                        \
        if (s == S1) return launch_one<S1>(G, grid, block, p, st);                             \
        if (s == S2) return launch_one<S2>(G, grid, block, p, st);                             \
        if (S3 >= 0 && s == S3) return launch_one<(S3 >= 0 ? S3 : S1)>(G, grid, block, p, st); \
        if (S4 >= 0 && s == S4) return launch_one<(S4 >= 0 ? S4 : S1)>(G, grid, block, p, st); \
        return cudaErrorInvalidValue;                                                          \
    }                                                                                          \
    int occupancy_family_##NAME(int s, int G, int block) {                                     \
        if (s == S1) return occupancy_one<S1>(G, block);                                       \
        if (s == S2) return occupancy_one<S2>(G, block);                                       \
        if (S3 >= 0 && s == S3) return occupancy_one<(S3 >= 0 ? S3 : S1)>(G, block);          \
        if (S4 >= 0 && s == S4) return occupancy_one<(S4 >= 0 ? S4 : S1)>(G, block);          \
        return -1;                                                                             \
    }                                                                                          \
    }
