/* Launch arguments shared by the kernels and the C-ABI layer. */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ov {

struct LaunchArgs {
    int64_t ncells;
    double* y;             /* [neq][ncells] */
    double* t;             /* [ncells] */
    double* dt;            /* [ncells] */
    const double* t_stop;  /* [ncells] */
    const uint8_t* mask;   /* [ncells] or null */
    int32_t* status;       /* [ncells] or null */
    int32_t* stats;        /* [ncells][OV_NSTATS] or null */
    unsigned long long* queue; /* work counter, zero at launch */
    double rtol, atol, dt_min;
    int32_t check_neg;
    int32_t max_attempts;
};

/* one launcher per network variant and arithmetic mode; returns the CUDA
   error of the launch.  G: 1 or 32; lu: 0 = FP64 LU, 1 = FP32 LU.
   block/grid 0: default (persistent grid from the occupancy). */
typedef cudaError_t (*launch_fn)(const LaunchArgs& a, int G, int lu, int block, int grid,
                                 cudaStream_t stream);

}  // namespace ov
