/* Peak-throughput probes for the roofline denominators (measurement utility,
 * no counterpart in the reference).  Each thread runs 8 independent
 * fused-multiply-add chains; FLOPs = 2 * 8 * iters * threads. */
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/odevec_b200.h"

namespace {

template <class T>
__global__ void fma_chains(T* out, int iters, T a, T b)
{
    T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
      x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, a, b);
        x1 = fma(x1, a, b);
        x2 = fma(x2, a, b);
        x3 = fma(x3, a, b);
        x4 = fma(x4, a, b);
        x5 = fma(x5, a, b);
        x6 = fma(x6, a, b);
        x7 = fma(x7, a, b);
    }
    T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-1.2345)
        out[blockIdx.x] = s; /* never true; keeps the chains alive */
}

}  // namespace

extern "C" int32_t odevec_probe_fma(int32_t fp64, int32_t blocks, int32_t threads, int32_t iters,
                                    void* scratch, void* stream, float* ms, double* flops)
{
    if (blocks <= 0 || threads <= 0 || threads > 1024 || iters <= 0 || !scratch || !ms || !flops)
        return OV_API_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    if (fp64)
        fma_chains<double><<<blocks, threads, 0, st>>>((double*)scratch, iters, 0.999999, 1e-7);
    else
        fma_chains<float><<<blocks, threads, 0, st>>>((float*)scratch, iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1, st);
    cudaError_t err = cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *flops = 2.0 * 8.0 * (double)iters * (double)blocks * (double)threads;
    return err == cudaSuccess ? OV_API_OK : OV_API_ECUDA;
}
