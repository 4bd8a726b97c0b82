// Throughput ceiling of the track-length tally's FP64 reductions on this GPU.
//
// The transport kernel scores every voxel visit with two FP64 reductions
// (kerma and H*(10) of one voxel, adjacent in a 16-byte cell) whose
// addresses follow the photons' paths.  No vendor figure gives the rate of
// such reductions, so this kernel measures it: every thread issues `per`
// visits, each two `red.global.add.f64` into one 16-byte cell of a region
// of `n_cells` cells, the cell chosen by a hash of (thread, visit) that is
//   * spread:  uniform over the region (a tally grid whose cells are hit at
//              random; region in or out of L2),
//   * hot:     one of `hot` cells (the busiest voxels of a beam),
//   * walk:    `run` consecutive cells along a line from a random start,
//              strided by `stride` cells (a photon crossing a row of voxels).
// The result is visits per second and reductions per second of one launch,
// timed with CUDA events; the region must be zeroed by the caller.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/chatcarlo_b200.h"

namespace {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    // a 32-bit integer hash (xorshift-multiply finaliser of MurmurHash3)
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ void red2(double* cell, double a, double b) {
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(cell), "d"(a) : "memory");
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(cell + 1), "d"(b) : "memory");
}

__global__ void atomics_kernel(double* __restrict__ cells, long long n_cells, int mode, int per, int hot, int run,
                               long long stride) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (mode == 2) {
        for (int v = 0; v < per; v += run) {
            const uint32_t h = mix32(tid * 0x9E3779B9u + (uint32_t)v);
            const long long span = (long long)run * stride;
            const long long start = n_cells > span ? (long long)(h % (uint32_t)(n_cells - span)) : 0;
            for (int k = 0; k < run && v + k < per; ++k) {
                const long long c = start + (long long)k * stride;
                red2(cells + 2 * c, 1.0, 0.5);
            }
        }
        return;
    }
    for (int v = 0; v < per; ++v) {
        const uint32_t h = mix32(tid * 0x9E3779B9u + (uint32_t)v * 0x85ebca6bu + 0x27d4eb2fu);
        const long long c = mode == 1 ? (long long)(h % (uint32_t)hot)
                                      : (long long)(((unsigned long long)h * (unsigned long long)n_cells) >> 32);
        red2(cells + 2 * c, 1.0, 0.5);
    }
}

}  // namespace

extern "C" int cc_measure_fp64_reductions(int device, double* d_cells, int64_t n_cells, int32_t mode,
                                          int32_t blocks, int32_t threads, int32_t per, int32_t hot, int32_t run,
                                          int64_t stride, int32_t repeats, double* visits_per_s) {
    if (!d_cells || n_cells < 1 || blocks < 1 || threads < 32 || per < 1 || repeats < 1 || !visits_per_s)
        return CC_E_INVALID;
    if (mode < 0 || mode > 2 || (mode == 1 && (hot < 1 || hot > n_cells)) ||
        (mode == 2 && (run < 1 || stride < 1 || (long long)run * stride > n_cells)) || n_cells > 0xFFFFFFFFll)
        return CC_E_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return CC_E_DEVICE;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return CC_E_DEVICE;
    atomics_kernel<<<blocks, threads>>>(d_cells, n_cells, mode, per, hot, run, stride);   // warm-up
    cudaEventRecord(e0);
    for (int r = 0; r < repeats; ++r) atomics_kernel<<<blocks, threads>>>(d_cells, n_cells, mode, per, hot, run, stride);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess || ms <= 0.f) return CC_E_DEVICE;
    *visits_per_s = (double)blocks * threads * per * repeats / (ms * 1e-3);
    return CC_OK;
}
