// Device helpers shared by the kernels: warp reductions with a fixed
// combination order (results are run-to-run deterministic), bounded waits
// on shared-memory ready bits, and status codes.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace lusp {

// Per-system status words (bit flags).
enum : int {
    ST_OK = 0,
    ST_SINGULAR = 1,       // a zero or non-finite pivot
    ST_PIVOT_WEAK = 2,     // |pivot| < pivot_tol * max |L(:,k)| before scaling
    ST_STAGNATED = 4,      // IR residual stopped decreasing
    ST_NOT_CONVERGED = 8,  // max_outer reached above rtol
    ST_NONFINITE = 16,     // NaN/Inf in a residual
    ST_WAIT_TIMEOUT = 32,  // a bounded wait gave up (never expected)
    ST_CAPACITY = 64,      // a work area was too small (never expected)
    ST_ESCALATED = 128,    // the result comes from an fp64 rung of the ladder
    ST_SHIFTED = 256,      // ... from the P-hard rung (factor of A + shift diag|A|)
    ST_LADDER_FULL = 512,  // the ladder had no free slot: P-fast result kept
    ST_FP16_OFF = 1024,    // fp16 inner products asked for, but the Ruiz-scaled
                           // values leave the fp16 normal range: fp32 used
};

// Spin bound for waits on shared-memory ready bits inside one CTA: about a
// second with the 64 ns back-off, far above any legitimate wait.
constexpr long long kSpinLimit = 1ll << 24;

// Wait until bit j of a shared-memory bitset is set.  Gives up after
// kSpinLimit polls, or at once when *abort is set (an earlier wait of this
// CTA timed out), so a missing producer costs one timeout, not one per
// waiter.  Returns false when it gave up; the caller records
// ST_WAIT_TIMEOUT and carries on without blocking.
__device__ __forceinline__ bool wait_ready(const unsigned* bits, int j, int* abort) {
    const volatile unsigned* w = bits + (j >> 5);
    const unsigned m = 1u << (j & 31);
    if (*w & m) return true;
    const volatile int* ab = abort;
    long long it = 0;
    while (!(*w & m)) {
        if (*ab) return false;
        if (++it > kSpinLimit) {
            atomicExch(abort, 1);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ void set_ready(unsigned* bits, int j) {
    atomicOr(bits + (j >> 5), 1u << (j & 31));
}

// Block-wide sum with a fixed order: warp butterflies, then warp 0 adds the
// per-warp partials in warp order.  scratch: >= 33 doubles of shared memory.
// All threads must call; all receive the result.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double s = lane < nw ? scratch[lane] : 0.0;
        s = warp_sum(s);
        if (lane == 0) scratch[32] = s;
    }
    __syncthreads();
    return scratch[32];
}

// Two block-wide sums in one reduction (same order as block_sum for each).
// Blocks of at most 16 warps; scratch: >= 34 doubles.
__device__ __forceinline__ void block_sum2(double& a, double& b, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    __syncthreads();
    if (lane == 0) {
        scratch[warp] = a;
        scratch[16 + warp] = b;
    }
    __syncthreads();
    if (warp == 0) {
        double s = lane < nw ? scratch[lane] : 0.0;
        double t = lane < nw ? scratch[16 + lane] : 0.0;
        s = warp_sum(s);
        t = warp_sum(t);
        if (lane == 0) {
            scratch[32] = s;
            scratch[33] = t;
        }
    }
    __syncthreads();
    a = scratch[32];
    b = scratch[33];
}

// Block-wide maximum / minimum (all threads call, all receive the result).
__device__ __forceinline__ double block_max(double v, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double s = lane < nw ? scratch[lane] : -INFINITY;
        s = warp_max(s);
        if (lane == 0) scratch[32] = s;
    }
    __syncthreads();
    return scratch[32];
}

__device__ __forceinline__ double block_min(double v, double* scratch) {
    return -block_max(-v, scratch);
}

template <typename T> struct ValTraits;
template <> struct ValTraits<double> {
    static __device__ __forceinline__ double load(const double* p) { return *p; }
    static __device__ __forceinline__ double to(double v) { return v; }
};
template <> struct ValTraits<float> {
    static __device__ __forceinline__ double load(const float* p) { return (double)*p; }
    static __device__ __forceinline__ float to(double v) { return (float)v; }
};

}  // namespace lusp
