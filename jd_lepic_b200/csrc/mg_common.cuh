// mg_common.cuh -- execution teams and fixed-order reductions shared by the multigrid
// kernels.  A team is either the whole cooperative grid (bounded software grid barrier) or
// CTA 0 alone (block barrier); every reduction has a fixed order, so results are identical
// in every CTA and reproducible run to run.
#pragma once
#include "lepic_internal.cuh"

#define MG_THREADS 256

// ---------------------------------------------------------------------------------------
// Teams: the whole grid (grid barrier) or CTA 0 alone (block barrier).
struct BigTeam {
    DevCounters *c;
    double *partials;
    __device__ long long rank() const { return blockIdx.x * (long long)blockDim.x + threadIdx.x; }
    __device__ long long size() const { return (long long)gridDim.x * blockDim.x; }
    __device__ bool sync() const { return grid_barrier(c, gridDim.x); }
};
struct SmallTeam {
    __device__ long long rank() const { return threadIdx.x; }
    __device__ long long size() const { return blockDim.x; }
    __device__ bool sync() const { __syncthreads(); return true; }
};

// fixed-order block sum; every thread gets the result
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double s[MG_THREADS];
    __shared__ double s_res;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int w = MG_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] = s[threadIdx.x] + s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) s_res = s[0];
    __syncthreads();
    double r = s_res;
    __syncthreads();
    return r;
}

__device__ __forceinline__ bool team_sum(const BigTeam &T, double v, double *out) {
    double b = block_sum(v);
    if (threadIdx.x == 0) T.partials[blockIdx.x] = b;
    if (!T.sync()) return false;
    __shared__ double s_tot;
    if (threadIdx.x < 32) {
        double a = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) a = a + ((volatile double *)T.partials)[i];
        for (int o = 16; o > 0; o >>= 1) a = a + __shfl_xor_sync(0xffffffffu, a, o);
        if (threadIdx.x == 0) s_tot = a;
    }
    __syncthreads();
    *out = s_tot;
    __syncthreads();
    return true;
}
__device__ __forceinline__ bool team_sum(const SmallTeam &, double v, double *out) {
    *out = block_sum(v);
    return true;
}

