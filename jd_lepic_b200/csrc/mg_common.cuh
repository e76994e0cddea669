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
    double *partials;          // 2 * gridDim.x doubles
    unsigned extra = 0;        // CTAs the barrier waits for beyond the launch (a test hook, 0 in use)
    mutable unsigned phase = 0;
    __device__ long long rank() const { return blockIdx.x * (long long)blockDim.x + threadIdx.x; }
    __device__ long long size() const { return (long long)gridDim.x * blockDim.x; }
    __device__ bool sync() const { return grid_barrier(c, gridDim.x + extra); }
};
struct SmallTeam {
    __device__ long long rank() const { return threadIdx.x; }
    __device__ long long size() const { return blockDim.x; }
    __device__ bool sync() const { __syncthreads(); return true; }
};

// Grid-stride walk over the (row, column) pairs of a rows x width index range without a
// division per element: the stride is split once into whole rows and a remainder, and the pair
// advances incrementally (flat index = row * width + column).
struct Walk2 {
    int j, k, dj, dk, width, rows;
    // 32-bit throughout: team sizes and node counts stay below 2^31 (checked at create)
    __device__ __forceinline__ Walk2(long long rank_, long long size_, int width_, int rows_)
        : width(width_), rows(rows_) {
        const unsigned rank = (unsigned)rank_, size = (unsigned)size_, w = (unsigned)width_;
        const unsigned tot = w * (unsigned)rows_;
        if (rank >= tot) { j = rows_; k = 0; dj = dk = 0; return; }
        j = (int)(rank / w);
        k = (int)(rank - (unsigned)j * w);
        const unsigned st = size < tot ? size : tot;
        dj = (int)(st / w);
        dk = (int)(st - (unsigned)dj * w);
    }
    __device__ __forceinline__ bool ok() const { return j < rows; }
    __device__ __forceinline__ void next() {
        k += dk;
        j += dj;
        if (k >= width) { k -= width; j++; }
    }
    __device__ __forceinline__ int flat() const { return j * width + k; }
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

// Consecutive sums alternate between two halves of `partials` (2 * gridDim.x doubles), so a CTA
// that runs ahead into the next sum never overwrites a partial another CTA is still reading.
__device__ __forceinline__ bool team_sum(const BigTeam &T, double v, double *out) {
    double b = block_sum(v);
    double *part = T.partials + (T.phase & 1) * gridDim.x;
    T.phase++;
    if (threadIdx.x == 0) part[blockIdx.x] = b;
    if (!T.sync()) return false;
    __shared__ double s_tot;
    if (threadIdx.x < 32) {
        double a = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) a = a + ((volatile double *)part)[i];
        for (int o = 16; o > 0; o >>= 1) a = a + __shfl_xor_sync(0xffffffffu, a, o);
        if (threadIdx.x == 0) s_tot = a;
    }
    __syncthreads();
    *out = s_tot;
    __syncthreads();
    return true;
}
// N sums behind one grid barrier.  Sum v of half h sits at partials + (2 v + h) * gridDim.x, so
// value 0 uses team_sum's layout and a CTA that runs ahead into any later sum (the other half)
// writes none of the slots still being read; `partials` holds 2 N * gridDim.x doubles.  Each
// sum is reduced in the same fixed order as team_sum's.
template <int N>
__device__ __forceinline__ bool team_sums(const BigTeam &T, const double (&v)[N], double (&out)[N]) {
    double b[N];
#pragma unroll
    for (int q = 0; q < N; q++) b[q] = block_sum(v[q]);
    const unsigned h = T.phase & 1;
    T.phase++;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < N; q++) T.partials[(2 * q + h) * gridDim.x + blockIdx.x] = b[q];
    }
    if (!T.sync()) return false;
    __shared__ double s_tot[N];
    if (threadIdx.x < 32) {
#pragma unroll
        for (int q = 0; q < N; q++) {
            const volatile double *part = T.partials + (2 * q + h) * gridDim.x;
            double a = 0.0;
            for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) a = a + part[i];
            for (int o = 16; o > 0; o >>= 1) a = a + __shfl_xor_sync(0xffffffffu, a, o);
            if (threadIdx.x == 0) s_tot[q] = a;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < N; q++) out[q] = s_tot[q];
    __syncthreads();
    return true;
}
__device__ __forceinline__ bool team_sum(const SmallTeam &, double v, double *out) {
    *out = block_sum(v);
    return true;
}

