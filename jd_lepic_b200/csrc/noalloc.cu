// noalloc.cu -- charge deposition that allocates no device memory.
//
// Some hosts cannot call cudaMalloc: an application whose whole device memory is reserved up
// front and handed out by its own allocator (or by another framework's caching allocator), or
// code on a path where the implicit device synchronisation of an allocation is not allowed.
// Such a caller owns its particle arrays, its node-factor grid and its output grid already;
// this entry point needs no other memory of its own.  The temporary integer accumulator lives
// in the file-scope device array below, of fixed size, which every GPU that loads the library
// holds until the process exits.
//
// The deposit is the same integer CIC as the fused push kernel (push.cu): per-particle weights
// are exact products of the fixed-point cell offsets, rounded to 2^-44, summed in uint64, and
// scaled once to np = kq * (k1 * acc * 2^-44); the result is bit-identical to the context path.
// A position outside the box (X >= nx << shift or Y >= ny << shift) is skipped, so no write
// can land outside the (nx+3)(ny+3) nodes of the accumulator.
// Compiled with -fmad=false like the other FP64 grid kernels.
#include <mutex>
#include "lepic_internal.cuh"

#define LEPIC_NOALLOC_MAX_NODES (1 << 20)  // (nx+3)*(ny+3) limit: 8 MiB of uint64

static __device__ __align__(256) unsigned long long g_noalloc_acc[LEPIC_NOALLOC_MAX_NODES];

// Host code must not use g_noalloc_acc directly (it names a host-side shadow, not device
// memory): its device address is looked up once per device and cached here, with the
// device's SM count for the launch shape.
static unsigned long long *g_noalloc_ptr[64];
static int g_noalloc_sms[64];
static std::mutex g_noalloc_mu;

__global__ void k_na_zero(unsigned long long *acc, long long nn) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn; t += (long long)gridDim.x * blockDim.x)
        acc[t] = 0ull;
}

__global__ void k_na_deposit(const uint32_t *X, const uint32_t *Y, const float *VX, long long n, int S, int nx,
                             int ny, unsigned long long *acc) {
    const uint32_t mask = (1u << S) - 1u;
    const uint64_t A = 1ull << S;
    const int sh = 2 * S - LEPIC_DEP_SHIFT;
    const int W = nx + 3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (VX && isnan(VX[i])) continue; // a hole left by a lost particle
        const uint32_t x = X[i], y = Y[i];
        const uint32_t cx = x >> S, cy = y >> S;
        if (cx >= (uint32_t)nx || cy >= (uint32_t)ny) continue; // outside the box: not deposited
        const uint64_t fx = x & mask, fy = y & mask, ax = A - fx, ay = A - fy;
        uint64_t w[4] = {ax * ay, fx * ay, fx * fy, ax * fy};
        for (int k = 0; k < 4; k++) {
            if (sh > 0) w[k] = (w[k] + (1ull << (sh - 1))) >> sh;
            else if (sh < 0) w[k] <<= -sh;
        }
        // cx <= nx-1 and cy <= ny-1, so the four nodes (cx+1..cx+2, cy+1..cy+2) are inside
        unsigned long long *q = acc + ((long long)cx + 1) + ((long long)cy + 1) * W;
        if (w[0]) atomicAdd(q, (unsigned long long)w[0]);
        if (w[1]) atomicAdd(q + 1, (unsigned long long)w[1]);
        if (w[2]) atomicAdd(q + W + 1, (unsigned long long)w[2]);
        if (w[3]) atomicAdd(q + W, (unsigned long long)w[3]);
    }
}

__global__ void k_na_finish(const unsigned long long *acc, const double *kq, double k1, long long nn, double *out) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn; t += (long long)gridDim.x * blockDim.x) {
        double w = (double)acc[t] * 5.684341886080802e-14; // 2^-44
        out[t] = kq[t] * (k1 * w);
    }
}

extern "C" int lepic_gpu_deposit_noalloc(const uint32_t *X, const uint32_t *Y, const float *VX, int64_t n,
                                         int32_t nx, int32_t ny, int32_t shift, double k1, const double *kq,
                                         double *np_out, void *stream) {
    if (n < 0 || nx < 1 || ny < 1 || shift < 1 || shift > 24 || !kq || !np_out || (n > 0 && (!X || !Y)))
        return LEPIC_EINVAL;
    if ((long long)nx << shift > (1ll << 32) || (long long)ny << shift > (1ll << 32)) return LEPIC_EINVAL;
    const long long nn = (long long)(nx + 3) * (ny + 3);
    if (nn > LEPIC_NOALLOC_MAX_NODES) return LEPIC_ECAPACITY; // larger than the static scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return LEPIC_ECUDA;
    unsigned long long *acc;
    int sms;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void *p = nullptr;
            int m = 0;
            if (cudaGetSymbolAddress(&p, g_noalloc_acc) != cudaSuccess || !p) return LEPIC_ECUDA;
            if (cudaDeviceGetAttribute(&m, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || m < 1)
                return LEPIC_ECUDA;
            g_noalloc_sms[dev] = m;
            g_noalloc_ptr[dev] = (unsigned long long *)p;
        }
        acc = g_noalloc_ptr[dev];
        sms = g_noalloc_sms[dev];
    }
    // an error left pending by earlier work of the caller is reported here and not cleared;
    // nothing is enqueued then
    if (cudaPeekAtLastError() != cudaSuccess) return LEPIC_ECUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = 4 * sms;
    k_na_zero<<<grid, 256, 0, st>>>(acc, nn); // the array keeps the previous call's sums
    if (n > 0) k_na_deposit<<<grid * 4, 256, 0, st>>>(X, Y, VX, n, shift, nx, ny, acc);
    k_na_finish<<<grid, 256, 0, st>>>(acc, kq, k1, nn, np_out);
    return cudaGetLastError() == cudaSuccess ? LEPIC_OK : LEPIC_ECUDA;
}
