// cnn.cu -- the learned warm start of the Poisson solve: a 4-level convolutional network
// (3x3 convolutions, channels 16/32/64/64) that maps (residual of the previous potential,
// previous potential) to a correction of the potential, trained online on the pairs the
// solver itself produces.  The solver (FP64 conjugate gradients with the FP32 V-cycle) then
// refines the corrected potential to the same residual as always, so it stays both the
// fallback and the arbiter of the answer.  No counterpart in the reference, whose solve starts from the
// previous step's potential (iterative_solver.f90:1-69, called at main.f90:829).
//
// Tensor-core path: every convolution (forward, and the input gradient as a forward
// convolution with rotated, transposed weights) is an implicit GEMM on the 5th-generation
// tensor cores: D[128 pixels][Cout] += A[128 pixels][16 channels] * B[16 channels][Cout] per
// tcgen05.mma (kind::f16, BF16 operands, FP32 accumulator in tensor memory), 9 taps x Cin/16
// instructions per output row.  A and B are staged in shared memory in the no-swizzle
// K-major canonical layout: a row of 130 input pixels (128 + halo) is stored as Cin/8 chunks
// of [pixel][8 channels], so the operand of tap (dy, dx) is the same rows shifted by dx
// pixels (16 bytes) -- the 9 taps read one staged copy, no im2col.  Rows rotate through a
// 4-slot ring so every input row is loaded once per strip while the tensor core works on
// the previous one.  The weight gradient runs on the CUDA cores (FP32 accumulation of BF16
// operands); it is only evaluated on the small training crops.
//
// Activations: NHWC BF16, channels padded to a multiple of 16.  Images are H x W with H and
// W multiples of 8 (three 2x2 poolings).
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <mutex>
#include <vector>
#include "cnn.cuh"

typedef __nv_bfloat16 bf16;

#define CONV_THREADS 128
#define CONV_PITCH 130
#define DW_THREADS 256

// ---------------------------------------------------------------------------------------
// network description (the same order as the parameter vector)
static const int L_CIN[CNN_LAYERS] = {2, 16, 16, 32, 32, 64, 64, 64, 64, 64, 32, 16};
static const int L_COUT[CNN_LAYERS] = {16, 16, 32, 32, 64, 64, 64, 64, 64, 32, 16, 1};
static inline int pad16(int c) { return (c + 15) / 16 * 16; }

// ---------------------------------------------------------------------------------------
// PTX helpers (tcgen05, mbarrier, proxy fences)
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor, no swizzle: start, leading-dimension byte offset (between
// the two 8-element K chunks of one instruction), stride byte offset (between 8-row groups)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait on an mbarrier phase; false after ~2^31 cycles (about a second)
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > (1ll << 31)) return false;
    }
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 columns of FP32: thread t of the warp gets lane (warp base + t), 16 columns
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

// ---------------------------------------------------------------------------------------
// BF16 packing helpers
__device__ __forceinline__ float2 bf2_to_f2(uint32_t u) {
    __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162 *>(&u);
    return __bfloat1622float2(h);
}
__device__ __forceinline__ uint32_t f2_to_bf2(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ uint32_t avg4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, float s) {
    const float2 fa = bf2_to_f2(a), fb = bf2_to_f2(b), fc = bf2_to_f2(c), fd = bf2_to_f2(d);
    return f2_to_bf2(((fa.x + fb.x) + (fc.x + fd.x)) * s, ((fa.y + fb.y) + (fc.y + fd.y)) * s);
}
__device__ __forceinline__ uint4 avg4v(uint4 a, uint4 b, uint4 c, uint4 d, float s) {
    return make_uint4(avg4(a.x, b.x, c.x, d.x, s), avg4(a.y, b.y, c.y, d.y, s), avg4(a.z, b.z, c.z, d.z, s),
                      avg4(a.w, b.w, c.w, d.w, s));
}
// keep the BF16 halves of v whose mask halves are > 0
__device__ __forceinline__ uint32_t mask_bf2(uint32_t v, uint32_t m) {
    const float2 f = bf2_to_f2(m);
    return v & ((f.x > 0.0f ? 0x0000FFFFu : 0u) | (f.y > 0.0f ? 0xFFFF0000u : 0u));
}

// ---------------------------------------------------------------------------------------
// convolution parameters
enum { IN_DIRECT = 0, IN_POOL = 1, IN_UP = 2, IN_X2 = 3 };  // IN_X2: 2 channels per pixel, zero-padded to CIN
enum { EPI_RELU = 0, EPI_OUTF = 1, EPI_GRAD = 2 };

struct ConvP {
    const bf16 *in;      // input tensor [N][inH][inW][CIN] ([N][H][W][2] for IN_X2)
    int in_mode, inH, inW;
    int N, H, W, R;      // output (and convolution input) size; rows per work unit
    const bf16 *w;       // packed weights [tap][CIN/8][COUT][8]
    const float *bias;   // [COUT] or null
    int epi;
    bf16 *out;           // EPI_RELU: relu(acc + b); EPI_GRAD: bf16(acc) masked by `mask`
    bf16 *out2;          // EPI_RELU: relu(acc + b) + skip; EPI_GRAD: bf16(acc) unmasked
    const bf16 *skip;    // [N][H][W][COUT]
    const bf16 *mask;    // [N][H][W][COUT]
    float *outf;         // EPI_OUTF: channel 0 of acc + b, [N][H][W]
    int *err;
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One input row (pixels x0-1 .. x0+128) into ring slot `slot` of the staging buffer.  Plain
// and upsampled inputs are copied with cp.async (zero-filled outside the image; the caller
// commits and waits); pooled and 2-channel inputs go through registers, all loads of a
// thread issued before its stores.
template <int CIN, int NT>
__device__ __forceinline__ void load_row(const ConvP &P, unsigned char *s_in, int n, int yy, int x0, int slot) {
    constexpr int NCH = CIN / 8;
    constexpr int ITEMS = (CONV_PITCH * NCH + NT - 1) / NT;
    const bool row_ok = yy >= 0 && yy < P.H;
    unsigned char *base = s_in + (size_t)slot * NCH * CONV_PITCH * 16;
    if (P.in_mode == IN_DIRECT || P.in_mode == IN_UP) {
        const int ys = P.in_mode == IN_UP ? (yy >> 1) : yy;
        for (int i = threadIdx.x; i < CONV_PITCH * NCH; i += NT) {
            const int p = i / NCH, c8 = i - p * NCH;
            const int xx = x0 - 1 + p;
            const bool ok = row_ok && xx >= 0 && xx < P.W;
            const int xs = P.in_mode == IN_UP ? (xx >> 1) : xx;
            const bf16 *src = ok ? P.in + (((size_t)n * P.inH + ys) * P.inW + xs) * CIN + 8 * c8 : P.in;
            cp_async16(smem_u32(base + ((size_t)c8 * CONV_PITCH + p) * 16), src, ok);
        }
        return;
    }
    constexpr int BATCH = 2;
#pragma unroll
    for (int b0 = 0; b0 < ITEMS; b0 += BATCH) {
        uint4 v[BATCH];
        int dst[BATCH];
#pragma unroll
        for (int k = 0; k < BATCH; k++) {
            const int i = threadIdx.x + (b0 + k) * NT;
            v[k] = make_uint4(0u, 0u, 0u, 0u);
            dst[k] = -1;
            if (b0 + k < ITEMS && i < CONV_PITCH * NCH) {
                const int p = i / NCH, c8 = i - p * NCH;
                const int xx = x0 - 1 + p;
                dst[k] = (c8 * CONV_PITCH + p) * 16;
                if (row_ok && xx >= 0 && xx < P.W) {
                    if (P.in_mode == IN_X2) {
                        if (c8 == 0)
                            v[k].x = __ldg(reinterpret_cast<const uint32_t *>(P.in) + ((size_t)n * P.inH + yy) * P.inW + xx);
                    } else {
                        const size_t r0 = ((size_t)n * P.inH + 2 * yy) * P.inW + 2 * xx;
                        const uint4 *q0 = reinterpret_cast<const uint4 *>(P.in + r0 * CIN) + c8;
                        const uint4 *q1 = reinterpret_cast<const uint4 *>(P.in + (r0 + P.inW) * CIN) + c8;
                        v[k] = avg4v(__ldg(q0), __ldg(q0 + NCH), __ldg(q1), __ldg(q1 + NCH), 0.25f);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < BATCH; k++)
            if (dst[k] >= 0) *reinterpret_cast<uint4 *>(base + dst[k]) = v[k];
    }
}

template <int COUT>
__device__ __forceinline__ void conv_epilogue(const ConvP &P, const float *s_bias, uint32_t tmem, int n, int y,
                                              int x0) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x = x0 + warp * 32 + lane;
    const bool ok = x < P.W;
    const size_t pix = ((size_t)n * P.H + y) * P.W + (ok ? x : 0);
    const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
    if (P.epi == EPI_OUTF) {
        float v[16];
        tmem_ld16(tbase, v);
        if (ok) P.outf[pix] = v[0] + s_bias[0];
        return;
    }
    // the skip (or mask) values of this pixel, fetched before the accumulator reads
    const bf16 *side = P.epi == EPI_RELU ? P.skip : P.mask;
    uint4 sd[COUT / 8];
#pragma unroll
    for (int k = 0; k < COUT / 8; k++)
        sd[k] = (side && ok) ? __ldg(reinterpret_cast<const uint4 *>(side + pix * COUT) + k) : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 16) {
        float v[16];
        tmem_ld16(tbase + c0, v);
        if (!ok) continue;
        const uint32_t sv[8] = {sd[c0 / 8].x, sd[c0 / 8].y, sd[c0 / 8].z, sd[c0 / 8].w,
                                sd[c0 / 8 + 1].x, sd[c0 / 8 + 1].y, sd[c0 / 8 + 1].z, sd[c0 / 8 + 1].w};
        uint32_t o[8];
        if (P.epi == EPI_RELU) {
#pragma unroll
            for (int k = 0; k < 16; k += 4) {
                const float4 b4 = *reinterpret_cast<const float4 *>(s_bias + c0 + k);
                v[k] = fmaxf(v[k] + b4.x, 0.0f);
                v[k + 1] = fmaxf(v[k + 1] + b4.y, 0.0f);
                v[k + 2] = fmaxf(v[k + 2] + b4.z, 0.0f);
                v[k + 3] = fmaxf(v[k + 3] + b4.w, 0.0f);
            }
#pragma unroll
            for (int k = 0; k < 8; k++) o[k] = f2_to_bf2(v[2 * k], v[2 * k + 1]);
            if (P.out) {
                uint4 *dst = reinterpret_cast<uint4 *>(P.out + pix * COUT + c0);
                dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
                dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
            }
            if (P.skip) {
                uint32_t q[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const float2 f = bf2_to_f2(sv[k]);
                    q[k] = f2_to_bf2(v[2 * k] + f.x, v[2 * k + 1] + f.y);
                }
                uint4 *dst = reinterpret_cast<uint4 *>(P.out2 + pix * COUT + c0);
                dst[0] = make_uint4(q[0], q[1], q[2], q[3]);
                dst[1] = make_uint4(q[4], q[5], q[6], q[7]);
            }
        } else { // EPI_GRAD
#pragma unroll
            for (int k = 0; k < 8; k++) o[k] = f2_to_bf2(v[2 * k], v[2 * k + 1]);
            if (P.out2) {
                uint4 *dst = reinterpret_cast<uint4 *>(P.out2 + pix * COUT + c0);
                dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
                dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
            }
            if (P.out) {
                if (P.mask) {
#pragma unroll
                    for (int k = 0; k < 8; k++) o[k] = mask_bf2(o[k], sv[k]);
                }
                uint4 *dst = reinterpret_cast<uint4 *>(P.out + pix * COUT + c0);
                dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
                dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
            }
        }
    }
}

// Persistent 3x3 convolution: a work unit is (image, 128-pixel strip, R rows); per output row
// one elected thread issues 9 * CIN/16 tcgen05.mma into tensor memory while all threads stage
// the next input row, then every thread drains its pixel's accumulator row (one TMEM lane).
template <int CIN, int COUT>
__global__ void __launch_bounds__(CONV_THREADS, (CIN == 16 && COUT == 16) ? 10 : 1) k_conv(ConvP P) {
    constexpr int NCH = CIN / 8;
    constexpr int W_BYTES = 9 * CIN * COUT * 2;
    constexpr uint32_t NCOLS = COUT < 32 ? 32 : COUT;
    constexpr uint32_t IDESC = idesc_bf16(128, COUT);
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *s_w = smem;
    unsigned char *s_in = smem + W_BYTES;
    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    __shared__ __align__(16) float s_bias[COUT];
    const int tid = threadIdx.x;
    if (tid < COUT) s_bias[tid] = P.bias ? P.bias[tid] : 0.0f;
    if (tid < 32) tmem_alloc(smem_u32(&s_tmem), NCOLS);
    if (tid == 0) {
        mbar_init(smem_u32(&s_mbar), 1);
        s_fail = 0;
    }
    {
        const uint4 *wg = reinterpret_cast<const uint4 *>(P.w);
        uint4 *ws = reinterpret_cast<uint4 *>(s_w);
        for (int i = tid; i < W_BYTES / 16; i += CONV_THREADS) ws[i] = __ldg(wg + i);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t a_base = smem_u32(s_in), b_base = smem_u32(s_w), mbar = smem_u32(&s_mbar);
    uint32_t phase = 0;
    const int nstrip = (P.W + 127) / 128, nrb = (P.H + P.R - 1) / P.R;
    const long long nunits = (long long)P.N * nstrip * nrb;
    for (long long u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int n = (int)(u / ((long long)nstrip * nrb));
        const int rem = (int)(u - (long long)n * nstrip * nrb);
        const int rb = rem / nstrip, xs = rem - rb * nstrip;
        const int x0 = xs * 128, y0 = rb * P.R, y1 = min(y0 + P.R, P.H);
        // slot of input row yy: (yy + 1) & 3
        load_row<CIN, CONV_THREADS>(P, s_in, n, y0 - 1, x0, (y0) & 3);
        load_row<CIN, CONV_THREADS>(P, s_in, n, y0, x0, (y0 + 1) & 3);
        load_row<CIN, CONV_THREADS>(P, s_in, n, y0 + 1, x0, (y0 + 2) & 3);
        cp_async_commit();
        cp_async_wait_all();
        fence_async_smem();
        __syncthreads();
        for (int y = y0; y < y1; y++) {
            if (tid == 0) {
                tc_fence_after();
#pragma unroll
                for (int tap = 0; tap < 9; tap++) {
                    const int dy = tap / 3, dx = tap - 3 * (tap / 3);
                    const int slot = (y + dy) & 3;
#pragma unroll
                    for (int q = 0; q < CIN / 16; q++) {
                        const uint32_t a = a_base + (uint32_t)(((slot * NCH + 2 * q) * CONV_PITCH + dx) * 16);
                        const uint32_t b = b_base + (uint32_t)(((tap * NCH + 2 * q) * COUT) * 16);
                        umma_bf16(tmem, sdesc(a, CONV_PITCH * 16, 128), sdesc(b, COUT * 16, 128), IDESC,
                                  (tap | q) ? 1u : 0u);
                    }
                }
                umma_commit(mbar);
            }
            if (y + 1 < y1) load_row<CIN, CONV_THREADS>(P, s_in, n, y + 2, x0, (y + 3) & 3);
            cp_async_commit();
            const bool done = mbar_wait(mbar, phase);
            phase ^= 1u;
            tc_fence_after();
            if (done) conv_epilogue<COUT>(P, s_bias, tmem, n, y, x0);
            else s_fail = 1;
            cp_async_wait_all();
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            if (s_fail) break;
        }
        if (s_fail) break;
    }
    __syncthreads();
    if (s_fail && tid == 0) atomicOr(P.err, 1);
    if (tid < 32) tmem_dealloc(tmem, NCOLS);
}

// ---------------------------------------------------------------------------------------
// weight gradient on the CUDA cores: dW[n][c][tap] = sum_p G[p][n] * X[p + tap][c] per work
// unit (image, strip, R rows) into per-unit partials, reduced in unit order afterwards
struct DwP {
    ConvP X;              // the convolution input as the forward pass read it (in, in_mode, sizes)
    const bf16 *G;        // output gradient [N][H][W][COUT]
    float *part;          // [units][COUT*CIN*9]
    float *partb;         // [units][COUT]
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(DW_THREADS) k_conv_dw(DwP D) {
    constexpr int NCH = CIN / 8, NB = COUT / 4, CB = CIN / 4, NBLK = 9 * NB * CB;
    constexpr int SLOT_BYTES = NCH * CONV_PITCH * 16;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *s_in = smem;
    bf16 *s_g = reinterpret_cast<bf16 *>(smem + 4 * SLOT_BYTES);
    const ConvP &P = D.X;
    const int tid = threadIdx.x;
    const int nstrip = (P.W + 127) / 128, nrb = (P.H + P.R - 1) / P.R;
    const int u = blockIdx.x;
    const int n = u / (nstrip * nrb);
    const int rem = u - n * nstrip * nrb;
    const int rb = rem / nstrip, xs = rem - rb * nstrip;
    const int x0 = xs * 128, y0 = rb * P.R, y1 = min(y0 + P.R, P.H);
    const int widx = blockIdx.y * DW_THREADS + tid;
    const bool active = widx < NBLK;
    const int tap = active ? widx / (NB * CB) : 0;
    const int r2 = active ? widx - tap * (NB * CB) : 0;
    const int nb = r2 / CB, cb = r2 - nb * CB;
    const int dy = tap / 3, dx = tap - 3 * dy;
    const bool bias_thr = blockIdx.y == 0 && tid < COUT;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
    float db = 0.0f;
    load_row<CIN, DW_THREADS>(P, s_in, n, y0 - 1, x0, y0 & 3);
    load_row<CIN, DW_THREADS>(P, s_in, n, y0, x0, (y0 + 1) & 3);
    for (int y = y0; y < y1; y++) {
        load_row<CIN, DW_THREADS>(P, s_in, n, y + 1, x0, (y + 2) & 3);
        cp_async_commit();
        for (int i = tid; i < 128 * (COUT / 8); i += DW_THREADS) {
            const int p = i / (COUT / 8), c8 = i - p * (COUT / 8);
            const int xx = x0 + p;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (xx < P.W) v = __ldg(reinterpret_cast<const uint4 *>(D.G + (((size_t)n * P.H + y) * P.W + xx) * COUT) + c8);
            reinterpret_cast<uint4 *>(s_g)[i] = v;
        }
        cp_async_wait_all();
        __syncthreads();
        if (active) {
            const int slot = (y + dy) & 3;
            const unsigned char *xb = s_in + ((size_t)(slot * NCH + (cb >> 1)) * CONV_PITCH + dx) * 16 + (cb & 1) * 8;
            for (int m = 0; m < 128; m++) {
                const uint2 gq = *reinterpret_cast<const uint2 *>(s_g + m * COUT + nb * 4);
                const uint2 xq = *reinterpret_cast<const uint2 *>(xb + m * 16);
                const float2 g01 = bf2_to_f2(gq.x), g23 = bf2_to_f2(gq.y);
                const float2 x01 = bf2_to_f2(xq.x), x23 = bf2_to_f2(xq.y);
                const float g[4] = {g01.x, g01.y, g23.x, g23.y}, xv[4] = {x01.x, x01.y, x23.x, x23.y};
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) acc[i][j] = fmaf(g[i], xv[j], acc[i][j]);
            }
        }
        if (bias_thr)
            for (int m = 0; m < 128; m++) db += __bfloat162float(s_g[m * COUT + tid]);
        __syncthreads();
    }
    if (active) {
        float *dst = D.part + (size_t)u * (COUT * CIN * 9);
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) dst[((nb * 4 + i) * CIN + cb * 4 + j) * 9 + tap] = acc[i][j];
    }
    if (bias_thr) D.partb[(size_t)u * COUT + tid] = db;
}

// sum of the per-unit partials into the parameter-gradient vector: one warp per parameter,
// lane l adds units l, l+32, ... and a fixed shuffle tree combines the lanes (deterministic)
__global__ void k_dw_reduce(const float *part, const float *partb, int units, int cinp, int coutp, int cin, int cout,
                            float *gw, float *gb) {
    const int nw = cout * cin * 9;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int k = blockIdx.x * wpb + (threadIdx.x >> 5); k < nw + cout; k += gridDim.x * wpb) {
        float s = 0.0f;
        if (k < nw) {
            const int n = k / (cin * 9), r = k - n * cin * 9, c = r / 9, tap = r - 9 * c;
            const size_t src = ((size_t)n * cinp + c) * 9 + tap;
            for (int u = lane; u < units; u += 32) s += part[(size_t)u * coutp * cinp * 9 + src];
        } else {
            const int n = k - nw;
            for (int u = lane; u < units; u += 32) s += partb[(size_t)u * coutp + n];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            if (k < nw) gw[k] = s;
            else gb[k - nw] = s;
        }
    }
}

// ---------------------------------------------------------------------------------------
// elementwise kernels of the backward pass

// gd = bf16(2x2 sum of gu) (adjoint of nearest upsampling); gdm = gd * [mask > 0]
__global__ void k_pool_sum(const bf16 *gu, int N, int H, int W, int C, bf16 *gd, bf16 *gdm, const bf16 *mask) {
    const long long tot = (long long)N * H * W * (C / 8);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(t % (C / 8));
        const long long pix = t / (C / 8);
        const int x = (int)(pix % W), y = (int)((pix / W) % H), n = (int)(pix / ((long long)W * H));
        const size_t r0 = ((size_t)n * (2 * H) + 2 * y) * (2 * W) + 2 * x;
        const uint4 *q0 = reinterpret_cast<const uint4 *>(gu + r0 * C) + c8;
        const uint4 *q1 = reinterpret_cast<const uint4 *>(gu + (r0 + 2 * W) * C) + c8;
        uint4 v = avg4v(q0[0], q0[C / 8], q1[0], q1[C / 8], 1.0f);
        if (gd) reinterpret_cast<uint4 *>(gd)[t] = v;
        if (gdm) {
            const uint4 m = reinterpret_cast<const uint4 *>(mask)[t];
            reinterpret_cast<uint4 *>(gdm)[t] =
                make_uint4(mask_bf2(v.x, m.x), mask_bf2(v.y, m.y), mask_bf2(v.z, m.z), mask_bf2(v.w, m.w));
        }
    }
}

// out = bf16(gskip + 0.25 up(gp)) * [e > 0]  (skip gradient plus the adjoint of 2x2 averaging)
__global__ void k_merge(const bf16 *gskip, const bf16 *gp, const bf16 *e, int N, int H, int W, int C, bf16 *out) {
    const long long tot = (long long)N * H * W * (C / 8);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(t % (C / 8));
        const long long pix = t / (C / 8);
        const int x = (int)(pix % W), y = (int)((pix / W) % H), n = (int)(pix / ((long long)W * H));
        const uint4 a = reinterpret_cast<const uint4 *>(gskip)[t];
        const uint4 b = reinterpret_cast<const uint4 *>(gp + ((((size_t)n * (H / 2) + y / 2) * (W / 2) + x / 2) * C))[c8];
        const uint4 m = reinterpret_cast<const uint4 *>(e)[t];
        const uint32_t av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w}, mv[4] = {m.x, m.y, m.z, m.w};
        uint32_t o[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float2 fa = bf2_to_f2(av[k]), fb = bf2_to_f2(bv[k]);
            o[k] = mask_bf2(f2_to_bf2(fa.x + 0.25f * fb.x, fa.y + 0.25f * fb.y), mv[k]);
        }
        reinterpret_cast<uint4 *>(out)[t] = make_uint4(o[0], o[1], o[2], o[3]);
    }
}

// energy-norm loss: e = (pred - t) m; G[p][0] = bf16(dL/dpred), other channels 0; per-block
// partial sums of the loss
__global__ void k_loss(const float *pred, const float *t, const uint8_t *m, int N, int H, int W, bf16 *G,
                       double *partial) {
    __shared__ double red[256];
    const long long tot = (long long)N * H * W;
    const float inv = 1.0f / (float)tot;
    double acc = 0.0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < tot; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % W), y = (int)((p / W) % H);
        auto err = [&](long long q) { return (pred[q] - t[q]) * (float)m[q]; };
        const float ep = err(p);
        float g = 0.0f;
        if (x > 0) g += ep - err(p - 1);
        if (x + 1 < W) { const float d = ep - err(p + 1); g += d; acc += (double)d * d; }
        if (y > 0) g += ep - err(p - W);
        if (y + 1 < H) { const float d = ep - err(p + W); g += d; acc += (double)d * d; }
        g *= 2.0f * inv * (float)m[p];
        uint4 *dst = reinterpret_cast<uint4 *>(G + p * 16);
        dst[0] = make_uint4(f2_to_bf2(g, 0.0f), 0u, 0u, 0u);
        dst[1] = make_uint4(0u, 0u, 0u, 0u);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0] * (double)inv;
}

// sum of n partials by one block of 256 threads in a fixed order (deterministic)
__device__ __forceinline__ double block_sum256(const double *partial, int n) {
    __shared__ double red[256];
    double s = 0.0;
    for (int k = threadIdx.x; k < n; k += 256) s += partial[k];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    return red[0];
}

__global__ void __launch_bounds__(256) k_sum_partials(const double *partial, int n, double *out) {
    const double s = block_sum256(partial, n);
    if (threadIdx.x == 0) *out = s;
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters
__global__ void k_adam(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float gk = g[k];
        const float mk = b1 * m[k] + (1.0f - b1) * gk;
        const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    }
}

// packed BF16 weights of one layer: forward [tap][cinp/8][coutp][8] from W[cout][cin][9], and
// the input-gradient form (a forward convolution with cin' = coutp, cout' = cinp, rotated taps)
struct PackLayer {
    int ow, ob, cin, cout, cinp, coutp;
    bf16 *fwd, *bwd;
    float *bias;
};
struct PackAll { PackLayer L[CNN_LAYERS]; };

__global__ void k_pack(const float *prm, PackAll A) {
    const PackLayer &L = A.L[blockIdx.y];
    const int tot = 9 * L.cinp * L.coutp;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += gridDim.x * blockDim.x) {
        // forward: k = ((tap * cinp/8 + c8) * coutp + n) * 8 + j
        {
            const int j = k & 7, r = k >> 3;
            const int n = r % L.coutp, r2 = r / L.coutp;
            const int c8 = r2 % (L.cinp / 8), tap = r2 / (L.cinp / 8);
            const int c = c8 * 8 + j;
            float w = 0.0f;
            if (n < L.cout && c < L.cin) w = prm[L.ow + (n * L.cin + c) * 9 + tap];
            L.fwd[k] = __float2bfloat16_rn(w);
        }
        // input gradient: k = ((tap' * coutp/8 + c8') * cinp + n') * 8 + j, W'[n'][c'][tap'] = W[c'][n'][8 - tap']
        {
            const int j = k & 7, r = k >> 3;
            const int np_ = r % L.cinp, r2 = r / L.cinp;
            const int c8 = r2 % (L.coutp / 8), tapp = r2 / (L.coutp / 8);
            const int co = c8 * 8 + j;
            float w = 0.0f;
            if (co < L.cout && np_ < L.cin) w = prm[L.ow + (co * L.cin + np_) * 9 + (8 - tapp)];
            L.bwd[k] = __float2bfloat16_rn(w);
        }
    }
    if (blockIdx.x == 0)
        for (int n = threadIdx.x; n < L.coutp; n += blockDim.x) L.bias[n] = n < L.cout ? prm[L.ob + n] : 0.0f;
}

// crops of the full-size training pair: image b = rows oy[b].., columns ox[b]..
struct CropP { int oy[CNN_MAX_BATCH], ox[CNN_MAX_BATCH]; };
__global__ void k_crop(const bf16 *x, const float *t, const uint8_t *m, int Hf, int Wf, int S, int B, CropP C,
                       bf16 *xc, float *tc, uint8_t *mc) {
    const long long tot = (long long)B * S * S;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < tot; p += (long long)gridDim.x * blockDim.x) {
        const int xx = (int)(p % S), yy = (int)((p / S) % S), b = (int)(p / ((long long)S * S));
        const size_t src = (size_t)(C.oy[b] + yy) * Wf + (C.ox[b] + xx);
        reinterpret_cast<uint32_t *>(xc)[p] = reinterpret_cast<const uint32_t *>(x)[src];
        tc[p] = t[src];
        mc[p] = m[src];
    }
}

// ---------------------------------------------------------------------------------------
// host side
#define NCUDA(call)                                                                     \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess) {                                                        \
            net->last_err = std::string(#call) + ": " + cudaGetErrorString(_e);         \
            return LEPIC_ECUDA;                                                         \
        }                                                                               \
    } while (0)

struct Acts {   // activations of one forward pass (N images of H x W)
    int N = 0, H = 0, W = 0;
    bool train = false;
    bf16 *x = nullptr;                                     // [N][H][W][2]
    bf16 *e0a, *e0, *e1a, *e1, *e2a, *e2, *e3a, *e3;       // encoder
    bf16 *d2a, *d2, *d1a, *d1, *d0a, *d0;                  // decoder
    float *out = nullptr;                                  // [N][H][W]
    // backward
    bf16 *G, *gd0, *gd0a, *gu0, *gd1, *gd1a, *gu1, *gd2, *gd2a, *gu2, *ge3, *ge3a, *gp3, *ge2, *ge2a, *gp2,
        *ge1, *ge1a, *gp1, *ge0, *ge0a;
    float *t = nullptr;
    uint8_t *m = nullptr;
    std::vector<void *> owned;
};

struct CnnNet {
    int dev = 0, num_sms = 0;
    cudaStream_t stream = nullptr;
    int nparams = 0;
    int ow[CNN_LAYERS], ob[CNN_LAYERS];
    float *prm = nullptr, *grad = nullptr, *am = nullptr, *av = nullptr;
    int adam_t = 0;
    bf16 *wf[CNN_LAYERS] = {nullptr}, *wb[CNN_LAYERS] = {nullptr};
    float *bias[CNN_LAYERS] = {nullptr};
    float *part = nullptr, *partb = nullptr;
    size_t part_cap = 0, partb_cap = 0;
    double *lpart = nullptr, *dsum = nullptr;
    int *derr = nullptr;
    Acts full, crop;
    std::string last_err;
    float lr = 1e-3f;
    unsigned long long rng = 0x9E3779B97F4A7C15ull;
};

static unsigned long long splitmix(unsigned long long &s) {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static int grid_for(long long work, int threads, int num_sms) {
    long long g = (work + threads - 1) / threads;
    return (int)std::max(1ll, std::min(g, (long long)num_sms * 8));
}

// resident CTAs per SM for a kernel of `smem` dynamic bytes and `threads` threads, bounded by
// the shared memory of an SM and, for the convolution, by its 512 tensor-memory columns
static int ctas_per_sm(CnnNet *net, size_t smem, int threads, int tmem_cols) {
    int smem_sm = 0;
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, net->dev);
    int k = (int)((size_t)smem_sm / (smem + 1024 + 256));     // + per-CTA reserved and static
    k = std::min(k, 2048 / threads);
    if (tmem_cols > 0) k = std::min(k, 512 / tmem_cols);
    return std::max(1, k);
}

template <int CIN, int COUT>
static int launch_conv(CnnNet *net, ConvP &P) {
    const size_t smem = (size_t)9 * CIN * COUT * 2 + (size_t)4 * (CIN / 8) * CONV_PITCH * 16;
    constexpr int NCOLS = COUT < 32 ? 32 : COUT;
    static int per_sm_cache[64] = {0};
    static std::mutex mu;
    int per_sm;
    {
        std::lock_guard<std::mutex> lk(mu);
        int &c = per_sm_cache[net->dev & 63];
        if (!c) {
            NCUDA(cudaFuncSetAttribute(k_conv<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            NCUDA(cudaFuncSetAttribute(k_conv<CIN, COUT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
            c = ctas_per_sm(net, smem, CONV_THREADS, NCOLS);
        }
        per_sm = c;
    }
    // rows per work unit: about one unit per resident CTA (one prologue each, no tail)
    const int nstrip = (P.W + 127) / 128;
    const long long slots = (long long)net->num_sms * per_sm;
    const long long strips = (long long)P.N * nstrip;
    P.R = (int)std::max(4ll, std::min((long long)P.H, (strips * P.H + slots - 1) / slots));
    const int nrb = (P.H + P.R - 1) / P.R;
    const long long units = strips * nrb;
    const int grid = (int)std::min(units, slots);
    P.err = net->derr;
    k_conv<CIN, COUT><<<grid, CONV_THREADS, smem, net->stream>>>(P);
    NCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int conv_dispatch(CnnNet *net, int cin, int cout, ConvP &P) {
#define CASE(a, b) if (cin == a && cout == b) return launch_conv<a, b>(net, P)
    CASE(16, 16); CASE(16, 32); CASE(32, 32); CASE(32, 64); CASE(64, 64); CASE(64, 32); CASE(32, 16);
#undef CASE
    net->last_err = "no convolution kernel for this channel pair";
    return LEPIC_ENOKERNEL;
}

template <int CIN, int COUT>
static int launch_dw(CnnNet *net, DwP &D, int units) {
    const size_t smem = (size_t)4 * (CIN / 8) * CONV_PITCH * 16 + (size_t)128 * COUT * 2;
    static bool set[64] = {false};
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!set[net->dev & 63]) {
            NCUDA(cudaFuncSetAttribute(k_conv_dw<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            NCUDA(cudaFuncSetAttribute(k_conv_dw<CIN, COUT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
            set[net->dev & 63] = true;
        }
    }
    constexpr int NBLK = 9 * (COUT / 4) * (CIN / 4);
    dim3 grid(units, (NBLK + DW_THREADS - 1) / DW_THREADS);
    k_conv_dw<CIN, COUT><<<grid, DW_THREADS, smem, net->stream>>>(D);
    NCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int dw_dispatch(CnnNet *net, int cin, int cout, DwP &D, int units) {
#define CASE(a, b) if (cin == a && cout == b) return launch_dw<a, b>(net, D, units)
    CASE(16, 16); CASE(16, 32); CASE(32, 32); CASE(32, 64); CASE(64, 64); CASE(64, 32); CASE(32, 16);
#undef CASE
    net->last_err = "no weight-gradient kernel for this channel pair";
    return LEPIC_ENOKERNEL;
}

static int conv_rows(int H) { return H >= 1024 ? 16 : H >= 256 ? 8 : 4; }

static ConvP conv_params(const bf16 *in, int mode, int N, int H, int W) {
    ConvP P;
    memset(&P, 0, sizeof(P));
    P.in = in;
    P.in_mode = mode;
    P.N = N; P.H = H; P.W = W;
    P.inH = mode == IN_POOL ? 2 * H : mode == IN_UP ? H / 2 : H;
    P.inW = mode == IN_POOL ? 2 * W : mode == IN_UP ? W / 2 : W;
    P.R = conv_rows(H);
    return P;
}

// forward conv of layer l with ReLU epilogue (act -> out; act + skip -> out2)
static int fwd_relu(CnnNet *net, int l, const bf16 *in, int mode, int N, int H, int W, bf16 *act, const bf16 *skip,
                    bf16 *sum) {
    ConvP P = conv_params(in, mode, N, H, W);
    P.w = net->wf[l];
    P.bias = net->bias[l];
    P.epi = EPI_RELU;
    P.out = act;
    P.skip = skip;
    P.out2 = sum;
    return conv_dispatch(net, pad16(L_CIN[l]), pad16(L_COUT[l]), P);
}

// input-gradient conv of layer l: out = bf16(convT(g)) masked by `mask`, out2 = unmasked
static int bwd_data(CnnNet *net, int l, const bf16 *g, int N, int H, int W, bf16 *out, const bf16 *mask, bf16 *out2) {
    ConvP P = conv_params(g, IN_DIRECT, N, H, W);
    P.w = net->wb[l];
    P.epi = EPI_GRAD;
    P.out = out;
    P.mask = mask;
    P.out2 = out2;
    return conv_dispatch(net, pad16(L_COUT[l]), pad16(L_CIN[l]), P);
}

static int bwd_weights(CnnNet *net, int l, const bf16 *in, int mode, const bf16 *g, int N, int H, int W) {
    DwP D;
    memset(&D, 0, sizeof(D));
    D.X = conv_params(in, mode, N, H, W);
    D.G = g;
    const int cinp = pad16(L_CIN[l]), coutp = pad16(L_COUT[l]);
    const int nstrip = (W + 127) / 128, nrb = (H + D.X.R - 1) / D.X.R;
    const int units = N * nstrip * nrb;
    const size_t need = (size_t)units * cinp * coutp * 9, needb = (size_t)units * coutp;
    if (need > net->part_cap || needb > net->partb_cap) {
        net->last_err = "weight-gradient scratch too small";
        return LEPIC_ECAPACITY;
    }
    D.part = net->part;
    D.partb = net->partb;
    int r = dw_dispatch(net, cinp, coutp, D, units);
    if (r) return r;
    const int nw = L_COUT[l] * L_CIN[l] * 9 + L_COUT[l];
    k_dw_reduce<<<grid_for((long long)nw * 32, 256, net->num_sms), 256, 0, net->stream>>>(
        net->part, net->partb, units, cinp, coutp, L_CIN[l], L_COUT[l], net->grad + net->ow[l], net->grad + net->ob[l]);
    NCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int acts_alloc(CnnNet *net, Acts &A, int N, int H, int W, bool train) {
    A.N = N; A.H = H; A.W = W; A.train = train;
    const size_t p0 = (size_t)N * H * W, p1 = p0 / 4, p2 = p0 / 16, p3 = p0 / 64;
    auto bf = [&](size_t n, bf16 **dst) -> int {
        void *q = nullptr;
        NCUDA(cudaMalloc(&q, n * sizeof(bf16)));
        A.owned.push_back(q);
        *dst = (bf16 *)q;
        return LEPIC_OK;
    };
    int r = 0;
    r |= bf(p0 * 2, &A.x);
    r |= bf(p0 * 16, &A.e0a); r |= bf(p0 * 16, &A.e0);
    r |= bf(p1 * 32, &A.e1a); r |= bf(p1 * 32, &A.e1);
    r |= bf(p2 * 64, &A.e2a); r |= bf(p2 * 64, &A.e2);
    r |= bf(p3 * 64, &A.e3a); r |= bf(p3 * 64, &A.e3);
    r |= bf(p2 * 64, &A.d2); r |= bf(p1 * 32, &A.d1); r |= bf(p0 * 16, &A.d0);
    if (train) {
        r |= bf(p2 * 64, &A.d2a); r |= bf(p1 * 32, &A.d1a); r |= bf(p0 * 16, &A.d0a);
        r |= bf(p0 * 16, &A.G); r |= bf(p0 * 16, &A.gd0); r |= bf(p0 * 16, &A.gd0a); r |= bf(p0 * 32, &A.gu0);
        r |= bf(p1 * 32, &A.gd1); r |= bf(p1 * 32, &A.gd1a); r |= bf(p1 * 64, &A.gu1);
        r |= bf(p2 * 64, &A.gd2); r |= bf(p2 * 64, &A.gd2a); r |= bf(p2 * 64, &A.gu2);
        r |= bf(p3 * 64, &A.ge3); r |= bf(p3 * 64, &A.ge3a); r |= bf(p3 * 64, &A.gp3);
        r |= bf(p2 * 64, &A.ge2); r |= bf(p2 * 64, &A.ge2a); r |= bf(p2 * 32, &A.gp2);
        r |= bf(p1 * 32, &A.ge1); r |= bf(p1 * 32, &A.ge1a); r |= bf(p1 * 16, &A.gp1);
        r |= bf(p0 * 16, &A.ge0); r |= bf(p0 * 16, &A.ge0a);
        void *q = nullptr;
        NCUDA(cudaMalloc(&q, p0 * sizeof(float))); A.owned.push_back(q); A.t = (float *)q;
        NCUDA(cudaMalloc(&q, p0)); A.owned.push_back(q); A.m = (uint8_t *)q;
    } else {
        A.d2a = A.d1a = A.d0a = nullptr;
    }
    void *q = nullptr;
    NCUDA(cudaMalloc(&q, p0 * sizeof(float)));
    A.owned.push_back(q);
    A.out = (float *)q;
    if (r) return LEPIC_ECUDA;
    NCUDA(cudaMemsetAsync(A.x, 0, p0 * 2 * sizeof(bf16), net->stream));
    return LEPIC_OK;
}

static void acts_free(Acts &A) {
    for (void *q : A.owned) cudaFree(q);
    A.owned.clear();
    A.N = A.H = A.W = 0;
}

// forward pass over A.x; the decoder's pre-skip activations are stored only when training
static int net_forward(CnnNet *net, Acts &A) {
    const int N = A.N, H = A.H, W = A.W;
    int r;
    if ((r = fwd_relu(net, 0, A.x, IN_X2, N, H, W, A.e0a, nullptr, nullptr))) return r;
    if ((r = fwd_relu(net, 1, A.e0a, IN_DIRECT, N, H, W, A.e0, nullptr, nullptr))) return r;
    if ((r = fwd_relu(net, 2, A.e0, IN_POOL, N, H / 2, W / 2, A.e1a, nullptr, nullptr))) return r;
    if ((r = fwd_relu(net, 3, A.e1a, IN_DIRECT, N, H / 2, W / 2, A.e1, nullptr, nullptr))) return r;
    if ((r = fwd_relu(net, 4, A.e1, IN_POOL, N, H / 4, W / 4, A.e2a, nullptr, nullptr))) return r;
    if ((r = fwd_relu(net, 5, A.e2a, IN_DIRECT, N, H / 4, W / 4, A.e2, nullptr, nullptr))) return r;
    if ((r = fwd_relu(net, 6, A.e2, IN_POOL, N, H / 8, W / 8, A.e3a, nullptr, nullptr))) return r;
    if ((r = fwd_relu(net, 7, A.e3a, IN_DIRECT, N, H / 8, W / 8, A.e3, nullptr, nullptr))) return r;
    if ((r = fwd_relu(net, 8, A.e3, IN_UP, N, H / 4, W / 4, A.d2a, A.e2, A.d2))) return r;
    if ((r = fwd_relu(net, 9, A.d2, IN_UP, N, H / 2, W / 2, A.d1a, A.e1, A.d1))) return r;
    if ((r = fwd_relu(net, 10, A.d1, IN_UP, N, H, W, A.d0a, A.e0, A.d0))) return r;
    ConvP P = conv_params(A.d0, IN_DIRECT, N, H, W);
    P.w = net->wf[11];
    P.bias = net->bias[11];
    P.epi = EPI_OUTF;
    P.outf = A.out;
    return conv_dispatch(net, 16, 16, P);
}

static int elem_grid(CnnNet *net, long long n) { return grid_for(n, 256, net->num_sms); }

// backward pass from A.G (loss gradient) into net->grad
static int net_backward(CnnNet *net, Acts &A) {
    const int N = A.N, H = A.H, W = A.W;
    const long long p0 = (long long)N * H * W;
    int r;
    // output conv
    if ((r = bwd_weights(net, 11, A.d0, IN_DIRECT, A.G, N, H, W))) return r;
    if ((r = bwd_data(net, 11, A.G, N, H, W, A.gd0a, A.d0a, A.gd0))) return r;
    // decoder level 0 (u0 = up(d1))
    if ((r = bwd_weights(net, 10, A.d1, IN_UP, A.gd0a, N, H, W))) return r;
    if ((r = bwd_data(net, 10, A.gd0a, N, H, W, A.gu0, nullptr, nullptr))) return r;
    k_pool_sum<<<elem_grid(net, p0 / 4 * 4), 256, 0, net->stream>>>(A.gu0, N, H / 2, W / 2, 32, A.gd1, A.gd1a, A.d1a);
    // decoder level 1 (u1 = up(d2))
    if ((r = bwd_weights(net, 9, A.d2, IN_UP, A.gd1a, N, H / 2, W / 2))) return r;
    if ((r = bwd_data(net, 9, A.gd1a, N, H / 2, W / 2, A.gu1, nullptr, nullptr))) return r;
    k_pool_sum<<<elem_grid(net, p0 / 16 * 8), 256, 0, net->stream>>>(A.gu1, N, H / 4, W / 4, 64, A.gd2, A.gd2a, A.d2a);
    // decoder level 2 (u2 = up(e3))
    if ((r = bwd_weights(net, 8, A.e3, IN_UP, A.gd2a, N, H / 4, W / 4))) return r;
    if ((r = bwd_data(net, 8, A.gd2a, N, H / 4, W / 4, A.gu2, nullptr, nullptr))) return r;
    k_pool_sum<<<elem_grid(net, p0 / 64 * 8), 256, 0, net->stream>>>(A.gu2, N, H / 8, W / 8, 64, nullptr, A.ge3, A.e3);
    // encoder level 3
    if ((r = bwd_weights(net, 7, A.e3a, IN_DIRECT, A.ge3, N, H / 8, W / 8))) return r;
    if ((r = bwd_data(net, 7, A.ge3, N, H / 8, W / 8, A.ge3a, A.e3a, nullptr))) return r;
    if ((r = bwd_weights(net, 6, A.e2, IN_POOL, A.ge3a, N, H / 8, W / 8))) return r;
    if ((r = bwd_data(net, 6, A.ge3a, N, H / 8, W / 8, A.gp3, nullptr, nullptr))) return r;
    // encoder level 2
    k_merge<<<elem_grid(net, p0 / 16 * 8), 256, 0, net->stream>>>(A.gd2, A.gp3, A.e2, N, H / 4, W / 4, 64, A.ge2);
    if ((r = bwd_weights(net, 5, A.e2a, IN_DIRECT, A.ge2, N, H / 4, W / 4))) return r;
    if ((r = bwd_data(net, 5, A.ge2, N, H / 4, W / 4, A.ge2a, A.e2a, nullptr))) return r;
    if ((r = bwd_weights(net, 4, A.e1, IN_POOL, A.ge2a, N, H / 4, W / 4))) return r;
    if ((r = bwd_data(net, 4, A.ge2a, N, H / 4, W / 4, A.gp2, nullptr, nullptr))) return r;
    // encoder level 1
    k_merge<<<elem_grid(net, p0 / 4 * 4), 256, 0, net->stream>>>(A.gd1, A.gp2, A.e1, N, H / 2, W / 2, 32, A.ge1);
    if ((r = bwd_weights(net, 3, A.e1a, IN_DIRECT, A.ge1, N, H / 2, W / 2))) return r;
    if ((r = bwd_data(net, 3, A.ge1, N, H / 2, W / 2, A.ge1a, A.e1a, nullptr))) return r;
    if ((r = bwd_weights(net, 2, A.e0, IN_POOL, A.ge1a, N, H / 2, W / 2))) return r;
    if ((r = bwd_data(net, 2, A.ge1a, N, H / 2, W / 2, A.gp1, nullptr, nullptr))) return r;
    // encoder level 0
    k_merge<<<elem_grid(net, p0 * 2), 256, 0, net->stream>>>(A.gd0, A.gp1, A.e0, N, H, W, 16, A.ge0);
    if ((r = bwd_weights(net, 1, A.e0a, IN_DIRECT, A.ge0, N, H, W))) return r;
    if ((r = bwd_data(net, 1, A.ge0, N, H, W, A.ge0a, A.e0a, nullptr))) return r;
    if ((r = bwd_weights(net, 0, A.x, IN_X2, A.ge0a, N, H, W))) return r;
    NCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int net_loss(CnnNet *net, Acts &A) {
    const long long np = (long long)A.N * A.H * A.W;
    const int grid = std::min(grid_for(np, 256, net->num_sms), 1024);
    k_loss<<<grid, 256, 0, net->stream>>>(A.out, A.t, A.m, A.N, A.H, A.W, A.G, net->lpart);
    k_sum_partials<<<1, 256, 0, net->stream>>>(net->lpart, grid, net->dsum);
    NCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int net_pack(CnnNet *net) {
    PackAll A;
    for (int l = 0; l < CNN_LAYERS; l++) {
        A.L[l].ow = net->ow[l]; A.L[l].ob = net->ob[l];
        A.L[l].cin = L_CIN[l]; A.L[l].cout = L_COUT[l];
        A.L[l].cinp = pad16(L_CIN[l]); A.L[l].coutp = pad16(L_COUT[l]);
        A.L[l].fwd = net->wf[l]; A.L[l].bwd = net->wb[l]; A.L[l].bias = net->bias[l];
    }
    k_pack<<<dim3(36, CNN_LAYERS), 256, 0, net->stream>>>(net->prm, A);
    NCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int net_adam(CnnNet *net) {
    net->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)net->adam_t), c2 = 1.0f - powf(b2, (float)net->adam_t);
    k_adam<<<grid_for(net->nparams, 256, net->num_sms), 256, 0, net->stream>>>(net->prm, net->grad, net->am, net->av,
                                                                               net->nparams, net->lr, b1, b2, 1e-8f,
                                                                               c1, c2);
    NCUDA(cudaGetLastError());
    return net_pack(net);
}

int cnn_net_create(CnnNet **out, int dev, cudaStream_t stream, unsigned long long seed) {
    CnnNet *net = new CnnNet();
    *out = net;
    net->dev = dev;
    net->stream = stream;
    NCUDA(cudaDeviceGetAttribute(&net->num_sms, cudaDevAttrMultiProcessorCount, dev));
    int n = 0;
    for (int l = 0; l < CNN_LAYERS; l++) {
        net->ow[l] = n; n += L_COUT[l] * L_CIN[l] * 9;
        net->ob[l] = n; n += L_COUT[l];
    }
    net->nparams = n;
    NCUDA(cudaMalloc(&net->prm, sizeof(float) * n));
    NCUDA(cudaMalloc(&net->grad, sizeof(float) * n));
    NCUDA(cudaMalloc(&net->am, sizeof(float) * n));
    NCUDA(cudaMalloc(&net->av, sizeof(float) * n));
    NCUDA(cudaMemsetAsync(net->grad, 0, sizeof(float) * n, stream));
    NCUDA(cudaMemsetAsync(net->am, 0, sizeof(float) * n, stream));
    NCUDA(cudaMemsetAsync(net->av, 0, sizeof(float) * n, stream));
    for (int l = 0; l < CNN_LAYERS; l++) {
        const size_t k = (size_t)9 * pad16(L_CIN[l]) * pad16(L_COUT[l]);
        NCUDA(cudaMalloc(&net->wf[l], k * sizeof(bf16)));
        NCUDA(cudaMalloc(&net->wb[l], k * sizeof(bf16)));
        NCUDA(cudaMalloc(&net->bias[l], pad16(L_COUT[l]) * sizeof(float)));
    }
    NCUDA(cudaMalloc(&net->lpart, sizeof(double) * 1024));
    NCUDA(cudaMalloc(&net->dsum, sizeof(double)));
    NCUDA(cudaMalloc(&net->derr, sizeof(int)));
    NCUDA(cudaMemsetAsync(net->derr, 0, sizeof(int), stream));
    // He-normal initialisation (Box-Muller on a SplitMix64 stream), zero biases
    std::vector<float> h(n, 0.0f);
    unsigned long long s = seed ^ 0x5DEECE66Dull;
    for (int l = 0; l < CNN_LAYERS; l++) {
        const double sd = sqrt(2.0 / (9.0 * L_CIN[l]));
        for (int k = net->ow[l]; k < net->ob[l]; k++) {
            const double u1 = ((splitmix(s) >> 11) + 1.0) * (1.0 / 9007199254740993.0);
            const double u2 = (splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
            h[k] = (float)(sd * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
        }
    }
    NCUDA(cudaMemcpyAsync(net->prm, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice, stream));
    net->rng = seed * 0x2545F4914F6CDD1Dull + 1;
    int r = net_pack(net);
    if (r) return r;
    NCUDA(cudaStreamSynchronize(stream));
    return LEPIC_OK;
}

void cnn_net_destroy(CnnNet *net) {
    if (!net) return;
    acts_free(net->full);
    acts_free(net->crop);
    cudaFree(net->prm); cudaFree(net->grad); cudaFree(net->am); cudaFree(net->av);
    for (int l = 0; l < CNN_LAYERS; l++) { cudaFree(net->wf[l]); cudaFree(net->wb[l]); cudaFree(net->bias[l]); }
    cudaFree(net->part); cudaFree(net->partb); cudaFree(net->lpart); cudaFree(net->dsum); cudaFree(net->derr);
    delete net;
}

// weight-gradient scratch for a batch of N images of H x W
static int ensure_part(CnnNet *net, int N, int H, int W) {
    size_t need = 0, needb = 0;
    for (int l = 0; l < CNN_LAYERS; l++) {
        const int lev = l <= 1 || l >= 10 ? 0 : l <= 3 || l == 9 ? 1 : l <= 5 || l == 8 ? 2 : 3;
        const int h = H >> lev, w = W >> lev;
        const size_t units = (size_t)N * ((w + 127) / 128) * ((h + conv_rows(h) - 1) / conv_rows(h));
        need = std::max(need, units * pad16(L_CIN[l]) * pad16(L_COUT[l]) * 9);
        needb = std::max(needb, units * pad16(L_COUT[l]));
    }
    if (need > net->part_cap) {
        cudaFree(net->part);
        net->part = nullptr;
        net->part_cap = 0;
        NCUDA(cudaMalloc(&net->part, need * sizeof(float)));
        net->part_cap = need;
    }
    if (needb > net->partb_cap) {
        cudaFree(net->partb);
        net->partb = nullptr;
        net->partb_cap = 0;
        NCUDA(cudaMalloc(&net->partb, needb * sizeof(float)));
        net->partb_cap = needb;
    }
    return LEPIC_OK;
}

static int check_err(CnnNet *net) {
    int e = 0;
    NCUDA(cudaMemcpyAsync(&e, net->derr, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
    NCUDA(cudaStreamSynchronize(net->stream));
    if (e) {
        net->last_err = "tensor-core convolution timed out waiting for its MMA";
        cudaMemsetAsync(net->derr, 0, sizeof(int), net->stream);
        return LEPIC_ETIMEOUT;
    }
    return LEPIC_OK;
}

// ---------------------------------------------------------------------------------------
// C ABI of the network alone (the gradient check and the weights' round trip)
extern "C" int lepic_cnn_create(void **net_out, uint64_t seed) {
    if (!net_out) return LEPIC_EINVAL;
    *net_out = nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return LEPIC_ECUDA;
    int maj = 0;
    cudaDeviceGetAttribute(&maj, cudaDevAttrComputeCapabilityMajor, dev);
    if (maj != 10) return LEPIC_ENOKERNEL;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return LEPIC_ECUDA;
    CnnNet *net = nullptr;
    int r = cnn_net_create(&net, dev, s, seed);
    if (r) {
        cnn_net_destroy(net);
        cudaStreamDestroy(s);
        return r;
    }
    *net_out = net;
    return LEPIC_OK;
}

extern "C" int lepic_cnn_destroy(void *p) {
    CnnNet *net = (CnnNet *)p;
    if (!net) return LEPIC_EINVAL;
    cudaStream_t s = net->stream;
    cudaStreamSynchronize(s);
    cnn_net_destroy(net);
    cudaStreamDestroy(s);
    return LEPIC_OK;
}

extern "C" int lepic_cnn_nparams(void) {
    int n = 0;
    for (int l = 0; l < CNN_LAYERS; l++) n += L_COUT[l] * L_CIN[l] * 9 + L_COUT[l];
    return n;
}

extern "C" int lepic_cnn_params(void *p, float *host, int64_t n, int32_t set) {
    CnnNet *net = (CnnNet *)p;
    if (!net || !host || n != net->nparams) return LEPIC_EINVAL;
    if (set) {
        NCUDA(cudaMemcpyAsync(net->prm, host, sizeof(float) * n, cudaMemcpyHostToDevice, net->stream));
        int r = net_pack(net);
        if (r) return r;
    } else {
        NCUDA(cudaMemcpyAsync(host, net->prm, sizeof(float) * n, cudaMemcpyDeviceToHost, net->stream));
    }
    NCUDA(cudaStreamSynchronize(net->stream));
    return LEPIC_OK;
}

// forward + loss + gradient on host data: x [N][H][W][2], t and m [N][H][W] (m: 0/1)
extern "C" int lepic_cnn_loss_grad(void *p, const float *x, const float *t, const float *m, int32_t N, int32_t H,
                                   int32_t W, float *out, float *grad, double *loss) {
    CnnNet *net = (CnnNet *)p;
    if (!net || !x || N < 1 || H < 8 || W < 8 || H % 8 || W % 8 || N > CNN_MAX_BATCH) return LEPIC_EINVAL;
    if ((t == nullptr) != (m == nullptr) || (grad && !t)) return LEPIC_EINVAL;
    Acts &A = net->crop;
    if (A.N != N || A.H != H || A.W != W || !A.train) {
        acts_free(A);
        int r = acts_alloc(net, A, N, H, W, true);
        if (r) return r;
        if ((r = ensure_part(net, N, H, W))) return r;
    }
    const size_t np = (size_t)N * H * W;
    std::vector<bf16> hx(np * 2);
    for (size_t k = 0; k < np * 2; k++) hx[k] = __float2bfloat16_rn(x[k]);
    NCUDA(cudaMemcpyAsync(A.x, hx.data(), np * 2 * sizeof(bf16), cudaMemcpyHostToDevice, net->stream));
    std::vector<uint8_t> hm(np, 1);
    if (t) NCUDA(cudaMemcpyAsync(A.t, t, np * sizeof(float), cudaMemcpyHostToDevice, net->stream));
    if (m) {
        for (size_t k = 0; k < np; k++) hm[k] = m[k] > 0.0f ? 1 : 0;
        NCUDA(cudaMemcpyAsync(A.m, hm.data(), np, cudaMemcpyHostToDevice, net->stream));
    }
    int r = net_forward(net, A);
    if (r) return r;
    if (t) {
        if ((r = net_loss(net, A))) return r;
        if (grad && (r = net_backward(net, A))) return r;
    }
    if (out) NCUDA(cudaMemcpyAsync(out, A.out, np * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
    if (grad) NCUDA(cudaMemcpyAsync(grad, net->grad, sizeof(float) * net->nparams, cudaMemcpyDeviceToHost, net->stream));
    double L = 0.0;
    if (t) NCUDA(cudaMemcpyAsync(&L, net->dsum, sizeof(double), cudaMemcpyDeviceToHost, net->stream));
    if ((r = check_err(net))) return r;
    if (loss) *loss = L;
    return LEPIC_OK;
}

// one Adam step with the gradient of the last lepic_cnn_loss_grad
extern "C" int lepic_cnn_adam_step(void *p, float lr) {
    CnnNet *net = (CnnNet *)p;
    if (!net || !(lr > 0)) return LEPIC_EINVAL;
    net->lr = lr;
    int r = net_adam(net);
    if (r) return r;
    NCUDA(cudaStreamSynchronize(net->stream));
    return LEPIC_OK;
}

extern "C" const char *lepic_cnn_last_error(void *p) {
    CnnNet *net = (CnnNet *)p;
    return net ? net->last_err.c_str() : "null network";
}

// ---------------------------------------------------------------------------------------
// the learned warm start inside the Poisson solve
//
// image pixel (y, x) = node (i, j) = (x + 1, y + 1) of the (nx+1) x (ny+1) node grid, padded
// with zeros to a multiple of 8 in each direction.

struct PrepP {
    const double *u, *b;
    const int8_t *bc;
    int nx, ny, Hc, Wc;
    double aw, an, ac;
};

// r0 = b - A u at unknown nodes (FP64, the solver's operator) into rbuf; sum r0^2 per block
__global__ void k_prep_resid(PrepP P, float *rbuf, double *partial) {
    __shared__ double red[256];
    const int tot = P.Hc * P.Wc;
    const int W = P.nx + 3;
    double acc = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < tot; p += gridDim.x * blockDim.x) {
        const int y = p / P.Wc, x = p - y * P.Wc;
        float rv = 0.0f;
        if (x <= P.nx && y <= P.ny) {
            const int n = (x + 1) + (y + 1) * W;
            if (P.bc[n] <= 0) {
                const double *u = P.u;
                const double r = P.b[x + y * (P.nx + 1)] -
                                 (P.aw * u[n - 1] + P.an * u[n + W] + P.an * u[n - W] + P.aw * u[n + 1] + P.ac * u[n]);
                acc += r * r;
                rv = (float)r;
            }
        }
        if (rbuf) rbuf[p] = rv;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// sums the partials (fixed order); scal[0] = ||r||^2, scal[1] = sigma = rms over unknowns
__global__ void __launch_bounds__(256) k_prep_sigma(const double *partial, int n, double count, double *scal) {
    const double s = block_sum256(partial, n);
    if (threadIdx.x == 0) {
        scal[0] = s;
        scal[1] = sqrt(s / count);
    }
}

// network input: channel 0 = r0 / sigma, channel 1 = u / u_scale
__global__ void k_prep_input(PrepP P, const float *rbuf, const double *scal, double u_scale, bf16 *xin) {
    const int tot = P.Hc * P.Wc;
    const double sig = scal[1];
    const float inv_s = sig > 0.0 ? (float)(1.0 / sig) : 0.0f;
    const float inv_u = (float)(1.0 / u_scale);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < tot; p += gridDim.x * blockDim.x) {
        const int y = p / P.Wc, x = p - y * P.Wc;
        float uv = 0.0f;
        if (x <= P.nx && y <= P.ny) uv = (float)P.u[(x + 1) + (y + 1) * (P.nx + 3)] * inv_u;
        reinterpret_cast<uint32_t *>(xin)[p] = f2_to_bf2(rbuf[p] * inv_s, uv);
    }
}

// u += out * sigma / |ac| at unknown nodes (the network's correction, applied in FP64)
__global__ void k_apply(PrepP P, const float *out, const double *scal, double *u) {
    const int tot = (P.nx + 1) * (P.ny + 1);
    const double f = scal[1] / fabs(P.ac);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
        const int y = t / (P.nx + 1), x = t - y * (P.nx + 1);
        const int n = (x + 1) + (y + 1) * (P.nx + 3);
        if (P.bc[n] <= 0) u[n] += (double)out[y * P.Wc + x] * f;
    }
}

// keep the corrected potential only if it lowered the residual: scal[2] = new ||r||^2
__global__ void k_accept(PrepP P, const double *scal, const double *uprev, double *u, int *accepted) {
    const bool keep = scal[2] < scal[0];
    if (blockIdx.x == 0 && threadIdx.x == 0) *accepted = keep ? 1 : 0;
    if (keep) return;
    const long long nn = (long long)(P.nx + 3) * (P.ny + 3);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn; t += (long long)gridDim.x * blockDim.x)
        u[t] = uprev[t];
}

// training pair: target = (u_solved - u_prev) |ac| / sigma at unknown nodes
__global__ void k_target(PrepP P, const double *u, const double *uprev, const double *scal, float *t, uint8_t *m) {
    const long long tot = (long long)P.Hc * P.Wc;
    const double sig = scal[1];
    const double f = sig > 0.0 ? fabs(P.ac) / sig : 0.0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < tot; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % P.Wc), y = (int)(p / P.Wc);
        float tv = 0.0f;
        uint8_t mv = 0;
        if (x <= P.nx && y <= P.ny) {
            const long long n = (x + 1) + (long long)(y + 1) * (P.nx + 3);
            if (P.bc[n] <= 0) {
                tv = (float)((u[n] - uprev[n]) * f);
                mv = 1;
            }
        }
        t[p] = tv;
        m[p] = mv;
    }
}

struct LearnState {
    CnnNet *net = nullptr;
    int Hc = 0, Wc = 0;
    float *rbuf = nullptr, *tfull = nullptr;
    uint8_t *mfull = nullptr;
    double *uprev = nullptr, *scal = nullptr, *partial = nullptr;
    int *accepted = nullptr;
    double u_scale = 1.0;
    lepic_cnn_config cfg;
    lepic_cnn_stats st;
};

static void learn_defaults(lepic_cnn_config &c) {
    c.enable_training = 1;
    c.warmup_solves = 50;
    c.steps_warmup = 2;
    c.train_every = 4;
    c.steps_after = 1;
    c.crop = 256;
    c.batch = 4;
    c.lr = 2e-3f;
    c.seed = 1234;
}

static int learn_init(lepic_ctx *c) {
    if (c->learn) return LEPIC_OK;
    LearnState *L = new LearnState();
    c->learn = L;
    learn_defaults(L->cfg);
    memset(&L->st, 0, sizeof(L->st));
    int r = cnn_net_create(&L->net, c->dev, c->stream, L->cfg.seed);
    if (r) { c->last_err = L->net ? L->net->last_err : "network create failed"; return r; }
    const int nx = c->cfg.nx, ny = c->cfg.ny;
    L->Hc = (ny + 1 + 7) / 8 * 8;
    L->Wc = (nx + 1 + 7) / 8 * 8;
    const size_t np = (size_t)L->Hc * L->Wc;
    LCUDA(cudaMalloc(&L->rbuf, np * sizeof(float)));
    LCUDA(cudaMalloc(&L->tfull, np * sizeof(float)));
    LCUDA(cudaMalloc(&L->mfull, np));
    LCUDA(cudaMalloc(&L->uprev, sizeof(double) * c->nn));
    LCUDA(cudaMalloc(&L->scal, sizeof(double) * 4));
    LCUDA(cudaMalloc(&L->partial, sizeof(double) * 1024));
    LCUDA(cudaMalloc(&L->accepted, sizeof(int)));
    LCUDA(cudaMemsetAsync(L->scal, 0, sizeof(double) * 4, c->stream));
    LCUDA(cudaMemsetAsync(L->accepted, 0, sizeof(int), c->stream));
    r = acts_alloc(L->net, L->net->full, 1, L->Hc, L->Wc, false);
    if (r) { c->last_err = L->net->last_err; return r; }
    L->u_scale = c->phi_scale > 0 ? c->phi_scale : 1.0;
    return LEPIC_OK;
}

void learn_free(lepic_ctx *c) {
    LearnState *L = (LearnState *)c->learn;
    if (!L) return;
    cnn_net_destroy(L->net);
    cudaFree(L->rbuf); cudaFree(L->tfull); cudaFree(L->mfull); cudaFree(L->uprev);
    cudaFree(L->scal); cudaFree(L->partial); cudaFree(L->accepted);
    delete L;
    c->learn = nullptr;
}

static PrepP prep_params(lepic_ctx *c, LearnState *L) {
    PrepP P;
    const MGLevel &a = c->lev[0];
    P.u = a.u; P.b = a.b; P.bc = a.bc;
    P.nx = c->cfg.nx; P.ny = c->cfg.ny; P.Hc = L->Hc; P.Wc = L->Wc;
    const double eps0 = c->cfg.eps0;
    P.aw = eps0 / (a.hx * a.hx);
    P.an = eps0 / (a.hy * a.hy);
    P.ac = -(P.an + P.an + P.aw + P.aw);
    return P;
}

static int learn_train(lepic_ctx *c, LearnState *L, int steps) {
    CnnNet *net = L->net;
    const int S = std::max(8, std::min(L->cfg.crop, std::min(L->Hc, L->Wc)) / 8 * 8);
    const int B = std::max(1, std::min(L->cfg.batch, CNN_MAX_BATCH));
    Acts &A = net->crop;
    if (A.N != B || A.H != S || A.W != S || !A.train) {
        acts_free(A);
        int r = acts_alloc(net, A, B, S, S, true);
        if (r) { c->last_err = net->last_err; return r; }
        if ((r = ensure_part(net, B, S, S))) { c->last_err = net->last_err; return r; }
    }
    net->lr = L->cfg.lr;
    for (int s = 0; s < steps; s++) {
        CropP C;
        for (int b = 0; b < B; b++) {
            const int ry = (L->Hc - S) / 8 + 1, rx = (L->Wc - S) / 8 + 1;
            C.oy[b] = (int)(splitmix(net->rng) % (unsigned long long)ry) * 8;
            C.ox[b] = (int)(splitmix(net->rng) % (unsigned long long)rx) * 8;
        }
        k_crop<<<grid_for((long long)B * S * S, 256, net->num_sms), 256, 0, c->stream>>>(
            net->full.x, L->tfull, L->mfull, L->Hc, L->Wc, S, B, C, A.x, A.t, A.m);
        LCUDA(cudaGetLastError());
        int r;
        if ((r = net_forward(net, A)) || (r = net_loss(net, A)) || (r = net_backward(net, A)) || (r = net_adam(net))) {
            c->last_err = net->last_err;
            return r;
        }
        L->st.train_steps++;
    }
    return LEPIC_OK;
}

// Poisson solve with the learned warm start: predict, keep the prediction only if it lowers
// the residual, refine with the mixed-precision CG, then learn from the solved pair.
int learned_solve(lepic_ctx *c, double eps) {
    if (c->cfg.flag_pbc || c->cfg.flag_nmn) return mg_mixed_solve(c, eps, false); // same scope as the CG
    int r = learn_init(c);
    if (r) return r;
    LearnState *L = (LearnState *)c->learn;
    CnnNet *net = L->net;
    PrepP P = prep_params(c, L);
    const long long np = (long long)L->Hc * L->Wc;
    const int g = std::min(grid_for(np, 256, c->num_sms), 1024);
    const double count = c->n_unknown > 0 ? (double)c->n_unknown : 1.0; // counted at create
    LCUDA(cudaMemcpyAsync(L->uprev, c->phi, sizeof(double) * c->nn, cudaMemcpyDeviceToDevice, c->stream));
    k_prep_resid<<<g, 256, 0, c->stream>>>(P, L->rbuf, L->partial);
    k_prep_sigma<<<1, 256, 0, c->stream>>>(L->partial, g, count, L->scal);
    k_prep_input<<<grid_for(np, 256, c->num_sms), 256, 0, c->stream>>>(P, L->rbuf, L->scal, L->u_scale, net->full.x);
    LCUDA(cudaGetLastError());
    r = net_forward(net, net->full);
    if (r) { c->last_err = net->last_err; return r; }
    k_apply<<<grid_for((long long)(c->cfg.nx + 1) * (c->cfg.ny + 1), 256, c->num_sms), 256, 0, c->stream>>>(
        P, net->full.out, L->scal, c->phi);
    // the new residual norm into scal[2]
    k_prep_resid<<<g, 256, 0, c->stream>>>(P, nullptr, L->partial);
    k_prep_sigma<<<1, 256, 0, c->stream>>>(L->partial, g, count, L->scal + 2);
    k_accept<<<grid_for(c->nn, 256, c->num_sms), 256, 0, c->stream>>>(P, L->scal, L->uprev, c->phi, L->accepted);
    LCUDA(cudaGetLastError());
    r = mg_mixed_solve(c, eps, false);   // from the network's start, not an extrapolation
    if (r) return r;
    L->st.solves++;
    const bool train = L->cfg.enable_training &&
                       (L->st.solves <= L->cfg.warmup_solves || (L->st.solves % std::max(1, L->cfg.train_every)) == 0);
    if (train) {
        k_target<<<grid_for(np, 256, c->num_sms), 256, 0, c->stream>>>(P, c->phi, L->uprev, L->scal, L->tfull,
                                                                        L->mfull);
        LCUDA(cudaGetLastError());
        r = learn_train(c, L, L->st.solves <= L->cfg.warmup_solves ? L->cfg.steps_warmup : L->cfg.steps_after);
        if (r) return r;
    }
    return LEPIC_OK;
}

// per-solve statistics need a synchronisation: read on request only
int learned_stats(lepic_ctx *c, lepic_cnn_stats *out) {
    LearnState *L = (LearnState *)c->learn;
    if (!L) {
        memset(out, 0, sizeof(*out));
        return LEPIC_OK;
    }
    double scal[4] = {0, 0, 0, 0};
    int acc = 0;
    double loss = 0;
    LCUDA(cudaMemcpyAsync(scal, L->scal, sizeof(scal), cudaMemcpyDeviceToHost, c->stream));
    LCUDA(cudaMemcpyAsync(&acc, L->accepted, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    LCUDA(cudaMemcpyAsync(&loss, L->net->dsum, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    LCUDA(cudaStreamSynchronize(c->stream));
    int r = check_err(L->net);
    if (r) { c->last_err = L->net->last_err; return r; }
    *out = L->st;
    out->last_accepted = acc;
    out->last_res_ratio = scal[0] > 0 ? sqrt(scal[2] / scal[0]) : 0.0;
    out->last_loss = loss;
    return LEPIC_OK;
}

int learned_configure(lepic_ctx *c, const lepic_cnn_config *cfg) {
    if (cfg->batch < 1 || cfg->batch > CNN_MAX_BATCH || cfg->crop < 8 || !(cfg->lr > 0) || cfg->train_every < 1)
        return LEPIC_EINVAL;
    int r = learn_init(c);
    if (r) return r;
    ((LearnState *)c->learn)->cfg = *cfg;
    return LEPIC_OK;
}

// ---------------------------------------------------------------------------------------
// C ABI of the learned warm start of a context
extern "C" int lepic_gpu_cnn_configure(lepic_ctx *c, const lepic_cnn_config *cfg) {
    if (!c || !cfg) return LEPIC_EINVAL;
    return learned_configure(c, cfg);
}

extern "C" int lepic_gpu_cnn_stats(lepic_ctx *c, lepic_cnn_stats *st) {
    if (!c || !st) return LEPIC_EINVAL;
    return learned_stats(c, st);
}

extern "C" void *lepic_gpu_cnn_net(lepic_ctx *c) {
    if (!c || !c->learn) return nullptr;
    return ((LearnState *)c->learn)->net;
}
