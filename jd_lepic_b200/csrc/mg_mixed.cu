// mg_mixed.cu -- mixed-precision Poisson solve, one persistent cooperative kernel:
// conjugate gradients in FP64 on the reference's discrete operator (5-point, Dirichlet walls
// and embedded conductors from bcnd), preconditioned by one FP32 V-cycle of the reference's
// multigrid components (red-black SOR smoothing, full-weighting restriction, bilinear
// prolongation, injection-coarsened masks, mg.f90 / sors.f90), run symmetrically
// (red-black before, black-red after the coarse correction) so that it is a valid CG
// preconditioner.
//
//   r = b - A u (FP64);  z = V32(r);  p = z
//   loop:  Ap = A p;  a = (r.z)/(p.Ap);  u += a p;  r -= a Ap          (FP64)
//          stop when ||r||_2 <= eps ||b - A u_D||_2 (checked on the true residual)
//          z = V32(r);  b = (r.z)_new/(r.z)_old;  p = z + b p
// Every quantity that decides the answer (u, r, p, Ap, the dot products) is FP64; the
// FP32 cycle only chooses search directions, so the converged u solves the FP64 system.
// Why CG around the cycle: with embedded conductors (the aperture plate) the injected coarse
// masks misrepresent the conductor and a stand-alone V-cycle contracts by ~0.5 per cycle or
// diverges; CG removes those few conductor modes (11-12 iterations from a cold start to 1e-8,
// independent of the grid size, in a CPU emulation of this exact algorithm).
// Roofline: per iteration the finest level moves ~5 FP64 passes (~170 B/node) plus the FP32
// cycle (~60 B/node); the coarsest levels that fit together in about 96 KB (e, r and mask)
// run on CTA 0 out of its shared memory.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <thread>
#include <vector>
#include "mg_common.cuh"

__device__ __forceinline__ float rfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return fma(a, b, c); }

namespace mx32 {
using R = float;
#include "mg_mixed_cycle.cuh"
}
namespace mx64 {
using R = double;
#include "mg_mixed_cycle.cuh"
}

// The extrapolated warm start: at the unknowns u = 2 u - u_prev, where u is this solve's
// input (the last solution) and u_prev the previous solve's input; u_prev <- u in the same
// pass.  Dirichlet nodes keep their values.
__global__ void k_warm_xtrap(double *u, double *hist, const int8_t *bc, long long nn, int have) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn; t += (long long)gridDim.x * blockDim.x) {
        const double cur = u[t];
        const double prev = hist[t];
        hist[t] = cur;
        if (have && bc[t] <= 0) u[t] = 2.0 * cur - prev;
    }
}

#define MX_DIRECT_MAX 2048   // unknowns of the exactly solved level (33^2 nodes fit)

// The inverse of level l's operator on its unknowns (nodes with bcnd <= 0 inside the level):
// B = -A is symmetric positive definite (the 5-point stencil with the walls' zero correction),
// factored by a Cholesky decomposition within its band (unknowns in row order: the band is one
// row of the level), then B^-1 column by column; M = A^-1 = -B^-1 is kept in FP32 (and in FP64
// for mode 4's cycle).  Computed once per level on the host (at most MX_DIRECT_MAX unknowns),
// then reused by every solve.
static int coarse_inverse(lepic_ctx *c, int l) {
    if (c->mx_clev == l) return LEPIC_OK;
    c->mx_clev = l;
    c->mx_cn = 0;
    const MGLevel &L = c->lev[l];
    const int W = L.nx + 3, nn = W * (L.ny + 3);
    std::vector<int8_t> bc((size_t)nn);
    LCUDA(cudaMemcpy(bc.data(), L.bc, (size_t)nn, cudaMemcpyDeviceToHost));
    std::vector<int> id((size_t)nn, -1), node, ridx;
    for (int j = 1; j <= L.ny + 1; j++)
        for (int i = 1; i <= L.nx + 1; i++) {
            const int t = i + j * W;
            if (bc[t] > 0) continue;
            id[t] = (int)node.size();
            node.push_back(t);
            ridx.push_back((i - 1) + (j - 1) * (L.nx + 1));
        }
    const int n = (int)node.size();
    if (n == 0 || n > MX_DIRECT_MAX) return LEPIC_OK;   // the CTA-0 cycle stays
    const double aw = c->cfg.eps0 / (L.hx * L.hx), an = c->cfg.eps0 / (L.hy * L.hy);
    std::vector<double> Bm((size_t)n * n, 0.0), G((size_t)n * n, 0.0);
    int bw = 0;
    for (int k = 0; k < n; k++) {
        const int t = node[k];
        Bm[(size_t)k * n + k] = 2.0 * aw + 2.0 * an;
        const int nb[4] = {t - 1, t + 1, t - W, t + W};
        const double cf[4] = {aw, aw, an, an};
        for (int q = 0; q < 4; q++) {
            const int m = id[nb[q]];
            if (m >= 0) {
                Bm[(size_t)k * n + m] = -cf[q];
                bw = std::max(bw, std::abs(m - k));
            }
        }
    }
    for (int j = 0; j < n; j++) {   // G lower triangular, zero below the band
        double d = Bm[(size_t)j * n + j];
        for (int k = std::max(0, j - bw); k < j; k++) d -= G[(size_t)j * n + k] * G[(size_t)j * n + k];
        if (!(d > 0.0)) return LEPIC_OK;   // not positive definite: the CTA-0 cycle stays
        const double gjj = std::sqrt(d);
        G[(size_t)j * n + j] = gjj;
        for (int i = j + 1; i <= std::min(n - 1, j + bw); i++) {
            double s = Bm[(size_t)i * n + j];
            for (int k = std::max(0, i - bw); k < j; k++) s -= G[(size_t)i * n + k] * G[(size_t)j * n + k];
            G[(size_t)i * n + j] = s / gjj;
        }
    }
    std::vector<float> M((size_t)n * n);
    std::vector<double> M64((size_t)n * n);
    // the columns are independent: host threads take every nth one
    auto columns = [&](int first, int stride) {
        std::vector<double> y((size_t)n), xv((size_t)n);
        for (int col = first; col < n; col += stride) {
            for (int i = 0; i < col; i++) y[i] = 0.0;
            for (int i = col; i < n; i++) {   // G y = e_col
                double s = i == col ? 1.0 : 0.0;
                for (int k = std::max(col, i - bw); k < i; k++) s -= G[(size_t)i * n + k] * y[k];
                y[i] = s / G[(size_t)i * n + i];
            }
            for (int i = n - 1; i >= 0; i--) {   // G^T x = y
                double s = y[i];
                for (int k = i + 1; k <= std::min(n - 1, i + bw); k++) s -= G[(size_t)k * n + i] * xv[k];
                xv[i] = s / G[(size_t)i * n + i];
            }
            for (int i = 0; i < n; i++) {
                M[(size_t)i * n + col] = (float)(-xv[i]);
                M64[(size_t)i * n + col] = -xv[i];
            }
        }
    };
    const int nth = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < 512 || nth == 1) {
        columns(0, 1);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nth; t++) pool.emplace_back(columns, t, nth);
        for (auto &th : pool) th.join();
    }
    if (c->mx_cinv) { cudaFree(c->mx_cinv); c->mx_cinv = nullptr; }
    if (c->mx_cinv64) { cudaFree(c->mx_cinv64); c->mx_cinv64 = nullptr; }
    if (c->mx_cidx) { cudaFree(c->mx_cidx); c->mx_cidx = nullptr; }
    if (cudaMalloc((void **)&c->mx_cinv, sizeof(float) * (size_t)n * n) != cudaSuccess ||
        cudaMalloc((void **)&c->mx_cinv64, sizeof(double) * (size_t)n * n) != cudaSuccess ||
        cudaMalloc((void **)&c->mx_cidx, sizeof(int) * 2 * (size_t)n) != cudaSuccess) {
        c->last_err = "mixed solver: cudaMalloc of the coarse inverse failed";
        return LEPIC_ENOMEM;
    }
    LCUDA(cudaMemcpy(c->mx_cinv, M.data(), sizeof(float) * (size_t)n * n, cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(c->mx_cinv64, M64.data(), sizeof(double) * (size_t)n * n, cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(c->mx_cidx, node.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(c->mx_cidx + n, ridx.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
    c->mx_cn = n;
    return LEPIC_OK;
}

// the two instantiations of the cycle: FP32 (mode 1) and FP64 (mode 4)
template <typename R> struct MxOf;
template <> struct MxOf<float> {
    using P = mx32::MXP;
    static void *kernel() { return (void *)mx32::k_mg_mixed; }
    static float *e(MGLevel &a) { return a.e32; }
    static float *e2(MGLevel &a) { return a.e32b; }
    static float *r(MGLevel &a) { return a.r32; }
    static const float *cinv(lepic_ctx *c) { return c->mx_cinv; }
};
template <> struct MxOf<double> {
    using P = mx64::MXP;
    static void *kernel() { return (void *)mx64::k_mg_mixed; }
    static double *e(MGLevel &a) { return a.e64; }
    static double *e2(MGLevel &a) { return a.e64b; }
    static double *r(MGLevel &a) { return a.r64; }
    static const double *cinv(lepic_ctx *c) { return c->mx_cinv64; }
};

template <typename R>
static int mixed_launch(lepic_ctx *c, double eps, int *grid_cache) {
    using Mx = MxOf<R>;
    typename Mx::P P;
    memset(&P, 0, sizeof(P));
    const double eps0 = c->cfg.eps0;
    for (int l = 0; l < c->nlev; l++) {
        MGLevel &a = c->lev[l];
        auto &d = P.L[l];
        d.nx = a.nx; d.ny = a.ny;
        double aw = eps0 / (a.hx * a.hx), an = eps0 / (a.hy * a.hy), ac = -(an + an + aw + aw);
        d.awd = aw; d.and_ = an; d.acd = ac;
        d.aw = (R)aw; d.an = (R)an; d.ac = (R)ac;
        d.e = Mx::e(a); d.e2 = Mx::e2(a); d.r = Mx::r(a); d.bc = a.bc; d.u = a.u; d.b = a.b;
    }
    P.ng = c->nlev;
    // the coarsest levels whose e, r and mask fit together in CTA 0's shared-memory budget
    // run on chip; the finer ones use the whole grid
    const long long budget = c->opt.mx_onchip_bytes;  // 20 KiB: 32^2 nodes and coarser (best at 2048^2)
    const long long rs = (long long)sizeof(R);
    auto level_bytes = [&](int l) {
        const long long nn = (long long)(c->lev[l].nx + 3) * (c->lev[l].ny + 3);
        const long long nr = (long long)(c->lev[l].nx + 1) * (c->lev[l].ny + 1);
        return ((nn * rs + 15) / 16) * 16 + ((nr * rs + 15) / 16) * 16 + ((nn + 15) / 16) * 16;
    };
    int Ls = c->nlev;
    long long total = 0;
    for (int l = c->nlev - 1; l >= 1; l--) {
        if (total + level_bytes(l) > budget * rs / 4) break;   // the FP32 budget's levels in both
        total += level_bytes(l);
        Ls = l;
    }
    long long off = 0;
    for (int l = Ls; l < c->nlev; l++) {
        const long long nn = (long long)(c->lev[l].nx + 3) * (c->lev[l].ny + 3);
        const long long nr = (long long)(c->lev[l].nx + 1) * (c->lev[l].ny + 1);
        P.soff_e[l] = (int)off; off += ((nn * rs + 15) / 16) * 16;
        P.soff_r[l] = (int)off; off += ((nr * rs + 15) / 16) * 16;
        P.soff_b[l] = (int)off; off += ((nn + 15) / 16) * 16;
    }
    P.Ls = Ls;
    P.cn = 0;
    if (c->opt.mx_coarse_direct && Ls >= 1 && Ls <= c->nlev - 1) {
        const int r = coarse_inverse(c, Ls);
        if (r != LEPIC_OK) return r;
        if (c->mx_cn > 0 && c->mx_clev == Ls) { P.cinv = Mx::cinv(c); P.cidx = c->mx_cidx; P.cn = c->mx_cn; }
    }
    // two over-relaxed sweeps (omega 1.15) before and after the coarse correction; the reverse
    // colour order after it keeps the cycle a symmetric preconditioner.  Measured at 2048^2
    // over 100 steps from the extrapolated start (2 iterations): 1.32 ms per solve against
    // 1.37 with three plain sweeps; two plain sweeps need a third iteration in some steps, and
    // omega 1.3 in others.  From phi_(n-1) alone: 4 iterations, against 5 with two plain
    // sweeps and 4 with three.
    // two sweeps each way on the coarsest level (3^2 nodes at 2048^2): eight gave the same
    // iteration counts and residuals and cost CTA 0's 28 more barriers per cycle
    P.omega = (R)c->opt.mx_omega;
    P.nu1 = c->opt.mx_nu1; P.nu2 = c->opt.mx_nu2; P.nuc = c->opt.mx_nuc; P.max_iter = c->opt.mx_max_iter;
    // tiles: region (TX + 2H) x (TY + 2H) with H = 2 nu + 2 (down) or 2 nu (up); e, r (R) and the
    // mask per node, sharing the dynamic shared memory with the small cycle
    const int Hmax = 2 * std::max(P.nu1 + 1, P.nu2);
    auto region_bytes = [&](int tx, int ty) {
        const long long cap = ((long long)((tx + 2 * Hmax + 3) & ~3) * (ty + 2 * Hmax) + 15) / 16 * 16;
        const long long cc = (long long)((tx + 2 * Hmax) / 2 + 3) * ((ty + 2 * Hmax) / 2 + 3);
        return cap * (2 * rs + 1) + cc * rs + 16;
    };
    int cap_tx = MX_TX, cap_ty = MX_TY;
    while (cap_ty > 8 && region_bytes(cap_tx, cap_ty) > 64 * 1024) cap_ty /= 2;
    P.tile_cap = (((cap_tx + 2 * Hmax + 3) & ~3) * (cap_ty + 2 * Hmax) + 15) / 16 * 16;   // rows padded to 4
    {
        // per level the tile that ends the pass soonest: the tiles go round the grid's CTAs, so
        // a pass lasts (rounds) x (one tile's region, halo included, plus a fixed latency per
        // tile: a tile is a chain of dependent loads and block barriers); 561 tiles on 444
        // CTAs, for instance, take two rounds where 442 slightly larger ones take one
        const int grid_est = *grid_cache > 0 ? *grid_cache : c->num_sms * c->opt.ctas_per_sm;
        for (int l = 0; l < c->nlev; l++) {
            long long best = -1;
            int btx = 16, bty = 8;
            for (int tx = 16; tx <= cap_tx; tx += 16)
                for (int ty = 8; ty <= cap_ty; ty += 4) {
                    const long long nt = (long long)((c->lev[l].nx + 1 + tx - 1) / tx) * ((c->lev[l].ny + 1 + ty - 1) / ty);
                    const long long rounds = (nt + grid_est - 1) / grid_est;
                    const long long cost = rounds * ((long long)(tx + 2 * Hmax) * (ty + 2 * Hmax) + 1000);
                    if (best < 0 || cost < best) { best = cost; btx = tx; bty = ty; }
                }
            P.tx[l] = btx;
            P.ty[l] = bty;
        }
    }
    const long long tile_bytes = region_bytes(cap_tx, cap_ty);
    P.tiled = (Ls <= c->nlev - 1 && Ls >= 1 && c->opt.mx_tiled && tile_bytes <= 64 * 1024) ? 1 : 0;
    P.smem_bytes = (int)std::max(off, P.tiled ? tile_bytes : 0ll);
    P.eps = eps;
    P.alpha = fabs((double)(c->cfg.nx + 1) * (c->cfg.ny + 1) * P.L[0].acd);
    P.pbc = c->cfg.flag_pbc;
    P.nmn = c->cfg.flag_nmn;
    P.r64 = c->cg_r; P.p64 = c->cg_p; P.ap64 = c->cg_ap;
    P.partials = c->partials;
    P.cnt = c->dcnt;
    P.bar_extra = (unsigned)c->opt.barrier_extra;
    const size_t smem = (size_t)P.smem_bytes;
    if (*grid_cache == 0) {
        LCUDA(cudaFuncSetAttribute(Mx::kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        int occ = 0;
        LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, Mx::kernel(), MG_THREADS, smem));
        if (occ < 1) { c->last_err = "mixed multigrid kernel does not fit on an SM"; return LEPIC_ECUDA; }
        *grid_cache = c->num_sms * std::max(1, std::min(occ, (int)c->opt.ctas_per_sm));
    }
    void *args[] = {&P};
    LCUDA(cudaMemsetAsync(&c->dcnt->bar_arrived, 0, sizeof(unsigned long long) + sizeof(int), c->stream));
    LCUDA(cudaLaunchCooperativeKernel(Mx::kernel(), dim3(*grid_cache), dim3(MG_THREADS), args, smem, c->stream));
    return LEPIC_OK;
}

// the FP64 cycle's level arrays, at its first use
static int alloc_fp64_cycle(lepic_ctx *c) {
    if (c->lev[0].e64) return LEPIC_OK;
    for (int l = 0; l < c->nlev; l++) {
        MGLevel &L = c->lev[l];
        const size_t nnl = (size_t)(L.nx + 3) * (L.ny + 3), nr = (size_t)(L.nx + 1) * (L.ny + 1);
        if (cudaMalloc((void **)&L.e64, sizeof(double) * nnl) != cudaSuccess ||
            cudaMalloc((void **)&L.e64b, sizeof(double) * nnl) != cudaSuccess ||
            cudaMalloc((void **)&L.r64, sizeof(double) * nr) != cudaSuccess) {
            c->last_err = "FP64-cycle solve: cudaMalloc failed";
            return LEPIC_ENOMEM;
        }
        LCUDA(cudaMemsetAsync(L.e64, 0, sizeof(double) * nnl, c->stream));
        LCUDA(cudaMemsetAsync(L.e64b, 0, sizeof(double) * nnl, c->stream));
        LCUDA(cudaMemsetAsync(L.r64, 0, sizeof(double) * nr, c->stream));
    }
    return LEPIC_OK;
}

// fp64: the same CG with the V-cycle in FP64 (mode 4) instead of FP32 (mode 1)
int mg_mixed_solve(lepic_ctx *c, double eps, bool xtrap, bool fp64) {
    if (c->cfg.flag_pbc || c->cfg.flag_nmn) // the CG operator is symmetric only with Dirichlet rows
        return mg_solve(c, eps, 2);
    if (xtrap && c->warm_xtrap) {
        k_warm_xtrap<<<c->num_sms * 8, 256, 0, c->stream>>>(c->phi, c->phi_hist, c->bc8, c->nn, c->have_hist);
        LCUDA(cudaGetLastError());
        c->have_hist = 1;
    }
    if (!fp64) return mixed_launch<float>(c, eps, &c->mg_grid_mixed);
    const int r = alloc_fp64_cycle(c);
    if (r != LEPIC_OK) return r;
    return mixed_launch<double>(c, eps, &c->mg_grid_mixed64);
}
