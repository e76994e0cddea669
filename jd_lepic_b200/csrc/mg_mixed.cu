// mg_mixed.cu -- mixed-precision Poisson solve: FP32 V-cycles inside FP64 iterative
// refinement, one persistent cooperative kernel.
//
//   loop:  r = b - A u          FP64 (the only place the solution's accuracy is decided)
//          stop when ||r||_2 <= eps * ||b - A u_D||_2   (u_D: u with the unknowns zeroed)
//          A e = r              one FP32 V-cycle from e = 0: red-black SOR smoothing (nu1/nu2
//                               sweeps), full-weighting restriction, bilinear prolongation,
//                               with the reference's boundary rules (mg.f90, sors.f90)
//          u = u + e            FP64
// The smoother, transfer operators and masks are the reference's; only the arithmetic type
// of the correction cycle changes, so the FP64 outer loop converges to the same discrete
// solution as the FP64 solver.  The coarse levels (at most `small_nodes` nodes) run on CTA 0.
// Roofline: per outer iteration the finest level moves ~110 B/node (FP64 u, b once; FP32 e, r
// for the sweeps); at 2049^2 nodes the working set is L2-resident.
#include <algorithm>
#include <cstdlib>
#include "mg_common.cuh"

struct MXL {
    int nx, ny;
    float aw, an, ac;         // FP32 stencil of this level
    double awd, and_, acd;    // FP64 stencil (finest level only)
    float *e, *r;
    const int8_t *bc;
    double *u, *b;
};

struct MXP {
    MXL L[LEPIC_MAXLEV];
    int ng, Ls;
    float omega;
    int nu1, nu2, nuc, max_outer;
    double eps, alpha;
    int pbc, nmn;
    double *partials;
    DevCounters *cnt;
};

template <class Team>
__device__ void sweep32(const Team &T, const MXL &L, int color, float omega) {
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    const float aw = L.aw, ae = L.aw, an = L.an, as = L.an, ac = L.ac;
    const float inv_ac = 1.0f / ac;
    const int hw = nx / 2 + 1;
    const long long tot = (long long)(ny + 1) * hw;
    for (long long w = T.rank(); w < tot; w += T.size()) {
        int j = (int)(w / hw) + 1;
        int k = (int)(w % hw);
        int i = ((((j + 1 + color) & 1) != 0) ? 1 : 2) + 2 * k;
        if (i > nx + 1) continue;
        const long long n = i + (long long)j * W;
        const int bc = L.bc[n];
        if (bc > 0) continue;
        const float rij = L.r[(i - 1) + (long long)(j - 1) * (nx + 1)];
        float *e = L.e;
        float s;
        if (bc == -2) {
            s = rij - an * e[n + W] - as * e[n - W] - 2.0f * ae * e[n + 1];
        } else {
            if (bc == 0 && j == ny + 1) continue;
            s = rij - aw * e[n - 1] - an * e[n + W] - as * e[n - W] - ae * e[n + 1];
        }
        e[n] = (1.0f - omega) * e[n] + omega * s * inv_ac;
    }
}

template <class Team>
__device__ void pbc32(const Team &T, const MXL &L) {
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    for (long long i = T.rank(); i <= nx + 2; i += T.size()) {
        if (L.bc[i + 1 * W] <= 0) L.e[i] = L.e[i + (long long)ny * W];
        if (L.bc[i + (long long)(ny + 1) * W] <= 0) L.e[i + (long long)(ny + 1) * W] = L.e[i + W];
    }
}

template <class Team>
__device__ bool smooth32(const Team &T, const MXP &P, int l, int nsweep) {
    for (int k = 0; k < nsweep; k++)
        for (int color = 0; color < 2; color++) {
            sweep32(T, P.L[l], color, P.omega);
            if (!T.sync()) return false;
            if (P.pbc) {
                pbc32(T, P.L[l]);
                if (!T.sync()) return false;
            }
        }
    return true;
}

__device__ __forceinline__ float getres32(const MXL &L, int ir, int jr, int flag) {
    const int W = L.nx + 3;
    float aw = L.aw, ae = L.aw;
    const float an = L.an, as = L.an, ac = L.ac;
    const long long n = ir + (long long)jr * W;
    const float *e = L.e;
    float uw;
    if (ir == 1 && flag == 1) { uw = 0.0f; aw = 0.0f; ae = 2.0f * ae; }
    else uw = e[n - 1];
    return L.r[(ir - 1) + (long long)(jr - 1) * (L.nx + 1)] -
           (aw * uw + ae * e[n + 1] + an * e[n + W] + as * e[n - W] + ac * e[n]);
}

__device__ __forceinline__ float rpbc32(const MXL &F, int x, int nmn) {
    const int W = F.nx + 3, ny = F.ny;
    bool set;
    if (x & 1) set = F.bc[x + (long long)(ny + 1) * W] <= 0;
    else set = (x - 1 >= 1 && F.bc[x - 1 + (long long)(ny + 1) * W] <= 0) ||
               (x + 1 <= F.nx + 1 && F.bc[x + 1 + (long long)(ny + 1) * W] <= 0);
    return set ? getres32(F, x, ny, nmn) : 0.0f;
}

// mg.f90:335-444 applied to the correction equation
template <class Team>
__device__ void restrict32(const Team &T, const MXL &F, const MXL &C, int pbc, int nmn) {
    const int nx = F.nx, ny = F.ny, W = nx + 3, nx2 = C.nx, ny2 = C.ny, W2 = nx2 + 3;
    const long long tot = (long long)(nx2 + 1) * (ny2 + 1);
    for (long long t = T.rank(); t < tot; t += T.size()) {
        int i = (int)(t % (nx2 + 1)) + 1, j = (int)(t / (nx2 + 1)) + 1;
        int ir = 2 * i - 1, jr = 2 * j - 1;
        float out = 0.0f;
        if (C.bc[i + (long long)j * W2] <= 0) {
            const int8_t *bc = F.bc;
#define FB(a, b) bc[(a) + (long long)(b) * W]
            float r1 = 0, r2 = 0, r3 = 0, r4 = 0, r5 = 0, r6 = 0, r7 = 0, r8 = 0;
            float r9 = getres32(F, ir, jr, nmn);
            if (ir != nx + 1 && jr != ny + 1 && FB(ir + 1, jr + 1) <= 0) r1 = getres32(F, ir + 1, jr + 1, nmn);
            if (ir != nx + 1 && FB(ir + 1, jr) <= 0) r2 = getres32(F, ir + 1, jr, nmn);
            if (FB(ir + 1, jr - 1) <= 0) {
                if (ir != nx + 1 && jr != 1) r3 = getres32(F, ir + 1, jr - 1, nmn);
                else if (jr == 1 && pbc) r3 = rpbc32(F, ir + 1, nmn);
            }
            if (FB(ir, jr - 1) <= 0) {
                if (jr != 1) r4 = getres32(F, ir, jr - 1, nmn);
                else if (pbc) r4 = rpbc32(F, ir, nmn);
            }
            if (FB(ir - 1, jr - 1) <= 0 && ir != 1) {
                if (jr != 1) r5 = getres32(F, ir - 1, jr - 1, nmn);
                else if (pbc) r5 = rpbc32(F, ir - 1, nmn);
            }
            if (FB(ir - 1, jr) <= 0 && ir != 1) r6 = getres32(F, ir - 1, jr, nmn);
            if (FB(ir - 1, jr + 1) <= 0 && ir != 1 && jr != ny + 1) r7 = getres32(F, ir - 1, jr + 1, nmn);
            if (FB(ir, jr + 1) <= 0 && jr != ny + 1) r8 = getres32(F, ir, jr + 1, nmn);
#undef FB
            out = (4.0f * r9 + 2.0f * (r2 + r4 + r6 + r8) + r1 + r3 + r5 + r7) * 0.0625f;
        }
        C.r[t] = out;
    }
    const long long tot2 = (long long)W2 * (ny2 + 3);
    for (long long t = T.rank(); t < tot2; t += T.size()) C.e[t] = 0.0f;
}

template <class Team>
__device__ void prolong32(const Team &T, const MXL &C, const MXL &F) {
    const int W = F.nx + 3, nx2 = C.nx, ny2 = C.ny, W2 = nx2 + 3;
    const long long tot = (long long)(nx2 + 1) * (ny2 + 1);
    for (long long t = T.rank(); t < tot; t += T.size()) {
        int i = (int)(t % (nx2 + 1)) + 1, j = (int)(t / (nx2 + 1)) + 1;
        const float *e = C.e;
        float r1 = e[i + (long long)j * W2], r2 = e[i + (long long)(j - 1) * W2];
        float r3 = e[i - 1 + (long long)(j - 1) * W2], r4 = e[i - 1 + (long long)j * W2];
        long long n = (2 * i - 1) + (long long)(2 * j - 1) * W;
        float *u = F.e;
        const int8_t *bc = F.bc;
        if (bc[n] <= 0) u[n] += r1;
        if (bc[n - W] <= 0) u[n - W] += 0.5f * (r1 + r2);
        if (bc[n - W - 1] <= 0) u[n - W - 1] += 0.25f * (r1 + r2 + r3 + r4);
        if (bc[n - 1] <= 0) u[n - 1] += 0.5f * (r1 + r4);
    }
}

// finest level, FP64: r32 = b - A u (getres form) at unknowns, e = 0; returns ||r||^2 over
// bcnd == -1 nodes (5-point form) and the L1 sum of the reference's residual
template <class Team>
__device__ bool fine_residual(const Team &T, const MXP &P, double *rr, double *l1) {
    const MXL &L = P.L[0];
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    const double aw = L.awd, ae = L.awd, an = L.and_, as = L.and_, ac = L.acd;
    const long long tot = (long long)(nx + 1) * (ny + 1);
    double a = 0.0, s1 = 0.0;
    for (long long t = T.rank(); t < tot; t += T.size()) {
        int i = (int)(t % (nx + 1)) + 1, j = (int)(t / (nx + 1)) + 1;
        const long long n = i + (long long)j * W;
        const int bc = L.bc[n];
        float out = 0.0f;
        if (bc <= 0) {
            const double *u = L.u;
            double uw = u[n - 1], awx = aw, aex = ae;
            if (i == 1 && P.nmn == 1) { uw = 0.0; awx = 0.0; aex = 2.0 * ae; }
            double r = L.b[t] - (awx * uw + aex * u[n + 1] + an * u[n + W] + as * u[n - W] + ac * u[n]);
            out = (float)r;
            if (bc == -1) {
                double rs = L.b[t] - (aw * u[n - 1] + an * u[n + W] + as * u[n - W] + ae * u[n + 1] + ac * u[n]);
                a += rs * rs;
                s1 += fabs(rs);
            }
        }
        L.r[t] = out;
    }
    const long long nn = (long long)W * (ny + 3);
    for (long long t = T.rank(); t < nn; t += T.size()) L.e[t] = 0.0f;
    if (!team_sum(T, a, rr)) return false;
    return team_sum(T, s1, l1);
}

template <class Team>
__device__ bool b0_norm(const Team &T, const MXL &L, double *bb) {
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    const double aw = L.awd, an = L.and_;
    const long long tot = (long long)(nx + 1) * (ny + 1);
    double b = 0.0;
    for (long long t = T.rank(); t < tot; t += T.size()) {
        int i = (int)(t % (nx + 1)) + 1, j = (int)(t / (nx + 1)) + 1;
        const long long n = i + (long long)j * W;
        if (L.bc[n] != -1) continue;
        const double *u = L.u;
        const int8_t *bc = L.bc;
        double d = L.b[t] - ((bc[n - 1] > 0 ? aw * u[n - 1] : 0.0) + (bc[n + W] > 0 ? an * u[n + W] : 0.0) +
                             (bc[n - W] > 0 ? an * u[n - W] : 0.0) + (bc[n + 1] > 0 ? aw * u[n + 1] : 0.0));
        b += d * d;
    }
    return team_sum(T, b, bb);
}

__device__ void small_cycle(const MXP &P) {
    SmallTeam T;
    const int ng = P.ng;
    for (int l = P.Ls; l <= ng - 2; l++) {
        smooth32(T, P, l, P.nu1);
        restrict32(T, P.L[l], P.L[l + 1], P.pbc, P.nmn);
        __syncthreads();
    }
    smooth32(T, P, ng - 1, P.nuc);
    for (int l = ng - 2; l >= P.Ls; l--) {
        prolong32(T, P.L[l + 1], P.L[l]);
        __syncthreads();
        smooth32(T, P, l, P.nu2);
    }
}

__device__ bool vcycle32(const MXP &P) {
    BigTeam B{P.cnt, P.partials};
    const int ng = P.ng, Ls = P.Ls;
    for (int l = 0; l < Ls && l <= ng - 2; l++) {
        if (!smooth32(B, P, l, P.nu1)) return false;
        restrict32(B, P.L[l], P.L[l + 1], P.pbc, P.nmn);
        if (!B.sync()) return false;
    }
    int top;
    if (Ls <= ng - 1) {
        if (blockIdx.x == 0) small_cycle(P);
        if (!B.sync()) return false;
        top = Ls;
    } else {
        if (!smooth32(B, P, ng - 1, P.nuc)) return false;
        top = ng - 1;
    }
    for (int l = top - 1; l >= 0; l--) {
        prolong32(B, P.L[l + 1], P.L[l]);
        if (!B.sync()) return false;
        if (!smooth32(B, P, l, P.nu2)) return false;
    }
    return true;
}

__global__ void __launch_bounds__(MG_THREADS) k_mg_mixed(MXP P) {
    BigTeam B{P.cnt, P.partials};
    double bb = 0.0, rr = 0.0, l1 = 0.0;
    if (!b0_norm(B, P.L[0], &bb)) return;
    const double b0 = sqrt(bb);
    int outer = 0;
    for (;;) {
        if (!fine_residual(B, P, &rr, &l1)) return;
        if (sqrt(rr) <= P.eps * b0 || outer >= P.max_outer) break;
        if (!vcycle32(P)) return;
        const MXL &L = P.L[0];
        const long long nn = (long long)(L.nx + 3) * (L.ny + 3);
        for (long long t = B.rank(); t < nn; t += B.size())
            if (L.bc[t] <= 0) L.u[t] = L.u[t] + (double)L.e[t];
        if (!B.sync()) return;
        outer++;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.cnt->mg_cycles = outer;
        P.cnt->mg_sweeps_fine = outer * (P.nu1 + P.nu2);
        P.cnt->mg_res_l1 = l1 / P.alpha;
        P.cnt->mg_ktot = 0.0;
        P.cnt->mg_res_l2 = sqrt(rr);
        P.cnt->mg_b_l2 = b0;
        if (outer >= P.max_outer && !(sqrt(rr) <= P.eps * b0)) set_err(P.cnt, LERR_NOTCONV, 600);
    }
}

int mg_mixed_solve(lepic_ctx *c, double eps) {
    MXP P;
    memset(&P, 0, sizeof(P));
    const double eps0 = c->cfg.eps0;
    for (int l = 0; l < c->nlev; l++) {
        MGLevel &a = c->lev[l];
        MXL &d = P.L[l];
        d.nx = a.nx; d.ny = a.ny;
        double aw = eps0 / (a.hx * a.hx), an = eps0 / (a.hy * a.hy), ac = -(an + an + aw + aw);
        d.awd = aw; d.and_ = an; d.acd = ac;
        d.aw = (float)aw; d.an = (float)an; d.ac = (float)ac;
        d.e = a.e32; d.r = a.r32; d.bc = a.bc; d.u = a.u; d.b = a.b;
    }
    P.ng = c->nlev;
    long long small_nodes = 4500;
    if (const char *e = getenv("LEPIC_MG_SMALL_NODES")) small_nodes = atoll(e);
    int Ls = c->nlev;
    for (int l = 0; l < c->nlev; l++)
        if ((long long)(c->lev[l].nx + 1) * (c->lev[l].ny + 1) <= small_nodes) { Ls = l; break; }
    P.Ls = Ls;
    P.omega = 1.15f;
    P.nu1 = 2; P.nu2 = 2; P.nuc = 40; P.max_outer = 200;
    if (const char *e = getenv("LEPIC_MX_OMEGA")) P.omega = (float)atof(e);
    if (const char *e = getenv("LEPIC_MX_NU1")) P.nu1 = atoi(e);
    if (const char *e = getenv("LEPIC_MX_NU2")) P.nu2 = atoi(e);
    P.eps = eps;
    P.alpha = fabs((double)(c->cfg.nx + 1) * (c->cfg.ny + 1) * P.L[0].acd);
    P.pbc = c->cfg.flag_pbc;
    P.nmn = c->cfg.flag_nmn;
    P.partials = c->partials;
    P.cnt = c->dcnt;
    if (c->mg_grid_mixed == 0) {
        int occ = 0;
        LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mg_mixed, MG_THREADS, 0));
        if (occ < 1) { c->last_err = "mixed multigrid kernel does not fit on an SM"; return LEPIC_ECUDA; }
        int per_sm = 2;
        if (const char *e = getenv("LEPIC_MG_CTAS_PER_SM")) per_sm = atoi(e);
        c->mg_grid_mixed = c->num_sms * std::max(1, std::min(occ, per_sm));
    }
    void *args[] = {&P};
    LCUDA(cudaMemsetAsync(&c->dcnt->bar_count, 0, 3 * sizeof(unsigned int), c->stream));
    LCUDA(cudaLaunchCooperativeKernel((void *)k_mg_mixed, dim3(c->mg_grid_mixed), dim3(MG_THREADS), args, 0,
                                      c->stream));
    return LEPIC_OK;
}
