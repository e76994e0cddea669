// mg.cu -- the reference's Poisson solver (iterative_solver.f90 -> mg.f90 -> sors.f90) as
// ONE persistent cooperative kernel: every V-cycle, every red-black SOR sweep and every
// convergence decision runs on the device; no host round trip per sweep or per cycle.
//
// Compiled with -fmad=false: the SOR update, the residual and the restriction weights are
// rounded exactly as the Fortran expressions are written, so with the same sweep counts the
// result equals the FP64 CPU restatement bit for bit.  The L1 residual sums are reduced in a
// fixed order (per-thread, fixed block tree, fixed cross-block order), so a solve is
// reproducible run to run.
//
// Levels whose node count is at most `small_nodes` are processed by CTA 0 alone with
// block barriers; larger levels use the whole cooperative grid with a bounded software grid
// barrier.  Roofline: each fine-level half-sweep streams u (8 B, 5-point), b (8 B) and the
// int8 mask; at 2049^2 nodes the working set (u, b, mask: ~72 MB) is L2-resident, so the fine
// sweeps are L2-bandwidth bound and the coarse levels are barrier-latency bound.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include "lepic_internal.cuh"

struct MGDev {
    int nx, ny;
    double aw, an, ac;    // mg.h:11-15 (ae = aw, as = an)
    double hx, hy;
    double *u;
    double *b;
    const int8_t *bc;
};

struct MGP {
    MGDev L[LEPIC_MAXLEV];
    int ng, Ls;           // levels >= Ls are handled by CTA 0
    double omega, eps, alpha;
    int ncycl, pbc, nmn, mode;
    double *partials;
    DevCounters *cnt;
    unsigned bar_extra;        // lepic_options::barrier_extra
};

#include "mg_common.cuh"

// ---------------------------------------------------------------------------------------
// sors.f90:80-118 / :210-248, one colour.  red (color 0): i+j odd; black (color 1): i+j even.
template <class Team>
__device__ void half_sweep(const Team &T, const MGDev &L, int color, double omega) {
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    const double aw = L.aw, ae = L.aw, an = L.an, as = L.an, ac = L.ac;
    const int hw = nx / 2 + 1;
    for (Walk2 w(T.rank(), T.size(), hw, ny + 1); w.ok(); w.next()) {
        const int j = w.j + 1;
        const int is = (((j + 1 + color) & 1) != 0) ? 1 : 2;
        const int i = is + 2 * w.k;
        if (i > nx + 1) continue;
        const int n = i + j * W;
        int bc = L.bc[n];
        if (bc > 0) continue;
        double bij = L.b[(i - 1) + (j - 1) * (nx + 1)];
        double *u = L.u;
        if (bc == -2) {
            u[n] = (1.0 - omega) * u[n] + omega * (bij - an * u[n + W] - as * u[n - W] - 2.0 * ae * u[n + 1]) / ac;
            continue;
        }
        if (bc == 0 && j == ny + 1) continue;
        u[n] = (1.0 - omega) * u[n] +
               omega * (bij - aw * u[n - 1] - an * u[n + W] - as * u[n - W] - ae * u[n + 1]) / ac;
    }
}

// sors.f90:185-200 periodic ghost rows
template <class Team>
__device__ void pbc_rows(const Team &T, const MGDev &L) {
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    for (int i = (int)T.rank(); i <= nx + 2; i += (int)T.size()) {
        if (L.bc[i + 1 * W] <= 0) L.u[i] = L.u[i + ny * W];
        if (L.bc[i + (ny + 1) * W] <= 0) L.u[i + (ny + 1) * W] = L.u[i + W];
    }
}

// sors.f90:338-357 L1 residual over bcnd == -1 nodes
template <class Team>
__device__ bool residual_l1(const Team &T, const MGDev &L, double *res) {
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    const double aw = L.aw, ae = L.aw, an = L.an, as = L.an, ac = L.ac;
    double acc = 0.0;
    for (Walk2 w(T.rank(), T.size(), nx + 1, ny + 1); w.ok(); w.next()) {
        const int t = w.flat();
        const int n = (w.k + 1) + (w.j + 1) * W;
        double rij = 0.0;
        if (L.bc[n] == -1) {
            const double *u = L.u;
            rij = L.b[t] - (aw * u[n - 1] + an * u[n + W] + as * u[n - W] + ae * u[n + 1] + ac * u[n]);
        }
        acc = acc + fabs(rij);
    }
    return team_sum(T, acc, res);
}

// sors.f90:1-435 on one rank; returns false when a barrier failed
template <class Team>
__device__ bool sor_rb(const Team &T, const MGP &P, int l, int kmg, int dig, double *res_out,
                       int *ksor_out) {
    const MGDev &L = P.L[l];
    double res = 0.0, res_s = 0.0;
    int ksor = 0;
    int nr = 10;
    if (kmg == 1 && dig == 0) nr = 1000000;
    for (int k = 1; k <= nr; k++) {
        for (int color = 0; color < 2; color++) {
            half_sweep(T, L, color, P.omega);
            if (!T.sync()) return false;
            if (P.pbc) {
                pbc_rows(T, L);
                if (!T.sync()) return false;
            }
        }
        if (!residual_l1(T, L, &res)) return false;
        ksor = ksor + 1;
        if (dig == 0) {
            if (res <= P.eps * P.alpha) break;
        } else {
            if (res_s > 0.0 && (res / res_s) <= 0.6) break;
        }
        res_s = res;
    }
    *res_out = res;
    *ksor_out = ksor;
    return true;
}

// mg.f90:512-547
__device__ __forceinline__ double getres(const MGDev &L, int ir, int jr, int flag) {
    const int W = L.nx + 3;
    double aw = L.aw, ae = L.aw, an = L.an, as = L.an;
    const double ac = L.ac;
    const int n = ir + jr * W;
    const double *u = L.u;
    double uij = u[n], un = u[n + W], us = u[n - W], ue = u[n + 1], uw;
    if (ir == 1 && flag == 1) {
        uw = 0.0;
        aw = 0;
        ae = 2.0 * ae;
    } else {
        uw = u[n - 1];
    }
    double urhs = L.b[(ir - 1) + (jr - 1) * (L.nx + 1)];
    return urhs - (aw * uw + ae * ue + an * un + as * us + ac * uij);
}

// r_pbc(x) of mg.f90:298-311 (zero where the reference leaves it unset)
__device__ __forceinline__ double r_pbc(const MGDev &F, int x, int nmn) {
    const int W = F.nx + 3, ny = F.ny;
    bool set;
    if (x & 1) set = F.bc[x + (ny + 1) * W] <= 0;
    else set = (x - 1 >= 1 && F.bc[x - 1 + (ny + 1) * W] <= 0) ||
               (x + 1 <= F.nx + 1 && F.bc[x + 1 + (ny + 1) * W] <= 0);
    return set ? getres(F, x, ny, nmn) : 0.0;
}

// mg.f90:235-509 on one rank: full-weighting restriction of the fine residual, coarse
// correction zeroed (the coarse mask is the precomputed injection).
template <class Team>
__device__ void restriction(const Team &T, const MGDev &F, const MGDev &C, int pbc, int nmn) {
    const int nx = F.nx, ny = F.ny, W = nx + 3, nx2 = C.nx, ny2 = C.ny, W2 = nx2 + 3;
    for (Walk2 w(T.rank(), T.size(), nx2 + 1, ny2 + 1); w.ok(); w.next()) {
        const int t = w.flat();
        const int i = w.k + 1, j = w.j + 1;
        int ir = 2 * i - 1, jr = 2 * j - 1;
        double out = 0.0;
        if (C.bc[i + j * W2] <= 0) {
            double r1 = 0, r2 = 0, r3 = 0, r4 = 0, r5 = 0, r6 = 0, r7 = 0, r8 = 0, r9 = 0;
            const int8_t *bc = F.bc;
#define FB(a, b) bc[(a) + (b) * W]
            r9 = getres(F, ir, jr, nmn);
            if (ir != nx + 1 && jr != ny + 1)
                if (FB(ir + 1, jr + 1) <= 0) r1 = getres(F, ir + 1, jr + 1, nmn);
            if (ir != nx + 1)
                if (FB(ir + 1, jr) <= 0) r2 = getres(F, ir + 1, jr, nmn);
            if (FB(ir + 1, jr - 1) <= 0) {
                if (ir != nx + 1 && jr != 1) r3 = getres(F, ir + 1, jr - 1, nmn);
                else if (jr == 1) r3 = pbc ? r_pbc(F, ir + 1, nmn) : 0.0;
            }
            if (FB(ir, jr - 1) <= 0) {
                if (jr != 1) r4 = getres(F, ir, jr - 1, nmn);
                else r4 = pbc ? r_pbc(F, ir, nmn) : 0.0;
            }
            if (FB(ir - 1, jr - 1) <= 0 && ir != 1) {
                if (jr != 1) r5 = getres(F, ir - 1, jr - 1, nmn);
                else r5 = pbc ? r_pbc(F, ir - 1, nmn) : 0.0;
            }
            if (FB(ir - 1, jr) <= 0)
                if (ir != 1) r6 = getres(F, ir - 1, jr, nmn);
            if (FB(ir - 1, jr + 1) <= 0)
                if (ir != 1 && jr != ny + 1) r7 = getres(F, ir - 1, jr + 1, nmn);
            if (FB(ir, jr + 1) <= 0)
                if (jr != ny + 1) r8 = getres(F, ir, jr + 1, nmn);
#undef FB
            out = (4.0 * r9 + 2.0 * (r2 + r4 + r6 + r8) + r1 + r3 + r5 + r7) / 16.0;
        }
        C.b[t] = out;
    }
    const int tot2 = W2 * (ny2 + 3);
    for (int t = (int)T.rank(); t < tot2; t += (int)T.size()) C.u[t] = 0.0;
}

// mg.f90:549-616 (each fine node has exactly one writer)
template <class Team>
__device__ void prolongation(const Team &T, const MGDev &C, const MGDev &F) {
    const int W = F.nx + 3, nx2 = C.nx, ny2 = C.ny, W2 = nx2 + 3;
    for (Walk2 w(T.rank(), T.size(), nx2 + 1, ny2 + 1); w.ok(); w.next()) {
        const int i = w.k + 1, j = w.j + 1;
        const double *e = C.u;
        double r1 = e[i + j * W2], r2 = e[i + (j - 1) * W2];
        double r3 = e[i - 1 + (j - 1) * W2], r4 = e[i - 1 + j * W2];
        int ir = 2 * i - 1, jr = 2 * j - 1;
        double *u = F.u;
        const int8_t *bc = F.bc;
        const int n = ir + jr * W;
        if (bc[n] <= 0) u[n] = u[n] + r1;
        if (bc[n - W] <= 0) u[n - W] = u[n - W] + (r1 + r2) / 2.0;
        if (bc[n - W - 1] <= 0) u[n - W - 1] = u[n - W - 1] + (r1 + r2 + r3 + r4) / 4.0;
        if (bc[n - 1] <= 0) u[n - 1] = u[n - 1] + (r1 + r4) / 2.0;
    }
}

// The part of a V-cycle on levels >= Ls, run by CTA 0: S(Ls)..R.. S*(ng-1) P.. S(Ls)
__device__ void small_region(const MGP &P, int k, double *res, int *iter) {
    SmallTeam T;
    int ks;
    const int ng = P.ng;
    for (int l = P.Ls; l <= ng - 2; l++) {
        sor_rb(T, P, l, k, l + 1 - ng, res, &ks);
        iter[l] += ks;
        restriction(T, P.L[l], P.L[l + 1], P.pbc, P.nmn);
        __syncthreads();
    }
    sor_rb(T, P, ng - 1, k, 0, res, &ks);
    iter[ng - 1] += ks;
    if (ng - 1 > P.Ls) {
        prolongation(T, P.L[ng - 1], P.L[ng - 2]);
        __syncthreads();
    }
    for (int l = ng - 2; l >= P.Ls; l--) {
        sor_rb(T, P, l, k, ng - l - 1, res, &ks);
        iter[l] += ks;
        if (l > P.Ls) {
            prolongation(T, P.L[l], P.L[l - 1]);
            __syncthreads();
        }
    }
}

// mg.f90:85-225 -- one V-cycle; *res is the L1 residual of the last finest-level sweep
__device__ bool vcycle(const MGP &P, int k, double *res, int *iter) {
    BigTeam B{P.cnt, P.partials, P.bar_extra};
    const int ng = P.ng, Ls = P.Ls;
    int ks;
    for (int l = 0; l < Ls && l <= ng - 2; l++) {
        if (!sor_rb(B, P, l, k, l + 1 - ng, res, &ks)) return false;
        iter[l] += ks;
        restriction(B, P.L[l], P.L[l + 1], P.pbc, P.nmn);
        if (!B.sync()) return false;
    }
    int top;
    if (Ls <= ng - 1) {
        if (blockIdx.x == 0) {
            double r = 0.0;
            small_region(P, k, &r, iter);
            if (threadIdx.x == 0) P.cnt->mg_res_l1 = r;
        }
        if (!B.sync()) return false;
        *res = ((volatile double *)&P.cnt->mg_res_l1)[0];
        top = Ls;
    } else {
        if (!sor_rb(B, P, ng - 1, k, 0, res, &ks)) return false;
        iter[ng - 1] += ks;
        top = ng - 1;
    }
    if (top >= 1) {
        prolongation(B, P.L[top], P.L[top - 1]);
        if (!B.sync()) return false;
    }
    for (int l = top - 1; l >= 0; l--) {
        if (!sor_rb(B, P, l, k, ng - l - 1, res, &ks)) return false;
        iter[l] += ks;
        if (l >= 1) {
            prolongation(B, P.L[l], P.L[l - 1]);
            if (!B.sync()) return false;
        }
    }
    return true;
}

// ||b - A u||_2^2 and ||b - A u_D||_2^2 (u_D: u with the unknowns zeroed) over bcnd == -1
template <class Team>
__device__ bool l2_norms(const Team &T, const MGDev &L, double *rr, double *bb) {
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    const double aw = L.aw, ae = L.aw, an = L.an, as = L.an, ac = L.ac;
    double a = 0.0, b = 0.0;
    for (Walk2 w(T.rank(), T.size(), nx + 1, ny + 1); w.ok(); w.next()) {
        const int t = w.flat();
        const int n = (w.k + 1) + (w.j + 1) * W;
        if (L.bc[n] != -1) continue;
        const double *u = L.u;
        const int8_t *bc = L.bc;
        double r = L.b[t] - (aw * u[n - 1] + an * u[n + W] + as * u[n - W] + ae * u[n + 1] + ac * u[n]);
        double d = L.b[t] - ((bc[n - 1] > 0 ? aw * u[n - 1] : 0.0) + (bc[n + W] > 0 ? an * u[n + W] : 0.0) +
                             (bc[n - W] > 0 ? as * u[n - W] : 0.0) + (bc[n + 1] > 0 ? ae * u[n + 1] : 0.0));
        a = a + r * r;
        b = b + d * d;
    }
    if (!team_sum(T, a, rr)) return false;
    return team_sum(T, b, bb);
}

// iterative_solver.f90:18-66.  mode 0: stop on the reference's normalised L1 residual;
// mode 2: same cycles, stop on ||b-Au||_2/||b-Au_D||_2 <= eps.
__global__ void __launch_bounds__(MG_THREADS) k_mg_solve(MGP P) {
    BigTeam B{P.cnt, P.partials, P.bar_extra};
    int iter[LEPIC_MAXLEV];
    for (int i = 0; i < LEPIC_MAXLEV; i++) iter[i] = 0;
    double res = 0.0, res_s = 0.0, rr = 0.0, bb = 0.0;
    int k = 1;
    if (P.mode == 2 && !l2_norms(B, P.L[0], &rr, &bb)) return;
    const double b0 = sqrt(bb);
    bool conv = false;
    for (;;) {
        if (!vcycle(P, k, &res, iter)) return;
        res = res / P.alpha;
        bool diverged = false;
        if (k == 1) res_s = res;
        else if (fabs(res / res_s) > 10.0) diverged = true;
        if (diverged) {
            if (blockIdx.x == 0 && threadIdx.x == 0) set_err(P.cnt, LERR_DIVERGED, 500);
            return; // every CTA takes the same decision
        }
        if (P.mode == 2) {
            if (!l2_norms(B, P.L[0], &rr, &bb)) return;
            conv = sqrt(rr) <= P.eps * b0;
        } else {
            conv = res <= P.eps;
        }
        if (conv || k == P.ncycl) break;
        k = k + 1;
    }
    if (!l2_norms(B, P.L[0], &rr, &bb)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // ncycl cycles without reaching eps: the reference goes on with this potential
        // (iterative_solver.f90:56); the call reports it and phi holds the last cycle's result
        if (!conv) set_err(P.cnt, LERR_NOTCONV, 501);
        double ktot = 0.0;
        for (int i = 1; i <= P.ng; i++) ktot = ktot + (double)iter[i - 1] / pow(2.0, 2 * (i - 1));
        P.cnt->mg_cycles = k;
        P.cnt->mg_sweeps_fine = iter[0];
        P.cnt->mg_res_l1 = res;
        P.cnt->mg_ktot = ktot;
        P.cnt->mg_res_l2 = sqrt(rr);
        P.cnt->mg_b_l2 = sqrt(bb);
    }
}

// Stats only: the L1 and L2 residuals of the current phi.
__global__ void __launch_bounds__(MG_THREADS) k_mg_stats(MGP P) {
    BigTeam B{P.cnt, P.partials, P.bar_extra};
    double res = 0.0, rr = 0.0, bb = 0.0;
    if (!residual_l1(B, P.L[0], &res)) return;
    if (!l2_norms(B, P.L[0], &rr, &bb)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.cnt->mg_res_l1 = res / P.alpha;
        P.cnt->mg_res_l2 = sqrt(rr);
        P.cnt->mg_b_l2 = sqrt(bb);
    }
}

// ---------------------------------------------------------------------------------------
static MGP mg_params(lepic_ctx *c, double eps, int mode) {
    MGP P;
    memset(&P, 0, sizeof(P));
    const double eps0 = c->cfg.eps0;
    for (int l = 0; l < c->nlev; l++) {
        MGLevel &a = c->lev[l];
        MGDev &d = P.L[l];
        d.nx = a.nx; d.ny = a.ny; d.hx = a.hx; d.hy = a.hy;
        d.aw = eps0 / (a.hx * a.hx);
        d.an = eps0 / (a.hy * a.hy);
        d.ac = -(d.an + d.an + d.aw + d.aw);
        d.u = a.u; d.b = a.b; d.bc = a.bc;
    }
    P.ng = c->nlev;
    const long long small_nodes = c->opt.mg_small_nodes;
    int Ls = c->nlev;
    for (int l = 0; l < c->nlev; l++)
        if ((long long)(c->lev[l].nx + 1) * (c->lev[l].ny + 1) <= small_nodes) { Ls = l; break; }
    P.Ls = Ls;
    P.omega = c->cfg.omega;
    P.eps = eps;
    P.alpha = fabs((double)(c->cfg.nx + 1) * (c->cfg.ny + 1) * P.L[0].ac) * 1.0;
    P.ncycl = c->cfg.ncycl;
    P.pbc = c->cfg.flag_pbc;
    P.nmn = c->cfg.flag_nmn;
    P.mode = mode;
    P.partials = c->partials;
    P.cnt = c->dcnt;
    P.bar_extra = (unsigned)c->opt.barrier_extra;
    return P;
}

int mg_init(lepic_ctx *c) {
    int occ = 0;
    LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mg_solve, MG_THREADS, 0));
    if (occ < 1) { c->last_err = "multigrid kernel does not fit on an SM"; return LEPIC_ECUDA; }
    c->mg_grid = c->num_sms * std::max(1, std::min(occ, (int)c->opt.ctas_per_sm));
    return LEPIC_OK;
}

static int launch_coop(lepic_ctx *c, void *fn, int grid, MGP &P) {
    void *args[] = {&P};
    LCUDA(cudaMemsetAsync(&c->dcnt->bar_arrived, 0, sizeof(unsigned long long) + sizeof(int), c->stream));
    LCUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(MG_THREADS), args, 0, c->stream));
    return LEPIC_OK;
}

int mg_solve(lepic_ctx *c, double eps, int mode) {
    MGP P = mg_params(c, eps, mode);
    return launch_coop(c, (void *)k_mg_solve, c->mg_grid, P);
}

int mg_residual_stats(lepic_ctx *c) {
    MGP P = mg_params(c, 0.0, 0);
    return launch_coop(c, (void *)k_mg_stats, c->mg_grid, P);
}
