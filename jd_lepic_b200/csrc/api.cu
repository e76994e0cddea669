// api.cu -- the C ABI (include/lepic_gpu.h): context, particle I/O, the device loader and the
// step driver.  Every entry point returns a status and never aborts; device-side failures
// are raised as bits in DevCounters::err and reported by the next synchronising call.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#include "cnn.cuh"

#define LEPIC_ABI_VERSION 4

extern "C" int32_t lepic_gpu_abi_version(void) { return LEPIC_ABI_VERSION; }

static int ceil_log2(long long v) {
    int k = 0;
    while ((1ll << k) < v) k++;
    return k;
}

template <class T>
static int dalloc(lepic_ctx *c, T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void **)p, sizeof(T) * count);
    if (e != cudaSuccess) {
        c->last_err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        *p = nullptr;
        return LEPIC_ENOMEM;
    }
    return LEPIC_OK;
}
#define LALLOC(ptr, n)                      \
    do {                                    \
        int _r = dalloc(c, &(ptr), (n));    \
        if (_r != LEPIC_OK) return _r;      \
    } while (0)

static void free_all(lepic_ctx *c) {
    auto F = [](void *p) { if (p) cudaFree(p); };
    F(c->bcnd); F(c->bc8); F(c->cellwall); F(c->cellwall_w); F(c->kq); F(c->Bf); F(c->phi); F(c->rhs); F(c->Ed_base); F(c->Ef);
    F(c->ss_diag); F(c->phi_hist); F(c->uB); F(c->dq); F(c->rf_ev); F(c->sec_ev); F(c->ev_count);
    F(c->npd); F(c->np_red); F(c->np_mx);
    for (int s = 0; s < LEPIC_MAXSP; s++) {
        SpeciesBuf &B = c->sp[s];
        for (int k = 0; k < 2; k++) { F(B.X[k]); F(B.Y[k]); F(B.VX[k]); F(B.VY[k]); F(B.VZ[k]); F(B.Z[k]); }
        F(B.acc); F(B.items); F(B.prod); F(B.cell_off); F(B.claim); F(B.pind);
    }
    F(c->keys); F(c->perm); F(c->counts); F(c->offsets); F(c->cursor); F(c->blocksums); F(c->bigseg);
    for (int l = 0; l < c->nlev; l++) {
        if (l > 0) { F(c->lev[l].u); F(c->lev[l].b); F(c->lev[l].bc); }
        F(c->lev[l].e32); F(c->lev[l].e32b); F(c->lev[l].r32);
        F(c->lev[l].e64); F(c->lev[l].e64b); F(c->lev[l].r64);
    }
    F(c->partials);
    F(c->cg_r); F(c->cg_p); F(c->cg_ap); F(c->mx_cinv); F(c->mx_cinv64); F(c->mx_cidx);
    F(c->sig_Er); F(c->sig); F(c->Eth); F(c->col_info); F(c->prod_sort);
    F(c->dcnt); F(c->tally); F(c->rg_scratch); F(c->rg_kfac); F(c->sigv_mx_d); F(c->nu_max_d);
    if (c->hcnt) cudaFreeHost(c->hcnt);
    if (c->cstream) { cudaStreamSynchronize(c->cstream); cudaStreamDestroy(c->cstream); }
    if (c->ev_snap) cudaEventDestroy(c->ev_snap);
    if (c->ev_down) cudaEventDestroy(c->ev_down);
    if (c->ev_up) cudaEventDestroy(c->ev_up);
    F(c->snap);
    if (c->stream) cudaStreamDestroy(c->stream);
}

static int create_impl(lepic_ctx *c, const lepic_config *cfg, const int32_t *bcnd, const double *phi_init,
                       const double *Bi, const lepic_xs_tables *xs) {
    c->cfg = *cfg;
    const lepic_config &g = c->cfg;
    if (g.nx < 2 || g.ny < 2 || g.dx <= 0 || g.dy <= 0 || g.zmax <= 0 || g.dt <= 0 || g.ntype < 1 ||
        g.ntype > LEPIC_MAXSP || g.nsp < g.ntype || g.nsp > LEPIC_MAXSP || g.ng < 1 || g.ng > LEPIC_MAXLEV ||
        !bcnd || !phi_init) {
        c->last_err = "invalid configuration";
        return LEPIC_EINVAL;
    }
    if ((long long)(g.nx + 3) * (g.ny + 3) >= (1ll << 30)) { // node indices are 32-bit in the solvers
        c->last_err = "grid too large: (nx+3)*(ny+3) must stay below 2^30 nodes";
        return LEPIC_EINVAL;
    }
    if ((g.nx % (1 << (g.ng - 1))) != 0 || (g.ny % (1 << (g.ng - 1))) != 0) {
        c->last_err = "nx and ny must be divisible by 2^(ng-1) (main.f90:268-277)";
        return LEPIC_EINVAL;
    }
    if (g.flag_B == 2 && !Bi) { c->last_err = "flag_B = 2 needs a B map"; return LEPIC_EINVAL; }
    for (int s = 0; s < g.ntype; s++)
        if (g.capacity[s] < 1 || g.capacity[s] > 0x7fffff00ll) { c->last_err = "capacity out of range"; return LEPIC_EINVAL; }
    LCUDA(cudaGetDevice(&c->dev));
    cudaDeviceProp prop;
    LCUDA(cudaGetDeviceProperties(&prop, c->dev));
    if (prop.major < 10) { c->last_err = "this library is built for sm_100a (B200)"; return LEPIC_ENOKERNEL; }
    c->num_sms = prop.multiProcessorCount;
    LCUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const int nx = g.nx, ny = g.ny;
    c->S = std::min(24, 32 - ceil_log2(std::max(nx, ny)));
    c->nn = (long long)(nx + 3) * (ny + 3);
    if (g.tile_w > 0 && g.tile_h > 0) { c->tw = std::min(g.tile_w, nx); c->th = std::min(g.tile_h, ny); }
    else { c->tw = nx; c->th = 1; }
    c->ntx = (nx + c->tw - 1) / c->tw;
    c->nty = (ny + c->th - 1) / c->th;
    c->ntiles = c->ntx * c->nty;
    c->nkeys = (long long)c->ntiles * c->tw * c->th;
    const long long nn = c->nn;
    const int W = nx + 3;
    // static grids
    std::vector<int8_t> bc8(nn);
    std::vector<double> kq(nn);
    for (long long n = 0; n < nn; n++) {
        int b = bcnd[n];
        bc8[n] = (int8_t)std::max(-4, std::min(1, b));
        kq[n] = (b != -1) ? 2.0 : 1.0; // main.f90:334-344
    }
    std::vector<uint8_t> cw((size_t)(nx + 2) * (ny + 2));
    std::vector<uint8_t> cww((size_t)W * (ny + 2), 0);   // the same with the node rows' stride
    for (int iy = 0; iy <= ny + 1; iy++)
        for (int ix = 0; ix <= nx + 1; ix++) {
            bool wall = bcnd[ix + iy * W] >= 1 && bcnd[ix + 1 + iy * W] >= 1 && bcnd[ix + 1 + (iy + 1) * W] >= 1 &&
                        bcnd[ix + (iy + 1) * W] >= 1;
            cw[ix + (size_t)iy * (nx + 2)] = wall ? 1 : 0;
            cww[ix + (size_t)iy * W] = wall ? 1 : 0;
        }
    // the masks are 16 bytes longer: the mixed solver's tiles read them in whole words
    LALLOC(c->bcnd, nn); LALLOC(c->bc8, nn + 16); LALLOC(c->cellwall, cw.size()); LALLOC(c->cellwall_w, cww.size()); LALLOC(c->kq, nn);
    LCUDA(cudaMemcpy(c->bcnd, bcnd, sizeof(int32_t) * nn, cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(c->bc8, bc8.data(), nn, cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(c->cellwall, cw.data(), cw.size(), cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(c->cellwall_w, cww.data(), cww.size(), cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(c->kq, kq.data(), sizeof(double) * nn, cudaMemcpyHostToDevice));
    if (g.flag_B == 2) {
        std::vector<float4> bf(nn);
        for (long long n = 0; n < nn; n++)
            bf[n] = make_float4((float)Bi[4 * n], (float)Bi[4 * n + 1], (float)Bi[4 * n + 2], (float)Bi[4 * n + 3]);
        LALLOC(c->Bf, nn);
        LCUDA(cudaMemcpy(c->Bf, bf.data(), sizeof(float4) * nn, cudaMemcpyHostToDevice));
    }
    LALLOC(c->phi, nn); LALLOC(c->rhs, (size_t)(nx + 1) * (ny + 1));
    LALLOC(c->Ed_base, 2 * nn); LALLOC(c->Ef, nn);
    c->Ed = c->Ed_base;
    LALLOC(c->npd, nn); LALLOC(c->np_red, (size_t)g.ntype * nn); LALLOC(c->np_mx, LEPIC_MAXSP);
    LCUDA(cudaMemcpy(c->phi, phi_init, sizeof(double) * nn, cudaMemcpyHostToDevice));
    {
        double m = 0.0;
        for (long long n = 0; n < nn; n++) m = std::max(m, fabs(phi_init[n]));
        c->phi_scale = m > 0.0 ? m : 1.0;
        long long cnt = 0;
        for (int j = 1; j <= ny + 1; j++)
            for (int i = 1; i <= nx + 1; i++) cnt += bcnd[i + (long long)j * (nx + 3)] <= 0;
        c->n_unknown = cnt;
    }
    LCUDA(cudaMemset(c->rhs, 0, sizeof(double) * (nx + 1) * (ny + 1)));
    LCUDA(cudaMemset(c->Ed_base, 0, sizeof(double2) * 2 * nn));
    LCUDA(cudaMemset(c->Ef, 0, sizeof(float4) * nn));
    // particles
    long long maxcap = 0;
    for (int s = 0; s < g.ntype; s++) {
        SpeciesBuf &B = c->sp[s];
        B.cap = g.capacity[s];
        maxcap = std::max(maxcap, B.cap);
        // storage rounded up to whole groups of 8 slots: the push reads and writes 8 consecutive
        // slots per thread with 16-byte vectors (the capacity itself is unchanged)
        const long long cap8 = (B.cap + 7) / 8 * 8;
        for (int k = 0; k < 2; k++) {
            LALLOC(B.X[k], cap8); LALLOC(B.Y[k], cap8);
            LALLOC(B.VX[k], cap8); LALLOC(B.VY[k], cap8); LALLOC(B.VZ[k], cap8);
        }
        B.cur = 0;
        LALLOC(B.acc, nn);
        LCUDA(cudaMemset(B.acc, 0, sizeof(unsigned long long) * nn));
        B.max_items = c->ntiles + (int)(B.cap / 2048) + 16;
        LALLOC(B.items, B.max_items);
        B.prod_cap = (int)std::min<long long>(1 << 24, std::max<long long>(65536, B.cap / 50));
        LALLOC(B.prod, B.prod_cap);
    }
    c->scratch_cap = maxcap;
    LALLOC(c->keys, maxcap); LALLOC(c->perm, maxcap);
    LALLOC(c->counts, c->nkeys + 1); LALLOC(c->offsets, c->nkeys + 1); LALLOC(c->cursor, c->nkeys + 1);
    LALLOC(c->blocksums, (c->nkeys + 2047) / 2048 + 1); LALLOC(c->bigseg, c->nkeys + 1);
    // multigrid levels (level 0 shares phi, rhs and the mask)
    c->nlev = g.ng;
    std::vector<int8_t> prev = bc8;
    for (int l = 0; l < c->nlev; l++) {
        MGLevel &L = c->lev[l];
        memset(&L, 0, sizeof(L));
        L.nx = nx >> l; L.ny = ny >> l;
        L.hx = g.dx * (double)(1 << l); L.hy = g.dy * (double)(1 << l);
        long long nnl = (long long)(L.nx + 3) * (L.ny + 3);
        if (l == 0) {
            L.u = c->phi; L.b = c->rhs; L.bc = c->bc8;
        } else {
            const int Wf = c->lev[l - 1].nx + 3, W2 = L.nx + 3;
            const int nxf = c->lev[l - 1].nx, nyf = c->lev[l - 1].ny;
            std::vector<int8_t> cur(nnl, 1);
            for (int j = 1; j <= L.ny + 1; j++)
                for (int i = 1; i <= L.nx + 1; i++) {
                    int ir = 2 * i - 1, jr = 2 * j - 1;
                    cur[i + j * W2] = prev[ir + jr * Wf];
                    if (ir == 1) cur[0 + j * W2] = prev[0 + jr * Wf];
                    if (ir == nxf + 1) cur[L.nx + 2 + j * W2] = prev[nxf + 2 + jr * Wf];
                    if (jr == 1) cur[i + 0 * W2] = prev[ir + 0 * Wf];
                    if (jr == nyf + 1) cur[i + (L.ny + 2) * W2] = prev[ir + (nyf + 2) * Wf];
                }
            cur[0] = prev[0];
            cur[L.nx + 2] = prev[nxf + 2];
            cur[(L.ny + 2) * W2] = prev[(nyf + 2) * Wf];
            cur[L.nx + 2 + (L.ny + 2) * W2] = prev[nxf + 2 + (nyf + 2) * Wf];
            LALLOC(L.u, nnl); LALLOC(L.b, (size_t)(L.nx + 1) * (L.ny + 1)); LALLOC(L.bc, nnl + 16);
            LCUDA(cudaMemset(L.u, 0, sizeof(double) * nnl));
            LCUDA(cudaMemset(L.b, 0, sizeof(double) * (L.nx + 1) * (L.ny + 1)));
            LCUDA(cudaMemcpy(L.bc, cur.data(), nnl, cudaMemcpyHostToDevice));
            prev.swap(cur);
        }
        LALLOC(L.e32, nnl); LALLOC(L.e32b, nnl); LALLOC(L.r32, (size_t)(L.nx + 1) * (L.ny + 1));
        LCUDA(cudaMemset(L.e32, 0, sizeof(float) * nnl));
        LCUDA(cudaMemset(L.e32b, 0, sizeof(float) * nnl));
        LCUDA(cudaMemset(L.r32, 0, sizeof(float) * (L.nx + 1) * (L.ny + 1)));
    }
    // grid-wide sums: up to 3 values x 2 halves per CTA of a cooperative grid of at most 8 CTAs
    // of 256 threads per SM
    LALLOC(c->partials, (size_t)c->num_sms * 48);
    LALLOC(c->cg_r, nn); LALLOC(c->cg_p, nn); LALLOC(c->cg_ap, nn);
    LCUDA(cudaMemset(c->cg_r, 0, sizeof(double) * nn));
    LCUDA(cudaMemset(c->cg_p, 0, sizeof(double) * nn));
    LCUDA(cudaMemset(c->cg_ap, 0, sizeof(double) * nn));
    // collision tables
    if (xs && xs->ncol > 0 && xs->npt > 1) {
        c->has_xs = true;
        c->npt = xs->npt; c->ncol = xs->ncol;
        LALLOC(c->sig_Er, xs->npt); LALLOC(c->sig, (size_t)xs->npt * xs->ncol); LALLOC(c->Eth, xs->ncol);
        LALLOC(c->col_info, (size_t)xs->ncol * 10);
        LCUDA(cudaMemcpy(c->sig_Er, xs->sig_Er, sizeof(double) * xs->npt, cudaMemcpyHostToDevice));
        LCUDA(cudaMemcpy(c->sig, xs->sig, sizeof(double) * xs->npt * xs->ncol, cudaMemcpyHostToDevice));
        LCUDA(cudaMemcpy(c->Eth, xs->Eth, sizeof(double) * xs->ncol, cudaMemcpyHostToDevice));
        LCUDA(cudaMemcpy(c->col_info, xs->col_info, sizeof(int) * xs->ncol * 10, cudaMemcpyHostToDevice));
        for (int s = 0; s < g.nsp; s++) {
            c->p_ncol[s] = xs->p_ncol[s];
            if (xs->p_ncol[s] > 16 || xs->p_ncol[s] < 0) {
                c->last_err = "more than 16 reactions for one incident species";
                return LEPIC_EINVAL;
            }
            for (int q = 0; q < xs->p_ncol[s]; q++) c->hsig_list[s * LEPIC_MAXCOL + q] = xs->sig_list[s * LEPIC_MAXCOL + q];
        }
        // collisions.f90:98-106 with neutral targets: nu_max = min(sum n_t*(sigma v)_max, nu_uplim)
        for (int s = 0; s < g.ntype; s++) {
            double nu = 0.0;
            for (int q = 0; q < c->p_ncol[s]; q++) {
                int ic = c->hsig_list[s * LEPIC_MAXCOL + q];
                int n_re = xs->col_info[ic * 10 + 0];
                int tt = xs->col_info[ic * 10 + 2 + n_re - 1];
                nu = nu + g.np_mx[tt] * xs->sigv_mx[s * LEPIC_MAXCOL + ic];
            }
            c->nu_max[s] = std::min(nu, g.nu_uplim[s]);
        }
        for (int ic = 0; ic < xs->ncol && ic < LEPIC_MAXCOL; ic++) {
            const int n_re = xs->col_info[ic * 10 + 0];
            c->hcol_tt[ic] = xs->col_info[ic * 10 + 2 + n_re - 1];
        }
        // charged targets (DSMC): per-cell lists of the target species and a claim per slot
        for (int s = 0; s < g.ntype; s++)
            for (int q = 0; q < c->p_ncol[s]; q++) {
                const int ic = c->hsig_list[s * LEPIC_MAXCOL + q];
                const int n_re = xs->col_info[ic * 10 + 0];
                const int tt = xs->col_info[ic * 10 + 2 + n_re - 1];
                if (tt < g.ntype && g.charge[tt] != 0.0 && g.mass[s] > 0.0) {
                    c->dsmc = true;
                    SpeciesBuf &T = c->sp[tt];
                    if (!T.cell_off) LALLOC(T.cell_off, c->nkeys + 1);
                    if (!T.claim) LALLOC(T.claim, T.cap);
                }
            }
        LALLOC(c->sigv_mx_d, LEPIC_MAXSP * LEPIC_MAXCOL);
        LALLOC(c->nu_max_d, LEPIC_MAXSP);
        LCUDA(cudaMemcpy(c->sigv_mx_d, xs->sigv_mx, sizeof(double) * LEPIC_MAXSP * LEPIC_MAXCOL, cudaMemcpyHostToDevice));
        for (int s = 0; s < LEPIC_MAXSP; s++)
            if (c->sp[s].cell_off) LCUDA(cudaMemset(c->sp[s].cell_off, 0, sizeof(int) * (c->nkeys + 1)));
        c->flag_ionrep = xs->flag_ionrep;
        c->fEk = xs->fEk;
        int pmax = 1;
        for (int s = 0; s < g.ntype; s++) pmax = std::max(pmax, c->sp[s].prod_cap);
        LALLOC(c->prod_sort, pmax);
    }
    LALLOC(c->dcnt, 1);
    LCUDA(cudaMemset(c->dcnt, 0, sizeof(DevCounters)));
    LALLOC(c->tally, 1);
    LCUDA(cudaMemset(c->tally, 0, sizeof(TallyDev)));
    LALLOC(c->rg_scratch, 2 * LEPIC_MAXRG);
    LALLOC(c->rg_kfac, LEPIC_MAXSP);
    LCUDA(cudaMallocHost((void **)&c->hcnt, sizeof(DevCounters)));
    memset(c->hcnt, 0, sizeof(DevCounters));
    int r = mg_init(c);
    if (r != LEPIC_OK) return r;
    LCUDA(cudaDeviceSynchronize());
    return LEPIC_OK;
}

static lepic_options default_options() {
    lepic_options o;
    memset(&o, 0, sizeof(o));
    o.mx_nu1 = 2; o.mx_nu2 = 2; o.mx_nuc = 2;
    o.mx_omega = 1.15f;
    o.mx_onchip_bytes = 20 * 1024;
    o.mx_tiled = 1;
    o.mx_max_iter = 200;
    o.mx_coarse_direct = 1;
    o.mg_small_nodes = 4500;
    o.ctas_per_sm = 3;
    o.barrier_extra = 0;
    o.fortran_max_subrecord = 2147483639ll;
    o.sort_defer = 1;
    return o;
}

extern "C" int lepic_gpu_get_options(lepic_ctx *c, lepic_options *out) {
    if (!c || !out) return LEPIC_EINVAL;
    *out = c->opt;
    return LEPIC_OK;
}

extern "C" int lepic_gpu_set_options(lepic_ctx *c, const lepic_options *in) {
    if (!c || !in) return LEPIC_EINVAL;
    const lepic_options &o = *in;
    if (o.mx_nu1 < 1 || o.mx_nu1 > 8 || o.mx_nu2 < 1 || o.mx_nu2 > 8 || o.mx_nuc < 1 || o.mx_nuc > 64 ||
        !(o.mx_omega > 0.0f && o.mx_omega < 2.0f) || o.mx_onchip_bytes < 0 || o.mx_onchip_bytes > 96 * 1024 ||
        (o.mx_tiled != 0 && o.mx_tiled != 1) || o.mx_max_iter < 1 ||
        (o.mx_coarse_direct != 0 && o.mx_coarse_direct != 1) || o.mg_small_nodes < 0 || o.ctas_per_sm < 1 ||
        o.ctas_per_sm > 8 || o.barrier_extra < 0 || o.barrier_extra > 1024 || o.fortran_max_subrecord < 8 ||
        o.fortran_max_subrecord > 2147483639ll || (o.sort_defer != 0 && o.sort_defer != 1)) {
        c->last_err = "set_options: a value is out of range";
        return LEPIC_EINVAL;
    }
    // the work list of a cooperative launch depends on these: wait for launches in flight
    LCUDA(cudaStreamSynchronize(c->stream));
    const bool relaunch = o.ctas_per_sm != c->opt.ctas_per_sm;
    c->opt = o;
    if (relaunch) {
        c->mg_grid_mixed = 0;  // sized again at the next mixed solve
        c->mg_grid_mixed64 = 0;
        int r = mg_init(c);
        if (r != LEPIC_OK) return r;
    }
    return LEPIC_OK;
}

// the reason of the last failed lepic_gpu_create (lepic_gpu_last_error(NULL))
static std::string g_create_err = "no context";

extern "C" int lepic_gpu_create(const lepic_config *cfg, const int32_t *bcnd, const double *phi_init,
                                const double *Bi, const lepic_xs_tables *xs, lepic_ctx **out) {
    if (!cfg || !out) return LEPIC_EINVAL;
    *out = nullptr;
    lepic_ctx *c = new (std::nothrow) lepic_ctx();
    if (!c) return LEPIC_ENOMEM;
    c->opt = default_options();
    int r = create_impl(c, cfg, bcnd, phi_init, Bi, xs);
    if (r != LEPIC_OK) {
        g_create_err = "lepic_gpu_create: " + c->last_err;
        free_all(c);
        delete c;
        return r;
    }
    *out = c;
    return LEPIC_OK;
}

extern "C" int lepic_gpu_destroy(lepic_ctx *c) {
    if (!c) return LEPIC_EINVAL;
    cudaStreamSynchronize(c->stream);
    learn_free(c);
    sources_free(c);
    avg_free(c);
    free_all(c);
    delete c;
    return LEPIC_OK;
}

extern "C" void *lepic_gpu_stream(lepic_ctx *c) { return c ? (void *)c->stream : nullptr; }
extern "C" const char *lepic_gpu_last_error(lepic_ctx *c) { return c ? c->last_err.c_str() : g_create_err.c_str(); }

// Reads the device counters; maps a raised device error to a status (then clears it).  A
// download still in flight on the copy stream is completed first: every call that
// synchronises the context leaves the host arrays of the asynchronous downloads filled.
static int sync_counters(lepic_ctx *c) {
    LCUDA(cudaMemcpyAsync(c->hcnt, c->dcnt, sizeof(DevCounters), cudaMemcpyDeviceToHost, c->stream));
    LCUDA(cudaStreamSynchronize(c->stream));
    if (c->down_pending) {
        LCUDA(cudaEventSynchronize(c->ev_down));
        c->down_pending = 0;
    }
    if (c->up_pending) {
        LCUDA(cudaEventSynchronize(c->ev_up));
        c->up_pending = 0;
    }
    int e = c->hcnt->err;
    if (e) {
        int where = c->hcnt->err_where;
        LCUDA(cudaMemsetAsync(&c->dcnt->err, 0, 2 * sizeof(int), c->stream));
        LCUDA(cudaStreamSynchronize(c->stream));
        c->last_err = "device error bits " + std::to_string(e) + " raised at site " + std::to_string(where);
        if (e & LERR_TIMEOUT) return LEPIC_ETIMEOUT;
        if (e & LERR_DIVERGED) return LEPIC_EDIVERGED;
        if (e & LERR_CAPACITY) return LEPIC_ECAPACITY;
        if (e & LERR_RANGE) return LEPIC_ERANGE;
        if (e & LERR_NOTCONV) return LEPIC_ENOTCONV;
        return LEPIC_ECUDA;
    }
    return LEPIC_OK;
}

extern "C" int lepic_gpu_sync(lepic_ctx *c) {
    if (!c) return LEPIC_EINVAL;
    return sync_counters(c);
}

// ---------------------------------------------------------------------------------------
// particles
int particles_put(lepic_ctx *c, int sp, const double *vxp, long long n) {
    SpeciesBuf &B = c->sp[sp];
    if (n < 0 || n > B.cap) { c->last_err = "particle count exceeds capacity"; return LEPIC_ECAPACITY; }
    const lepic_config &g = c->cfg;
    const double sx = (double)(1u << c->S) / g.dx, sy = (double)(1u << c->S) / g.dy;
    const long long xl = (long long)g.nx << c->S, yl = (long long)g.ny << c->S;
    std::vector<uint32_t> X(n), Y(n);
    std::vector<float> VX(n), VY(n), VZ(n), Z(B.Z[0] ? n : 0);
    for (long long k = 0; k < n; k++) {
        const double *p = vxp + 6 * k;
        long long xi = llround(p[0] * sx), yi = llround(p[1] * sy);
        if (xi < 0 || xi >= xl || yi < 0 || yi >= yl) { c->last_err = "particle outside the box"; return LEPIC_EINVAL; }
        X[k] = (uint32_t)xi; Y[k] = (uint32_t)yi;
        VX[k] = (float)p[3]; VY[k] = (float)p[4]; VZ[k] = (float)p[5];
        if (B.Z[0]) Z[k] = (float)p[2];
    }
    const int cur = B.cur;
    if (n > 0 && B.Z[0]) LCUDA(cudaMemcpyAsync(B.Z[cur], Z.data(), 4 * n, cudaMemcpyHostToDevice, c->stream));
    if (n > 0) {
        LCUDA(cudaMemcpyAsync(B.X[cur], X.data(), 4 * n, cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaMemcpyAsync(B.Y[cur], Y.data(), 4 * n, cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaMemcpyAsync(B.VX[cur], VX.data(), 4 * n, cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaMemcpyAsync(B.VY[cur], VY.data(), 4 * n, cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaMemcpyAsync(B.VZ[cur], VZ.data(), 4 * n, cudaMemcpyHostToDevice, c->stream));
    }
    LCUDA(cudaStreamSynchronize(c->stream));
    long long v = n;
    int zero = 0;
    LCUDA(cudaMemcpy(&c->dcnt->n_slots[sp], &v, sizeof(v), cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(&c->dcnt->n_alive[sp], &v, sizeof(v), cudaMemcpyHostToDevice));
    v = 0;
    LCUDA(cudaMemcpy(&c->dcnt->n_sorted[sp], &v, sizeof(v), cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(&c->dcnt->n_items[sp], &zero, sizeof(int), cudaMemcpyHostToDevice));
    B.ordered = false;
    return LEPIC_OK;
}

int particles_get(lepic_ctx *c, int sp, double *vxp, long long cap, long long *n_out) {
    int r = sync_counters(c);
    if (r != LEPIC_OK) return r;
    SpeciesBuf &B = c->sp[sp];
    const long long ns = c->hcnt->n_slots[sp];
    std::vector<uint32_t> X(ns), Y(ns);
    std::vector<float> VX(ns), VY(ns), VZ(ns), Z(B.Z[0] ? ns : 0);
    const int cur = B.cur;
    if (ns > 0 && B.Z[0]) LCUDA(cudaMemcpy(Z.data(), B.Z[cur], 4 * ns, cudaMemcpyDeviceToHost));
    if (ns > 0) {
        LCUDA(cudaMemcpy(X.data(), B.X[cur], 4 * ns, cudaMemcpyDeviceToHost));
        LCUDA(cudaMemcpy(Y.data(), B.Y[cur], 4 * ns, cudaMemcpyDeviceToHost));
        LCUDA(cudaMemcpy(VX.data(), B.VX[cur], 4 * ns, cudaMemcpyDeviceToHost));
        LCUDA(cudaMemcpy(VY.data(), B.VY[cur], 4 * ns, cudaMemcpyDeviceToHost));
        LCUDA(cudaMemcpy(VZ.data(), B.VZ[cur], 4 * ns, cudaMemcpyDeviceToHost));
    }
    const lepic_config &g = c->cfg;
    const double ux = g.dx * std::ldexp(1.0, -c->S), uy = g.dy * std::ldexp(1.0, -c->S);
    long long k = 0;
    for (long long i = 0; i < ns; i++) {
        if (std::isnan(VX[i])) continue;
        if (vxp && k < cap) {
            double *p = vxp + 6 * k;
            p[0] = (double)X[i] * ux; p[1] = (double)Y[i] * uy; p[2] = B.Z[0] ? (double)Z[i] : 0.0;
            p[3] = VX[i]; p[4] = VY[i]; p[5] = VZ[i];
        }
        k++;
    }
    if (n_out) *n_out = k;
    if (vxp && k > cap) { c->last_err = "output capacity too small"; return LEPIC_ECAPACITY; }
    return LEPIC_OK;
}

struct LoadP {
    int nx, ny, S, ntype, profile;
    long long n;
    unsigned long long xload;  // x_load in fixed-point units (nx << S can be 2^32)
    unsigned long long ylim;   // ny << S
    double n_peak, n_floor, sig2, xc, yc, dx, dy;
    const uint8_t *cellwall;
    uint32_t *X[LEPIC_MAXSP], *Y[LEPIC_MAXSP];
    float *VX[LEPIC_MAXSP], *VY[LEPIC_MAXSP], *VZ[LEPIC_MAXSP];
    float *Z[LEPIC_MAXSP];     // null without the 3rd dimension
    double zmax;
    double vt[LEPIC_MAXSP];
    uint32_t k0, k1;
    DevCounters *cnt;
};

__global__ void k_load(LoadP P) {
    const double pi = 3.141592653589793;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.n; i += (long long)gridDim.x * blockDim.x) {
        uint32_t X = 0, Y = 0;
        bool ok = false;
        for (uint32_t a = 0; a < 100000u && !ok; a++) {
            U4 r = philox4x32_10(U4{(uint32_t)i, a, 0x4C4F4144u, (uint32_t)(i >> 32)}, P.k0, P.k1);
            X = (uint32_t)(((unsigned long long)r.x * P.xload) >> 32);
            Y = (uint32_t)(((unsigned long long)r.y * P.ylim) >> 32);
            int ix = (int)(X >> P.S) + 1, iy = (int)(Y >> P.S) + 1;
            if (P.cellwall[ix + (long long)iy * (P.nx + 2)]) continue; // load_part.f90:115-116
            if (P.profile == 1) {
                double x = ((double)X + 0.5) * P.dx * ldexp(1.0, -P.S) - P.xc;
                double y = ((double)Y + 0.5) * P.dy * ldexp(1.0, -P.S) - P.yc;
                double nloc = P.n_floor + (P.n_peak - P.n_floor) * exp(-(x * x + y * y) / (2.0 * P.sig2));
                if (u01(r.z) * P.n_peak > nloc) continue;
            }
            ok = true;
        }
        if (!ok) set_err(P.cnt, LERR_RANGE, 400);
        for (int s = 0; s < P.ntype; s++) {
            U4 r = philox4x32_10(U4{(uint32_t)i, (uint32_t)s, 0x56454C4Fu, (uint32_t)(i >> 32)}, P.k0, P.k1);
            double vp = P.vt[s] * sqrt(-log(1.0 - u01(r.x)));
            double sn, cs;
            sincos(2.0 * pi * u01(r.y), &sn, &cs);
            double vpz = P.vt[s] * sqrt(-log(1.0 - u01(r.z)));
            double sz, cz;
            sincos(2.0 * pi * u01(r.w), &sz, &cz);
            P.X[s][i] = X; P.Y[s][i] = Y;
            P.VX[s][i] = (float)(vp * cs); P.VY[s][i] = (float)(vp * sn); P.VZ[s][i] = (float)(vpz * cz);
            if (P.Z[s]) {   // z = rnd zmax, one z for the sample (load_part.f90:108, 141-143)
                const U4 q = philox4x32_10(U4{(uint32_t)i, 0u, 0x5A504F53u, (uint32_t)(i >> 32)}, P.k0, P.k1);
                P.Z[s][i] = (float)(u01(q.x) * P.zmax);
            }
        }
    }
}

int particles_load(lepic_ctx *c, const lepic_load_spec *sp) {
    const lepic_config &g = c->cfg;
    for (int s = 0; s < g.ntype; s++)
        if (sp->n_samples > c->sp[s].cap) { c->last_err = "load exceeds capacity"; return LEPIC_ECAPACITY; }
    LoadP P;
    memset(&P, 0, sizeof(P));
    P.nx = g.nx; P.ny = g.ny; P.S = c->S; P.ntype = g.ntype; P.profile = sp->profile; P.n = sp->n_samples;
    double xl = std::min(sp->x_load, g.dx * g.nx);
    if (xl <= 0) xl = g.dx * g.nx;
    P.xload = (unsigned long long)std::min<double>((double)((long long)g.nx << c->S),
                                                   std::floor(xl / g.dx * (double)(1u << c->S)));
    P.ylim = (unsigned long long)g.ny << c->S;
    P.n_peak = sp->n_peak; P.n_floor = sp->n_floor; P.sig2 = sp->sigma * sp->sigma;
    P.xc = 0.5 * g.dx * g.nx; P.yc = 0.5 * g.dy * g.ny; P.dx = g.dx; P.dy = g.dy;
    P.cellwall = c->cellwall;
    for (int s = 0; s < g.ntype; s++) {
        SpeciesBuf &B = c->sp[s];
        P.X[s] = B.X[B.cur]; P.Y[s] = B.Y[B.cur]; P.VX[s] = B.VX[B.cur]; P.VY[s] = B.VY[B.cur]; P.VZ[s] = B.VZ[B.cur];
        P.Z[s] = B.Z[B.cur];
        // vt0 = sqrt(2kT/m); load_gauss draws each component with sigma = vt0/sqrt(2)
        P.vt[s] = g.vt0[s];
    }
    P.k0 = (uint32_t)sp->seed; P.k1 = (uint32_t)(sp->seed >> 32) ^ 0x1234567u;
    P.zmax = g.zmax;
    P.cnt = c->dcnt;
    k_load<<<c->num_sms * 8, 256, 0, c->stream>>>(P);
    LCUDA(cudaGetLastError());
    for (int s = 0; s < g.ntype; s++) {
        long long v = sp->n_samples, z = 0;
        int zero = 0;
        LCUDA(cudaMemcpyAsync(&c->dcnt->n_slots[s], &v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaMemcpyAsync(&c->dcnt->n_alive[s], &v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaMemcpyAsync(&c->dcnt->n_sorted[s], &z, sizeof(z), cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaMemcpyAsync(&c->dcnt->n_items[s], &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaStreamSynchronize(c->stream));
        c->sp[s].ordered = false;
    }
    return sync_counters(c);
}

extern "C" int lepic_gpu_put_particles(lepic_ctx *c, int32_t ptype, const double *vxp, int64_t n) {
    if (!c || ptype < 0 || ptype >= c->cfg.ntype || (n > 0 && !vxp)) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    return particles_put(c, ptype, vxp, n);
}
// The reference's own particle array vxp(6, nmax, ntype, nproc) with np_tot(ntype, nproc): a
// species' slabs are concatenated in slab order on the way in; on the way out its live
// particles are dealt to the nproc slabs in equal parts, in slot order, as sorting.f90:92-251
// rebalances them.
extern "C" int lepic_gpu_put_particles_slabs(lepic_ctx *c, const double *vxp, const int32_t *np_tot, int64_t nmax,
                                             int32_t ntype, int32_t nproc) {
    if (!c || !vxp || !np_tot || nmax < 0 || ntype != c->cfg.ntype || nproc < 1) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    for (int s = 0; s < ntype; s++) {
        long long n = 0;
        for (int p = 0; p < nproc; p++) {
            const int32_t k = np_tot[s + (long long)ntype * p];
            if (k < 0 || k > nmax) { c->last_err = "np_tot outside 0..nmax"; return LEPIC_EINVAL; }
            n += k;
        }
        std::vector<double> buf((size_t)6 * n);
        long long o = 0;
        for (int p = 0; p < nproc; p++) {
            const int32_t k = np_tot[s + (long long)ntype * p];
            const double *src = vxp + 6 * nmax * ((long long)s + (long long)ntype * p);
            std::memcpy(buf.data() + 6 * o, src, sizeof(double) * 6 * (size_t)k);
            o += k;
        }
        int r = particles_put(c, s, buf.data(), n);
        if (r != LEPIC_OK) return r;
    }
    return LEPIC_OK;
}

extern "C" int lepic_gpu_get_particles_slabs(lepic_ctx *c, double *vxp, int32_t *np_tot, int64_t nmax,
                                             int32_t ntype, int32_t nproc) {
    if (!c || !vxp || !np_tot || nmax < 0 || ntype != c->cfg.ntype || nproc < 1) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    for (int s = 0; s < ntype; s++) {
        long long n = 0;
        int r = particles_get(c, s, nullptr, 0, &n);
        if (r != LEPIC_OK) return r;
        if ((n + nproc - 1) / nproc > nmax) { c->last_err = "a slab would exceed nmax"; return LEPIC_ECAPACITY; }
        std::vector<double> buf((size_t)6 * std::max(n, 1ll));
        r = particles_get(c, s, buf.data(), n, &n);
        if (r != LEPIC_OK) return r;
        long long o = 0;
        for (int p = 0; p < nproc; p++) {
            const long long k = n / nproc + (p < n % nproc ? 1 : 0);
            double *dst = vxp + 6 * nmax * ((long long)s + (long long)ntype * p);
            std::memcpy(dst, buf.data() + 6 * o, sizeof(double) * 6 * (size_t)k);
            np_tot[s + (long long)ntype * p] = (int32_t)k;
            o += k;
        }
    }
    return LEPIC_OK;
}

extern "C" int lepic_gpu_get_particles(lepic_ctx *c, int32_t ptype, double *vxp, int64_t cap, int64_t *n_out) {
    if (!c || ptype < 0 || ptype >= c->cfg.ntype) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    long long n = 0;
    int r = particles_get(c, ptype, vxp, cap, &n);
    if (n_out) *n_out = n;
    return r;
}
extern "C" int lepic_gpu_load_particles(lepic_ctx *c, const lepic_load_spec *spec) {
    if (!c || !spec || spec->n_samples < 0) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    return particles_load(c, spec);
}

// ---------------------------------------------------------------------------------------
extern "C" int lepic_gpu_charge_deposition(lepic_ctx *c) {
    if (!c) return LEPIC_EINVAL;
    return push_deposit(c, 0, false);
}

extern "C" int lepic_gpu_calc_rhs(lepic_ctx *c, double *rhs_out) {
    if (!c) return LEPIC_EINVAL;
    int r = field_calc_rhs(c);
    if (r != LEPIC_OK || !rhs_out) return r;
    LCUDA(cudaMemcpyAsync(rhs_out, c->rhs, sizeof(double) * (c->cfg.nx + 1) * (c->cfg.ny + 1),
                          cudaMemcpyDeviceToHost, c->stream));
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

extern "C" int lepic_gpu_dens_red(lepic_ctx *c, double *np_red_out, double *np_mx_out) {
    if (!c) return LEPIC_EINVAL;
    int r = field_dens_red(c);
    if (r != LEPIC_OK) return r;
    if (np_red_out)
        LCUDA(cudaMemcpyAsync(np_red_out, c->np_red, sizeof(double) * c->cfg.ntype * c->nn, cudaMemcpyDeviceToHost,
                              c->stream));
    if (np_mx_out)
        LCUDA(cudaMemcpyAsync(np_mx_out, c->np_mx, sizeof(double) * c->cfg.ntype, cudaMemcpyDeviceToHost, c->stream));
    if (np_red_out || np_mx_out) LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

// The context's stream waits for copies on the copy stream: the work that reads or writes phi
// for a staged upload into phi (lepic_gpu_stage_solver_input); an upload from a host array, and
// the reuse of the download snapshot, for the last download (into that array, out of the
// snapshot).  A download alone holds up nothing else: the E field and the push run beside it.
int wait_upload(lepic_ctx *c) {
    if (c->up_pending) LCUDA(cudaStreamWaitEvent(c->stream, c->ev_up, 0));
    return LEPIC_OK;
}
static int wait_download(lepic_ctx *c) {
    if (c->down_pending) LCUDA(cudaStreamWaitEvent(c->stream, c->ev_down, 0));
    return LEPIC_OK;
}
static int wait_copies(lepic_ctx *c) {
    if (const int r = wait_upload(c)) return r;
    return wait_download(c);
}

static int solve(lepic_ctx *c, double eps, int mode) {
    if (const int r = wait_upload(c)) return r;
    if (mode == LEPIC_POISSON_MIXED_IR) return mg_mixed_solve(c, eps, true);
    if (mode == LEPIC_POISSON_FP64_PCG) return mg_mixed_solve(c, eps, true, true);
    c->have_hist = 0;   // any other solver: the next mixed solve starts from its answer as it is
    if (mode == LEPIC_POISSON_FP64_MG) return mg_solve(c, eps, 0);
    if (mode == 2) return mg_solve(c, eps, 2);
    if (mode == LEPIC_POISSON_LEARNED) return learned_solve(c, eps);
    c->last_err = "unknown Poisson mode";
    return LEPIC_EINVAL;
}

// Enqueues the download of `bytes` from the device array `src` into the host array `out`
// without waiting for it: a device-to-device snapshot on the context's stream (ordered after
// the work that produced src, ~10 us for a 2049^2 potential), then the device-to-host copy of the
// snapshot on the copy stream, where it runs beside the kernels enqueued next.  The snapshot is
// reused by the next download only after this one has completed.
static int copy_stream(lepic_ctx *c);
static int download_async(lepic_ctx *c, void *out, const void *src, size_t bytes) {
    if (const int r = copy_stream(c)) return r;
    if (c->snap_bytes < bytes) {
        int r = sync_counters(c);   // no copy may still read the old snapshot
        if (r != LEPIC_OK) return r;
        if (c->snap) cudaFree(c->snap);
        c->snap = nullptr;
        c->snap_bytes = 0;
        if (cudaMalloc(&c->snap, bytes) != cudaSuccess) { c->last_err = "download snapshot: cudaMalloc failed"; return LEPIC_ENOMEM; }
        c->snap_bytes = bytes;
    }
    int r = wait_copies(c);
    if (r != LEPIC_OK) return r;
    LCUDA(cudaMemcpyAsync(c->snap, src, bytes, cudaMemcpyDeviceToDevice, c->stream));
    LCUDA(cudaEventRecord(c->ev_snap, c->stream));
    LCUDA(cudaStreamWaitEvent(c->cstream, c->ev_snap, 0));
    LCUDA(cudaMemcpyAsync(out, c->snap, bytes, cudaMemcpyDeviceToHost, c->cstream));
    LCUDA(cudaEventRecord(c->ev_down, c->cstream));
    c->down_pending = 1;
    return LEPIC_OK;
}

// the copy stream and its events, created with the first overlapped copy
static int copy_stream(lepic_ctx *c) {
    if (!c->cstream) {
        LCUDA(cudaStreamCreateWithFlags(&c->cstream, cudaStreamNonBlocking));
        LCUDA(cudaEventCreateWithFlags(&c->ev_snap, cudaEventDisableTiming));
        LCUDA(cudaEventCreateWithFlags(&c->ev_down, cudaEventDisableTiming));
        LCUDA(cudaEventCreateWithFlags(&c->ev_up, cudaEventDisableTiming));
    }
    return LEPIC_OK;
}

extern "C" int lepic_gpu_stage_solver_input(lepic_ctx *c, const double *phi_in) {
    if (!c || !phi_in) return LEPIC_EINVAL;
    int r = copy_stream(c);
    if (r != LEPIC_OK) return r;
    // after the work enqueued so far (the E field that reads phi) and after the copy stream's
    // earlier copies (a download into phi_in), then the copy into phi; the next work that reads
    // or writes phi waits for it
    LCUDA(cudaEventRecord(c->ev_snap, c->stream));
    LCUDA(cudaStreamWaitEvent(c->cstream, c->ev_snap, 0));
    LCUDA(cudaMemcpyAsync(c->phi, phi_in, sizeof(double) * c->nn, cudaMemcpyHostToDevice, c->cstream));
    LCUDA(cudaEventRecord(c->ev_up, c->cstream));
    c->up_pending = 1;
    return LEPIC_OK;
}

extern "C" int lepic_gpu_iterative_solver_async(lepic_ctx *c, const double *phi_in, double *phi_out, double eps,
                                                int32_t mode) {
    if (!c || !(eps > 0)) return LEPIC_EINVAL;
    int r;
    if (phi_in) {
        if ((r = wait_copies(c)) != LEPIC_OK) return r;
        LCUDA(cudaMemcpyAsync(c->phi, phi_in, sizeof(double) * c->nn, cudaMemcpyHostToDevice, c->stream));
    }
    if ((r = solve(c, eps, mode)) != LEPIC_OK) return r;
    if (phi_out) return download_async(c, phi_out, c->phi, sizeof(double) * c->nn);
    return LEPIC_OK;
}

extern "C" int lepic_gpu_get_grid_async(lepic_ctx *c, int32_t which, double *out) {
    if (!c || !out) return LEPIC_EINVAL;
    if (which == LEPIC_GRID_PHI) return download_async(c, out, c->phi, sizeof(double) * c->nn);
    if (which == LEPIC_GRID_RHS)
        return download_async(c, out, c->rhs, sizeof(double) * (c->cfg.nx + 1) * (c->cfg.ny + 1));
    if (which == LEPIC_GRID_EI) return download_async(c, out, c->Ed, sizeof(double2) * c->nn);
    return LEPIC_EINVAL;
}

extern "C" int lepic_gpu_iterative_solver(lepic_ctx *c, double *phi_inout, double eps, int32_t mode,
                                          lepic_solve_stats *st) {
    if (!c || !(eps > 0)) return LEPIC_EINVAL;
    if (phi_inout) {
        int r = wait_copies(c);
        if (r != LEPIC_OK) return r;
        LCUDA(cudaMemcpyAsync(c->phi, phi_inout, sizeof(double) * c->nn, cudaMemcpyHostToDevice, c->stream));
    }
    int r = solve(c, eps, mode);
    if (r != LEPIC_OK) return r;
    if (phi_inout)
        LCUDA(cudaMemcpyAsync(phi_inout, c->phi, sizeof(double) * c->nn, cudaMemcpyDeviceToHost, c->stream));
    if (phi_inout || st) {
        r = sync_counters(c);
        if (st) {
            st->cycles = c->hcnt->mg_cycles;
            st->sweeps_fine = c->hcnt->mg_sweeps_fine;
            st->res_l1 = c->hcnt->mg_res_l1;
            st->res_l2_rel = c->hcnt->mg_b_l2 > 0 ? c->hcnt->mg_res_l2 / c->hcnt->mg_b_l2 : c->hcnt->mg_res_l2;
            st->ktot = c->hcnt->mg_ktot;
        }
        return r;
    }
    return LEPIC_OK;
}

extern "C" int lepic_gpu_calc_efield(lepic_ctx *c, double *Ei_out) {
    if (!c) return LEPIC_EINVAL;
    int r = field_calc_efield(c);
    if (r != LEPIC_OK || !Ei_out) return r;
    LCUDA(cudaMemcpyAsync(Ei_out, c->Ed, sizeof(double2) * c->nn, cudaMemcpyDeviceToHost, c->stream));
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

extern "C" int lepic_gpu_part_sorting(lepic_ctx *c, int32_t ptype, int32_t *plist_out) {
    if (!c || ptype < 0 || ptype >= c->cfg.ntype) return LEPIC_EINVAL;
    // the records move into sorted order in the next push (or, before any other call that reads
    // them, at that call's start): the same order, one pass over the records fewer
    int r = sort_species(c, ptype, c->opt.sort_defer == 1 && !push_needs_general(c, ptype));
    if (r != LEPIC_OK || !plist_out) return r;
    const int nx = c->cfg.nx, ny = c->cfg.ny;
    const long long pl_max = (long long)nx + (long long)nx * ny + 1;
    std::vector<int> off(c->nkeys + 1);
    LCUDA(cudaMemcpyAsync(off.data(), c->offsets, sizeof(int) * (c->nkeys + 1), cudaMemcpyDeviceToHost, c->stream));
    r = sync_counters(c);
    plist_out[0] = 0;
    for (long long i = 1; i <= pl_max; i++) plist_out[i] = (i <= c->nkeys) ? off[i] : off[c->nkeys];
    return r;
}

extern "C" int lepic_gpu_collisions(lepic_ctx *c, int32_t it, lepic_mcc_stats *st) {
    if (!c) return LEPIC_EINVAL;
    int r = mcc_collide(c, it, false);
    if (r != LEPIC_OK) return r;
    if (st) return lepic_gpu_get_mcc_stats(c, st);
    return LEPIC_OK;
}

extern "C" int lepic_gpu_push_deposit(lepic_ctx *c, int32_t it, lepic_push_stats *st) {
    if (!c) return LEPIC_EINVAL;
    int r = push_deposit(c, it, true);
    if (r != LEPIC_OK) return r;
    if (st) return lepic_gpu_get_push_stats(c, st);
    return LEPIC_OK;
}

// an error inside lepic_gpu_step: the records of a pending permutation are moved first
static int settle(lepic_ctx *c, int r) {
    materialize_all(c);
    return r;
}

extern "C" int lepic_gpu_step(lepic_ctx *c, int32_t it, double eps, int32_t mode) {
    if (!c) return LEPIC_EINVAL;
    const lepic_config &g = c->cfg;
    int r;
    if (c->dq && (r = dielectric_update(c)) != LEPIC_OK) return r;   // main.f90:756-809
    if ((r = field_calc_rhs(c)) != LEPIC_OK) return r;
    if ((r = solve(c, eps, mode)) != LEPIC_OK) return r;
    if ((r = field_calc_efield(c)) != LEPIC_OK) return r;
    // The sort leaves its permutation pending for the species the fast mover pushes (as
    // lepic_gpu_part_sorting does): the collisions read and write through it and the push moves
    // the records into sorted order as it writes them, which saves the sort's gather (44 B per
    // particle).  Whatever else would read the records in between moves them first.
    if (g.nsort > 0 && it % g.nsort == 1)
        for (int s = 0; s < g.ntype; s++)
            if ((r = sort_species(c, s, c->opt.sort_defer == 1 && !push_needs_general(c, s))) != LEPIC_OK)
                return settle(c, r);
    if ((r = avg_step(c, it)) != LEPIC_OK) return settle(c, r);  // main.f90:906-949
    if (it > 1 && g.ns_coll > 0 && it % g.ns_coll == 1)
        if ((r = mcc_collide(c, it, false)) != LEPIC_OK) return settle(c, r);
    if ((r = sources_before_push(c, it)) != LEPIC_OK) return settle(c, r);
    if ((r = push_deposit(c, it, true)) != LEPIC_OK) return settle(c, r);
    return sources_after_push(c, it);
}

extern "C" int lepic_gpu_get_grid(lepic_ctx *c, int32_t which, double *out) {
    if (!c || !out) return LEPIC_EINVAL;
    if (const int r = wait_upload(c)) return r;   // a staged upload into phi
    const long long nn = c->nn;
    if (which == LEPIC_GRID_PHI) {
        LCUDA(cudaMemcpyAsync(out, c->phi, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream));
    } else if (which == LEPIC_GRID_RHS) {
        LCUDA(cudaMemcpyAsync(out, c->rhs, sizeof(double) * (c->cfg.nx + 1) * (c->cfg.ny + 1), cudaMemcpyDeviceToHost,
                              c->stream));
    } else if (which == LEPIC_GRID_EI) {
        LCUDA(cudaMemcpyAsync(out, c->Ed, sizeof(double2) * nn, cudaMemcpyDeviceToHost, c->stream));
    } else if (which >= LEPIC_GRID_NP && which < LEPIC_GRID_NP + c->cfg.ntype) {
        int r = field_np_grid(c, which - LEPIC_GRID_NP, c->npd);
        if (r != LEPIC_OK) return r;
        LCUDA(cudaMemcpyAsync(out, c->npd, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream));
    } else {
        return LEPIC_EINVAL;
    }
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

extern "C" int lepic_gpu_set_warm_start(lepic_ctx *c, int32_t mode) {
    if (!c || (mode != 0 && mode != 1)) return LEPIC_EINVAL;
    if (mode == 1 && !c->phi_hist) {
        if (cudaMalloc((void **)&c->phi_hist, sizeof(double) * c->nn) != cudaSuccess) {
            c->last_err = "set_warm_start: cudaMalloc failed";
            return LEPIC_ENOMEM;
        }
    }
    c->warm_xtrap = mode;
    c->have_hist = 0;
    return LEPIC_OK;
}

extern "C" int lepic_gpu_set_grid(lepic_ctx *c, int32_t which, const double *in) {
    if (!c || !in) return LEPIC_EINVAL;
    if (wait_copies(c) != LEPIC_OK) return LEPIC_ECUDA;
    if (which == LEPIC_GRID_PHI) {
        LCUDA(cudaMemcpyAsync(c->phi, in, sizeof(double) * c->nn, cudaMemcpyHostToDevice, c->stream));
        c->have_hist = 0;   // a potential from elsewhere: the next solve starts from it as it is
    }
    else if (which == LEPIC_GRID_RHS)
        LCUDA(cudaMemcpyAsync(c->rhs, in, sizeof(double) * (c->cfg.nx + 1) * (c->cfg.ny + 1), cudaMemcpyHostToDevice,
                              c->stream));
    else
        return LEPIC_EINVAL;
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

extern "C" int lepic_gpu_get_push_stats(lepic_ctx *c, lepic_push_stats *st) {
    if (!c || !st) return LEPIC_EINVAL;
    int r = sync_counters(c);
    memset(st, 0, sizeof(*st));
    for (int s = 0; s < c->cfg.ntype; s++) {
        st->np_tot[s] = c->hcnt->n_alive[s];
        st->n_lost[s] = (int64_t)c->hcnt->n_lost[s];
        st->n_dead[s] = (int64_t)c->hcnt->n_dead[s];
        st->n_slots[s] = c->hcnt->n_slots[s];
    }
    return r;
}

extern "C" int lepic_gpu_get_mcc_stats(lepic_ctx *c, lepic_mcc_stats *st) {
    if (!c || !st) return LEPIC_EINVAL;
    int r = sync_counters(c);
    memset(st, 0, sizeof(*st));
    for (int s = 0; s < LEPIC_MAXSP; s++) {
        st->n_cand[s] = (int64_t)c->hcnt->n_cand[s];
        st->n_add[s] = (int64_t)c->hcnt->n_add[s];
        st->nu_max[s] = c->nu_max[s];
    }
    for (int q = 0; q < LEPIC_MAXCOL; q++) st->n_coll[q] = (int64_t)c->hcnt->n_coll[q];
    st->n_overflow = (int64_t)c->hcnt->n_overflow;
    return r;
}

extern "C" int lepic_gpu_deposit_grid(lepic_ctx *c, int32_t ptype, void **acc) {
    if (!c || !acc || ptype < 0 || ptype >= c->cfg.ntype) return LEPIC_EINVAL;
    *acc = c->sp[ptype].acc;
    return LEPIC_OK;
}

extern "C" int lepic_gpu_particle_arrays(lepic_ctx *c, int32_t ptype, void **X, void **Y, void **VX, void **VY,
                                         void **VZ, int64_t *n_slots, int32_t *shift) {
    if (!c || ptype < 0 || ptype >= c->cfg.ntype) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    SpeciesBuf &B = c->sp[ptype];
    if (X) *X = B.X[B.cur];
    if (Y) *Y = B.Y[B.cur];
    if (VX) *VX = B.VX[B.cur];
    if (VY) *VY = B.VY[B.cur];
    if (VZ) *VZ = B.VZ[B.cur];
    if (shift) *shift = c->S;
    if (n_slots) {
        int r = sync_counters(c);
        *n_slots = c->hcnt->n_slots[ptype];
        return r;
    }
    return LEPIC_OK;
}
