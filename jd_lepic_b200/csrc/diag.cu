// diag.cu -- device-side averages: part_moments (utils.f90:1-131), calc_avg (utils.f90:133-266)
// and the potential and field averages of main.f90:935-947, one averaging sample per call at
// MOD(it,navg) == 1 (main.f90:906-949).  data_pavg and phi_avg stay on the device in the
// reference's Fortran layouts; the host reads them when it writes its files.
//
// k_moments: one particle per thread in slot order (the particles are cell-sorted at this
// step, main.f90:891-906): the back-stepped position xp = x - vx dt/2 selects a cell of the
// coarse grid (size_na cells of the field grid per cell); the 16 contributions (4 nodes x
// n<v^2>, jx, jy, jz) of lanes that share a cell are combined by a segmented warp scan and the
// last lane of each segment adds them with FP64 atomics.  FP64 sums in atomic order: the
// averages agree with the FP64 restatement to rounding, not bit for bit.
// Roofline: 20 B per particle read (X, Y, VX, VY, VZ) per averaging sample, every navg steps.
#include <algorithm>
#include <cstring>
#include <vector>
#include "rho.cuh"

struct AvgState {
    int size_na = 0, na1 = 0, na2 = 0, navg = 0;
    long long ncell = 0;    // (na1 + 3) (na2 + 3): p_mts nodes 0 .. na + 2 per direction
    double *p_mts = nullptr;     // [ntype][4][ncell]: n<v^2>, jx, jy, jz (utils.f90:18)
    double *data = nullptr;      // data_pavg(7, na1+1, na2+1, ntype)
    double *phi_avg = nullptr;   // phi_avg(3, 0:nx+2, 0:ny+2)
    int cnt = 0;                 // cnt_avg(1)
};

static AvgState *avg_state(lepic_ctx *c) { return (AvgState *)c->avg; }

struct MomP {
    const uint32_t *X, *Y;
    const float *VX, *VY, *VZ;
    const DevCounters *cnt;
    int sp, S, nx, size_na, na1, na2, nmn, pbc, spec;
    double ux, uy, dt, xmax, ymax, ha1, ha2, k1;
    const double *kq;
    double *p_mts;       // this species' 4 x ncell block
    long long ncell;
};

// utils.f90:39-127 for one particle: the coarse cell key and the 16 contributions
__device__ __forceinline__ int moment_of(const MomP &P, long long k, double *c) {
    const float fvx = P.VX[k];
    if (isnan(fvx)) return -1;
    double vx = fvx, vy = P.VY[k], vz = P.VZ[k];
    double xp = (double)P.X[k] * P.ux - vx * P.dt / 2.0;
    double yp = (double)P.Y[k] * P.uy - vy * P.dt / 2.0;
    if (P.nmn == 1 && xp <= 0.0) { xp = -xp; vx = -vx; }  // :46-53
    if (P.pbc == 1) {                                      // :56-75
        const int k2 = (int)(yp / P.ymax);
        if (yp >= P.ymax) {
            if (P.spec == 0) yp = yp - k2 * P.ymax;
            else { yp = (k2 + 1) * P.ymax - yp; vy = -vy; }
        }
        if (yp <= 0.0) {
            if (P.spec == 0) yp = (1 - k2) * P.ymax + yp;
            else { yp = k2 * P.ymax - yp; vy = -vy; }
        }
    }
    if (xp > P.xmax || xp < 0.0 || yp > P.ymax || yp < 0.0) return -1;
    const double Eki = vx * vx + vy * vy + vz * vz;
    const int ix = (int)(xp / P.ha1) + 1, iy = (int)(yp / P.ha2) + 1;
    if (ix > P.na1 + 1 || iy > P.na2 + 1) return -1;   // beyond the coarse grid's last node
    const double px = (ix * P.ha1 - xp) / P.ha1, py = (iy * P.ha2 - yp) / P.ha2;
    const double ki[4] = {P.k1 * px * py, P.k1 * (1.0 - px) * py, P.k1 * (1.0 - px) * (1.0 - py),
                          P.k1 * px * (1.0 - py)};
    const int ixf = P.size_na * ix - (P.size_na - 1), iyf = P.size_na * iy - (P.size_na - 1);
    const int W = P.nx + 3;
    // the kq nodes of utils.f90:106-126: (ix_f, iy_f), (ix_f+1, iy_f), (ix_f+1, iy_f+1), (ix_f, iy_f+1)
    const long long f = ixf + (long long)iyf * W;
    const double kqv[4] = {P.kq[f], P.kq[f + 1], P.kq[f + 1 + W], P.kq[f + W]};
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double kt = kqv[q] * ki[q];
        c[4 * q + 0] = kt * Eki;
        c[4 * q + 1] = kt * vx;
        c[4 * q + 2] = kt * vy;
        c[4 * q + 3] = kt * vz;
    }
    return ix + iy * (P.na1 + 3);
}

__global__ void __launch_bounds__(256) k_moments(MomP P) {
    const long long n = P.cnt->n_slots[P.sp];
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long w0 = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5);
    for (long long base = w0 * 32; base < n; base += nwarps * 32) {   // warp-uniform trip count
        const long long k = base + lane;
        double c[16];
        int key = -1;
        if (k < n) key = moment_of(P, k, c);
        if (key < 0) {
#pragma unroll
            for (int q = 0; q < 16; q++) c[q] = 0.0;
        }
        // segmented inclusive scan: a segment is a run of equal keys in lane order (one run
        // per cell after the sort); segment ids from the run heads keep runs of a key that
        // repeats apart separate
        const int kprev = __shfl_up_sync(0xffffffffu, key, 1);
        const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || kprev != key);
        const int seg = __popc(heads & (0xffffffffu >> (31 - lane)));
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int so = __shfl_up_sync(0xffffffffu, seg, off);
            const bool take = lane >= off && so == seg;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const double o = __shfl_up_sync(0xffffffffu, c[q], off);
                if (take) c[q] += o;
            }
        }
        const bool last = lane == 31 || ((heads >> (lane + 1)) & 1u);
        if (key >= 0 && last) {
            const int ix = key % (P.na1 + 3), iy = key / (P.na1 + 3);
            const long long nodes[4] = {ix + (long long)iy * (P.na1 + 3), ix + 1 + (long long)iy * (P.na1 + 3),
                                        ix + 1 + (long long)(iy + 1) * (P.na1 + 3),
                                        ix + (long long)(iy + 1) * (P.na1 + 3)};
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int m = 0; m < 4; m++)
                    if (c[4 * q + m] != 0.0) atomicAdd(P.p_mts + m * P.ncell + nodes[q], c[4 * q + m]);
        }
    }
}

// calc_avg (utils.f90:176-262) for one species on the coarse nodes ix = 1..na1+1, iy = 1..na2+1:
// n from the field grid's node (ix_f, iy_f), the fluxes and n<v^2> from p_mts, and Tp from them
struct AvgP {
    RhoParams R;
    int sp, size_na, na1, na2;
    long long ncell;
    const double *p_mts;
    double *data;        // data_pavg(7, na1+1, na2+1, ntype)
    double m_over_qe;
    const unsigned int *ss_src, *ss_sink;   // this species' ss2D counts (plt_src = 0)
    double k_ss;                            // Nm / Vc, Vc = dx dy zmax (utils.f90:168, 200-204)
    const double *ssd_src, *ssd_sink;       // this species' ss2D densities (plt_src = 1), or null
};

__global__ void k_calc_avg(AvgP P) {
    const long long nodes = (long long)(P.na1 + 1) * (P.na2 + 1);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nodes;
         t += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(t % (P.na1 + 1)) + 1, iy = (int)(t / (P.na1 + 1)) + 1;
        const int ixf = P.size_na * ix - (P.size_na - 1), iyf = P.size_na * iy - (P.size_na - 1);
        const double np_ = np_val(P.R, P.sp, ixf, iyf);
        const long long m = ix + (long long)iy * (P.na1 + 3);
        const double p1 = P.p_mts[m], jx = P.p_mts[P.ncell + m], jy = P.p_mts[2 * P.ncell + m],
                     jz = P.p_mts[3 * P.ncell + m];
        double *d = P.data + 7 * (t + nodes * P.sp);
        d[0] += np_;
        d[2] += jx;
        d[3] += jy;
        d[4] += jz;
        double Tp = 0.0;
        if (np_ > 0) Tp = P.m_over_qe * (1.0 / 3.0) * (p1 / np_ - (jx * jx + jy * jy + jz * jz) / (np_ * np_));
        if (Tp > 0) d[1] += Tp;  // :251 (corners, few particles)
        const long long f = ixf + (long long)iyf * (P.R.nx + 3);   // sour_avg, sink_avg (:200-209)
        if (P.ssd_src) {
            d[5] += P.ssd_src[f];
            d[6] += P.ssd_sink[f];
        } else {
            d[5] += (double)P.ss_src[f] * P.k_ss;
            d[6] += (double)P.ss_sink[f] * P.k_ss;
        }
    }
}

// main.f90:935-947: phi_avg(1..3, ix, iy) += phi, Ex, Ey over the whole node grid
__global__ void k_phi_avg(const double *phi, const double2 *E, long long nn, double *out) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
         t += (long long)gridDim.x * blockDim.x) {
        const double2 e = E[t];
        out[3 * t] += phi[t];
        out[3 * t + 1] += e.x;
        out[3 * t + 2] += e.y;
    }
}

void avg_free(lepic_ctx *c) {
    if (c->ss_map) { cudaFree(c->ss_map); c->ss_map = nullptr; }
    AvgState *A = avg_state(c);
    if (!A) return;
    if (A->p_mts) cudaFree(A->p_mts);
    if (A->data) cudaFree(A->data);
    if (A->phi_avg) cudaFree(A->phi_avg);
    delete A;
    c->avg = nullptr;
}

extern "C" int lepic_gpu_set_avg(lepic_ctx *c, int32_t size_na, int32_t navg) {
    if (!c || size_na < 1 || navg < 0) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    const lepic_config &g = c->cfg;
    if (g.nx / size_na < 1 || g.ny / size_na < 1) { c->last_err = "size_na larger than the grid"; return LEPIC_EINVAL; }
    avg_free(c);
    AvgState *A = new (std::nothrow) AvgState;
    if (!A) return LEPIC_ENOMEM;
    c->avg = A;
    A->size_na = size_na;
    A->na1 = g.nx / size_na;   // read_input.f90:111
    A->na2 = g.ny / size_na;
    A->navg = navg;
    A->ncell = (long long)(A->na1 + 3) * (A->na2 + 3);
    const size_t nd = (size_t)7 * (A->na1 + 1) * (A->na2 + 1) * g.ntype;
    if (cudaMalloc((void **)&A->p_mts, sizeof(double) * 4 * A->ncell * g.ntype) != cudaSuccess ||
        cudaMalloc((void **)&A->data, sizeof(double) * nd) != cudaSuccess ||
        cudaMalloc((void **)&A->phi_avg, sizeof(double) * 3 * c->nn) != cudaSuccess ||
        cudaMalloc((void **)&c->ss_map, sizeof(unsigned int) * 2 * g.ntype * c->nn) != cudaSuccess) {
        avg_free(c);
        c->last_err = "set_avg: cudaMalloc failed";
        return LEPIC_ENOMEM;
    }
    LCUDA(cudaMemsetAsync(A->data, 0, sizeof(double) * nd, c->stream));
    LCUDA(cudaMemsetAsync(A->phi_avg, 0, sizeof(double) * 3 * c->nn, c->stream));
    LCUDA(cudaMemsetAsync(c->ss_map, 0, sizeof(unsigned int) * 2 * g.ntype * c->nn, c->stream));
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

int avg_sample(lepic_ctx *c, int it) {
    AvgState *A = avg_state(c);
    const lepic_config &g = c->cfg;
    if (c->plt_src == 1) {   // main.f90:921-927: ss2D from the collision frequencies of this state
        LCUDA(cudaMemsetAsync(c->ss_diag, 0, sizeof(double) * 2 * g.ntype * c->nn, c->stream));
        const int r = mcc_collide(c, it, true);
        if (r != LEPIC_OK) return r;
    }
    LCUDA(cudaMemsetAsync(A->p_mts, 0, sizeof(double) * 4 * A->ncell * g.ntype, c->stream));
    for (int s = 0; s < g.ntype; s++) {
        SpeciesBuf &B = c->sp[s];
        MomP P;
        memset(&P, 0, sizeof(P));
        P.X = B.X[B.cur]; P.Y = B.Y[B.cur]; P.VX = B.VX[B.cur]; P.VY = B.VY[B.cur]; P.VZ = B.VZ[B.cur];
        P.cnt = c->dcnt; P.sp = s; P.S = c->S; P.nx = g.nx;
        P.size_na = A->size_na; P.na1 = A->na1; P.na2 = A->na2;
        P.nmn = g.flag_nmn; P.pbc = g.flag_pbc; P.spec = g.flag_spec;
        P.ux = g.dx * std::ldexp(1.0, -c->S); P.uy = g.dy * std::ldexp(1.0, -c->S);
        P.dt = g.dt; P.xmax = g.nx * g.dx; P.ymax = g.ny * g.dy;
        P.ha1 = A->size_na * g.dx; P.ha2 = A->size_na * g.dy;   // ha = size_na*h
        P.k1 = g.Nm[s] / (P.ha1 * P.ha2 * g.zmax);
        P.kq = c->kq;
        P.p_mts = A->p_mts + (size_t)4 * A->ncell * s;
        P.ncell = A->ncell;
        k_moments<<<c->num_sms * 8, 256, 0, c->stream>>>(P);
        LCUDA(cudaGetLastError());
    }
    const long long nodes = (long long)(A->na1 + 1) * (A->na2 + 1);
    for (int s = 0; s < g.ntype; s++) {
        AvgP P;
        P.R = rho_params(c);
        P.sp = s; P.size_na = A->size_na; P.na1 = A->na1; P.na2 = A->na2; P.ncell = A->ncell;
        P.p_mts = A->p_mts + (size_t)4 * A->ncell * s;
        P.data = A->data;
        P.m_over_qe = g.mass[s] / g.qe;
        P.ss_src = c->ss_map + (size_t)(2 * s) * c->nn;
        P.ss_sink = c->ss_map + (size_t)(2 * s + 1) * c->nn;
        P.k_ss = g.Nm[s] / (g.dx * g.dy * g.zmax);
        P.ssd_src = c->plt_src == 1 ? c->ss_diag + (size_t)(2 * s) * c->nn : nullptr;
        P.ssd_sink = c->plt_src == 1 ? c->ss_diag + (size_t)(2 * s + 1) * c->nn : nullptr;
        k_calc_avg<<<(int)std::min<long long>(div_up(nodes, 256), (long long)c->num_sms * 8), 256, 0, c->stream>>>(P);
        LCUDA(cudaGetLastError());
    }
    // main.f90:931: the counts start again after each sample
    if (c->plt_src == 0) LCUDA(cudaMemsetAsync(c->ss_map, 0, sizeof(unsigned int) * 2 * g.ntype * c->nn, c->stream));
    k_phi_avg<<<(int)std::min<long long>(div_up(c->nn, 256), (long long)c->num_sms * 8), 256, 0, c->stream>>>(
        c->phi, c->Ed, c->nn, A->phi_avg);
    LCUDA(cudaGetLastError());
    A->cnt++;
    return zloss_after_avg(c, A->data, A->na1, A->na2, A->size_na, A->cnt);   // main.f90:950-960
}

extern "C" int lepic_gpu_calc_avg(lepic_ctx *c) {
    if (!c || !avg_state(c)) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    return avg_sample(c, 0x40000000 + avg_state(c)->cnt);   // the diagnostic pass's draws: a stream per sample
}

extern "C" int lepic_gpu_set_source_option(lepic_ctx *c, int32_t plt_src) {
    if (!c || (plt_src != 0 && plt_src != 1)) return LEPIC_EINVAL;
    if (plt_src == 1 && !c->ss_diag) {
        if (cudaMalloc((void **)&c->ss_diag, sizeof(double) * 2 * c->cfg.ntype * c->nn) != cudaSuccess) {
            c->last_err = "set_source_option: cudaMalloc failed";
            return LEPIC_ENOMEM;
        }
        LCUDA(cudaMemsetAsync(c->ss_diag, 0, sizeof(double) * 2 * c->cfg.ntype * c->nn, c->stream));
    }
    if (plt_src == 0 && c->ss_map)
        LCUDA(cudaMemsetAsync(c->ss_map, 0, sizeof(unsigned int) * 2 * c->cfg.ntype * c->nn, c->stream));
    c->plt_src = plt_src;
    return lepic_gpu_sync(c);
}

extern "C" int lepic_gpu_get_avg(lepic_ctx *c, double *data_pavg, double *phi_avg, int32_t *cnt_avg, int32_t reset) {
    if (!c || !avg_state(c)) return LEPIC_EINVAL;
    AvgState *A = avg_state(c);
    const size_t nd = (size_t)7 * (A->na1 + 1) * (A->na2 + 1) * c->cfg.ntype;
    if (data_pavg) LCUDA(cudaMemcpyAsync(data_pavg, A->data, sizeof(double) * nd, cudaMemcpyDeviceToHost, c->stream));
    if (phi_avg) LCUDA(cudaMemcpyAsync(phi_avg, A->phi_avg, sizeof(double) * 3 * c->nn, cudaMemcpyDeviceToHost, c->stream));
    if (cnt_avg) *cnt_avg = A->cnt;
    if (reset) {  // main.f90:1290-1296 after a write
        LCUDA(cudaMemsetAsync(A->data, 0, sizeof(double) * nd, c->stream));
        LCUDA(cudaMemsetAsync(A->phi_avg, 0, sizeof(double) * 3 * c->nn, c->stream));
        A->cnt = 0;
    }
    return lepic_gpu_sync(c);
}

// ss2D(2, 0:nx+2, 0:ny+2, ntype) of one rank as the reference holds it between samples
extern "C" int lepic_gpu_get_source_maps(lepic_ctx *c, double *ss2D) {
    if (!c || !ss2D) return LEPIC_EINVAL;
    if (!c->ss_map) { c->last_err = "source maps need lepic_gpu_set_avg"; return LEPIC_EINVAL; }
    const int nt = c->cfg.ntype;
    const long long nn = c->nn;
    if (c->plt_src == 1) {   // the densities of the last sample's diagnostic pass
        std::vector<double> h((size_t)2 * nt * nn);
        LCUDA(cudaMemcpyAsync(h.data(), c->ss_diag, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
        int r = lepic_gpu_sync(c);
        if (r) return r;
        for (int s = 0; s < nt; s++)
            for (long long n = 0; n < nn; n++)
                for (int k = 0; k < 2; k++) ss2D[k + 2 * (n + nn * s)] = h[(size_t)(2 * s + k) * nn + n];
        return LEPIC_OK;
    }
    std::vector<unsigned int> h((size_t)2 * nt * nn);
    LCUDA(cudaMemcpyAsync(h.data(), c->ss_map, sizeof(unsigned int) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    int r = lepic_gpu_sync(c);
    if (r) return r;
    for (int s = 0; s < nt; s++)
        for (long long n = 0; n < nn; n++)
            for (int k = 0; k < 2; k++) ss2D[k + 2 * (n + nn * s)] = (double)h[(size_t)(2 * s + k) * nn + n];
    return LEPIC_OK;
}

int avg_step(lepic_ctx *c, int it) {
    AvgState *A = avg_state(c);
    if (!A || A->navg < 1 || it % A->navg != 1) return LEPIC_OK;
    const int r = materialize_all(c);   // the moments read the records in sorted order
    if (r != LEPIC_OK) return r;
    return avg_sample(c, it);
}

// ---------------------------------------------------------------------------------------
// loss, power and collision tallies (the device side lives in push.cu, mcc.cu, sources.cu)
extern "C" int lepic_gpu_set_regions(lepic_ctx *c, int32_t n_rg, const double *xl_rg, const double *xr_rg,
                                     double yl_rg, double yr_rg) {
    if (!c || n_rg < 0 || n_rg > LEPIC_MAXRG || (n_rg > 0 && (!xl_rg || !xr_rg))) return LEPIC_EINVAL;
    const lepic_config &g = c->cfg;
    const double xmax = g.nx * g.dx, ymax = g.ny * g.dy;
    for (int i = 0; i < n_rg; i++) {  // main.f90:319-324
        const double xl = std::max(xl_rg[i], 0.0), xr = std::min(xr_rg[i], xmax);
        c->ixl_rg[i] = (int)std::lround(xl / g.dx) + 1;
        c->ixr_rg[i] = (int)std::lround(xr / g.dx) + 1;
    }
    c->iyl_rg = (int)std::lround(std::max(yl_rg, 0.0) / g.dy) + 1;  // :325-328
    c->iyr_rg = (int)std::lround(std::min(yr_rg, ymax) / g.dy) + 1;
    c->n_rg = n_rg;
    return LEPIC_OK;
}

// takes the loss holes not yet seen by a sort into the tallies and turns them into plain holes
__global__ void k_loss_scan(const uint32_t *X, const uint32_t *Y, float *VX, const float *VY, const float *VZ,
                            const int32_t *bcnd, TallyDev *tal, const DevCounters *cnt, int sp) {
    const long long n = cnt->n_slots[sp];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float vx = VX[i];
        if (isnan(vx) && loss_hole_tally(tal, sp, bcnd, vx, X[i], Y[i], VY[i], VZ[i])) VX[i] = __int_as_float(HOLE_NAN);
    }
}

int sources_power(lepic_ctx *c, double *P_heat, double *P_inj, double *P_src);
int sources_reset_power(lepic_ctx *c);

extern "C" int lepic_gpu_get_tallies(lepic_ctx *c, lepic_tallies *out, int32_t reset) {
    if (!c || !out) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    for (int s = 0; s < c->cfg.ntype; s++) {
        SpeciesBuf &B = c->sp[s];
        k_loss_scan<<<c->num_sms * 8, 256, 0, c->stream>>>(B.X[B.cur], B.Y[B.cur], B.VX[B.cur], B.VY[B.cur], B.VZ[B.cur],
                                                           c->bcnd, c->tally, c->dcnt, s);
        LCUDA(cudaGetLastError());
    }
    TallyDev *h = new (std::nothrow) TallyDev;
    if (!h) return LEPIC_ENOMEM;
    cudaError_t e = cudaMemcpyAsync(h, c->tally, sizeof(TallyDev), cudaMemcpyDeviceToHost, c->stream);
    int r = e == cudaSuccess ? lepic_gpu_sync(c) : LEPIC_ECUDA;
    const lepic_config &g = c->cfg;
    memset(out, 0, sizeof(*out));
    double P_heat = 0.0, P_inj[LEPIC_MAXSP] = {0}, P_src[LEPIC_MAXSP] = {0};
    if (r == LEPIC_OK) r = sources_power(c, &P_heat, P_inj, P_src);
    for (int s = 0; s < g.ntype; s++) {
        const double Ek = 0.5 * g.Nm[s] * g.mass[s];
        double lost = 0.0;
        for (int l = 0; l < LEPIC_MAXLABEL; l++) {
            out->n_loss[s][l] = (int64_t)h->n_loss[s][l];
            out->P_w[s][l] = Ek * h->v2_loss[s][l];
            lost += out->P_w[s][l];
        }
        out->P_loss[0][s] = lost + P_src[s] + h->P1z[s] + h->P1r[s];
        out->P_loss[1][s] = s == 0 ? P_heat : 0.0;
        out->P_loss[2][s] = h->P3[s];
        out->P_loss[3][s] = P_inj[s] + h->P4r[s];
    }
    memcpy(out->cnt_col, h->cnt_col, sizeof(out->cnt_col));
    out->n_rg = c->n_rg;
    delete h;
    if (r == LEPIC_OK && reset) {
        // the per-step inv_np_rg stays; everything cumulative is zeroed
        LCUDA(cudaMemsetAsync(c->tally, 0, offsetof(TallyDev, inv_np_rg), c->stream));
        r = sources_reset_power(c);
        if (r == LEPIC_OK) LCUDA(cudaStreamSynchronize(c->stream));
    }
    return r;
}
