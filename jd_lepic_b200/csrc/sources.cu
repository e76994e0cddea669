// sources.cu -- the particle sources of the per-step region: electron heating
// (e_heating.f90:1-112), the heating-region tallies of charge_deposition
// (part_expmover.f90:583-605) with the self-consistent temperature update
// (main.f90:984-1011), and volume injection (part_injection.f90:1-237).
//
// Random numbers: Philox4x32-10 streams keyed by the source seed, one counter per decision
// (group of 4 slots and step for the heating decision, one word per slot; slot and step for
// the new velocity; species, injected index, attempt and step for injection), so
// every particle's draws are independent of the launch shape and of the other particles.
// The reference draws from one sequential ran2 stream per OpenMP thread; the two differ in
// which numbers are drawn, not in the distributions (the oracle holds both forms).
//
// Tallies are summed per thread in FP64, reduced per CTA by a fixed tree, and the CTA
// partials of a fixed grid are added in CTA order by one finishing CTA: the sums do not
// depend on scheduling, so a run is bit-reproducible.
//
// Roofline (HBM): heating and the tally read X, Y of every electron slot (8 B) and the
// velocities of the electrons in the heating region (12 B); heating writes the velocities of
// the heated ones (12 B).  Injection writes 20 B per injected particle plus 4 atomics.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include "lepic_internal.cuh"

#define SRC_THREADS 256
#define SRC_BLOCKS 592          // fixed grids of the scanning kernels (bit-reproducible sums):
#define HEAT_BLOCKS 444         // 4 and 3 CTAs per SM of a B200
#define INJ_THREADS 128
#define INJ_BLOCKS 64
#define INJ_MAX_ATTEMPTS 65536  // rejection-sampling attempts per injected particle

#define TAG_HEAT 0x48454154u    // heating decision
#define TAG_HEATV 0x48564C31u   // heating velocity
#define TAG_INJN 0x494E4A4Eu    // injection count rounding
#define TAG_INJP 0x494E4A50u    // injection position attempt
#define TAG_INJV 0x494E4A56u    // injection velocity
#define TAG_INJF 0x494E4A46u    // opt_inj = 4: shifted-flux attempt
#define TAG_INJG 0x494E4A47u    // opt_inj = 4: transverse velocity and time offset
#define TAG_FXN 0x46584E31u     // emission count rounding
#define TAG_FXP 0x46585031u     // emission attempt position
#define TAG_FXV 0x46585631u     // emission velocity and time offset
#define EMIT_THREADS 512

// device tallies and per-call state of the sources
struct SrcDev {
    double P_heat;
    unsigned long long n_heated, n_heat_calls;
    double P_inj[LEPIC_MAXSP], P_src[LEPIC_MAXSP];
    unsigned long long n_inj[LEPIC_MAXSP], n_inj_last[LEPIC_MAXSP];
    unsigned long long lost_mark[LEPIC_MAXSP];  // n_lost at the last injection (|opt_inj| = 2)
    long long inj_start[LEPIC_MAXSP];           // first slot of this call's injected particles
    long long inj_count[LEPIC_MAXSP];
    long long Nh[LEPIC_MAXICP];
    double sum_dEk[LEPIC_MAXICP];
    double vt[LEPIC_MAXICP];
    double Pabs[LEPIC_MAXICP];
    unsigned long long n_emit[LEPIC_MAXSP], n_emit_last[LEPIC_MAXSP], n_emit_out;
};

struct SrcState {
    lepic_source_config cfg;
    SrcDev *d = nullptr;
    double *part = nullptr;      // SRC_BLOCKS * (2 * LEPIC_MAXICP) CTA partials
    int tally_it = INT_MIN;      // the step whose end the last region tally reflects
};

// The region of read_input.f90:43-55: slit or disk, centre xa, half width dr.
// For the slit, the tests are monotone in the fixed-point X and Y (x = X ux is monotone, and
// so is each side of (x - xa)^2), so the host turns them into exact integer intervals by a
// binary search over the same FP64 expressions the device would evaluate: the kernels then
// compare integers, with the same result bit for bit.
struct Region {
    int disk;
    double xl, xr, yl, yr, xa, dr, ymid;
    uint32_t hx0, hx1, hy0, hy1;    // slit heating test (e_heating.f90:52-54): X, Y intervals
    uint32_t tx0, tx1, ty0, ty1;    // slit tally test (part_expmover.f90:585-587); lo > hi: empty
};

// first X in [a, b] where pred turns true (pred false then true on [a, b]); b + 1 if never
template <class F>
static long long first_true(long long a, long long b, F pred) {
    long long lo = a, hi = b + 1;
    while (lo < hi) {
        const long long m = lo + (hi - lo) / 2;
        if (pred(m)) hi = m;
        else lo = m + 1;
    }
    return lo;
}

static Region make_region(const lepic_source_config &s, const lepic_config &g, int S) {
    Region R;
    R.disk = s.flag_c;
    R.xl = s.xl_pow; R.xr = s.xr_pow; R.yl = s.yl_pow; R.yr = s.yr_pow;
    R.xa = (s.xl_pow + s.xr_pow) / 2.0;
    R.dr = (s.xr_pow - s.xl_pow) / 2.0;
    R.ymid = (double)g.ny * g.dy / 2.0;
    const double ux = g.dx * std::ldexp(1.0, -S), uy = g.dy * std::ldexp(1.0, -S);
    const long long xm = ((long long)g.nx << S) - 1, ym = ((long long)g.ny << S) - 1;
    const double dr2 = R.dr * R.dr;
    auto xv = [&](long long X) { return (double)X * ux; };
    auto yv = [&](long long Y) { return (double)Y * uy; };
    // heating: (x - xa)^2 <= dr^2 around the centre, yl <= y <= yr
    auto hin = [&](long long X) { const double x = xv(X); return (x - R.xa) * (x - R.xa) <= dr2; };
    const long long xc = std::min(xm, std::max(0ll, (long long)std::llround(R.xa / ux)));
    // intervals [lo, hi] of [0, 2^32); an empty one is stored as lo = 1, hi = 0
    auto put = [](long long lo, long long hi, uint32_t &a, uint32_t &b) {
        if (lo > hi) { a = 1; b = 0; }
        else { a = (uint32_t)lo; b = (uint32_t)hi; }
    };
    long long h0 = 1, h1 = 0;
    if (hin(xc)) {
        h0 = first_true(0, xc, hin);
        h1 = first_true(xc, xm, [&](long long X) { return !hin(X); }) - 1;
    }
    put(h0, h1, R.hx0, R.hx1);
    put(first_true(0, ym, [&](long long Y) { return yv(Y) >= R.yl; }),
        first_true(0, ym, [&](long long Y) { return yv(Y) > R.yr; }) - 1, R.hy0, R.hy1);
    // tally: xl <= x <= xr, yl <= y <= yr
    put(first_true(0, xm, [&](long long X) { return xv(X) >= R.xl; }),
        first_true(0, xm, [&](long long X) { return xv(X) > R.xr; }) - 1, R.tx0, R.tx1);
    R.ty0 = R.hy0;
    R.ty1 = R.hy1;
    return R;
}

static SrcState *state(lepic_ctx *c) { return (SrcState *)c->src; }

// one CTA's sums of NV values per thread (in shared memory, column = thread), reduced by a
// fixed tree and written to the CTA's partial row
template <int NT>
__device__ void cta_reduce_rows(double *col, int nv, double *out_row) {
    __syncthreads();
    for (int h = NT / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h)
            for (int v = 0; v < nv; v++) col[v * NT + threadIdx.x] += col[v * NT + threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < nv; v++) out_row[v] = col[v * NT];
}

// ---------------------------------------------------------------------------------------
// eheating (e_heating.f90:33-108) over the electron slots.  Each thread takes groups of 4
// consecutive slots (one 16-byte load of X and of Y per group, two groups in flight); only
// the electrons in the region load VX (the hole test), only the heated ones VY, VZ.
struct HeatP {
    const uint32_t *X, *Y;
    float *VX, *VY, *VZ;
    const DevCounters *cnt;
    const SrcDev *src;
    Region R;
    double ux, uy, ymax, dt, nudt, Pabs_cor, Ek;  // Ek = 0.5 Nm m
    double vt_const;                             // > 0: every band heats at this speed
    int n_icp, gpp, type;
    uint32_t it, k0, k1;
};

// the new velocity of a heated electron (e_heating.f90:67-103); returns its energy gain.
// Out of line: the rare path keeps its registers away from the scan loop.
__device__ __noinline__ double heat_apply(float *VX, float *VY, float *VZ, long long k, double vt, int type, double Ek,
                                          uint32_t it, uint32_t k0, uint32_t k1) {
    const float vx = VX[k], vy = VY[k], vz = VZ[k];
    const U4 q = philox4x32_10(U4{(uint32_t)k, (uint32_t)(k >> 32), TAG_HEATV, it}, k0, k1);
    double dvx, dvy, dvz, unused;
    gauss_pair(vt, q.x, q.y, &dvx, &dvy);
    gauss_pair(vt, q.z, q.w, &dvz, &unused);
    const double v2old = (double)vx * vx + (double)vy * vy + (double)vz * vz;
    float nx_, ny_, nz_;
    if (type == 1) {
        nx_ = (float)dvx; ny_ = (float)dvy; nz_ = (float)dvz;
    } else {
        nx_ = (float)((double)vx + dvx); ny_ = (float)((double)vy + dvy); nz_ = (float)((double)vz + dvz);
    }
    VX[k] = nx_; VY[k] = ny_; VZ[k] = nz_;
    return Ek * ((double)nx_ * nx_ + (double)ny_ * ny_ + (double)nz_ * nz_ - v2old);
}

// the heating region test of e_heating.f90:51-58 (the slit as integer intervals)
__device__ __forceinline__ bool heat_in(const HeatP &P, uint32_t Xk, uint32_t Yk, double dr2) {
    if (P.R.disk == 0) return Xk >= P.R.hx0 && Xk <= P.R.hx1 && Yk >= P.R.hy0 && Yk <= P.R.hy1;
    const double x = (double)Xk * P.ux, y = (double)Yk * P.uy;
    return (x - P.R.xa) * (x - P.R.xa) + (y - P.R.ymid) * (y - P.R.ymid) <= dr2;
}
// rp2 as the reference forms it, for the Gaussian profile
__device__ __forceinline__ double heat_rp2(const HeatP &P, uint32_t Xk, uint32_t Yk) {
    const double x = (double)Xk * P.ux;
    if (P.R.disk == 0) return (x - P.R.xa) * (x - P.R.xa);
    const double y = (double)Yk * P.uy;
    return (x - P.R.xa) * (x - P.R.xa) + (y - P.R.ymid) * (y - P.R.ymid);
}

// one group of 4 consecutive slots (k0 = 4 g): the region and hole tests give a candidate
// mask; if it is not empty, one Philox draw decides the group (slot k takes word k & 3)
__device__ __forceinline__ void heat_group(const HeatP &P, long long k0, const uint32_t *xs, const uint32_t *ys,
                                           long long n, double dr2, double &dE, unsigned &cnt) {
    unsigned mask = 0;
#pragma unroll
    for (int p = 0; p < 4; p++)
        if (k0 + p < n && heat_in(P, xs[p], ys[p], dr2) && !isnan(P.VX[k0 + p])) mask |= 1u << p;  // NaN: a hole
    if (!mask) return;
    const long long g = k0 >> 2;
    const U4 r = philox4x32_10(U4{(uint32_t)g, (uint32_t)(g >> 32), TAG_HEAT, P.it}, P.k0, P.k1);
    const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int p = 0; p < 4; p++) {
        if (!(mask >> p & 1u)) continue;
        double nu_tmp = P.nudt / P.dt;
        if (P.gpp) nu_tmp = (P.nudt / P.dt) * 9.0 * P.Pabs_cor * exp(-9.0 * heat_rp2(P, xs[p], ys[p]) / dr2);
        if (!(u01(w[p]) <= nu_tmp * P.dt)) continue;
        int band = 0;
        if (P.n_icp > 1) {
            band = (int)(P.n_icp * ((double)ys[p] * P.uy) / P.ymax);
            band = band < 0 ? 0 : (band >= P.n_icp ? P.n_icp - 1 : band);
        }
        const double vt = P.vt_const > 0.0 ? P.vt_const : P.src->vt[band];
        dE += heat_apply(P.VX, P.VY, P.VZ, k0 + p, vt, P.type, P.Ek, P.it, P.k0, P.k1);
        cnt++;
    }
}

// the slot groups of one thread, software-pipelined: the next group's X, Y (one 16-byte
// load each) are issued before the current group is processed; f(k0, xs, ys)
template <int NBLK, class F>
__device__ __forceinline__ void scan_groups(const uint32_t *X, const uint32_t *Y, long long n, F f) {
    const long long ngroups = (n + 3) >> 2;
    const long long stride = (long long)NBLK * SRC_THREADS;
    long long g = blockIdx.x * (long long)SRC_THREADS + threadIdx.x;
    if (g >= ngroups) return;
    // storage is whole groups of 8 slots: a group's vector stays inside the allocation
    uint4 xc = __ldcs(reinterpret_cast<const uint4 *>(X) + g), yc = __ldcs(reinterpret_cast<const uint4 *>(Y) + g);
    for (; g < ngroups; g += stride) {
        const long long h = g + stride;
        uint4 xn = xc, yn = yc;
        if (h < ngroups) {
            xn = __ldcs(reinterpret_cast<const uint4 *>(X) + h);
            yn = __ldcs(reinterpret_cast<const uint4 *>(Y) + h);
        }
        const uint32_t xs[4] = {xc.x, xc.y, xc.z, xc.w}, ys[4] = {yc.x, yc.y, yc.z, yc.w};
        f(g << 2, xs, ys);
        xc = xn;
        yc = yn;
    }
}

__global__ void __launch_bounds__(SRC_THREADS, 3) k_eheat(HeatP P, double *part) {
    __shared__ double col[2 * SRC_THREADS];
    const long long n = P.cnt->n_slots[0];
    double dE = 0.0;
    unsigned cnt = 0;
    const double dr2 = P.R.dr * P.R.dr;
    scan_groups<HEAT_BLOCKS>(P.X, P.Y, n, [&](long long k0, const uint32_t *xs, const uint32_t *ys) {
        heat_group(P, k0, xs, ys, n, dr2, dE, cnt);
    });
    col[threadIdx.x] = dE;
    col[SRC_THREADS + threadIdx.x] = (double)cnt;
    cta_reduce_rows<SRC_THREADS>(col, 2, part + 2 * blockIdx.x);
}

// heating-region tally of charge_deposition (part_expmover.f90:583-605)
struct TallyP {
    const uint32_t *X, *Y;
    const float *VX, *VY, *VZ;
    const DevCounters *cnt;
    Region R;
    double ux, uy, ymax, Ek;
    int n_icp, type;
};

__global__ void __launch_bounds__(SRC_THREADS, 4) k_heat_tally(TallyP P, double *part) {
    extern __shared__ double col[];   // [2 * n_icp][SRC_THREADS]: Nh then sum_dEk per band
    const int nv = 2 * P.n_icp;
    for (int v = 0; v < nv; v++) col[v * SRC_THREADS + threadIdx.x] = 0.0;
    const long long n = P.cnt->n_slots[0];
    const double dr2 = P.R.dr * P.R.dr;
    scan_groups<SRC_BLOCKS>(P.X, P.Y, n, [&](long long k0, const uint32_t *xs, const uint32_t *ys) {
#pragma unroll
        for (int p = 0; p < 4; p++) {
            const long long k = k0 + p;
            if (k >= n) break;
            if (P.R.disk == 0) {
                if (xs[p] < P.R.tx0 || xs[p] > P.R.tx1 || ys[p] < P.R.ty0 || ys[p] > P.R.ty1) continue;
            } else {
                const double x = (double)xs[p] * P.ux, y = (double)ys[p] * P.uy;
                if ((x - P.R.xa) * (x - P.R.xa) + (y - P.R.ymid) * (y - P.R.ymid) > dr2) continue;
            }
            const float vx = P.VX[k];
            if (isnan(vx)) continue;
            int band = 0;
            if (P.n_icp > 1) {
                band = (int)(P.n_icp * ((double)ys[p] * P.uy) / P.ymax);
                band = band < 0 ? 0 : (band >= P.n_icp ? P.n_icp - 1 : band);
            }
            col[band * SRC_THREADS + threadIdx.x] += 1.0;
            if (P.type == 1) {
                const float vy = P.VY[k], vz = P.VZ[k];
                col[(P.n_icp + band) * SRC_THREADS + threadIdx.x] +=
                    P.Ek * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
            }
        }
    });
    cta_reduce_rows<SRC_THREADS>(col, nv, part + (size_t)nv * blockIdx.x);
}

// Sums column v of the CTA partials part[b * nv + v] (b < nblocks) in a fixed order -- one
// CTA per value, a fixed stride per thread, then a fixed tree -- and applies the sum.
#define FIN_HEAT 0    // v = 0: P_heat +=, v = 1: n_heated +=, calls += 1
#define FIN_TALLY 1   // v < n_icp: Nh[v] =, else sum_dEk[v - n_icp] =
#define FIN_INJ 2     // v < MAXSP: P_inj[v] +=, else P_src[v - MAXSP] +=
__global__ void __launch_bounds__(256) k_finish(const double *part, int nblocks, int nv, int kind, SrcDev *src) {
    __shared__ double red[256];
    const int v = blockIdx.x;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 256) s += part[(size_t)b * nv + v];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    s = red[0];
    if (kind == FIN_HEAT) {
        if (v == 0) src->P_heat += s;
        else { src->n_heated += (unsigned long long)s; src->n_heat_calls += 1; }
    } else if (kind == FIN_TALLY) {
        const int nb = nv / 2;
        if (v < nb) src->Nh[v] = (long long)s;
        else src->sum_dEk[v - nb] = s;
    } else {
        if (v < LEPIC_MAXSP) src->P_inj[v] += s;
        else src->P_src[v - LEPIC_MAXSP] += s;
    }
}

// main.f90:1003-1010 for one rank: Te from the tallies, vt = sqrt(2 qe Te / |m|)
__global__ void k_te_update(SrcDev *src, int n_icp, int type, double nu_h, double Nm, double qe, double mass) {
    const int b = threadIdx.x;
    if (b >= n_icp) return;
    const long long nh = src->Nh[b];
    if (nh <= 0) return;  // the reference divides by zero here; the previous speed is kept
    double Te;
    if (type == 1) Te = (2.0 / 3.0) * (src->sum_dEk[b] + src->Pabs[b] / nu_h) / (Nm * qe * (double)nh);
    else Te = (2.0 / 3.0) * (src->Pabs[b] / nu_h) / (Nm * qe * (double)nh);
    src->vt[b] = sqrt(2.0 * qe * Te / fabs(mass));
}

// ---------------------------------------------------------------------------------------
// part_injection (part_injection.f90:49-233)
struct InjPlanP {
    DevCounters *cnt;
    SrcDev *src;
    int ntype, opt2, tag_neg, electrons_only;
    long long cap[LEPIC_MAXSP];
    double dN_fixed[LEPIC_MAXSP];  // |opt_inj| = 1: I_inj ns_inj dt ni0 / (qe Nm(1)) / nproc_mpi
    double ni0[LEPIC_MAXSP];
    uint32_t it, k0, k1;
};

// the counts of part_injection.f90:49-75 for every species, in the order of main.f90:1058
__global__ void k_inj_plan(InjPlanP P) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    long long lost[LEPIC_MAXSP];
    for (int s = 0; s < P.ntype; s++) lost[s] = (long long)(P.cnt->n_lost[s] - P.src->lost_mark[s]);
    long long pos_lost = 0;  // SUM(N_inj(2:ntype)) - N_inj(tag_neg)
    for (int s = 1; s < P.ntype; s++)
        if (s != P.tag_neg) pos_lost += lost[s];
    for (int s = 0; s < P.ntype; s++) {
        long long N;
        bool draw = true;
        double dN = 0.0;
        if (P.opt2) {
            if (s == 0 || s == P.tag_neg) dN = P.ni0[s] * (double)pos_lost;
            else { N = lost[s]; draw = false; }  // the positive ion's own losses
        } else {
            dN = P.dN_fixed[s];
        }
        if (draw) {
            N = (long long)dN;
            const U4 r = philox4x32_10(U4{(uint32_t)s, 0u, TAG_INJN, P.it}, P.k0, P.k1);
            if (u01(r.x) <= dN - (double)N) N += 1;
        }
        if (P.electrons_only && s > 0) N = 0;  // part_injection.f90:77-79
        const long long start = P.cnt->n_slots[s];
        if (start + N > P.cap[s]) {  // part_injection.f90:146-150
            set_err(P.cnt, LERR_CAPACITY, 700 + s);
            N = 0;
        }
        P.src->inj_start[s] = start;
        P.src->inj_count[s] = N;
        P.src->n_inj[s] += (unsigned long long)N;
        P.src->n_inj_last[s] = (unsigned long long)N;
        P.cnt->n_slots[s] = start + N;
        P.cnt->n_alive[s] += N;
    }
    for (int s = 0; s < P.ntype; s++) P.src->lost_mark[s] = P.cnt->n_lost[s];
}

struct InjP {
    SrcDev *src;
    DevCounters *cnt;
    int ntype, nx, ny, S, W;
    int opt, slit, flag_nmn, diffsrc;
    double vb[LEPIC_MAXSP], fmax[LEPIC_MAXSP];   // |opt_inj| = 3, 4: beam speed, flux maximum
    double sin_thB, cos_thB, ns_dt;
    Region R;
    double dx, dy, xmax, ymax;
    double vt[LEPIC_MAXSP], Ek[LEPIC_MAXSP], qphi[LEPIC_MAXSP];  // qphi = -Nm q
    const uint8_t *cellwall;
    const double *phi;
    uint32_t *X[LEPIC_MAXSP], *Y[LEPIC_MAXSP];
    float *VX[LEPIC_MAXSP], *VY[LEPIC_MAXSP], *VZ[LEPIC_MAXSP];
    float *Z[LEPIC_MAXSP];  // the 3rd dimension's z (null without it)
    double zmax;
    unsigned long long *acc[LEPIC_MAXSP];
    unsigned int *ss_map;   // ss2D counts (null: not accumulated), see lepic_ctx::ss_map
    long long ss_nn;
    uint32_t it, k0, k1;
};

__device__ __forceinline__ void inj_cic(int S, uint32_t X, uint32_t Y, uint64_t *w) {
    // the push's integer CIC weights (exact products of the offsets, scaled to 2^44)
    const uint32_t mask = (1u << S) - 1u, A = 1u << S;
    const uint32_t fx = X & mask, fy = Y & mask, ax = A - fx, ay = A - fy;
    w[0] = (uint64_t)ax * ay; w[1] = (uint64_t)fx * ay; w[2] = (uint64_t)fx * fy; w[3] = (uint64_t)ax * fy;
    const int sh = 2 * S - LEPIC_DEP_SHIFT;
    for (int k = 0; k < 4; k++) {
        if (sh > 0) w[k] = (w[k] + (1ull << (sh - 1))) >> sh;
        else if (sh < 0) w[k] <<= -sh;
    }
}

__global__ void __launch_bounds__(INJ_THREADS) k_inject(InjP P, double *part) {
    __shared__ double col[2 * LEPIC_MAXSP * INJ_THREADS];  // P_inj then P_src per species
    for (int v = 0; v < 2 * LEPIC_MAXSP; v++) col[v * INJ_THREADS + threadIdx.x] = 0.0;
    long long total = 0;
    for (int s = 0; s < P.ntype; s++) total += P.src->inj_count[s];
    const double dr2 = P.R.dr * P.R.dr;
    for (long long t = blockIdx.x * (long long)INJ_THREADS + threadIdx.x; t < total;
         t += (long long)INJ_BLOCKS * INJ_THREADS) {
        int s = 0;
        long long j = t;
        while (j >= P.src->inj_count[s]) { j -= P.src->inj_count[s]; s++; }
        // position: part_injection.f90:85-137, redrawn until the cell is not all walls
        double x = 0.0, y = 0.0;
        int ix = 1, iy = 1;
        bool ok = false;
        for (uint32_t a = 0; a < INJ_MAX_ATTEMPTS && !ok; a++) {
            const U4 r = philox4x32_10(U4{(uint32_t)j, (a << 3) | (uint32_t)s, TAG_INJP, P.it}, P.k0, P.k1);
            if (P.opt > 0) {
                x = u01(r.x) * (P.R.xl - P.R.xr) + P.R.xr;
                if (P.R.disk) {
                    y = u01(r.y) * (2.0 * P.R.dr) + P.R.ymid - P.R.dr;
                    if ((x - P.R.xa) * (x - P.R.xa) + (y - P.R.ymid) * (y - P.R.ymid) > dr2) continue;
                }
            } else if (!P.R.disk) {
                double g0, g1;
                gauss_pair(P.R.dr, r.x, r.y, &g0, &g1);
                x = g0 + P.R.xa;
                if (P.flag_nmn == 1 && P.R.xa == 0.0) x = fabs(x);
                if (x < P.R.xa - 4.0 * P.R.dr || x > P.R.xa + 4.0 * P.R.dr || x < 0.0 || x > P.xmax) continue;
            } else {
                double g0, g1;
                gauss_pair(P.R.dr, r.x, r.y, &g0, &g1);
                x = g0 + P.R.xa;
                y = g1 + P.R.ymid;
                if ((x - P.R.xa) * (x - P.R.xa) + (y - P.R.ymid) * (y - P.R.ymid) > 4.0 * dr2 || x < 0.0 ||
                    x > P.xmax || y < 0.0 || y > P.ymax)
                    continue;
            }
            if (!P.R.disk) y = u01(r.z) * (P.R.yl - P.R.yr) + P.R.yr;
            ix = (int)(x / P.dx) + 1;
            iy = (int)(y / P.dy) + 1;
            ix = ix < 1 ? 1 : (ix > P.nx + 1 ? P.nx + 1 : ix);
            iy = iy < 1 ? 1 : (iy > P.ny + 1 ? P.ny + 1 : iy);
            if (P.cellwall[ix + (long long)iy * (P.nx + 2)]) continue;
            ok = true;
        }
        const long long slot = P.src->inj_start[s] + j;
        if (!ok) {  // a region with no room: the slot stays a hole and the call fails
            set_err(P.cnt, LERR_RANGE, 710 + s);
            P.VX[s][slot] = __int_as_float(HOLE_NAN);
            P.X[s][slot] = 0; P.Y[s][slot] = 0; P.VY[s][slot] = 0.f; P.VZ[s][slot] = 0.f;
            continue;
        }
        // velocity: part_injection.f90:152-194, with its draw order: the first particle of a
        // call takes (vx, vy) and vz from the second pair (so vz = vx), the next takes its own
        // (vx, vy) and the saved second component of the previous particle's second pair
        const double vt = P.vt[s];
        double vx, vy, vz;
        if (P.opt == 4 || P.opt == -4) {
            // part_injection.f90:161-178: vx from the shifted-Maxwellian flux about vb cos(th_B)
            // (acceptance-rejection, :239-265), (vy, vz) Maxwellian with vy += vb sin(th_B), and
            // the particle moved off the cathode at x = 0 by vx times a random part of ns_inj dt
            const double vbt = P.vb[s] * P.cos_thB;
            const double vm = fmax(0.0, vbt - 4.0 * vt), vpm = vbt + 4.0 * vt;
            bool got = false;
            vx = vy = vz = 0.0;
            for (uint32_t a = 0; a < INJ_MAX_ATTEMPTS && !got; a++) {
                const U4 f = philox4x32_10(U4{(uint32_t)j, (a << 3) | (uint32_t)s, TAG_INJF, P.it}, P.k0, P.k1);
                const double v = vm + u01(f.x) * (vpm - vm);
                const double fv = v * exp(-(v - vbt) * (v - vbt) / (vt * vt));
                if (u01(f.y) > fv / P.fmax[s]) continue;
                gauss_pair(vt, f.z, f.w, &vy, &vz);
                const U4 g2 = philox4x32_10(U4{(uint32_t)j, (a << 3) | (uint32_t)s, TAG_INJG, P.it}, P.k0, P.k1);
                const double xn = v * (u01(g2.x) * P.ns_dt);
                if (xn < 0.0 || xn > P.xmax) continue;
                vx = v;
                vy = vy + P.vb[s] * P.sin_thB;
                x = xn;
                got = true;
            }
            if (!got) {
                set_err(P.cnt, LERR_RANGE, 720 + s);
                P.VX[s][slot] = __int_as_float(HOLE_NAN);
                P.X[s][slot] = 0; P.Y[s][slot] = 0; P.VY[s][slot] = 0.f; P.VZ[s][slot] = 0.f;
                continue;
            }
            ix = (int)floor(x / P.dx) + 1;
            ix = ix < 1 ? 1 : (ix > P.nx + 1 ? P.nx + 1 : ix);
        } else {
            const U4 q = philox4x32_10(U4{(uint32_t)j, (uint32_t)s, TAG_INJV, P.it}, P.k0, P.k1);
            if ((j & 1) == 0) {
                gauss_pair(vt, q.z, q.w, &vx, &vy);
                vz = vx;
            } else {
                gauss_pair(vt, q.x, q.y, &vx, &vy);
                const U4 qp = philox4x32_10(U4{(uint32_t)(j - 1), (uint32_t)s, TAG_INJV, P.it}, P.k0, P.k1);
                double unused;
                gauss_pair(vt, qp.z, qp.w, &unused, &vz);
            }
            if (P.opt == 3 || P.opt == -3) vz = vz + P.vb[s];  // :202 beam along z
        }
        // fixed point: x/h truncated, so the cell is the reference's INT(x/h)
        const double fx = x / P.dx * (double)(1u << P.S), fy = y / P.dy * (double)(1u << P.S);
        const long long xl = ((long long)P.nx << P.S) - 1, yl = ((long long)P.ny << P.S) - 1;
        const uint32_t Xf = (uint32_t)min((long long)fx, xl), Yf = (uint32_t)min((long long)fy, yl);
        const float fvx = (float)vx, fvy = (float)vy, fvz = (float)vz;
        P.X[s][slot] = Xf; P.Y[s][slot] = Yf;
        P.VX[s][slot] = fvx; P.VY[s][slot] = fvy; P.VZ[s][slot] = fvz;
        if (P.Z[s]) {   // z = rnd zmax (part_injection.f90:129)
            const U4 zq = philox4x32_10(U4{(uint32_t)j, (uint32_t)s, 0x495A504Fu, P.it}, P.k0, P.k1);
            P.Z[s][slot] = (float)(u01(zq.x) * P.zmax);
        }
        if (P.ss_map)   // part_injection.f90:205: the source at the particle's (ix, iy)
            atomicAdd(P.ss_map + (size_t)(2 * s) * P.ss_nn + ix + (long long)iy * P.W, 1u);
        // deposit (the injected particle is in this step's np)
        uint64_t w[4];
        inj_cic(P.S, Xf, Yf, w);
        const long long n00 = (long long)((Xf >> P.S) + 1) + (long long)((Yf >> P.S) + 1) * P.W;
        unsigned long long *a = P.acc[s];
        if (w[0]) atomicAdd(a + n00, (unsigned long long)w[0]);
        if (w[1]) atomicAdd(a + n00 + 1, (unsigned long long)w[1]);
        if (w[2]) atomicAdd(a + n00 + P.W + 1, (unsigned long long)w[2]);
        if (w[3]) atomicAdd(a + n00 + P.W, (unsigned long long)w[3]);
        col[s * INJ_THREADS + threadIdx.x] +=
            P.Ek[s] * ((double)fvx * fvx + (double)fvy * fvy + (double)fvz * fvz);
        if (P.diffsrc) {  // part_injection.f90:216-231
            const double px = ((double)ix * P.dx - x) / P.dx, py = ((double)iy * P.dy - y) / P.dy;
            const long long m = ix + (long long)iy * P.W;
            const double phip = px * py * P.phi[m] + (1.0 - px) * py * P.phi[m + 1] +
                                (1.0 - px) * (1.0 - py) * P.phi[m + P.W + 1] + px * (1.0 - py) * P.phi[m + P.W];
            col[(LEPIC_MAXSP + s) * INJ_THREADS + threadIdx.x] += P.qphi[s] * phip;
        }
    }
    cta_reduce_rows<INJ_THREADS>(col, 2 * LEPIC_MAXSP, part + (size_t)2 * LEPIC_MAXSP * blockIdx.x);
}

// ---------------------------------------------------------------------------------------
// part_flux_emitter (part_flux_emitter.f90:21-214).  Attempts are numbered a = 0, 1, ... and
// processed in order, 512 per round by one CTA; each draws from its own stream.  An attempt
// on a wall face (part_flux_emitter.f90:141-144) adds to the counts of plasma nodes on its
// left and right; those counts run over all attempts of the call, and the attempt is kept
// when they differ (the flux direction: part_flux_emitter.f90:145-157).  Block prefix sums
// give every attempt its running counts and every kept attempt its particle index, so the
// result is the sequential algorithm's; the call stops at the Nh-th particle.
struct EmitP {
    DevCounters *cnt;
    SrcDev *src;
    int nx, ny, S, W;
    double dx, dy, xmax, ymax, ns_dt;
    double xg1, Lg, y1c, th_c;
    int n_icp, chamfer;
    int sp[2];                      // species of flat-surface and chamfer emission
    double dNh;
    double vt[2], Ek[2];
    long long cap[2];
    const int32_t *bcnd;
    uint32_t *X[2], *Y[2];
    float *VX[2], *VY[2], *VZ[2];
    float *Z[2];            // the 3rd dimension's z (null without it)
    double zmax;
    long long max_attempts_extra;
    unsigned int *ss_map;   // ss2D counts (null: not accumulated), see lepic_ctx::ss_map
    long long ss_nn;
    uint32_t it, k0, k1;
};

// exclusive prefix (in thread order) and block total of a predicate
__device__ __forceinline__ int block_prefix(bool p, int *wcnt, int &total) {
    const unsigned b = __ballot_sync(0xffffffffu, p);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wcnt[w] = __popc(b);
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < EMIT_THREADS / 32; i++) {
        const int c = wcnt[i];
        off += i < w ? c : 0;
        tot += c;
    }
    __syncthreads();
    total = tot;
    return off + __popc(b & ((1u << lane) - 1u));
}

__global__ void __launch_bounds__(EMIT_THREADS) k_emit(EmitP P) {
    __shared__ int wcnt[EMIT_THREADS / 32];
    __shared__ long long s_l, s_r, s_tot, s_n[2], s_start[2], s_Nh, s_out[2];
    __shared__ double red[2][EMIT_THREADS];
    const double pi = 3.141592653589793;
    if (threadIdx.x == 0) {
        long long N = (long long)P.dNh;
        const U4 r = philox4x32_10(U4{0u, 0u, TAG_FXN, P.it}, P.k0, P.k1);  // part_flux_emitter.f90:47-51
        if (u01(r.x) <= P.dNh - (double)N) N += 1;
        s_Nh = N;
        s_l = s_r = s_tot = 0;
        for (int q = 0; q < 2; q++) { s_n[q] = 0; s_out[q] = 0; s_start[q] = P.cnt->n_slots[P.sp[q]]; }
    }
    __syncthreads();
    const long long Nh = s_Nh;
    const long long max_att = 64 * Nh + P.max_attempts_extra;
    double e[2] = {0.0, 0.0};
    for (long long base = 0; s_tot < Nh && base < max_att; base += EMIT_THREADS) {
        const long long a = base + threadIdx.x;
        bool wall = false, lh = false, rh = false;
        int q = 0, eix = 0, eiy = 0;   // the attempt's node (ix, iy)
        double x = P.xg1, y = 0.0, th = pi / 2.0;
        if (a < max_att) {
            const U4 r = philox4x32_10(U4{(uint32_t)a, (uint32_t)(a >> 32), TAG_FXP, P.it}, P.k0, P.k1);
            y = P.n_icp == 1 ? (P.ymax - P.Lg) / 2.0 + P.Lg * u01(r.x) : P.ymax * (1.0 - u01(r.x));
            const double h2 = P.ymax / 2.0;
            if (P.chamfer && ((y <= h2 && y > P.y1c) || (y > h2 && fabs(P.ymax - y) > P.y1c))) {
                q = 1;  // part_flux_emitter.f90:114-133
                double thp = P.th_c, d0 = y - P.y1c, d1 = P.y1c;
                if (y > h2) { thp = -P.th_c; d0 = fabs(y - P.ymax) - P.y1c; d1 = P.ymax - P.y1c; }
                x = P.xg1 + d0 * cos(thp);
                y = d1 + d0 * sin(thp);
            }
            // the rotation of the velocity (part_flux_emitter.f90:187-193), on the moved point
            if (P.chamfer && ((y <= h2 && y > P.y1c) || (y > h2 && fabs(P.ymax - y) > P.y1c)))
                th = y > h2 ? pi / 2.0 + P.th_c : P.th_c;
            const int ix = (int)(x / P.dx) + 1, iy = (int)(y / P.dy) + 1;
            eix = ix; eiy = iy;
            if (ix >= 1 && ix <= P.nx + 1 && iy >= 1 && iy <= P.ny + 1) {  // INT truncates toward 0
                const int32_t *b = P.bcnd;
                const long long m = ix + (long long)iy * P.W;
                wall = (b[m] >= 1 && b[m + P.W] >= 1) || (b[m + 1] >= 1 && b[m + 1 + P.W] >= 1);
                lh = wall && b[m - 1] == -1;
                rh = wall && b[m + 1] == -1;
            }
        }
        int tl, tr, tacc, tacc1;
        const long long cl = s_l + block_prefix(lh, wcnt, tl) + (lh ? 1 : 0);
        const long long cr = s_r + block_prefix(rh, wcnt, tr) + (rh ? 1 : 0);
        const bool acc = wall && cl != cr;
        const double dir = cl > cr ? 1.0 : -1.0;
        const long long j = s_tot + block_prefix(acc, wcnt, tacc);
        const int qe = (P.sp[1] != P.sp[0]) ? q : 0;   // the particle's species slot
        const long long idx1 = block_prefix(acc && qe == 1, wcnt, tacc1);
        const long long idx0 = (j - s_tot) - idx1;      // accepted before it with qe == 0
        if (acc && j < Nh) {
            const long long slot = s_start[qe] + s_n[qe] + (qe ? idx1 : idx0);
            if (P.ss_map)   // part_flux_emitter.f90:175: the source at the attempt's (ix, iy)
                atomicAdd(P.ss_map + (size_t)(2 * P.sp[qe]) * P.ss_nn + eix + (long long)eiy * P.W, 1u);
            const U4 v = philox4x32_10(U4{(uint32_t)j, (uint32_t)(j >> 32), TAG_FXV, P.it}, P.k0, P.k1);
            const double vt = P.vt[qe];
            const double vx = dir * vt * sqrt(-log(1.0 - u01(v.x)));
            double vy, vz;
            gauss_pair(vt, v.y, v.z, &vy, &vz);
            const double vxt = -vx * sin(th) + vy * cos(th), vyt = vx * cos(th) + vy * sin(th);
            const double dt_tmp = u01(v.w) * P.ns_dt;
            const double xn = x + vxt * dt_tmp, yn = y + vyt * dt_tmp;
            const float fvx = (float)vxt, fvy = (float)vyt, fvz = (float)vz;
            e[qe] += P.Ek[qe] * ((double)fvx * fvx + (double)fvy * fvy + (double)fvz * fvz);
            if (slot >= P.cap[qe]) {
                set_err(P.cnt, LERR_CAPACITY, 720 + qe);
            } else if (xn < 0.0 || xn >= P.xmax || yn < 0.0 || yn >= P.ymax) {
                // outside the box after the partial move: a wall loss of the next push
                P.VX[qe][slot] = __int_as_float(HOLE_NAN);
                P.X[qe][slot] = 0; P.Y[qe][slot] = 0; P.VY[qe][slot] = 0.f; P.VZ[qe][slot] = 0.f;
                atomicAdd((unsigned long long *)&s_out[qe], 1ull);
            } else {
                const double fx = xn / P.dx * (double)(1u << P.S), fy = yn / P.dy * (double)(1u << P.S);
                const long long xl = ((long long)P.nx << P.S) - 1, yl = ((long long)P.ny << P.S) - 1;
                P.X[qe][slot] = (uint32_t)min((long long)fx, xl);
                P.Y[qe][slot] = (uint32_t)min((long long)fy, yl);
                P.VX[qe][slot] = fvx; P.VY[qe][slot] = fvy; P.VZ[qe][slot] = fvz;
                if (P.Z[qe]) {   // z_inj = zmax (1 - rnd), moved with vz (part_flux_emitter.f90:139, 207)
                    const U4 zq = philox4x32_10(U4{(uint32_t)slot, (uint32_t)qe, 0x455A504Fu, P.it}, P.k0, P.k1);
                    P.Z[qe][slot] = (float)(P.zmax * (1.0 - u01(zq.x)) + vz * dt_tmp);
                }
            }
        }
        // the created particles of this round per species: those with j < Nh
        const long long made = min((long long)tacc, Nh - s_tot);
        int m1;
        block_prefix(acc && j < Nh && qe == 1, wcnt, m1);
        if (threadIdx.x == 0) {
            s_l += tl;
            s_r += tr;
            s_tot += made;
            s_n[1] += m1;
            s_n[0] += made - m1;
        }
        __syncthreads();
    }
    if (s_tot < Nh && threadIdx.x == 0) set_err(P.cnt, LERR_RANGE, 730);  // no wall face found
    // energy of the emitted particles (P_loss(4)), reduced by a fixed tree
    red[0][threadIdx.x] = e[0];
    red[1][threadIdx.x] = e[1];
    __syncthreads();
    for (int h = EMIT_THREADS / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            red[0][threadIdx.x] += red[0][threadIdx.x + h];
            red[1][threadIdx.x] += red[1][threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int nq = P.sp[1] != P.sp[0] ? 2 : 1;
        for (int q = 0; q < nq; q++) {
            const int sp = P.sp[q];
            const long long n = min(s_n[q], P.cap[q] - s_start[q]);
            P.cnt->n_slots[sp] = s_start[q] + n;
            P.cnt->n_alive[sp] += n - s_out[q];
            P.cnt->n_lost[sp] += (unsigned long long)s_out[q];
            P.src->n_emit[sp] += (unsigned long long)n;
            P.src->n_emit_last[sp] = (unsigned long long)n;
            P.src->n_emit_out += (unsigned long long)s_out[q];
            P.src->P_inj[sp] += red[q][0];
        }
    }
}

// ---------------------------------------------------------------------------------------
// host side
static void keys(const lepic_source_config &s, uint32_t *k0, uint32_t *k1) {
    *k0 = (uint32_t)s.seed;
    *k1 = (uint32_t)(s.seed >> 32) ^ 0x53524331u;
}

void sources_free(lepic_ctx *c) {
    SrcState *S = state(c);
    if (!S) return;
    if (S->d) cudaFree(S->d);
    if (S->part) cudaFree(S->part);
    delete S;
    c->src = nullptr;
}

static int check_config(lepic_ctx *c, const lepic_source_config &s) {
    const lepic_config &g = c->cfg;
    const double xmax = g.nx * g.dx, ymax = g.ny * g.dy;
    auto bad = [&](const char *m) { c->last_err = std::string("sources: ") + m; return LEPIC_EINVAL; };
    if (s.js > 0.0) {
        if (s.ptype_fx < 0 || s.ptype_fx >= g.ntype) return bad("ptype_fx out of range");
        if (s.tag_b < -1 || s.tag_b >= g.ntype) return bad("tag_b out of range");
        if (s.ns_Hm < 1) return bad("ns_Hm < 1");
        if (s.n_icp < 1 || s.n_icp > LEPIC_MAXICP) return bad("n_icp out of range");
        if (!(s.xg1 >= 0.0) || !(s.Lg > 0.0) || !(s.Lh >= 0.0) || s.n_holes < 0) return bad("emitter grid");
        if (s.Lh >= std::min(s.Lg, ymax)) return bad("Lh >= Lg (generate_boundary.f90:249-254)");
        if (!(s.THm > 0.0)) return bad("THm must be > 0 for the emitter");
        if (s.nproc_mpi < 1) return bad("nproc_mpi < 1");
        if (s.flag_chmfrd && s.chmfrd[1] == s.chmfrd[0] && s.chmfrd[3] == s.chmfrd[2]) return bad("chamfer of zero length");
    }
    if (!s.flag_heat && !s.flag_inj) return LEPIC_OK;
    if (s.flag_c != 0 && s.flag_c != 1) return bad("flag_c must be 0 or 1");
    if (!(s.xl_pow >= 0 && s.xr_pow > s.xl_pow)) return bad("need 0 <= xl_pow < xr_pow");
    const double xa = (s.xl_pow + s.xr_pow) / 2.0, dr = (s.xr_pow - s.xl_pow) / 2.0;
    if (s.flag_c == 0) {
        if (s.xr_pow > xmax || !(s.yl_pow >= 0 && s.yr_pow >= s.yl_pow && s.yr_pow <= ymax))
            return bad("slit region outside the box");
    } else if (xa + dr > xmax || ymax / 2.0 - dr < 0.0) {
        return bad("disk region outside the box");
    }
    if (s.flag_heat) {
        if (s.ns_heat < 1) return bad("ns_heat < 1");
        if (s.eheat_type != 1 && s.eheat_type != 2) return bad("eheat_type must be 1 or 2");
        if (s.n_icp < 1 || s.n_icp > LEPIC_MAXICP) return bad("n_icp out of range");
        if (!(s.nudt >= 0.0 && s.nudt <= 1.0)) return bad("nu*dt > 1 (main.f90:519-523)");
        if (s.flag_gpp && s.nudt * 9.0 * s.Pabs_cor > 1.0) return bad("nu0*dt > 1 for the Gaussian profile");
        if (s.te_update && !(s.nu_h > 0.0)) return bad("te_update needs nu_h > 0");
        for (int b = 0; b < s.n_icp; b++)
            if (!(s.vt[b] >= 0.0)) return bad("vt must be >= 0");
    }
    if (s.flag_inj) {
        if (s.ns_inj < 1) return bad("ns_inj < 1");
        const int a = std::abs(s.opt_inj);
        if (a < 1 || a > 4) return bad("opt_inj must be +-1 .. +-4");
        if (a >= 3 && !(s.THm >= 0.0)) return bad("THm < 0");
        if (a == 4) {
            if (!std::isfinite(s.th_B)) return bad("th_B is not finite");
            for (int sp = 0; sp < g.ntype; sp++)
                if (!(g.vt0[sp] > 0.0)) return bad("opt_inj 4 needs vt0 > 0 (init_shifted_maxwellian_flux)");
        }
        if (s.nproc_mpi < 1) return bad("nproc_mpi < 1");
        if (s.tag_neg < -1 || s.tag_neg >= g.ntype || s.tag_neg == 0) return bad("tag_neg out of range");
        if (s.I_inj < 0.0) return bad("I_inj < 0");
    }
    return LEPIC_OK;
}

extern "C" int lepic_gpu_set_sources(lepic_ctx *c, const lepic_source_config *cfg) {
    if (!c || !cfg) return LEPIC_EINVAL;
    int r = check_config(c, *cfg);
    if (r != LEPIC_OK) return r;
    SrcState *S = state(c);
    if (!S) {
        S = new (std::nothrow) SrcState;
        if (!S) return LEPIC_ENOMEM;
        c->src = S;
        if (cudaMalloc((void **)&S->d, sizeof(SrcDev)) != cudaSuccess ||
            cudaMalloc((void **)&S->part, sizeof(double) * SRC_BLOCKS * 2 * LEPIC_MAXICP) != cudaSuccess) {
            c->last_err = "sources: cudaMalloc failed";
            sources_free(c);
            return LEPIC_ENOMEM;
        }
        LCUDA(cudaMemsetAsync(S->d, 0, sizeof(SrcDev), c->stream));
    }
    S->cfg = *cfg;
    S->tally_it = INT_MIN;
    // heating speeds, and the loss mark from which |opt_inj| = 2 counts
    LCUDA(cudaMemcpyAsync(S->d->vt, cfg->vt, sizeof(double) * LEPIC_MAXICP, cudaMemcpyHostToDevice, c->stream));
    LCUDA(cudaMemcpyAsync(S->d->Pabs, cfg->Pabs, sizeof(double) * LEPIC_MAXICP, cudaMemcpyHostToDevice, c->stream));
    LCUDA(cudaMemcpyAsync(S->d->lost_mark, c->dcnt->n_lost, sizeof(unsigned long long) * LEPIC_MAXSP,
                          cudaMemcpyDeviceToDevice, c->stream));
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

extern "C" int lepic_gpu_set_heating(lepic_ctx *c, const double *vt, int32_t n_icp, double Pabs_cor) {
    if (!c || !vt || !state(c)) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    SrcState *S = state(c);
    if (n_icp != S->cfg.n_icp) { c->last_err = "set_heating: n_icp differs from the source config"; return LEPIC_EINVAL; }
    for (int b = 0; b < n_icp; b++)
        if (!(vt[b] >= 0.0)) return LEPIC_EINVAL;
    if (S->cfg.flag_gpp && S->cfg.nudt * 9.0 * Pabs_cor > 1.0) {
        c->last_err = "nu0*dt > 1 for the Gaussian profile (main.f90:1308-1311)";
        return LEPIC_EINVAL;
    }
    S->cfg.Pabs_cor = Pabs_cor;
    for (int b = 0; b < n_icp; b++) S->cfg.vt[b] = vt[b];
    LCUDA(cudaMemcpyAsync(S->d->vt, S->cfg.vt, sizeof(double) * LEPIC_MAXICP, cudaMemcpyHostToDevice, c->stream));
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

static int run_heating(lepic_ctx *c, int it) {
    SrcState *S = state(c);
    const lepic_source_config &s = S->cfg;
    const lepic_config &g = c->cfg;
    SpeciesBuf &B = c->sp[0];
    HeatP P;
    memset(&P, 0, sizeof(P));
    P.X = B.X[B.cur]; P.Y = B.Y[B.cur]; P.VX = B.VX[B.cur]; P.VY = B.VY[B.cur]; P.VZ = B.VZ[B.cur];
    P.cnt = c->dcnt; P.src = S->d;
    P.R = make_region(s, g, c->S);
    P.ux = g.dx * std::ldexp(1.0, -c->S); P.uy = g.dy * std::ldexp(1.0, -c->S);
    P.ymax = g.ny * g.dy; P.dt = g.dt; P.nudt = s.nudt; P.Pabs_cor = s.Pabs_cor;
    P.Ek = 0.5 * g.Nm[0] * g.mass[0];
    P.vt_const = s.flag_inj ? g.vt0[0] : 0.0;  // main.f90:1034
    P.n_icp = s.n_icp; P.gpp = s.flag_gpp; P.type = s.eheat_type;
    P.it = (uint32_t)it;
    keys(s, &P.k0, &P.k1);
    k_eheat<<<HEAT_BLOCKS, SRC_THREADS, 0, c->stream>>>(P, S->part);
    LCUDA(cudaGetLastError());
    k_finish<<<2, 256, 0, c->stream>>>(S->part, HEAT_BLOCKS, 2, FIN_HEAT, S->d);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int run_tally(lepic_ctx *c) {
    SrcState *S = state(c);
    const lepic_source_config &s = S->cfg;
    const lepic_config &g = c->cfg;
    SpeciesBuf &B = c->sp[0];
    TallyP P;
    memset(&P, 0, sizeof(P));
    P.X = B.X[B.cur]; P.Y = B.Y[B.cur]; P.VX = B.VX[B.cur]; P.VY = B.VY[B.cur]; P.VZ = B.VZ[B.cur];
    P.cnt = c->dcnt;
    P.R = make_region(s, g, c->S);
    P.ux = g.dx * std::ldexp(1.0, -c->S); P.uy = g.dy * std::ldexp(1.0, -c->S);
    P.ymax = g.ny * g.dy;
    P.Ek = 0.5 * g.Nm[0] * g.mass[0];
    P.n_icp = std::max(1, std::min(s.n_icp, LEPIC_MAXICP));
    P.type = s.eheat_type;
    const size_t smem = sizeof(double) * 2 * P.n_icp * SRC_THREADS;
    static bool attr[64] = {false};
    if (!attr[c->dev & 63]) {
        LCUDA(cudaFuncSetAttribute(k_heat_tally, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(double) * 2 * LEPIC_MAXICP * SRC_THREADS)));
        attr[c->dev & 63] = true;
    }
    k_heat_tally<<<SRC_BLOCKS, SRC_THREADS, smem, c->stream>>>(P, S->part);
    LCUDA(cudaGetLastError());
    k_finish<<<2 * P.n_icp, 256, 0, c->stream>>>(S->part, SRC_BLOCKS, 2 * P.n_icp, FIN_TALLY, S->d);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int run_injection(lepic_ctx *c, int it) {
    SrcState *S = state(c);
    const lepic_source_config &s = S->cfg;
    const lepic_config &g = c->cfg;
    InjPlanP Q;
    memset(&Q, 0, sizeof(Q));
    Q.cnt = c->dcnt; Q.src = S->d; Q.ntype = g.ntype;
    Q.opt2 = std::abs(s.opt_inj) == 2;
    Q.tag_neg = s.tag_neg;
    Q.electrons_only = std::abs(s.opt_inj) == 3 || (std::abs(s.opt_inj) == 4 && g.flag_nmn == 0);
    for (int sp = 0; sp < g.ntype; sp++) {
        Q.cap[sp] = c->sp[sp].cap;
        Q.ni0[sp] = s.ni0[sp];
        Q.dN_fixed[sp] = s.I_inj * s.ns_inj * g.dt * s.ni0[sp] / (g.qe * g.Nm[0]) / (double)s.nproc_mpi;
    }
    Q.it = (uint32_t)it;
    keys(s, &Q.k0, &Q.k1);
    k_inj_plan<<<1, 32, 0, c->stream>>>(Q);
    LCUDA(cudaGetLastError());

    InjP P;
    memset(&P, 0, sizeof(P));
    P.src = S->d; P.cnt = c->dcnt; P.ntype = g.ntype;
    P.nx = g.nx; P.ny = g.ny; P.S = c->S; P.W = g.nx + 3;
    P.opt = s.opt_inj; P.flag_nmn = g.flag_nmn; P.diffsrc = s.flag_diffsrc;
    P.R = make_region(s, g, c->S);
    P.dx = g.dx; P.dy = g.dy; P.xmax = g.nx * g.dx; P.ymax = g.ny * g.dy;
    P.sin_thB = std::sin(s.th_B); P.cos_thB = std::cos(s.th_B);
    P.ns_dt = (double)s.ns_inj * g.dt;
    for (int sp = 0; sp < g.ntype; sp++) {
        double vt = g.vt0[sp];
        if (std::abs(s.opt_inj) <= 2 && s.flag_Tp == 1 && sp == 0) vt = std::sqrt(2.0 * g.qe * s.THm / std::fabs(g.mass[0]));
        P.vt[sp] = vt;
        // part_injection.f90:34-47 and init_shifted_maxwellian_flux (:267-290)
        if (std::abs(s.opt_inj) == 3 || std::abs(s.opt_inj) == 4) {
            double vb = std::sqrt(2.0 * g.qe * s.THm / std::fabs(g.mass[sp]));
            if (std::abs(s.opt_inj) == 4 && sp == 0 && g.flag_nmn == 1) vb = 0.0;  // half-Maxwellian flux
            P.vb[sp] = vb;
            const double v0 = g.vt0[sp];
            const double vmax = (vb + std::sqrt(vb * vb + 2.0 * v0 * v0)) / 2.0;
            P.fmax[sp] = vmax * std::exp(-(vmax - vb) * (vmax - vb) / (v0 * v0));
        }
        P.Ek[sp] = 0.5 * g.Nm[sp] * g.mass[sp];
        P.qphi[sp] = -g.Nm[sp] * g.charge[sp];
        SpeciesBuf &B = c->sp[sp];
        P.X[sp] = B.X[B.cur]; P.Y[sp] = B.Y[B.cur];
        P.VX[sp] = B.VX[B.cur]; P.VY[sp] = B.VY[B.cur]; P.VZ[sp] = B.VZ[B.cur];
        P.Z[sp] = B.Z[B.cur];
        P.acc[sp] = B.acc;
    }
    P.cellwall = c->cellwall;
    P.ss_map = ss_counts(c); P.ss_nn = c->nn;
    P.phi = c->phi;
    P.zmax = g.zmax;
    P.it = (uint32_t)it;
    keys(s, &P.k0, &P.k1);
    k_inject<<<INJ_BLOCKS, INJ_THREADS, 0, c->stream>>>(P, S->part);
    LCUDA(cudaGetLastError());
    k_finish<<<2 * LEPIC_MAXSP, 256, 0, c->stream>>>(S->part, INJ_BLOCKS, 2 * LEPIC_MAXSP, FIN_INJ, S->d);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int run_emitter(lepic_ctx *c, int it) {
    SrcState *S = state(c);
    const lepic_source_config &s = S->cfg;
    const lepic_config &g = c->cfg;
    EmitP P;
    memset(&P, 0, sizeof(P));
    P.cnt = c->dcnt; P.src = S->d;
    P.nx = g.nx; P.ny = g.ny; P.S = c->S; P.W = g.nx + 3;
    P.dx = g.dx; P.dy = g.dy; P.xmax = g.nx * g.dx; P.ymax = g.ny * g.dy;
    P.ns_dt = (double)s.ns_Hm * g.dt;
    P.xg1 = std::min(s.xg1, P.xmax);
    P.Lg = std::min(s.Lg, P.ymax);
    P.n_icp = s.n_icp;
    // part_flux_emitter.f90:21-46: current I = js zmax Lgrd, particles per call
    double Lgrd = s.n_icp * (P.Lg - s.Lh * s.n_holes);
    P.chamfer = (s.ptype_fx == s.tag_neg && s.flag_chmfrd == 1) ? 1 : 0;
    if (P.chamfer) {
        const double x1 = s.chmfrd[0], x2 = s.chmfrd[1], y1 = s.chmfrd[2], y2 = s.chmfrd[3];
        const double d = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
        P.th_c = std::acos((x2 - x1) / d);
        P.y1c = y1;
        Lgrd = 2.0 * (y1 + d);
        if (Lgrd > P.ymax) { c->last_err = "flux emitter: Lgrd > ymax (part_flux_emitter.f90:38-41)"; return LEPIC_EINVAL; }
    }
    P.dNh = s.js * g.zmax * Lgrd * P.ns_dt / (g.Nm[s.ptype_fx] * g.qe) / (double)s.nproc_mpi;
    P.sp[0] = s.ptype_fx;
    P.sp[1] = (P.chamfer && s.tag_b >= 0) ? s.tag_b : s.ptype_fx;
    for (int q = 0; q < 2; q++) {
        const int sp = P.sp[q];
        P.vt[q] = std::sqrt(2.0 * g.qe * s.THm / std::fabs(g.mass[sp]));  // part_flux_emitter.f90:178
        P.Ek[q] = 0.5 * g.Nm[sp] * g.mass[sp];
        P.cap[q] = c->sp[sp].cap;
        SpeciesBuf &B = c->sp[sp];
        P.X[q] = B.X[B.cur]; P.Y[q] = B.Y[B.cur];
        P.VX[q] = B.VX[B.cur]; P.VY[q] = B.VY[B.cur]; P.VZ[q] = B.VZ[B.cur];
        P.Z[q] = B.Z[B.cur];
    }
    P.zmax = g.zmax;
    P.bcnd = c->bcnd;
    P.ss_map = ss_counts(c); P.ss_nn = c->nn;
    P.max_attempts_extra = 65536;
    P.it = (uint32_t)it;
    keys(s, &P.k0, &P.k1);
    k_emit<<<1, EMIT_THREADS, 0, c->stream>>>(P);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

static int te_update(lepic_ctx *c) {
    SrcState *S = state(c);
    const lepic_source_config &s = S->cfg;
    const lepic_config &g = c->cfg;
    k_te_update<<<1, LEPIC_MAXICP, 0, c->stream>>>(S->d, s.n_icp, s.eheat_type, s.nu_h, g.Nm[0], g.qe, g.mass[0]);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

extern "C" int lepic_gpu_eheating(lepic_ctx *c, int32_t it) {
    if (!c || !state(c) || !state(c)->cfg.flag_heat) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    return run_heating(c, it);
}

extern "C" int lepic_gpu_part_injection(lepic_ctx *c, int32_t it) {
    if (!c || !state(c) || !state(c)->cfg.flag_inj) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    return run_injection(c, it);
}

extern "C" int lepic_gpu_flux_emitter(lepic_ctx *c, int32_t it) {
    if (!c || !state(c) || !(state(c)->cfg.js > 0.0)) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    return run_emitter(c, it);
}

extern "C" int lepic_gpu_heating_tally(lepic_ctx *c) {
    if (!c || !state(c)) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    return run_tally(c);
}

extern "C" int lepic_gpu_source_tallies(lepic_ctx *c, lepic_source_tally *out, int32_t reset) {
    if (!c || !out || !state(c)) return LEPIC_EINVAL;
    SrcState *S = state(c);
    SrcDev h;
    LCUDA(cudaMemcpyAsync(&h, S->d, sizeof(SrcDev), cudaMemcpyDeviceToHost, c->stream));
    int r = lepic_gpu_sync(c);
    memset(out, 0, sizeof(*out));
    out->P_heat = h.P_heat;
    out->n_heated = (int64_t)h.n_heated;
    out->n_heat_calls = (int64_t)h.n_heat_calls;
    for (int s = 0; s < LEPIC_MAXSP; s++) {
        out->P_inj[s] = h.P_inj[s];
        out->P_src[s] = h.P_src[s];
        out->n_inj[s] = (int64_t)h.n_inj[s];
        out->n_inj_last[s] = (int64_t)h.n_inj_last[s];
    }
    out->n_icp = S->cfg.n_icp;
    for (int b = 0; b < LEPIC_MAXICP; b++) {
        out->Nh[b] = h.Nh[b];
        out->sum_dEk[b] = h.sum_dEk[b];
        out->vt[b] = h.vt[b];
    }
    for (int s2 = 0; s2 < LEPIC_MAXSP; s2++) {
        out->n_emit[s2] = (int64_t)h.n_emit[s2];
        out->n_emit_last[s2] = (int64_t)h.n_emit_last[s2];
    }
    out->n_emit_out = (int64_t)h.n_emit_out;
    if (reset) {
        SrcDev z = h;
        z.P_heat = 0.0; z.n_heated = 0; z.n_heat_calls = 0;
        for (int s = 0; s < LEPIC_MAXSP; s++) { z.P_inj[s] = 0.0; z.P_src[s] = 0.0; z.n_inj[s] = 0; z.n_emit[s] = 0; }
        z.n_emit_out = 0;
        LCUDA(cudaMemcpyAsync(S->d, &z, sizeof(SrcDev), cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaStreamSynchronize(c->stream));
    }
    return r;
}

// The source steps of lepic_gpu_step around the push (main.f90:984-1011, 1033-1068).
int sources_before_push(lepic_ctx *c, int it) {
    SrcState *S = state(c);
    if (!S || !S->cfg.flag_heat || it % S->cfg.ns_heat != 0) return LEPIC_OK;
    const int rm = materialize_all(c);   // the heating reads the records in sorted order
    if (rm != LEPIC_OK) return rm;
    const lepic_source_config &s = S->cfg;
    if (s.te_update && s.Pabs[0] > 0.0 && !s.flag_inj) {
        int r;
        if (S->tally_it != it - 1 && (r = run_tally(c)) != LEPIC_OK) return r;
        if ((r = te_update(c)) != LEPIC_OK) return r;
    }
    return run_heating(c, it);
}

int sources_after_push(lepic_ctx *c, int it) {
    SrcState *S = state(c);
    if (!S) return LEPIC_OK;
    const lepic_source_config &s = S->cfg;
    int r;
    if (s.flag_inj && it % s.ns_inj == 0)
        if ((r = run_injection(c, it)) != LEPIC_OK) return r;
    if (s.js > 0.0 && (s.ns_Hm == 1 || it % s.ns_Hm == 1))  // main.f90:1093-1096
        if ((r = run_emitter(c, it)) != LEPIC_OK) return r;
    if (s.flag_heat && s.Pabs[0] > 0.0 && (it + 1) % s.ns_heat == 0) {
        if ((r = run_tally(c)) != LEPIC_OK) return r;
        S->tally_it = it;
    }
    return LEPIC_OK;
}

// the sources' power tallies for lepic_gpu_get_tallies (zeros when no sources are set)
int sources_power(lepic_ctx *c, double *P_heat, double *P_inj, double *P_src) {
    SrcState *S = state(c);
    if (!S) return LEPIC_OK;
    SrcDev h;
    LCUDA(cudaMemcpyAsync(&h, S->d, sizeof(SrcDev), cudaMemcpyDeviceToHost, c->stream));
    LCUDA(cudaStreamSynchronize(c->stream));
    *P_heat = h.P_heat;
    for (int s = 0; s < LEPIC_MAXSP; s++) { P_inj[s] = h.P_inj[s]; P_src[s] = h.P_src[s]; }
    return LEPIC_OK;
}

int sources_reset_power(lepic_ctx *c) {
    SrcState *S = state(c);
    if (!S) return LEPIC_OK;
    LCUDA(cudaMemsetAsync(&S->d->P_heat, 0, sizeof(double), c->stream));
    LCUDA(cudaMemsetAsync(S->d->P_inj, 0, sizeof(double) * 2 * LEPIC_MAXSP, c->stream));  // P_inj, P_src
    return LEPIC_OK;
}

bool sources_reflux(const lepic_ctx *c, int sp, double *vb, double *fmax, double *vt, double *sin_thB,
                    double *cos_thB) {
    const SrcState *S = (const SrcState *)c->src;
    const lepic_config &g = c->cfg;
    if (!S || std::abs(S->cfg.opt_inj) != 4 || g.flag_nmn != 1) return false;
    // part_injection.f90:34-47 (electrons: a half-Maxwellian flux with the Neumann option) and
    // init_shifted_maxwellian_flux (:267-290)
    double b = std::sqrt(2.0 * g.qe * S->cfg.THm / std::fabs(g.mass[sp]));
    if (sp == 0) b = 0.0;
    const double v0 = g.vt0[sp];
    const double vmax = (b + std::sqrt(b * b + 2.0 * v0 * v0)) / 2.0;
    *vb = b;
    *fmax = vmax * std::exp(-(vmax - b) * (vmax - b) / (v0 * v0));
    *vt = v0;
    *sin_thB = std::sin(S->cfg.th_B);
    *cos_thB = std::cos(S->cfg.th_B);
    return true;
}
