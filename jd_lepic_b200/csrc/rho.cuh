// rho.cuh -- the np density of one node from the uint64 deposit accumulators (shared by the
// right-hand side, the density reduction and the averaging diagnostics).
#pragma once
#include "lepic_internal.cuh"

struct RhoParams {
    int nx, ny, ntype, pbc;
    const unsigned long long *acc[LEPIC_MAXSP];
    const double *kq;
    const int8_t *bc;
    double k1[LEPIC_MAXSP];      // Nm / (dx dy zmax)
    double charge[LEPIC_MAXSP];
};

// np(ix,iy,s) after the periodic fold of calc_rho.f90:1-35.  The reference accumulates
// kq*(k1*w) per particle; here the exact integer sum of w*2^44 is scaled once.
__device__ __forceinline__ double np_raw(const RhoParams &P, int s, int ix, int iy) {
    const long long n = ix + (long long)iy * (P.nx + 3);
    double w = (double)P.acc[s][n] * 5.684341886080802e-14; // 2^-44
    return P.kq[n] * (P.k1[s] * w);
}
__device__ __forceinline__ double np_val(const RhoParams &P, int s, int ix, int iy) {
    if (P.pbc) {
        const int W = P.nx + 3;
        if (iy == 1 && P.bc[ix + 1 * W] == 0)
            return 0.5 * (np_raw(P, s, ix, 1) + np_raw(P, s, ix, P.ny + 1));
        if (iy == P.ny + 1 && P.bc[ix + (P.ny + 1) * W] == 0) {
            if (P.bc[ix + 1 * W] == 0) return 0.5 * (np_raw(P, s, ix, 1) + np_raw(P, s, ix, P.ny + 1));
            return np_raw(P, s, ix, 1);
        }
    }
    return np_raw(P, s, ix, iy);
}

static inline RhoParams rho_params(lepic_ctx *c) {
    RhoParams P;
    P.nx = c->cfg.nx; P.ny = c->cfg.ny; P.ntype = c->cfg.ntype; P.pbc = c->cfg.flag_pbc;
    for (int s = 0; s < LEPIC_MAXSP; s++) { P.acc[s] = nullptr; P.k1[s] = 0; P.charge[s] = 0; }
    for (int s = 0; s < c->cfg.ntype; s++) {
        P.acc[s] = c->sp[s].acc;
        P.k1[s] = c->cfg.Nm[s] / (c->cfg.dx * c->cfg.dy * c->cfg.zmax);
        P.charge[s] = c->cfg.charge[s];
    }
    P.kq = c->kq; P.bc = c->bc8;
    return P;
}
