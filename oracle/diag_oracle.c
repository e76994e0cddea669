/*
 * diag_oracle.c -- CPU FP64 restatement of the reference's averaging diagnostics:
 * part_moments (utils.f90:1-131) and calc_avg (utils.f90:133-266), flag_1D = 0, nproc = 1.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (see lepic_oracle.h).
 * Parity against the reference's own outputs is unpinned (no Fortran compiler here); the
 * tests pin it with analytic moments (a drifting Maxwellian's flux and temperature).
 */
#include <string.h>
#include "lepic_oracle.h"

/* p_mts(4, 0:na1+2, 0:na2+2) of one species: index m*ncell + ix + iy*(na1+3), ncell =
 * (na1+3)(na2+3), m = 0: n<v^2>, 1..3: jx, jy, jz.  Zeroed here (utils.f90:25). */
void o_part_moments(const o_cfg *c, int size_na, int ptype, const double *vxp, int64_t n, const double *kq,
                    double *p_mts) {
    const int na1 = c->nx / size_na, na2 = c->ny / size_na;
    const int64_t ncell = (int64_t)(na1 + 3) * (na2 + 3);
    const int W = c->nx + 3;
    memset(p_mts, 0, sizeof(double) * 4 * ncell);
    const double ha1 = size_na * c->dx, ha2 = size_na * c->dy;
    const double k1 = c->Nm[ptype] / (ha1 * ha2 * c->zmax);
    for (int64_t i = 0; i < n; i++) {
        const double *p = vxp + 6 * i;
        double vx = p[3], vy = p[4], vz = p[5];
        double xp = p[0] - vx * c->dt / 2.0;
        double yp = p[1] - vy * c->dt / 2.0;
        if (c->flag_nmn == 1 && xp <= 0.0) { xp = -xp; vx = -vx; }
        if (c->flag_pbc == 1) {
            const int k2 = (int)(yp / c->ymax);
            if (yp >= c->ymax) {
                if (c->flag_spec == 0) yp = yp - k2 * c->ymax;
                else { yp = (k2 + 1) * c->ymax - yp; vy = -vy; }
            }
            if (yp <= 0.0) {
                if (c->flag_spec == 0) yp = (1 - k2) * c->ymax + yp;
                else { yp = k2 * c->ymax - yp; vy = -vy; }
            }
        }
        if (xp > c->xmax || xp < 0.0 || yp > c->ymax || yp < 0.0) continue;
        const double Eki = vx * vx + vy * vy + vz * vz;
        const int ix = (int)(xp / ha1) + 1, iy = (int)(yp / ha2) + 1;
        if (ix > na1 + 1 || iy > na2 + 1) continue;
        const double px = (ix * ha1 - xp) / ha1, py = (iy * ha2 - yp) / ha2;
        const double ki[4] = {k1 * px * py, k1 * (1.0 - px) * py, k1 * (1.0 - px) * (1.0 - py), k1 * px * (1.0 - py)};
        const int ixf = size_na * ix - (size_na - 1), iyf = size_na * iy - (size_na - 1);
        const int64_t f = ixf + (int64_t)iyf * W;
        const double kqv[4] = {kq[f], kq[f + 1], kq[f + 1 + W], kq[f + W]};
        const int64_t nodes[4] = {ix + (int64_t)iy * (na1 + 3), ix + 1 + (int64_t)iy * (na1 + 3),
                                  ix + 1 + (int64_t)(iy + 1) * (na1 + 3), ix + (int64_t)(iy + 1) * (na1 + 3)};
        for (int q = 0; q < 4; q++) {
            const double kt = kqv[q] * ki[q];
            p_mts[0 * ncell + nodes[q]] += kt * Eki;
            p_mts[1 * ncell + nodes[q]] += kt * vx;
            p_mts[2 * ncell + nodes[q]] += kt * vy;
            p_mts[3 * ncell + nodes[q]] += kt * vz;
        }
    }
}

/* calc_avg for ptype: npg is that species' np(0:nx+2, 0:ny+2); data_pavg(7, na1+1, na2+1,
 * ntype) accumulates (utils.f90:176-262; the ss2D columns 6, 7 are not formed) */
void o_calc_avg(const o_cfg *c, int size_na, int ptype, const double *npg, const double *p_mts, double *data_pavg,
                const double *ss_src, const double *ss_sink) {
    const int na1 = c->nx / size_na, na2 = c->ny / size_na;
    const int64_t ncell = (int64_t)(na1 + 3) * (na2 + 3);
    const int64_t nodes = (int64_t)(na1 + 1) * (na2 + 1);
    const int W = c->nx + 3;
    for (int iy = 1; iy <= na2 + 1; iy++)
        for (int ix = 1; ix <= na1 + 1; ix++) {
            const int ixf = size_na * ix - (size_na - 1), iyf = size_na * iy - (size_na - 1);
            const double np_ = npg[ixf + (int64_t)iyf * W];
            const int64_t m = ix + (int64_t)iy * (na1 + 3);
            const double p1 = p_mts[m], jx = p_mts[ncell + m], jy = p_mts[2 * ncell + m], jz = p_mts[3 * ncell + m];
            double *d = data_pavg + 7 * ((ix - 1) + (int64_t)(na1 + 1) * (iy - 1) + nodes * ptype);
            d[0] += np_;
            d[2] += jx;
            d[3] += jy;
            d[4] += jz;
            double Tp = 0.0;
            if (np_ > 0) Tp = c->mass[ptype] / c->qe * (1.0 / 3.0) * (p1 / np_ - (jx * jx + jy * jy + jz * jz) / (np_ * np_));
            if (Tp > 0) d[1] += Tp;
            if (ss_src) { /* utils.f90:200-204, plt_src = 0: counts times Nm/Vc at the fine node */
                const double k = c->Nm[ptype] / (c->dx * c->dy * c->zmax);
                d[5] += ss_src[ixf + (int64_t)iyf * W] * k;
                d[6] += ss_sink[ixf + (int64_t)iyf * W] * k;
            }
        }
}
