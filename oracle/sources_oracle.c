/*
 * sources_oracle.c -- CPU FP64 restatement of the reference's particle sources:
 * eheating (e_heating.f90:1-112), the heating-region tallies of charge_deposition
 * (part_expmover.f90:583-605), the temperature update (main.f90:1003-1010) and
 * part_injection (part_injection.f90:1-290, options |opt_inj| = 1 .. 4).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (see lepic_oracle.h).
 * Parity against the reference's own outputs is unpinned (no Fortran compiler here, and
 * the reference ships no tests for these routines); the tests pin the restatement with the
 * published Philox4x32-10 known answers and with distribution checks.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "lepic_oracle.h"

#define TAG_HEAT 0x48454154u
#define TAG_HEATV 0x48564C31u
#define TAG_INJN 0x494E4A4Eu
#define TAG_INJP 0x494E4A50u
#define TAG_INJV 0x494E4A56u
#define TAG_INJF 0x494E4A46u
#define TAG_INJG 0x494E4A47u
#define MAX_ATTEMPTS 65536u

/* Philox4x32-10: ten rounds of two 32x32->64 multiplies, Weyl key schedule */
void o_philox4x32_10(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += W0;
        k1 += W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

double o_u01(uint32_t v) { return ((double)v + 0.5) * 2.3283064365386963e-10; }

static void draw4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint64_t seed, uint32_t out[4]) {
    const uint32_t ctr[4] = {a, b, c, d};
    o_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x53524331u, out);
}

/* load_gauss with the two uniforms of a counter draw */
static void gauss_u(double vt, uint32_t a, uint32_t b, double *x, double *y) {
    const double rnd[2] = {o_u01(a), o_u01(b)};
    o_load_gauss(x, y, vt, rnd);
}

static int band_of(const o_cfg *c, const o_src *s, double y) {
    int b = (int)(s->n_icp * y / c->ymax);
    if (b < 0) b = 0;
    if (b >= s->n_icp) b = s->n_icp - 1;
    return b;
}

/* the heating test of e_heating.f90:51-65; returns 1 inside, with rp2 */
static int heat_region(const o_cfg *c, const o_src *s, double x, double y, double *rp2) {
    const double xa = (s->xl_pow + s->xr_pow) / 2.0, dr = (s->xr_pow - s->xl_pow) / 2.0;
    if (s->flag_c == 0) {
        *rp2 = (x - xa) * (x - xa);
        return *rp2 <= dr * dr && y >= s->yl_pow && y <= s->yr_pow;
    }
    *rp2 = (x - xa) * (x - xa) + (y - c->ymax / 2.0) * (y - c->ymax / 2.0);
    return *rp2 <= dr * dr;
}

/* e_heating.f90:33-108 */
void o_eheating(const o_cfg *c, const o_src *s, double *vxp, int64_t n, const double *vt,
                int32_t *iseed, double *P_heat, int64_t *n_heated) {
    const double dr = (s->xr_pow - s->xl_pow) / 2.0;
    double vz_sav = 0.0;
    double nu_tmp = s->nudt / c->dt;
    for (int64_t i = 0; i < n; i++) {
        double *p = vxp + 6 * i;
        double rp2;
        if (!heat_region(c, s, p[0], p[1], &rp2)) continue;
        if (s->flag_gpp == 1) nu_tmp = (s->nudt / c->dt) * 9.0 * s->Pabs_cor * exp(-9.0 * rp2 / (dr * dr));
        double rnd[2];
        rnd[0] = o_ran2(iseed);
        if (rnd[0] <= nu_tmp * c->dt) {
            const double v2old = p[3] * p[3] + p[4] * p[4] + p[5] * p[5];
            const int b = band_of(c, s, p[1]);
            double dvx, dvy, dvz;
            rnd[0] = o_ran2(iseed);
            rnd[1] = o_ran2(iseed);
            o_load_gauss(&dvx, &dvy, vt[b], rnd);
            if (vz_sav == 0.0) {
                rnd[0] = o_ran2(iseed);
                rnd[1] = o_ran2(iseed);
                o_load_gauss(&dvz, &vz_sav, vt[b], rnd);
            } else {
                dvz = vz_sav;
                vz_sav = 0.0;
            }
            if (s->eheat_type == 1) {
                p[3] = dvx; p[4] = dvy; p[5] = dvz;
            } else {
                p[3] += dvx; p[4] += dvy; p[5] += dvz;
            }
            *P_heat += 0.5 * c->Nm[0] * c->mass[0] * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5] - v2old);
            (*n_heated)++;
        }
    }
}

/* the same with the device's streams: the decision from word k & 3 of the draw of slot group
 * k / 4 and the step, then one velocity draw per heated slot */
void o_eheating_ctr(const o_cfg *c, const o_src *s, double *vxp, int64_t n, const double *vt,
                    uint64_t seed, int32_t it, double *P_heat, int64_t *n_heated) {
    const double dr = (s->xr_pow - s->xl_pow) / 2.0;
    const double Ek = 0.5 * c->Nm[0] * c->mass[0];
    for (int64_t k = 0; k < n; k++) {
        double *p = vxp + 6 * k;
        double rp2;
        if (!heat_region(c, s, p[0], p[1], &rp2)) continue;
        double nu_tmp = s->nudt / c->dt;
        if (s->flag_gpp == 1) nu_tmp = (s->nudt / c->dt) * 9.0 * s->Pabs_cor * exp(-9.0 * rp2 / (dr * dr));
        uint32_t r[4], q[4];
        const uint64_t g = (uint64_t)k >> 2;   /* one draw per group of 4 slots, word k & 3 */
        draw4((uint32_t)g, (uint32_t)(g >> 32), TAG_HEAT, (uint32_t)it, seed, r);
        if (!(o_u01(r[k & 3]) <= nu_tmp * c->dt)) continue;
        const int b = band_of(c, s, p[1]);
        draw4((uint32_t)k, (uint32_t)((uint64_t)k >> 32), TAG_HEATV, (uint32_t)it, seed, q);
        double dvx, dvy, dvz, unused;
        gauss_u(vt[b], q[0], q[1], &dvx, &dvy);
        gauss_u(vt[b], q[2], q[3], &dvz, &unused);
        const double v2old = p[3] * p[3] + p[4] * p[4] + p[5] * p[5];
        if (s->eheat_type == 1) {
            p[3] = (float)dvx; p[4] = (float)dvy; p[5] = (float)dvz;
        } else {
            p[3] = (float)(p[3] + dvx); p[4] = (float)(p[4] + dvy); p[5] = (float)(p[5] + dvz);
        }
        *P_heat += Ek * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5] - v2old);
        (*n_heated)++;
    }
}

/* part_expmover.f90:583-605 */
void o_heat_tally(const o_cfg *c, const o_src *s, const double *vxp, int64_t n, int64_t *Nh,
                  double *sum_dEk) {
    const double xa = (s->xl_pow + s->xr_pow) / 2.0, dr = (s->xr_pow - s->xl_pow) / 2.0;
    for (int b = 0; b < s->n_icp; b++) { Nh[b] = 0; sum_dEk[b] = 0.0; }
    for (int64_t i = 0; i < n; i++) {
        const double *p = vxp + 6 * i;
        const double x = p[0], y = p[1];
        if (s->flag_c == 0) {
            if (x < s->xl_pow || x > s->xr_pow || y < s->yl_pow || y > s->yr_pow) continue;
        } else if ((x - xa) * (x - xa) + (y - c->ymax / 2.0) * (y - c->ymax / 2.0) > dr * dr) {
            continue;
        }
        const int b = band_of(c, s, y);
        Nh[b]++;
        if (s->eheat_type == 1) sum_dEk[b] += 0.5 * c->Nm[0] * c->mass[0] * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5]);
    }
}

double o_te_update(const o_cfg *c, int eheat_type, double Pabs, double nu_h, int64_t Nh, double sum_dEk,
                   double vt_old) {
    if (Nh <= 0) return vt_old;
    double Te;
    if (eheat_type == 1) Te = (2.0 / 3.0) * (sum_dEk + Pabs / nu_h) / (c->Nm[0] * c->qe * (double)Nh);
    else Te = (2.0 / 3.0) * (Pabs / nu_h) / (c->Nm[0] * c->qe * (double)Nh);
    return sqrt(2.0 * c->qe * Te / fabs(c->mass[0]));
}

/* the cell test of part_injection.f90:131-137: 1 when all four corners are walls */
static int all_walls(const o_cfg *c, const int32_t *bcnd, int ix, int iy) {
    const int W = c->nx + 3;
    return bcnd[ix + iy * W] >= 1 && bcnd[ix + 1 + iy * W] >= 1 && bcnd[ix + 1 + (iy + 1) * W] >= 1 &&
           bcnd[ix + (iy + 1) * W] >= 1;
}

static double inj_vt(const o_cfg *c, const o_src *s, int ptype) {
    double vt = c->vt0[ptype];
    if (abs(s->opt_inj) <= 2 && s->flag_Tp == 1 && ptype == 0) vt = sqrt(2.0 * c->qe * s->THm / fabs(c->mass[0]));
    return vt;
}

/* the beam speed and the flux maximum of part_injection.f90:34-47 and
 * init_shifted_maxwellian_flux (part_injection.f90:267-290) */
static void inj_beam(const o_cfg *c, const o_src *s, int ptype, double *vb, double *fmax) {
    *vb = 0.0;
    *fmax = 0.0;
    const int a = abs(s->opt_inj);
    if (a != 3 && a != 4) return;
    *vb = sqrt(2.0 * c->qe * s->THm / fabs(c->mass[ptype]));
    if (a == 4 && ptype == 0 && c->flag_nmn == 1) *vb = 0.0;
    const double v0 = c->vt0[ptype];
    const double vmax = (*vb + sqrt(*vb * *vb + 2.0 * v0 * v0)) / 2.0;
    *fmax = vmax * exp(-(vmax - *vb) * (vmax - *vb) / (v0 * v0));
}

/* part_injection.f90:77-79: no ions under the beam, nor under cathode emission without the
 * divertor option */
static int inj_electrons_only(const o_cfg *c, const o_src *s) {
    return abs(s->opt_inj) == 3 || (abs(s->opt_inj) == 4 && c->flag_nmn == 0);
}

/* shifted_maxwellian_flux (part_injection.f90:239-265) from a ran2 stream */
static double shifted_flux_ran2(double vb, double vt, double fmax, int32_t *iseed) {
    const double vm = vb - 4.0 * vt > 0.0 ? vb - 4.0 * vt : 0.0, vp = vb + 4.0 * vt;
    for (;;) {
        const double r1 = o_ran2(iseed), r2 = o_ran2(iseed);
        const double v = vm + r1 * (vp - vm);
        const double f = v * exp(-(v - vb) * (v - vb) / (vt * vt));
        if (!(r2 > f / fmax)) return v;
    }
}

/* part_injection.f90:216-231 */
static double phi_at(const o_cfg *c, const double *phi, int ix, int iy, double x, double y) {
    const int W = c->nx + 3;
    const double px = (ix * c->dx - x) / c->dx, py = (iy * c->dy - y) / c->dy;
    return px * py * phi[ix + iy * W] + (1.0 - px) * py * phi[ix + 1 + iy * W] +
           (1.0 - px) * (1.0 - py) * phi[ix + 1 + (iy + 1) * W] + px * (1.0 - py) * phi[ix + (iy + 1) * W];
}

/* the count of part_injection.f90:49-75 before its stochastic rounding; *draw = 0 when the
 * count is an exact loss count (positive ions under |opt_inj| = 2) */
static double inj_dN(const o_cfg *c, const o_src *s, int ptype, const int64_t *lost, int *draw) {
    *draw = 1;
    if (abs(s->opt_inj) == 2) {
        if (ptype == 0 || ptype == s->tag_neg) {
            int64_t t = 0;
            for (int q = 1; q < c->ntype; q++)
                if (q != s->tag_neg) t += lost[q];
            return s->ni0[ptype] * (double)t;
        }
        *draw = 0;
        return (double)lost[ptype];
    }
    return s->I_inj * s->ns_inj * c->dt * s->ni0[ptype] / (c->qe * c->Nm[0]) / (double)s->nproc_mpi;
}

int o_part_injection(const o_cfg *c, const o_src *s, int ptype, const int32_t *bcnd,
                     const double *phi, int64_t *N_inj, double *vxp, int64_t *np, int64_t cap,
                     int32_t *iseed, double *P_inj, double *P_src) {
    const double xa = (s->xl_pow + s->xr_pow) / 2.0, dr = (s->xr_pow - s->xl_pow) / 2.0;
    const double ymid = c->ymax / 2.0;
    double vz_sav = 0.0, x_sav = 0.0;
    int draw;
    const double dN = inj_dN(c, s, ptype, N_inj, &draw);
    if (draw) {
        int64_t N = (int64_t)dN;
        if (o_ran2(iseed) <= dN - (double)N) N += 1;
        N_inj[ptype] = N;
    }
    if (inj_electrons_only(c, s))
        for (int q = 1; q < c->ntype; q++) N_inj[q] = 0;
    const double vt = inj_vt(c, s, ptype);
    double vb, fmx;
    inj_beam(c, s, ptype, &vb, &fmx);
    for (int64_t i = 0; i < N_inj[ptype]; i++) {
        double x = 0.0, y = 0.0, rnd[2];
        int ix, iy;
        for (;;) { /* label 70 */
            if (s->opt_inj > 0) {
                for (;;) { /* label 60 */
                    x = o_ran2(iseed) * (s->xl_pow - s->xr_pow) + s->xr_pow;
                    if (s->flag_c != 1) break;
                    y = o_ran2(iseed) * (2.0 * dr) + ymid - dr;
                    if (!((x - xa) * (x - xa) + (y - ymid) * (y - ymid) > dr * dr)) break;
                }
            } else if (s->flag_c == 0) {
                for (;;) { /* label 50 */
                    if (x_sav == 0) {
                        rnd[0] = o_ran2(iseed);
                        rnd[1] = o_ran2(iseed);
                        o_load_gauss(&x, &x_sav, dr, rnd);
                        x = x + xa;
                        x_sav = x_sav + xa;
                    } else {
                        x = x_sav;
                        x_sav = 0.0;
                    }
                    if (c->flag_nmn == 1 && xa == 0.0) x = fabs(x);
                    if (!(x < xa - 4.0 * dr || x > xa + 4.0 * dr || x < 0.0 || x > c->xmax)) break;
                }
            } else {
                for (;;) { /* label 40 */
                    rnd[0] = o_ran2(iseed);
                    rnd[1] = o_ran2(iseed);
                    o_load_gauss(&x, &y, dr, rnd);
                    x = x + xa;
                    y = y + ymid;
                    if (!((x - xa) * (x - xa) + (y - ymid) * (y - ymid) > 4.0 * dr * dr || x < 0.0 ||
                          x > c->xmax || y < 0.0 || y > c->ymax))
                        break;
                }
            }
            if (s->flag_c == 0) y = o_ran2(iseed) * (s->yl_pow - s->yr_pow) + s->yr_pow;
            (void)o_ran2(iseed); /* z */
            ix = (int)(x / c->dx) + 1;
            iy = (int)(y / c->dy) + 1;
            if (!all_walls(c, bcnd, ix, iy)) break;
        }
        if (*np + 1 > cap) return -2;
        double *p = vxp + 6 * (*np);
        (*np)++;
        double vx, vy, vz;
        if (abs(s->opt_inj) == 4) { /* part_injection.f90:161-178 */
            const double vb_tmp = vb * cos(s->th_B);
            for (;;) { /* label 75 */
                vx = shifted_flux_ran2(vb_tmp, vt, fmx, iseed);
                rnd[0] = o_ran2(iseed);
                rnd[1] = o_ran2(iseed);
                o_load_gauss(&vy, &vz, vt, rnd);
                vy = vy + vb * sin(s->th_B);
                const double dt_tmp = o_ran2(iseed) * ((double)s->ns_inj * c->dt);
                x = vx * dt_tmp;
                if (!(x < 0.0 || x > c->xmax)) break;
            }
            ix = (int)floor(x / c->dx) + 1;
        } else {
            rnd[0] = o_ran2(iseed);
            rnd[1] = o_ran2(iseed);
            o_load_gauss(&vx, &vy, vt, rnd);
            if (vz_sav == 0.0) {
                rnd[0] = o_ran2(iseed);
                rnd[1] = o_ran2(iseed);
                o_load_gauss(&vx, &vy, vt, rnd);
                vz = vx;
                vz_sav = vy;
            } else {
                vz = vz_sav;
                vz_sav = 0.0;
            }
        }
        if (abs(s->opt_inj) == 3) vz = vz + vb; /* part_injection.f90:202 */
        p[0] = x; p[1] = y; p[2] = 0.0;
        p[3] = vx; p[4] = vy; p[5] = vz;
        *P_inj += 0.5 * c->Nm[ptype] * c->mass[ptype] * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5]);
        if (s->flag_diffsrc == 1) *P_src -= c->Nm[ptype] * c->charge[ptype] * phi_at(c, phi, ix, iy, x, y);
    }
    return 0;
}

int o_part_injection_ctr(const o_cfg *c, const o_src *s, const int32_t *bcnd, const double *phi,
                         const int64_t *lost, uint64_t seed, int32_t it, int S, double **vxp,
                         int64_t *np, const int64_t *cap, int64_t *count, double *P_inj,
                         double *P_src) {
    const double xa = (s->xl_pow + s->xr_pow) / 2.0, dr = (s->xr_pow - s->xl_pow) / 2.0;
    const double ymid = c->ymax / 2.0;
    const uint32_t U = (uint32_t)it;
    int rc = 0;
    for (int sp = 0; sp < c->ntype; sp++) {
        int draw;
        const double dN = inj_dN(c, s, sp, lost, &draw);
        int64_t N = draw ? (int64_t)dN : lost[sp];
        if (draw) {
            uint32_t r[4];
            draw4((uint32_t)sp, 0u, TAG_INJN, U, seed, r);
            if (o_u01(r[0]) <= dN - (double)N) N += 1;
        }
        if (sp > 0 && inj_electrons_only(c, s)) N = 0;
        if (np[sp] + N > cap[sp]) { rc = -2; N = 0; }
        count[sp] = N;
    }
    for (int sp = 0; sp < c->ntype; sp++) {
        const double vt = inj_vt(c, s, sp);
        const double Ek = 0.5 * c->Nm[sp] * c->mass[sp];
        double vb, fmx;
        inj_beam(c, s, sp, &vb, &fmx);
        for (int64_t j = 0; j < count[sp]; j++) {
            double x = 0.0, y = 0.0;
            int ix = 1, iy = 1, ok = 0;
            for (uint32_t a = 0; a < MAX_ATTEMPTS && !ok; a++) {
                uint32_t r[4];
                draw4((uint32_t)j, (a << 3) | (uint32_t)sp, TAG_INJP, U, seed, r);
                if (s->opt_inj > 0) {
                    x = o_u01(r[0]) * (s->xl_pow - s->xr_pow) + s->xr_pow;
                    if (s->flag_c == 1) {
                        y = o_u01(r[1]) * (2.0 * dr) + ymid - dr;
                        if ((x - xa) * (x - xa) + (y - ymid) * (y - ymid) > dr * dr) continue;
                    }
                } else if (s->flag_c == 0) {
                    double g0, g1;
                    gauss_u(dr, r[0], r[1], &g0, &g1);
                    x = g0 + xa;
                    if (c->flag_nmn == 1 && xa == 0.0) x = fabs(x);
                    if (x < xa - 4.0 * dr || x > xa + 4.0 * dr || x < 0.0 || x > c->xmax) continue;
                } else {
                    double g0, g1;
                    gauss_u(dr, r[0], r[1], &g0, &g1);
                    x = g0 + xa;
                    y = g1 + ymid;
                    if ((x - xa) * (x - xa) + (y - ymid) * (y - ymid) > 4.0 * dr * dr || x < 0.0 || x > c->xmax ||
                        y < 0.0 || y > c->ymax)
                        continue;
                }
                if (s->flag_c == 0) y = o_u01(r[2]) * (s->yl_pow - s->yr_pow) + s->yr_pow;
                ix = (int)(x / c->dx) + 1;
                iy = (int)(y / c->dy) + 1;
                if (ix < 1) ix = 1;
                if (ix > c->nx + 1) ix = c->nx + 1;
                if (iy < 1) iy = 1;
                if (iy > c->ny + 1) iy = c->ny + 1;
                if (all_walls(c, bcnd, ix, iy)) continue;
                ok = 1;
            }
            if (!ok) return -3;
            double vx = 0.0, vy = 0.0, vz = 0.0;
            if (abs(s->opt_inj) == 4) {
                /* one attempt = one flux draw (TAG_INJF: v, its acceptance, vy, vz) and one
                 * time offset (TAG_INJG); a rejection or an x outside [0, xmax] starts the next */
                const double vbt = vb * cos(s->th_B);
                const double vm = vbt - 4.0 * vt > 0.0 ? vbt - 4.0 * vt : 0.0, vpm = vbt + 4.0 * vt;
                int got = 0;
                for (uint32_t a = 0; a < MAX_ATTEMPTS && !got; a++) {
                    uint32_t f[4], g[4];
                    draw4((uint32_t)j, (a << 3) | (uint32_t)sp, TAG_INJF, U, seed, f);
                    const double v = vm + o_u01(f[0]) * (vpm - vm);
                    const double fv = v * exp(-(v - vbt) * (v - vbt) / (vt * vt));
                    if (o_u01(f[1]) > fv / fmx) continue;
                    gauss_u(vt, f[2], f[3], &vy, &vz);
                    draw4((uint32_t)j, (a << 3) | (uint32_t)sp, TAG_INJG, U, seed, g);
                    const double xn = v * (o_u01(g[0]) * ((double)s->ns_inj * c->dt));
                    if (xn < 0.0 || xn > c->xmax) continue;
                    vx = v;
                    vy = vy + vb * sin(s->th_B);
                    x = xn;
                    got = 1;
                }
                if (!got) return -3;
                ix = (int)floor(x / c->dx) + 1;
                if (ix < 1) ix = 1;
                if (ix > c->nx + 1) ix = c->nx + 1;
            } else {
                uint32_t q[4];
                draw4((uint32_t)j, (uint32_t)sp, TAG_INJV, U, seed, q);
                if ((j & 1) == 0) {
                    gauss_u(vt, q[2], q[3], &vx, &vy);
                    vz = vx;
                } else {
                    uint32_t qp[4];
                    double unused;
                    gauss_u(vt, q[0], q[1], &vx, &vy);
                    draw4((uint32_t)(j - 1), (uint32_t)sp, TAG_INJV, U, seed, qp);
                    gauss_u(vt, qp[2], qp[3], &unused, &vz);
                }
                if (abs(s->opt_inj) == 3) vz = vz + vb;
            }
            double *p = vxp[sp] + 6 * (np[sp] + j);
            if (S > 0) {
                const double sc = ldexp(1.0, S);
                double fx = floor(x / c->dx * sc), fy = floor(y / c->dy * sc);
                const double xl = ldexp((double)c->nx, S) - 1.0, yl = ldexp((double)c->ny, S) - 1.0;
                if (fx > xl) fx = xl;
                if (fy > yl) fy = yl;
                p[0] = fx * (c->dx * ldexp(1.0, -S));
                p[1] = fy * (c->dy * ldexp(1.0, -S));
                p[3] = (float)vx; p[4] = (float)vy; p[5] = (float)vz;
            } else {
                p[0] = x; p[1] = y;
                p[3] = vx; p[4] = vy; p[5] = vz;
            }
            p[2] = 0.0;
            P_inj[sp] += Ek * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5]);
            if (s->flag_diffsrc == 1) P_src[sp] += (-c->Nm[sp] * c->charge[sp]) * phi_at(c, phi, ix, iy, x, y);
        }
        np[sp] += count[sp];
    }
    return rc;
}

/* ---- part_flux_emitter.f90 ------------------------------------------------------------ */
#define TAG_FXN 0x46584E31u
#define TAG_FXP 0x46585031u
#define TAG_FXV 0x46585631u

typedef struct {
    double xg1, Lg, y1c, th_c, dNh;
} emit_geo;

/* part_flux_emitter.f90:21-46 (nproc = 1) and generate_boundary.f90:246-248 */
static int emit_setup(const o_cfg *c, const o_emit *e, emit_geo *g) {
    g->xg1 = e->xg1 > c->xmax ? c->xmax : e->xg1;
    g->Lg = e->Lg > c->ymax ? c->ymax : e->Lg;
    double Lgrd = e->n_icp * (g->Lg - e->Lh * e->n_holes);
    g->y1c = 0.0;
    g->th_c = 0.0;
    if (e->chamfer) {
        const double x1 = e->chmfrd[0], x2 = e->chmfrd[1], y1 = e->chmfrd[2], y2 = e->chmfrd[3];
        const double d = sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
        g->th_c = acos((x2 - x1) / d);
        g->y1c = y1;
        Lgrd = 2.0 * (y1 + d);
        if (Lgrd > c->ymax) return -1;
    }
    const double I_sec = e->js * c->zmax * Lgrd;
    g->dNh = I_sec * ((double)e->ns_Hm * c->dt) / (c->Nm[e->sp_fx] * c->qe) / (double)e->nproc_mpi;
    return 0;
}

static int on_chamfer(const o_cfg *c, const emit_geo *g, double y) {
    return (y <= c->ymax / 2.0 && y > g->y1c) || (y > c->ymax / 2.0 && fabs(c->ymax - y) > g->y1c);
}

/* the emission point of one attempt (part_flux_emitter.f90:103-136): returns the species slot
 * q (1: chamfer), the point, the velocity rotation angle and the cell; 0 if off the grid */
static int emit_point(const o_cfg *c, const o_emit *e, const emit_geo *g, double r, int *q, double *x,
                      double *y, double *th, int *ix, int *iy) {
    const double pi = 4.0 * atan(1.0);
    *x = g->xg1;
    *y = e->n_icp == 1 ? (c->ymax - g->Lg) / 2.0 + g->Lg * r : c->ymax * (1.0 - r);
    *q = 0;
    if (e->chamfer && on_chamfer(c, g, *y)) {
        *q = 1;
        double thp = g->th_c, d0 = *y - g->y1c, d1 = g->y1c;
        if (*y > c->ymax / 2.0) {
            thp = -g->th_c;
            d0 = fabs(*y - c->ymax) - g->y1c;
            d1 = c->ymax - g->y1c;
        }
        *x = g->xg1 + d0 * cos(thp);
        *y = d1 + d0 * sin(thp);
    }
    *th = pi / 2.0;
    if (e->chamfer && on_chamfer(c, g, *y)) *th = *y > c->ymax / 2.0 ? pi / 2.0 + g->th_c : g->th_c;
    *ix = (int)(*x / c->dx) + 1;
    *iy = (int)(*y / c->dy) + 1;
    return *ix >= 1 && *ix <= c->nx + 1 && *iy >= 1 && *iy <= c->ny + 1;
}

/* the wall-face test and the running plasma-side counts (part_flux_emitter.f90:141-161);
 * returns 1 when the attempt is kept, with its direction */
static int emit_accept(const o_cfg *c, const int32_t *b, int ix, int iy, int64_t *cl, int64_t *cr, double *dir) {
    const int W = c->nx + 3;
    const int m = ix + iy * W;
    if (!((b[m] >= 1 && b[m + W] >= 1) || (b[m + 1] >= 1 && b[m + 1 + W] >= 1))) return 0;
    if (b[m - 1] == -1) (*cl)++;
    if (b[m + 1] == -1) (*cr)++;
    if (*cl == *cr) return 0;
    *dir = *cl > *cr ? 1.0 : -1.0;
    return 1;
}

int o_part_flux_emitter(const o_cfg *c, const o_emit *e, const int32_t *bcnd, double **vxp,
                        int64_t *np, const int64_t *cap, int32_t *iseed, int64_t *count,
                        double *P_inj) {
    emit_geo g;
    if (emit_setup(c, e, &g)) return -1;
    int64_t Nh = (int64_t)g.dNh;
    if (o_ran2(iseed) <= g.dNh - (double)Nh) Nh += 1;
    int64_t cl = 0, cr = 0;
    const int64_t max_att = 64 * Nh + 65536;
    int64_t att = 0;
    for (int s = 0; s < c->ntype; s++) count[s] = 0;
    for (int64_t i = 0; i < Nh; i++) {
        double x, y, th, dir = 1.0;
        int q, ix, iy;
        for (;;) { /* label 90 */
            if (att++ >= max_att) return -3;
            const double r = o_ran2(iseed);
            const int ok = emit_point(c, e, &g, r, &q, &x, &y, &th, &ix, &iy);
            (void)o_ran2(iseed); /* z_inj */
            if (ok && emit_accept(c, bcnd, ix, iy, &cl, &cr, &dir)) break;
        }
        const int sp = q ? e->sp_b : e->sp_fx;
        if (np[sp] + 1 > cap[sp]) return -2;
        const double vt = sqrt(2.0 * c->qe * e->THm / fabs(c->mass[sp]));
        double rnd[2], vy, vz;
        const double vx = dir * vt * sqrt(-log(1 - o_ran2(iseed)));
        rnd[0] = o_ran2(iseed);
        rnd[1] = o_ran2(iseed);
        o_load_gauss(&vy, &vz, vt, rnd);
        const double vxt = -vx * sin(th) + vy * cos(th), vyt = vx * cos(th) + vy * sin(th);
        const double dt_tmp = o_ran2(iseed) * ((double)e->ns_Hm * c->dt);
        double *p = vxp[sp] + 6 * np[sp];
        p[0] = x + vxt * dt_tmp; p[1] = y + vyt * dt_tmp; p[2] = 0.0;
        p[3] = vxt; p[4] = vyt; p[5] = vz;
        np[sp]++;
        count[sp]++;
        P_inj[sp] += 0.5 * c->Nm[sp] * c->mass[sp] * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5]);
    }
    return 0;
}

int o_part_flux_emitter_ctr(const o_cfg *c, const o_emit *e, const int32_t *bcnd, uint64_t seed,
                            int32_t it, int S, double **vxp, int64_t *np, const int64_t *cap,
                            int64_t *count, double *P_inj, int64_t *n_out) {
    emit_geo g;
    if (emit_setup(c, e, &g)) return -1;
    const uint32_t U = (uint32_t)it;
    uint32_t r[4];
    draw4(0u, 0u, TAG_FXN, U, seed, r);
    int64_t Nh = (int64_t)g.dNh;
    if (o_u01(r[0]) <= g.dNh - (double)Nh) Nh += 1;
    int64_t cl = 0, cr = 0, j = 0;
    const int64_t max_att = 64 * Nh + 65536;
    for (int s = 0; s < c->ntype; s++) count[s] = 0;
    *n_out = 0;
    for (int64_t a = 0; j < Nh && a < max_att; a++) {
        double x, y, th, dir = 1.0;
        int q, ix, iy;
        draw4((uint32_t)a, (uint32_t)((uint64_t)a >> 32), TAG_FXP, U, seed, r);
        if (!emit_point(c, e, &g, o_u01(r[0]), &q, &x, &y, &th, &ix, &iy)) continue;
        if (!emit_accept(c, bcnd, ix, iy, &cl, &cr, &dir)) continue;
        const int sp = q ? e->sp_b : e->sp_fx;
        uint32_t v[4];
        draw4((uint32_t)j, (uint32_t)((uint64_t)j >> 32), TAG_FXV, U, seed, v);
        j++;
        if (np[sp] + 1 > cap[sp]) return -2;
        const double vt = sqrt(2.0 * c->qe * e->THm / fabs(c->mass[sp]));
        const double vx = dir * vt * sqrt(-log(1.0 - o_u01(v[0])));
        double vy, vz;
        gauss_u(vt, v[1], v[2], &vy, &vz);
        const double vxt = -vx * sin(th) + vy * cos(th), vyt = vx * cos(th) + vy * sin(th);
        const double dt_tmp = o_u01(v[3]) * ((double)e->ns_Hm * c->dt);
        const double xn = x + vxt * dt_tmp, yn = y + vyt * dt_tmp;
        const float fvx = (float)vxt, fvy = (float)vyt, fvz = (float)vz;
        P_inj[sp] += 0.5 * c->Nm[sp] * c->mass[sp] * ((double)fvx * fvx + (double)fvy * fvy + (double)fvz * fvz);
        count[sp]++;
        if (xn < 0.0 || xn >= c->xmax || yn < 0.0 || yn >= c->ymax) {
            (*n_out)++;   /* a hole on the device: not among the live particles */
            continue;
        }
        double *p = vxp[sp] + 6 * np[sp];
        if (S > 0) {
            const double sc = ldexp(1.0, S);
            double fx = floor(xn / c->dx * sc), fy = floor(yn / c->dy * sc);
            const double xl = ldexp((double)c->nx, S) - 1.0, yl = ldexp((double)c->ny, S) - 1.0;
            if (fx > xl) fx = xl;
            if (fy > yl) fy = yl;
            p[0] = fx * (c->dx * ldexp(1.0, -S));
            p[1] = fy * (c->dy * ldexp(1.0, -S));
        } else {
            p[0] = xn; p[1] = yn;
        }
        p[2] = 0.0;
        p[3] = fvx; p[4] = fvy; p[5] = fvz;
        np[sp]++;
    }
    return j < Nh ? -3 : 0;
}
