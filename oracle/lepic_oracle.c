/*
 * lepic_oracle.c -- CPU FP64 restatement of the LePIC per-step routines.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for the CUDA path; see lepic_oracle.h).
 * Parity against the reference's own outputs is UNPINNED: the Fortran reference cannot be
 * built here and has no golden vectors.  Each function cites the reference lines it restates.
 *
 * Build with -ffp-contract=off so that every product and sum is rounded exactly as written
 * (the GPU FP64 multigrid and field kernels are compiled the same way and match bit for bit).
 */
#include "lepic_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NODE(i, j, nx) ((i) + (j) * ((nx) + 3))
#define RHS(i, j, nx) (((i) - 1) + ((j) - 1) * ((nx) + 1))

/* ------------------------------------------------------------------------------------ */
/* ran2.f90:1-15: irand = 16807*irand mod (2^31-1) by Schrage's method; returns irand/im  */
double o_ran2(int32_t *irand) {
    const int32_t ia = 16807, im = 2147483647, iq = 127773, ir = 2836;
    const double am = 1.0 / im;
    int32_t k = *irand / iq;
    *irand = ia * (*irand - k * iq) - ir * k;
    if (*irand < 0) *irand += im;
    return am * (*irand);
}

/* load_gauss.f90:16-39: Rayleigh magnitude vt*sqrt(-ln(1-r1)) at angle 2*pi*r2 */
void o_load_gauss(double *vx, double *vy, double vt, const double rnd[2]) {
    const double pi = 4.0 * atan(1.0);
    double vp = vt * sqrt(-log(1 - rnd[0]));
    double theta = 2.0 * pi * rnd[1];
    *vx = vp * cos(theta);
    *vy = vp * sin(theta);
}

/* part_expmover.f90:612-627 */
static void check_outofbounds(int *ix, int *iy, int nx, int ny) {
    if (*ix < 0) *ix = 0;
    if (*ix > nx + 1) *ix = nx + 1;
    if (*iy < 0) *iy = 0;
    if (*iy > ny + 1) *iy = ny + 1;
}

/* ------------------------------------------------------------------------------------ */
/* part_expmover.f90:1-517 */
void o_part_mover(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                  const int32_t *bcnd, double *vxp, int64_t *np_tot, int8_t *flag_dead,
                  o_push_tally *t) {
    o_part_mover_z(c, ptype, Ei, Bi, bcnd, vxp, np_tot, flag_dead, t, NULL);
}

void o_part_mover_z(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                    const int32_t *bcnd, double *vxp, int64_t *np_tot, int8_t *flag_dead,
                    o_push_tally *t, const o_zloss *zl) {
    o_part_mover_zd(c, ptype, Ei, Bi, bcnd, vxp, np_tot, flag_dead, t, zl, NULL);
}

static int o_label(int l) { return l < 0 ? 0 : (l > 15 ? 15 : l); }

void o_part_mover_zd(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                     const int32_t *bcnd, double *vxp, int64_t *np_tot, int8_t *flag_dead,
                     o_push_tally *t, const o_zloss *zl, const o_dielec *dl) {
    o_part_mover_x(c, ptype, Ei, Bi, bcnd, vxp, np_tot, flag_dead, t, zl, dl, NULL);
}

#define O_TAG_SECN 0x5345434Eu
#define O_TAG_SECV 0x53454356u
#define O_TAG_RFX 0x52465831u
#define O_TAG_RFX2 0x52465832u

void o_part_mover_x(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                    const int32_t *bcnd, double *vxp, int64_t *np_tot, int8_t *flag_dead,
                    o_push_tally *t, const o_zloss *zl, const o_dielec *dl, o_wallx *wx) {
    const int nx = c->nx, ny = c->ny;
    const double h1 = c->dx, h2 = c->dy, dt = c->dt;
    const double amu = 1.66053886e-27;
    int64_t np_lost = 0;
    const double k1 = dt * c->charge[ptype] / (2.0 * c->mass[ptype]); /* :61 */
    const int64_t n = *np_tot;
    for (int64_t i = 0; i < n; i++) {
        double *p = vxp + 6 * i;
        double xp = p[0], yp = p[1], zp = p[2], vx = p[3], vy = p[4], vz = p[5];
        if (flag_dead && flag_dead[i] == 1) { /* :84-98 */
            np_lost++;
            flag_dead[i] = 0;
            if (t) t->n_dead++;
            continue;
        }
        int ix = (int)(xp / h1) + 1; /* :103-104, INT truncates toward zero */
        int iy = (int)(yp / h2) + 1;
        double px = (ix * h1 - xp) / h1; /* :109-110 */
        double py = (iy * h2 - yp) / h2;
        double ki[4];
        ki[0] = px * py;
        ki[1] = (1.0 - px) * py;
        ki[2] = (1.0 - px) * (1.0 - py);
        ki[3] = px * (1.0 - py);
        const double *e00 = Ei + 2 * NODE(ix, iy, nx), *e10 = Ei + 2 * NODE(ix + 1, iy, nx);
        const double *e11 = Ei + 2 * NODE(ix + 1, iy + 1, nx), *e01 = Ei + 2 * NODE(ix, iy + 1, nx);
        double Exp = ki[0] * e00[0] + ki[1] * e10[0] + ki[2] * e11[0] + ki[3] * e01[0];
        double Eyp = ki[0] * e00[1] + ki[1] * e10[1] + ki[2] * e11[1] + ki[3] * e01[1];
        int flag_B_tmp = 0; /* :130-182 */
        double Bpx = 0, Bpy = 0, Bpz = 0;
        if (c->flag_B == 1) {
            Bpx = c->Bc[0]; Bpy = c->Bc[1]; Bpz = c->Bc[2];
            flag_B_tmp = 1;
        } else if (c->flag_B == 2) {
            if (Bi[4 * NODE(ix, iy, nx) + 3] > 1.e-5) {
                const double *b00 = Bi + 4 * NODE(ix, iy, nx), *b10 = Bi + 4 * NODE(ix + 1, iy, nx);
                const double *b11 = Bi + 4 * NODE(ix + 1, iy + 1, nx), *b01 = Bi + 4 * NODE(ix, iy + 1, nx);
                Bpx = ki[0] * b00[0] + ki[1] * b10[0] + ki[2] * b11[0] + ki[3] * b01[0];
                Bpy = ki[0] * b00[1] + ki[1] * b10[1] + ki[2] * b11[1] + ki[3] * b01[1];
                Bpz = ki[0] * b00[2] + ki[1] * b10[2] + ki[2] * b11[2] + ki[3] * b01[2];
                flag_B_tmp = 1;
            }
        }
        if (c->flag_B_pos == 1 && c->charge[ptype] > 0.0) flag_B_tmp = 0; /* :185 */
        if (flag_B_tmp == 1) { /* :187-206 Boris */
            double B_tot = sqrt(Bpx * Bpx + Bpy * Bpy + Bpz * Bpz);
            double k2 = k1 * (2.0 / (1.0 + (k1 * B_tot) * (k1 * B_tot)));
            double v1x = vx + k1 * Exp, v1y = vy + k1 * Eyp, v1z = vz;
            double v3x = v1x + k1 * (v1y * Bpz - v1z * Bpy);
            double v3y = v1y + k1 * (v1z * Bpx - v1x * Bpz);
            double v3z = v1z + k1 * (v1x * Bpy - v1y * Bpx);
            double v2x = v1x + k2 * (v3y * Bpz - v3z * Bpy);
            double v2y = v1y + k2 * (v3z * Bpx - v3x * Bpz);
            double v2z = v1z + k2 * (v3x * Bpy - v3y * Bpx);
            vx = v2x + k1 * Exp;
            vy = v2y + k1 * Eyp;
            vz = v2z;
        } else { /* :210-211 leap-frog */
            vx = vx + 2.0 * k1 * Exp;
            vy = vy + 2.0 * k1 * Eyp;
        }
        xp = xp + dt * vx; /* :216-219 */
        yp = yp + dt * vy;
        zp = zp + dt * vz;
        if (c->flag_pbc == 1) { /* :222-241 */
            int k4 = (int)(yp / c->ymax);
            if (yp >= c->ymax) {
                if (c->flag_spec == 0) yp = yp - k4 * c->ymax;
                else { yp = (k4 + 1) * c->ymax - yp; vy = -vy; }
            }
            if (yp <= 0.0) {
                if (c->flag_spec == 0) yp = (1 - k4) * c->ymax + yp;
                else { yp = k4 * c->ymax - yp; vy = -vy; }
            }
        }
        ix = (int)floor(xp / h1) + 1; /* :244-248 FLOOR */
        iy = (int)floor(yp / h2) + 1;
        check_outofbounds(&ix, &iy, nx, ny);
        int flag_lost = 0; /* :253-266 */
        if (bcnd[NODE(ix, iy, nx)] >= 1 && bcnd[NODE(ix + 1, iy, nx)] >= 1 &&
            bcnd[NODE(ix + 1, iy + 1, nx)] >= 1 && bcnd[NODE(ix, iy + 1, nx)] >= 1)
            flag_lost = 1;
        else if (c->charge[ptype] < 0 && c->mass[ptype] >= amu && xp < 0.0 && c->flag_nmn == 1)
            flag_lost = 3;
        else if (zl) { /* :269-309 the 3rd virtual dimension */
            if (c->charge[ptype] < 0) {
                if (zp <= 0.0 || zp >= c->zmax) {
                    const double Eki = 0.5 * c->mass[ptype] * vz * vz / c->qe;
                    if (Eki >= zl->phi[NODE(ix, iy, nx)] - zl->phi0) flag_lost = 2;
                    else {
                        vz = -vz;
                        zp = zp <= 0.0 ? 0.02 * c->zmax : 0.98 * c->zmax;
                    }
                }
            } else {
                int ixc = ix, iyc = iy;
                if (zl->size_na != 1) {
                    ixc = (int)(xp / (zl->size_na * h1)) + 1;
                    iyc = (int)(yp / (zl->size_na * h2)) + 1;
                }
                /* the device's draw: Philox keyed by (slot, step, tag, species); the product
                   nu_3D dt in FP32, as the device forms it */
                const float p = zl->nu_fac * zl->uB[(ixc - 1) + (int64_t)(iyc - 1) * (zl->na1 + 1)];
                uint32_t ctr[4] = {(uint32_t)i, zl->it, 0x5A4C4F53u, (uint32_t)ptype}, out[4];
                o_philox4x32_10(ctr, zl->k0, zl->k1, out);
                if (o_u01(out[0]) <= (double)p) flag_lost = 2;
            }
        }
        if (flag_lost >= 1) { /* :314-427 */
            np_lost++;
            if (dl && flag_lost == 1) { /* :337-350 dielectric charging */
                const int igrid = o_label(bcnd[NODE(ix, iy, nx)]);
                const int up = o_label(bcnd[NODE(ix, iy + 1, nx)]);
                int dt_tmp = dl->dtype[igrid];
                if (dl->dtype[up] > dt_tmp) dt_tmp = dl->dtype[up];
                if (dt_tmp == 1) {
                    const double k3 = c->Nm[ptype] * c->charge[ptype];
                    const double py = (iy * h2 - yp) / h2;
                    dl->dq[(int64_t)igrid * (ny + 3) + iy] += k3 * py;
                    dl->dq[(int64_t)igrid * (ny + 3) + iy + 1] += k3 * (1.0 - py);
                }
            }
            if (wx && wx->sec_label > 0 && flag_lost == 1 && c->charge[ptype] > 0 &&
                bcnd[NODE(ix, iy, nx)] == wx->sec_label) { /* :354-392 secondary emission */
                uint32_t ctr[4] = {(uint32_t)i, wx->it, O_TAG_SECN, (uint32_t)ptype}, r[4];
                o_philox4x32_10(ctr, wx->k0, wx->k1, r);
                int n_sec = (int)wx->gam_sec;
                if (o_u01(r[0]) <= wx->gam_sec - n_sec) n_sec++;
                for (int k = 0; k < n_sec; k++) {
                    uint32_t cv[4] = {(uint32_t)i, wx->it, O_TAG_SECV, ((uint32_t)ptype << 8) | (uint32_t)k}, v[4];
                    o_philox4x32_10(cv, wx->k0, wx->k1, v);
                    const double sgn = vx >= 0.0 ? 1.0 : -1.0; /* SIGN(1.d0, vpx_new) */
                    const double vxs = -sgn * wx->vt_sec * sqrt(-log(1.0 - o_u01(v[0])));
                    double vys, vzs;
                    const double g[2] = {o_u01(v[1]), o_u01(v[2])};
                    o_load_gauss(&vys, &vzs, wx->vt_sec, g);
                    if (wx->n_sec < wx->sec_cap) {
                        double *q = wx->sec_out + 6 * wx->n_sec;
                        q[0] = wx->xg_sec; q[1] = yp; q[2] = zp; q[3] = vxs; q[4] = vys; q[5] = vzs;
                    }
                    wx->n_sec++;
                    wx->P4sec += 0.5 * wx->Nm0 * wx->m0 * (vxs * vxs + vzs * vzs + vzs * vzs);
                }
            }
            if (t && flag_lost == 2) { /* :400-421 Nm q phi at the loss point */
                const double px2 = ((int)(xp / h1) + 1) * h1, py2 = ((int)(yp / h2) + 1) * h2;
                const int jx = (int)(xp / h1) + 1, jy = (int)(yp / h2) + 1;
                const double qx = (px2 - xp) / h1, qy = (py2 - yp) / h2;
                const double phip = qx * qy * zl->phi[NODE(jx, jy, nx)] + (1.0 - qx) * qy * zl->phi[NODE(jx + 1, jy, nx)] +
                                    (1.0 - qx) * (1.0 - qy) * zl->phi[NODE(jx + 1, jy + 1, nx)] +
                                    qx * (1.0 - qy) * zl->phi[NODE(jx, jy + 1, nx)];
                t->P1z += c->Nm[ptype] * c->charge[ptype] * phip;
            }
            if (t) {
                t->n_lost++;
                int igrid = flag_lost == 1 ? bcnd[NODE(ix, iy, nx)] : 0;
                if (igrid < 0) igrid = 0;
                if (igrid > 15) igrid = 15;
                t->n_loss[igrid]++;
                t->v2_loss[igrid] += vx * vx + vy * vy + vz * vz;
            }
            continue;
        }
        if (c->flag_nmn == 1 && xp <= 0.0) {
            int done = 0;
            if (wx && wx->reflux) { /* :445-470 refluxing */
                const double vbx = wx->vb * wx->cos_thB;
                const double vm = vbx - 4.0 * wx->vt > 0.0 ? vbx - 4.0 * wx->vt : 0.0, vpm = vbx + 4.0 * wx->vt;
                const double xmax = nx * h1;
                for (uint32_t a = 0; a < 4096 && !done; a++) {
                    uint32_t cf[4] = {(uint32_t)i, (a << 3) | (uint32_t)ptype, O_TAG_RFX, wx->it}, f[4];
                    o_philox4x32_10(cf, wx->k0, wx->k1, f);
                    const double v = vm + o_u01(f[0]) * (vpm - vm);
                    const double fv = v * exp(-(v - vbx) * (v - vbx) / (wx->vt * wx->vt));
                    if (o_u01(f[1]) > fv / wx->fmax) continue;
                    double vyn, vzn;
                    const double g[2] = {o_u01(f[2]), o_u01(f[3])};
                    o_load_gauss(&vyn, &vzn, wx->vt, g);
                    vyn += wx->vb * wx->sin_thB;
                    uint32_t cg[4] = {(uint32_t)i, (a << 3) | (uint32_t)ptype, O_TAG_RFX2, wx->it}, gg[4];
                    o_philox4x32_10(cg, wx->k0, wx->k1, gg);
                    const double xn = v * (o_u01(gg[0]) * dt);
                    if (xn < 0.0 || xn > xmax) continue;
                    const double ek = 0.5 * c->Nm[ptype] * c->mass[ptype];
                    wx->P1r += ek * (vx * vx + vy * vy + vz * vz);
                    wx->P4r += ek * (v * v + vyn * vyn + vzn * vzn);
                    xp = xn; vx = v; vy = vyn; vz = vzn;
                    done = 1;
                }
            }
            if (!done) { /* :454-459 specular reflection */
                xp = -xp;
                vx = -vx;
            }
        }
        double *q = vxp + 6 * (i - np_lost); /* :496-503 */
        q[0] = xp; q[1] = yp; q[2] = zp; q[3] = vx; q[4] = vy; q[5] = vz;
    }
    *np_tot = n - np_lost; /* :513 */
}

/* main.f90:756-809 with nproc = 1 and one MPI rank */
void o_dielectric_update(const o_cfg *c, double *phi, const int32_t *bcnd, const int32_t *dtype,
                         double *dq, double Ca) {
    const int nx = c->nx, ny = c->ny;
    const int iyl = c->flag_pbc == 1 ? 0 : 2, iyr = c->flag_pbc == 1 ? ny + 2 : ny;
    for (int iy = iyl; iy <= iyr; iy++) {
        const double kd = (iy == 1 || iy == ny + 1) ? 2.0 : 1.0; /* :763 half cell */
        for (int ix = 0; ix <= nx + 2; ix++) {
            const int igrid = bcnd[NODE(ix, iy, nx)];
            if (igrid >= 1 && dtype[o_label(igrid)] == 1)
                phi[NODE(ix, iy, nx)] += kd * dq[(int64_t)o_label(igrid) * (ny + 3) + iy] / (Ca * c->dy);
        }
    }
    for (int64_t k = 0; k < 16 * (int64_t)(ny + 3); k++) dq[k] = 0.0; /* :776 */
}

/* part_expmover.f90:520-610 (heating tally not restated) */
void o_charge_deposition(const o_cfg *c, int ptype, const double *vxp, int64_t np_tot,
                         const double *kq, double *npg) {
    const int nx = c->nx;
    const double h1 = c->dx, h2 = c->dy;
    for (int64_t i = 0; i < np_tot; i++) {
        const double xp = vxp[6 * i], yp = vxp[6 * i + 1];
        int ix = (int)(xp / h1) + 1;
        int iy = (int)(yp / h2) + 1;
        double px = (ix * h1 - xp) / h1;
        double py = (iy * h2 - yp) / h2;
        double k1 = c->Nm[ptype] / (h1 * h2 * c->zmax);
        double k1a = k1 * px * py;
        double k1b = k1 * (1.0 - px) * py;
        double k1c = k1 * (1.0 - px) * (1.0 - py);
        double k1d = k1 * px * (1.0 - py);
        npg[NODE(ix, iy, nx)] = npg[NODE(ix, iy, nx)] + kq[NODE(ix, iy, nx)] * k1a;
        npg[NODE(ix + 1, iy, nx)] = npg[NODE(ix + 1, iy, nx)] + kq[NODE(ix + 1, iy, nx)] * k1b;
        npg[NODE(ix + 1, iy + 1, nx)] =
            npg[NODE(ix + 1, iy + 1, nx)] + kq[NODE(ix + 1, iy + 1, nx)] * k1c;
        npg[NODE(ix, iy + 1, nx)] = npg[NODE(ix, iy + 1, nx)] + kq[NODE(ix, iy + 1, nx)] * k1d;
    }
}

/* calc_rho.f90:1-35 (one grid per species, one thread) */
void o_np_periodic(const o_cfg *c, double *npg, const int32_t *bcnd) {
    const int nx = c->nx, ny = c->ny;
    const int64_t nn = (int64_t)(nx + 3) * (ny + 3);
    for (int ix = 1; ix <= nx + 1; ix++) {
        for (int s = 0; s < c->ntype; s++) {
            double *g = npg + s * nn;
            if (bcnd[NODE(ix, 1, nx)] == 0) {
                g[NODE(ix, 1, nx)] = 0.5 * (g[NODE(ix, 1, nx)] + g[NODE(ix, ny + 1, nx)]);
                g[NODE(ix, 0, nx)] = g[NODE(ix, ny, nx)];
            }
            if (bcnd[NODE(ix, ny + 1, nx)] == 0) {
                g[NODE(ix, ny + 2, nx)] = g[NODE(ix, 2, nx)];
                g[NODE(ix, ny + 1, nx)] = g[NODE(ix, 1, nx)];
            }
        }
    }
}

/* calc_rho.f90:37-77 */
void o_calc_rhs(const o_cfg *c, const double *npg, double *rhs) {
    const int nx = c->nx, ny = c->ny;
    const int64_t nn = (int64_t)(nx + 3) * (ny + 3);
    for (int iy = 1; iy <= ny + 1; iy++)
        for (int ix = 1; ix <= nx + 1; ix++) {
            double r = 0.0;
            for (int s = 0; s < c->ntype; s++) r = r - c->charge[s] * npg[s * nn + NODE(ix, iy, nx)];
            rhs[RHS(ix, iy, nx)] = r;
        }
}

/* calc_rho.f90:134-199 */
void o_dens_red(o_cfg *c, const double *npg, double *np_red, const int32_t *bcnd) {
    const int nx = c->nx, ny = c->ny;
    const int64_t nn = (int64_t)(nx + 3) * (ny + 3);
    for (int s = 0; s < c->ntype; s++) {
        c->np_mx[s] = 0.0;
        for (int64_t k = 0; k < nn; k++) np_red[s * nn + k] = 0.0;
        for (int iy = 1; iy <= ny + 1; iy++)
            for (int ix = 1; ix <= nx + 1; ix++) np_red[s * nn + NODE(ix, iy, nx)] = npg[s * nn + NODE(ix, iy, nx)];
        for (int iy = 1; iy <= ny + 1; iy++)
            for (int ix = 1; ix <= nx + 1; ix++)
                if (bcnd[NODE(ix, iy, nx)] == -1 && np_red[s * nn + NODE(ix, iy, nx)] > c->np_mx[s])
                    c->np_mx[s] = np_red[s * nn + NODE(ix, iy, nx)];
    }
}

/* ------------------------------------------------------------------------------------ */
/* Efield.f90:1-128 in the single-thread loop order */
void o_calc_efield(const o_cfg *c, const double *phi, double *Ei, const int32_t *bcnd) {
    const int nx = c->nx, ny = c->ny;
    const double h1 = c->dx, h2 = c->dy;
#define EX(i, j) Ei[2 * NODE(i, j, nx)]
#define EY(i, j) Ei[2 * NODE(i, j, nx) + 1]
#define PHI(i, j) phi[NODE(i, j, nx)]
#define BC(i, j) bcnd[NODE(i, j, nx)]
    for (int iy = 1; iy <= ny + 1; iy++) /* :19-34 */
        for (int ix = 1; ix <= nx + 1; ix++)
            if (BC(ix, iy) <= 0) {
                EX(ix, iy) = -(PHI(ix + 1, iy) - PHI(ix - 1, iy)) / (2.0 * h1);
                EY(ix, iy) = -(PHI(ix, iy + 1) - PHI(ix, iy - 1)) / (2.0 * h2);
            }
    for (int iy = 1; iy <= ny + 1; iy++) /* :43-122 */
        for (int ix = 1; ix <= nx + 1; ix++) {
            int b = BC(ix, iy);
            if (b == -1) continue;
            if (b == -2) {
                EX(1, iy) = 0.0;
                if (iy > 1 && iy < ny + 1) {
                    EY(1, iy) = -(PHI(1, iy + 1) - PHI(1, iy - 1)) / (2.0 * h2);
                    continue;
                }
            }
            if (b == 0 || b == -2) {
                if (iy == 1) {
                    EY(ix, 1) = -(PHI(ix, 2) - PHI(ix, ny)) / (2.0 * h2);
                    EY(ix, 0) = EY(ix, ny);
                    EY(ix, ny + 1) = EY(ix, 1);
                    EY(ix, ny + 2) = EY(ix, 2);
                    EX(ix, 0) = EX(ix, ny);
                    EX(ix, ny + 2) = EX(ix, 2);
                    continue;
                }
            }
            if (b >= 1) {
                EX(ix, iy) = 0.0;
                EY(ix, iy) = 0.0;
                if (BC(ix + 1, iy) <= 0) EX(ix, iy) = 2.0 * EX(ix + 1, iy) - EX(ix + 2, iy);
                if (BC(ix - 1, iy) <= 0) EX(ix, iy) = 2.0 * EX(ix - 1, iy) - EX(ix - 2, iy);
                if (BC(ix, iy + 1) <= 0) EY(ix, iy) = 2.0 * EY(ix, iy + 1) - EY(ix, iy + 2);
                if (BC(ix, iy - 1) <= 0) EY(ix, iy) = 2.0 * EY(ix, iy - 1) - EY(ix, iy - 2);
            }
        }
#undef EX
#undef EY
#undef PHI
#undef BC
}

/* ------------------------------------------------------------------------------------ */
/* Multigrid.  Level arrays follow mg.f90:28-44: u/e (0:n+2)^2, r (1:n+1)^2, bcnd (0:n+2)^2. */

/* sors.f90:1-435 with nproc = 1 (jl = 1, jr = ny+1, no halo exchange) */
static int sor_rb_nt(int nx, int ny, double hx, double hy, double eps0, double *u,
                     const double *b, const int32_t *bcnd, double *res_out, double omega,
                     double eps, int kmg, int dig, int flag_pbc, int nt) {
    const double aw = eps0 / (hx * hx), ae = aw, an = eps0 / (hy * hy), as = an;
    const double ac = -(an + as + aw + ae); /* mg.h:11-15 */
    const int W = nx + 3;
    double res = 0.0, res_s = 0.0;
    int ksor = 0;
    int nr = 10;
    if (kmg == 1 && dig == 0) nr = 1000000; /* :64 */
    const double eta = 0.6;
    (void)nt;
    for (int k = 1; k <= nr; k++) {
        for (int color = 0; color < 2; color++) {
            /* red: j even -> is = 1, j odd -> is = 2 ; black: j even -> 2, j odd -> 1 */
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
            for (int j = 1; j <= ny + 1; j++) {
                int is = (j % 2 == 0) ? (color == 0 ? 1 : 2) : (color == 0 ? 2 : 1);
                for (int i = is; i <= nx + 1; i += 2) {
                    int bc = bcnd[i + j * W];
                    if (bc > 0) continue;
                    double bij = b[(i - 1) + (j - 1) * (nx + 1)];
                    if (bc == -2) {
                        u[i + j * W] = (1.0 - omega) * u[i + j * W] +
                                       omega * (bij - an * u[i + (j + 1) * W] - as * u[i + (j - 1) * W] -
                                                2.0 * ae * u[i + 1 + j * W]) / ac;
                        continue;
                    }
                    if (bc == 0 && j == ny + 1) continue;
                    u[i + j * W] = (1.0 - omega) * u[i + j * W] +
                                   omega * (bij - aw * u[i - 1 + j * W] - an * u[i + (j + 1) * W] -
                                            as * u[i + (j - 1) * W] - ae * u[i + 1 + j * W]) / ac;
                }
            }
            if (flag_pbc == 1) { /* :185-200 */
                for (int i = 0; i <= nx + 2; i++) {
                    if (bcnd[i + 1 * W] <= 0) u[i + 0 * W] = u[i + ny * W];
                    if (bcnd[i + (ny + 1) * W] <= 0) u[i + (ny + 1) * W] = u[i + 1 * W];
                }
            }
        }
        res = 0.0; /* :338-357 */
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static) reduction(+ : res)
        for (int j = 1; j <= ny + 1; j++)
            for (int i = 1; i <= nx + 1; i++) {
                double rij = 0.0;
                if (bcnd[i + j * W] == -1)
                    rij = b[(i - 1) + (j - 1) * (nx + 1)] -
                          (aw * u[i - 1 + j * W] + an * u[i + (j + 1) * W] + as * u[i + (j - 1) * W] +
                           ae * u[i + 1 + j * W] + ac * u[i + j * W]);
                res = res + fabs(rij);
            }
        ksor = ksor + 1; /* :371-379 */
        if (dig == 0) {
            if (res <= eps) break;
        } else {
            if (res_s > 0.0 && (res / res_s) <= eta) break;
        }
        res_s = res;
    }
    *res_out = res;
    return ksor;
}

int o_sor_rb(int nx, int ny, double hx, double hy, double eps0, double *u, const double *b,
             const int32_t *bcnd, double *res, double omega, double eps, int kmg, int dig,
             int flag_pbc) {
    return sor_rb_nt(nx, ny, hx, hy, eps0, u, b, bcnd, res, omega, eps, kmg, dig, flag_pbc, 1);
}

/* mg.f90:512-547 */
static inline double getres(const double *u, const double *b, int nx, double hx, double hy,
                            double eps0, int ir, int jr, int flag) {
    double aw = eps0 / (hx * hx), ae = aw, an = eps0 / (hy * hy), as = an;
    const double ac = -(an + as + aw + ae);
    const int W = nx + 3;
    double uij = u[ir + jr * W], un = u[ir + (jr + 1) * W], us = u[ir + (jr - 1) * W];
    double ue = u[ir + 1 + jr * W], uw;
    if (ir == 1 && flag == 1) {
        uw = 0.0;
        aw = 0;
        ae = 2.0 * ae;
    } else {
        uw = u[ir - 1 + jr * W];
    }
    double urhs = b[(ir - 1) + (jr - 1) * (nx + 1)];
    return urhs - (aw * uw + ae * ue + an * un + as * us + ac * uij);
}

/* mg.f90:235-509 with nproc = 1 */
static void restriction_nt(int nx, int ny, double hx, double hy, double eps0, const double *u,
                           const double *b, const int32_t *bcnd, int32_t *bcnd2h, double *r2h,
                           double *e2h, int flag_pbc, int flag_nmn, int nt) {
    const int W = nx + 3, nx2 = nx / 2, ny2 = ny / 2, W2 = nx2 + 3;
    double *r_pbc = NULL;
    if (flag_pbc == 1) { /* :298-311 */
        r_pbc = (double *)calloc((size_t)nx + 2, sizeof(double)); /* r_pbc(1:nx+1) */
        for (int i = 1; i <= nx2 + 1; i++) {
            int ir = 2 * i - 1;
            if (bcnd[ir + (ny + 1) * W] <= 0) {
                if (ir != nx + 1) r_pbc[ir + 1] = getres(u, b, nx, hx, hy, eps0, ir + 1, ny, flag_nmn);
                r_pbc[ir] = getres(u, b, nx, hx, hy, eps0, ir, ny, flag_nmn);
                if (ir != 1) r_pbc[ir - 1] = getres(u, b, nx, hx, hy, eps0, ir - 1, ny, flag_nmn);
            }
        }
    }
    /* ghost corners of the coarse mask are not written by the reference (stack garbage);
     * here they are injected from the fine ghost corners so that every run is defined */
    bcnd2h[0] = bcnd[0];
    bcnd2h[(nx2 + 2)] = bcnd[nx + 2];
    bcnd2h[(ny2 + 2) * W2] = bcnd[(ny + 2) * W];
    bcnd2h[(nx2 + 2) + (ny2 + 2) * W2] = bcnd[(nx + 2) + (ny + 2) * W];
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
    for (int j = 1; j <= ny2 + 1; j++) { /* :335-427 */
        for (int i = 1; i <= nx2 + 1; i++) {
            int ir = 2 * i - 1, jr = 2 * j - 1;
            bcnd2h[i + j * W2] = bcnd[ir + jr * W];
            if (ir == 1) bcnd2h[0 + j * W2] = bcnd[0 + jr * W];
            if (ir == nx + 1) bcnd2h[nx2 + 2 + j * W2] = bcnd[nx + 2 + jr * W];
            if (jr == 1) bcnd2h[i + 0 * W2] = bcnd[ir + 0 * W];
            if (jr == ny + 1) bcnd2h[i + (ny2 + 2) * W2] = bcnd[ir + (ny + 2) * W];
            if (bcnd2h[i + j * W2] <= 0) {
                double r1 = 0, r2 = 0, r3 = 0, r4 = 0, r5 = 0, r6 = 0, r7 = 0, r8 = 0, r9 = 0;
                r9 = getres(u, b, nx, hx, hy, eps0, ir, jr, flag_nmn);
                if (ir != nx + 1 && jr != ny + 1)
                    if (bcnd[ir + 1 + (jr + 1) * W] <= 0) r1 = getres(u, b, nx, hx, hy, eps0, ir + 1, jr + 1, flag_nmn);
                if (ir != nx + 1)
                    if (bcnd[ir + 1 + jr * W] <= 0) r2 = getres(u, b, nx, hx, hy, eps0, ir + 1, jr, flag_nmn);
                if (bcnd[ir + 1 + (jr - 1) * W] <= 0) {
                    if (ir != nx + 1 && jr != 1) r3 = getres(u, b, nx, hx, hy, eps0, ir + 1, jr - 1, flag_nmn);
                    else if (jr == 1) r3 = r_pbc ? r_pbc[ir + 1] : 0.0;
                }
                if (bcnd[ir + (jr - 1) * W] <= 0) {
                    if (jr != 1) r4 = getres(u, b, nx, hx, hy, eps0, ir, jr - 1, flag_nmn);
                    else r4 = r_pbc ? r_pbc[ir] : 0.0;
                }
                if (bcnd[ir - 1 + (jr - 1) * W] <= 0 && ir != 1) {
                    if (jr != 1) r5 = getres(u, b, nx, hx, hy, eps0, ir - 1, jr - 1, flag_nmn);
                    else r5 = r_pbc ? r_pbc[ir - 1] : 0.0;
                }
                if (bcnd[ir - 1 + jr * W] <= 0)
                    if (ir != 1) r6 = getres(u, b, nx, hx, hy, eps0, ir - 1, jr, flag_nmn);
                if (bcnd[ir - 1 + (jr + 1) * W] <= 0)
                    if (ir != 1 && jr != ny + 1) r7 = getres(u, b, nx, hx, hy, eps0, ir - 1, jr + 1, flag_nmn);
                if (bcnd[ir + (jr + 1) * W] <= 0)
                    if (jr != ny + 1) r8 = getres(u, b, nx, hx, hy, eps0, ir, jr + 1, flag_nmn);
                r2h[(i - 1) + (j - 1) * (nx2 + 1)] =
                    (4.0 * r9 + 2.0 * (r2 + r4 + r6 + r8) + r1 + r3 + r5 + r7) / 16.0;
            } else {
                r2h[(i - 1) + (j - 1) * (nx2 + 1)] = 0.0;
            }
        }
    }
    /* :424-444 the whole coarse correction starts at zero, ghosts included */
    memset(e2h, 0, sizeof(double) * (size_t)W2 * (ny2 + 3));
    free(r_pbc);
}

void o_restriction(int nx, int ny, double hx, double hy, double eps0, const double *u,
                   const double *b, const int32_t *bcnd, int32_t *bcnd2h, double *r2h,
                   double *e2h, int flag_pbc, int flag_nmn) {
    restriction_nt(nx, ny, hx, hy, eps0, u, b, bcnd, bcnd2h, r2h, e2h, flag_pbc, flag_nmn, 1);
}

/* mg.f90:549-616 (each fine node is written by exactly one coarse node) */
static void prolongation_nt(int nx, int ny, double *u, const double *e2h, const int32_t *bcnd,
                            int nt) {
    const int W = nx + 3, nx2 = nx / 2, ny2 = ny / 2, W2 = nx2 + 3;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
    for (int j = 1; j <= ny2 + 1; j++)
        for (int i = 1; i <= nx2 + 1; i++) {
            double r1 = e2h[i + j * W2], r2 = e2h[i + (j - 1) * W2];
            double r3 = e2h[i - 1 + (j - 1) * W2], r4 = e2h[i - 1 + j * W2];
            int ir = 2 * i - 1, jr = 2 * j - 1;
            if (bcnd[ir + jr * W] <= 0) u[ir + jr * W] = u[ir + jr * W] + r1;
            if (bcnd[ir + (jr - 1) * W] <= 0) u[ir + (jr - 1) * W] = u[ir + (jr - 1) * W] + (r1 + r2) / 2.0;
            if (bcnd[ir - 1 + (jr - 1) * W] <= 0)
                u[ir - 1 + (jr - 1) * W] = u[ir - 1 + (jr - 1) * W] + (r1 + r2 + r3 + r4) / 4.0;
            if (bcnd[ir - 1 + jr * W] <= 0) u[ir - 1 + jr * W] = u[ir - 1 + jr * W] + (r1 + r4) / 2.0;
        }
}

void o_prolongation(int nx, int ny, double *u, const double *e2h, const int32_t *bcnd) {
    prolongation_nt(nx, ny, u, e2h, bcnd, 1);
}

typedef struct { int nx, ny; double hx, hy; double *u; double *b; int32_t *bc; } mg_level;

/* mg.f90:1-232: one V-cycle (ig = 1 .. 2ng-1); returns the residual of the last fine sweep */
static double mg_vcycle(const o_cfg *c, mg_level *L, int ng, double omega, double eps, int k,
                        double *ktot, int *sweeps_fine, int nt) {
    int iter[16] = {0};
    double res = 0.0;
    for (int ig = 1; ig <= 2 * ng - 1; ig++) {
        for (int il = 1; il < ng; il++) {
            int down = (ig < ng && ig == il), up = (ig > ng && ig == 2 * ng - il);
            if (!(down || up)) continue;
            mg_level *a = &L[il - 1];
            int ks = sor_rb_nt(a->nx, a->ny, a->hx, a->hy, c->eps0, a->u, a->b, a->bc, &res, omega,
                               eps, k, ig - ng, c->flag_pbc, nt);
            iter[il - 1] += ks;
            if (il == 1 && sweeps_fine) *sweeps_fine += ks;
            if (down) {
                mg_level *d = &L[il];
                restriction_nt(a->nx, a->ny, a->hx, a->hy, c->eps0, a->u, a->b, a->bc, d->bc, d->b,
                               d->u, c->flag_pbc, c->flag_nmn, nt);
            }
            if (up && il >= 2) {
                mg_level *f = &L[il - 2];
                prolongation_nt(f->nx, f->ny, f->u, a->u, f->bc, nt);
            }
        }
        if (ig == ng) { /* :197-223 coarsest level */
            mg_level *a = &L[ng - 1];
            int ks = sor_rb_nt(a->nx, a->ny, a->hx, a->hy, c->eps0, a->u, a->b, a->bc, &res, omega,
                               eps, k, 0, c->flag_pbc, nt);
            iter[ng - 1] += ks;
            if (ng == 1 && sweeps_fine) *sweeps_fine += ks;
            if (ng >= 2) {
                mg_level *f = &L[ng - 2];
                prolongation_nt(f->nx, f->ny, f->u, a->u, f->bc, nt);
            }
        }
    }
    for (int i = 1; i <= ng; i++) *ktot += (double)iter[i - 1] / pow(2.0, 2 * (i - 1));
    return res;
}

/* ||b - A u||_2 and ||b - A u_D||_2 over the bcnd == -1 nodes (u_D: the walls' values only),
 * the relative residual the device's mixed and L2 modes stop on */
static void l2_norms(const o_cfg *c, const double *u, const double *b, const int32_t *bcnd, double *rr,
                     double *dd, int nt) {
    const int nx = c->nx, ny = c->ny;
    const double aw = c->eps0 / (c->dx * c->dx), an = c->eps0 / (c->dy * c->dy);
    const double ac = -(an + an + aw + aw);
    double sr = 0.0, sd = 0.0;
#pragma omp parallel for num_threads(nt) reduction(+ : sr, sd) schedule(static)
    for (int iy = 1; iy <= ny + 1; iy++)
        for (int ix = 1; ix <= nx + 1; ix++) {
            const int64_t n = NODE(ix, iy, nx);
            if (bcnd[n] != -1) continue;
            const int64_t W = nx + 3;
            const double bb = b[RHS(ix, iy, nx)];
            const double r = bb - (aw * u[n - 1] + an * u[n + W] + an * u[n - W] + aw * u[n + 1] + ac * u[n]);
            const double d = bb - ((bcnd[n - 1] > 0 ? aw * u[n - 1] : 0.0) + (bcnd[n + W] > 0 ? an * u[n + W] : 0.0) +
                                   (bcnd[n - W] > 0 ? an * u[n - W] : 0.0) + (bcnd[n + 1] > 0 ? aw * u[n + 1] : 0.0));
            sr += r * r;
            sd += d * d;
        }
    *rr = sqrt(sr);
    *dd = sqrt(sd);
}

static int solver_impl(const o_cfg *c, double *u, const double *b, const int32_t *bcnd, int ng,
                       int ncycl, double eps, o_solve_stats *st, int nt, int l2) {
    const int nx = c->nx, ny = c->ny;
    mg_level L[16];
    memset(L, 0, sizeof(L));
    L[0].nx = nx; L[0].ny = ny; L[0].hx = c->dx; L[0].hy = c->dy;
    L[0].u = u; L[0].b = (double *)b; L[0].bc = (int32_t *)bcnd;
    for (int l = 1; l < ng; l++) {
        L[l].nx = L[l - 1].nx / 2; L[l].ny = L[l - 1].ny / 2;
        L[l].hx = 2.0 * L[l - 1].hx; L[l].hy = 2.0 * L[l - 1].hy;
        size_t nn = (size_t)(L[l].nx + 3) * (L[l].ny + 3);
        L[l].u = (double *)calloc(nn, sizeof(double));
        L[l].b = (double *)calloc((size_t)(L[l].nx + 1) * (L[l].ny + 1), sizeof(double));
        L[l].bc = (int32_t *)calloc(nn, sizeof(int32_t));
    }
    const double aw = c->eps0 / (c->dx * c->dx), an = c->eps0 / (c->dy * c->dy);
    const double ac = -(an + an + aw + aw);
    const double alpha = fabs((double)(nx + 1) * (ny + 1) * ac) * 1.0; /* :22-23 */
    double ktot = 0.0, res = 0.0, res_s = 0.0;
    const double omega = 1.4;
    int k = 1, rc = 0, sweeps = 0;
    double rr = 0.0, b0 = 0.0;
    if (l2) l2_norms(c, u, b, bcnd, &rr, &b0, nt);
    for (;;) { /* :33-66 */
        res = mg_vcycle(c, L, ng, omega, alpha * eps, k, &ktot, &sweeps, nt);
        res = res / alpha;
        if (k == 1) res_s = res;
        else if (fabs(res / res_s) > 10.0) { rc = -1; break; }
        int conv = res <= eps;
        if (l2) {
            double dd;
            l2_norms(c, u, b, bcnd, &rr, &dd, nt);
            conv = rr <= eps * b0;
        }
        if (conv || k == ncycl) break;
        k = k + 1;
    }
    for (int l = 1; l < ng; l++) { free(L[l].u); free(L[l].b); free(L[l].bc); }
    if (st) { st->k = k; st->ktot = ktot; st->res = res; st->sweeps_fine = sweeps; }
    return rc;
}

int o_iterative_solver(const o_cfg *c, double *u, const double *b, const int32_t *bcnd, int ng,
                       int ncycl, double eps, o_solve_stats *st) {
    return solver_impl(c, u, b, bcnd, ng, ncycl, eps, st, 1, 0);
}

int o_iterative_solver_omp(const o_cfg *c, double *u, const double *b, const int32_t *bcnd,
                           int ng, int ncycl, double eps, o_solve_stats *st, int nthreads) {
    return solver_impl(c, u, b, bcnd, ng, ncycl, eps, st, nthreads < 1 ? 1 : nthreads, 0);
}

int o_iterative_solver_l2_omp(const o_cfg *c, double *u, const double *b, const int32_t *bcnd,
                              int ng, int ncycl, double eps, o_solve_stats *st, int nthreads) {
    return solver_impl(c, u, b, bcnd, ng, ncycl, eps, st, nthreads < 1 ? 1 : nthreads, 1);
}

/* ------------------------------------------------------------------------------------ */
/* sorting.f90:92-251, nproc = 1: stable counting sort; plist(ic) ends as the inclusive end */
void o_part_sorting(const o_cfg *c, double *vxp, int64_t np_tot, int32_t *plist,
                    double *scratch) {
    const int nx = c->nx, ny = c->ny;
    const int pl_max = nx + nx * ny + 1;
    memset(plist, 0, sizeof(int32_t) * (size_t)(pl_max + 1));
    for (int64_t i = 0; i < np_tot; i++) {
        const double *p = vxp + 6 * i;
        int ix = (int)(p[0] / c->dx) + 1, iy = (int)(p[1] / c->dy) + 1;
        int ic = (ix - 1) + nx * (iy - 1) + 1;
        plist[ic] += 1;
        memcpy(scratch + 6 * i, p, 6 * sizeof(double));
    }
    int32_t k = 0;
    for (int i = 1; i <= pl_max; i++) {
        int32_t j = plist[i];
        plist[i] = k;
        k += j;
    }
    for (int64_t i = 0; i < np_tot; i++) {
        const double *p = scratch + 6 * i;
        int ix = (int)(p[0] / c->dx) + 1, iy = (int)(p[1] / c->dy) + 1;
        int ic = (ix - 1) + nx * (iy - 1) + 1;
        plist[ic] += 1;
        int32_t j = plist[ic];
        memcpy(vxp + 6 * (int64_t)(j - 1), p, 6 * sizeof(double));
    }
}

/* indexx.f90:1-88 (Numerical Recipes), output 0-based */
void o_indexx(int n, const double *arr0, int *indx0) {
    const int M = 7, NSTACK = 50;
    int istack[51];
    int indx[O_MAXCOL + 2];
    const double *arr = arr0 - 1; /* 1-based views */
    int i, indxt, ir, itemp, j, jstack, k, l;
    double a;
    for (j = 1; j <= n; j++) indx[j] = j;
    jstack = 0; l = 1; ir = n;
    for (;;) {
        if (ir - l < M) {
            for (j = l + 1; j <= ir; j++) {
                indxt = indx[j]; a = arr[indxt];
                for (i = j - 1; i >= 1; i--) {
                    if (arr[indx[i]] <= a) break;
                    indx[i + 1] = indx[i];
                }
                if (i < 1) i = 0;
                indx[i + 1] = indxt;
            }
            if (jstack == 0) break;
            ir = istack[jstack]; l = istack[jstack - 1]; jstack -= 2;
        } else {
            k = (l + ir) / 2;
            itemp = indx[k]; indx[k] = indx[l + 1]; indx[l + 1] = itemp;
            if (arr[indx[l + 1]] > arr[indx[ir]]) { itemp = indx[l + 1]; indx[l + 1] = indx[ir]; indx[ir] = itemp; }
            if (arr[indx[l]] > arr[indx[ir]]) { itemp = indx[l]; indx[l] = indx[ir]; indx[ir] = itemp; }
            if (arr[indx[l + 1]] > arr[indx[l]]) { itemp = indx[l + 1]; indx[l + 1] = indx[l]; indx[l] = itemp; }
            i = l + 1; j = ir; indxt = indx[l]; a = arr[indxt];
            for (;;) {
                do i++; while (arr[indx[i]] < a);
                do j--; while (arr[indx[j]] > a);
                if (j < i) break;
                itemp = indx[i]; indx[i] = indx[j]; indx[j] = itemp;
            }
            indx[l] = indx[j]; indx[j] = indxt;
            jstack += 2;
            if (jstack > NSTACK) return;
            if (ir - i + 1 >= j - l) { istack[jstack] = ir; istack[jstack - 1] = i; ir = j - 1; }
            else { istack[jstack] = j - 1; istack[jstack - 1] = l; l = i; }
        }
    }
    for (j = 1; j <= n; j++) indx0[j - 1] = indx[j] - 1;
}

/* collisions.f90:1042-1070 */
void o_scatter(double *vx1, double *vy1, double *vz1, double vx, double vy, double vz,
               double costheta, double phi) {
    double sintheta = sqrt(fmax(1.0 - costheta * costheta, 0.0));
    double sinphi = sin(phi), cosphi = cos(phi);
    double v = sqrt(vx * vx + vy * vy + vz * vz), vv;
    if (v == 0) return;
    if (fabs(vy) > fabs(vz)) {
        vv = sqrt(vx * vx + vy * vy);
        *vx1 = vx * costheta + (vy * v * sinphi + vx * vz * cosphi) / vv * sintheta;
        *vy1 = vy * costheta + (-vx * v * sinphi + vy * vz * cosphi) / vv * sintheta;
        *vz1 = vz * costheta - vv * cosphi * sintheta;
    } else {
        vv = sqrt(vx * vx + vz * vz);
        *vx1 = vx * costheta + (vz * v * sinphi - vy * vx * cosphi) / vv * sintheta;
        *vy1 = vy * costheta + vv * cosphi * sintheta;
        *vz1 = vz * costheta - (vx * v * sinphi + vy * vz * cosphi) / vv * sintheta;
    }
}

/* collisions.f90:339-403: the target of species tt for the incident in 1-based cell ici of the
 * reference's row-major numbering: the incident's cell, else the first non-empty of ici+1,
 * ici-1, ici+nx, ici-nx (the linear index, which wraps rows at the box edges) inside 1..pl_max;
 * returns the cell (0: none) */
static int dsmc_cell(const int32_t *plist, int ici, int nx, int pl_max) {
    const int cand[5] = {ici, ici + 1, ici - 1, ici + nx, ici - nx};
    for (int k = 0; k < 5; k++) {
        const int ict = cand[k];
        if (ict <= 0 || ict > pl_max) continue;
        if (plist[ict] - plist[ict - 1] > 0) return ict;
    }
    return 0;
}

/* collisions.f90:1-207 and collision_OMP :209-1040, one thread (nproc = 1); charged targets
 * (DSMC, :339-418, :524-528, :767-797, :908-935, :942-1000) when d gives the targets' Plist */
int o_collisions_dsmc(o_cfg *c, const o_xs *xs, double **vxp, int64_t *np_tot, const int64_t *cap,
                      int8_t **flag_dead, int32_t *iseed, o_mcc_tally *t, const o_dsmc *d) {
    const double pi = c->pi, qe = c->qe, dt = c->dt;
    const int pl_max = c->nx + c->nx * c->ny + 1;
    const int64_t nn = (int64_t)(c->nx + 3) * (c->ny + 3);
    int64_t Nc[O_MAXSP] = {0}, np_add[O_MAXSP] = {0};
    int sav_ttype[O_MAXCOL];
    for (int i = 0; i < O_MAXCOL; i++) sav_ttype[i] = -1;
    for (int p = 0; p < c->ntype; p++) { /* :92-157 */
        c->mass[p] = c->mass[p];
        if (xs->p_ncol[p] == 0 || c->mass[p] <= 0) continue;
        double nu_max = 0.0;
        for (int icol = 0; icol < xs->p_ncol[p]; icol++) {
            int ind_col = xs->sig_list[p * O_MAXCOL + icol];
            const int32_t *ci = xs->col_info + ind_col * 10;
            int n_re = ci[0];
            int ttype = ci[2 + n_re - 1];
            sav_ttype[ind_col] = ttype;
            nu_max = nu_max + c->np_mx[ttype] * xs->sigv_mx[p * O_MAXCOL + ind_col];
        }
        nu_max = fmin(nu_max, c->nu_uplim[p]);
        if (t) t->nu_max[p] = nu_max;
        int64_t sum_np_tot = np_tot[p];
        double Pmax = nu_max * (double)(float)c->ns_coll * dt;
        if (Pmax > 1.0) return -1;
        double dNc = (double)sum_np_tot * Pmax / (double)(float)1;
        int64_t Nc_tmp = (int64_t)dNc;
        double rnd = o_ran2(iseed);
        if (rnd <= (dNc - (double)Nc_tmp)) Nc_tmp = Nc_tmp + 1;
        Nc[p] = Nc_tmp;
    }
    for (int p = 0; p < c->ntype; p++) { /* :162-181 and collision_OMP */
        if (xs->p_ncol[p] == 0 || c->mass[p] <= 0 || Nc[p] == 0 || np_tot[p] == 0) continue;
        if (t) t->n_cand[p] += Nc[p];
        /* :172 real() is default (single) precision in the reference */
        double nu_max_OMP = (double)((float)Nc[p] / (float)np_tot[p]) / ((double)(float)c->ns_coll * dt);
        double vz_sav = 0.0, vzb_sav = 0.0;
        const double mp = fabs(c->mass[p]);
        for (int64_t ic = 0; ic < Nc[p]; ic++) {
            double r0 = o_ran2(iseed);
            int64_t ip = (int64_t)((double)np_tot[p] * r0); /* 0-based: INT(N*r)+1-1 */
            if (ip == np_tot[p]) return -4;
            double *P = vxp[p] + 6 * ip;
            double vx[2], vy[2], vz[2];
            vx[0] = P[3]; vy[0] = P[4]; vz[0] = P[5];
            const int ixc = (int)(P[0] / c->dx) + 1, iyc = (int)(P[1] / c->dy) + 1; /* :286-292 */
            const int ici = (ixc - 1) + c->nx * (iyc - 1) + 1;
            int flag_err[O_MAXSP] = {0};
            int64_t sav_it[O_MAXSP];
            for (int q = 0; q < O_MAXSP; q++) sav_it[q] = -1;
            int flag_ttype[O_MAXSP] = {0};
            double vr[O_MAXSP] = {0}, Ekr[O_MAXSP] = {0}, mu[O_MAXSP] = {0};
            double vx_cm[O_MAXSP] = {0}, vy_cm[O_MAXSP] = {0}, vz_cm[O_MAXSP] = {0};
            double nu[O_MAXCOL] = {0}, sort_arr[O_MAXCOL] = {0}, sum_nu = 0.0;
            int c_ind = -1;
            for (int icol = 0; icol < xs->p_ncol[p]; icol++) {
                int ind_col = xs->sig_list[p * O_MAXCOL + icol];
                int ttype = sav_ttype[ind_col];
                const int charged = c->charge[ttype] != 0.0;
                if (charged && (!d || !d->plist[ttype])) continue; /* no target list: not restated */
                if (flag_err[ttype]) continue;                      /* :333 */
                if (flag_ttype[ttype] == 0) {
                    if (charged) { /* :339-418: the target particle and its velocity */
                        const int ict = dsmc_cell(d->plist[ttype], ici, c->nx, pl_max);
                        if (ict == 0) { flag_err[ttype] = 1; continue; }
                        const double r = o_ran2(iseed);
                        const int64_t it1 = (int64_t)((double)d->plist[ttype][ict] * (1.0 - r) +
                                                      (double)d->plist[ttype][ict - 1] * r + 1.0);
                        sav_it[ttype] = it1 - 1;
                        const double *T = vxp[ttype] + 6 * (it1 - 1);
                        vx[1] = T[3]; vy[1] = T[4]; vz[1] = T[5];
                    } else {
                    double rr[2];
                    rr[0] = o_ran2(iseed); rr[1] = o_ran2(iseed);
                    o_load_gauss(&vx[1], &vy[1], c->vt0[ttype], rr);
                    if (vz_sav == 0.0) {
                        rr[0] = o_ran2(iseed); rr[1] = o_ran2(iseed);
                        o_load_gauss(&vz[1], &vz_sav, c->vt0[ttype], rr);
                    } else {
                        vz[1] = vz_sav;
                        vz_sav = 0.0;
                    }
                    }
                    const double mt = fabs(c->mass[ttype]);
                    mu[ttype] = mp * mt / (mp + mt);
                    vr[ttype] = sqrt((vx[0] - vx[1]) * (vx[0] - vx[1]) + (vy[0] - vy[1]) * (vy[0] - vy[1]) +
                                     (vz[0] - vz[1]) * (vz[0] - vz[1]));
                    Ekr[ttype] = (0.5 * mu[ttype] * (vr[ttype] * vr[ttype])) / qe;
                    double sum_mass = mp + mt;
                    vx_cm[ttype] = (mp * vx[0] + mt * vx[1]) / sum_mass;
                    vy_cm[ttype] = (mp * vy[0] + mt * vy[1]) / sum_mass;
                    vz_cm[ttype] = (mp * vz[0] + mt * vz[1]) / sum_mass;
                    if (Ekr[ttype] > xs->sig_Er[xs->npt - 1] && t) t->n_overflow++;
                    flag_ttype[ttype] = 1;
                }
                /* :485-497 five bisection steps on the union grid (1-based indices) */
                int ipt_L = 1, ipt_R = xs->npt;
                const double *Er = xs->sig_Er - 1;
                for (int s = 0; s < 5; s++) {
                    int ipt_M = (int)((double)(float)(ipt_R - ipt_L) / 2.0) + ipt_L;
                    double Ek_L = Er[ipt_L], Ek_R = Er[ipt_R], Ek_M = Er[ipt_M];
                    if (Ekr[ttype] >= Ek_L && Ekr[ttype] <= Ek_M) ipt_R = ipt_M;
                    if (Ekr[ttype] > Ek_M && Ekr[ttype] <= Ek_R) ipt_L = ipt_M;
                }
                for (int ipt = ipt_L + 1; ipt <= ipt_R; ipt++) { /* :503-611 */
                    double Ek_L = Er[ipt - 1], Ek_R = Er[ipt];
                    if (Ekr[ttype] > Ek_L && Ekr[ttype] <= Ek_R) {
                        const double *sg = xs->sig + (int64_t)ind_col * xs->npt - 1;
                        double sig_L = sg[ipt - 1], sig_R = sg[ipt];
                        double sig_p = sig_L + (Ekr[ttype] - Ek_L) * (sig_R - sig_L) / (Ek_R - Ek_L);
                        double np_t = c->np_mx[ttype];
                        if (charged) { /* :524-528, the four nodes of the incident's cell */
                            const double *g = d->np_red + ttype * nn;
                            np_t = 0.25 * (g[NODE(ixc, iyc, c->nx)] + g[NODE(ixc + 1, iyc, c->nx)] +
                                           g[NODE(ixc, iyc + 1, c->nx)] + g[NODE(ixc + 1, iyc + 1, c->nx)]);
                        }
                        nu[icol] = np_t * sig_p * vr[ttype] / nu_max_OMP;
                        sum_nu = sum_nu + nu[icol];
                        sort_arr[icol] = nu[icol];
                        break;
                    }
                }
            }
            int indx[O_MAXCOL];
            o_indexx(xs->p_ncol[p], sort_arr, indx); /* :619 */
            double r1 = o_ran2(iseed); /* :624-647 */
            int flag_coll = 0;
            if (r1 <= sum_nu) {
                sum_nu = 0.0;
                for (int icol = 0; icol < xs->p_ncol[p]; icol++) {
                    sum_nu = sum_nu + nu[indx[icol]];
                    if (r1 <= sum_nu) {
                        flag_coll = 1;
                        c_ind = xs->sig_list[p * O_MAXCOL + indx[icol]];
                        break;
                    }
                }
            }
            if (!flag_coll) continue;
            const int32_t *ci = xs->col_info + c_ind * 10;
            int n_re = ci[0], n_by = ci[1], rt = ci[2 + n_re + n_by];
            int ttype = sav_ttype[c_ind];
            if (t) t->n_coll[c_ind]++;
            if (rt != 4) { /* :677-937 */
                double Eth = xs->Eth[c_ind];
                double Ee = 0.5 * mu[ttype] * (vr[ttype] * vr[ttype]) - Eth * qe;
                int opt_scat = 1;
                double Ek_b[16] = {0}, sum_mass = 0.0, th = 0, th_add = 0, sin_ph = 0, cos_ph = 0;
                double cos_th_s = 0, phi_s = 0;
                if (rt == 2 && xs->flag_ionrep >= 1 && n_by == 3) {
                    int cnt_ele = 0, flag_ion = 0;
                    for (int ib = 0; ib < n_by; ib++) {
                        int bt = ci[2 + n_re + ib];
                        if (bt == 0) {
                            cnt_ele++;
                            if (cnt_ele == 1) Ek_b[ib] = xs->fEk;
                            if (cnt_ele == 2) Ek_b[ib] = 1.0 - xs->fEk;
                        }
                        if (bt != 0 && c->charge[bt] != 0) flag_ion = 1;
                    }
                    if (cnt_ele == 2 && flag_ion == 1) {
                        opt_scat = 2;
                        Ee = 0.5 * c->mass[0] * (vx[0] * vx[0] + vy[0] * vy[0] + vz[0] * vz[0]) - Eth * qe;
                        if (Ee < 0.0) Ee = 0.0;
                    }
                } else {
                    for (int ib = 0; ib < n_by; ib++) sum_mass = sum_mass + 1.0 / fabs(c->mass[ci[2 + n_re + ib]]);
                    double rr0 = o_ran2(iseed), rr1 = o_ran2(iseed);
                    th_add = 2.0 * pi / (double)(float)n_by;
                    double cos_th = 1.0 - 2.0 * rr0;
                    th = acos(cos_th);
                    double phi = 2.0 * pi * rr1;
                    cos_ph = cos(phi);
                    sin_ph = sin(phi);
                    rr0 = o_ran2(iseed); rr1 = o_ran2(iseed);
                    cos_th_s = 1.0 - 2.0 * rr0;
                    phi_s = 2.0 * pi * rr1;
                }
                if (Ee < 0.0) return -3;
                int flag_add[16];
                for (int q = 0; q < 16; q++) flag_add[q] = 0;
                flag_add[0] = -1; flag_add[1] = -1;
                for (int q = n_re; q < n_re + n_by; q++) flag_add[q] = 0;
                for (int iby = 0; iby < n_by; iby++) { /* :767-902 */
                    int bt = ci[2 + n_re + iby];
                    if (c->mass[bt] <= 0) continue;
                    int opt_add = 1;
                    int64_t ib = -1;
                    if (iby == 0 && bt == p) { ib = ip; opt_add = 0; flag_add[0] = 0; }
                    if (rt == 1 || rt == 3) {
                        if (bt == p) ib = ip;
                        if (bt == ttype && bt != p) ib = sav_it[ttype]; /* :794-797 the target scatters too */
                        opt_add = 0;
                        flag_add[0] = 0; flag_add[1] = 0;
                    }
                    if (opt_add == 1) {
                        np_add[bt]++;
                        ib = np_tot[bt] + np_add[bt] - 1;
                        if (ib >= cap[bt]) return -2;
                        double *B = vxp[bt] + 6 * ib;
                        B[0] = P[0]; B[1] = P[1]; B[2] = P[2];
                        flag_add[n_re + iby] = 1;
                    }
                    if (ib < 0) continue; /* neither the incident, its target nor a new particle */
                    double vbx = 0, vby = 0, vbz = 0;
                    if (opt_scat == 1) {
                        double cos_th = cos(th), sin_th = sin(th);
                        th = th + th_add;
                        double ex = cos_th, ey = sin_th * sin_ph, ez = sin_th * cos_ph;
                        double ex1 = 0, ey1 = 0, ez1 = 0;
                        o_scatter(&ex1, &ey1, &ez1, ex, ey, ez, cos_th_s, phi_s);
                        double mb = fabs(c->mass[bt]);
                        double vp = sqrt(2.0 * (Ee / sum_mass) / (mb * mb));
                        vbx = vx_cm[ttype] + vp * ex;
                        vby = vy_cm[ttype] + vp * ey;
                        vbz = vz_cm[ttype] + vp * ez;
                    } else {
                        if (bt == 0) {
                            double rr0 = o_ran2(iseed), rr1 = o_ran2(iseed);
                            double cos_th = 1.0 - 2.0 * rr0;
                            double sin_th = 2.0 * sqrt(rr0 * (1.0 - rr0));
                            double phi = 2.0 * pi * rr1;
                            double ex1 = cos_th, ey1 = sin_th * sin(phi), ez1 = sin_th * cos(phi);
                            double vp = sqrt(2.0 * (Ee * Ek_b[iby] / fabs(c->mass[bt])));
                            vbx = vp * ex1; vby = vp * ey1; vbz = vp * ez1;
                        } else {
                            double rr[2];
                            rr[0] = o_ran2(iseed); rr[1] = o_ran2(iseed);
                            o_load_gauss(&vbx, &vby, c->vt0[bt], rr);
                            if (vzb_sav == 0.0) {
                                rr[0] = o_ran2(iseed); rr[1] = o_ran2(iseed);
                                o_load_gauss(&vbz, &vzb_sav, c->vt0[bt], rr);
                            } else {
                                vbz = vzb_sav;
                                vzb_sav = 0.0;
                            }
                        }
                    }
                    double *B = vxp[bt] + 6 * ib;
                    B[3] = vbx; B[4] = vby; B[5] = vbz;
                }
                for (int ire = 0; ire < n_re; ire++) { /* :908-935 */
                    int ct = ci[2 + ire];
                    if (c->mass[ct] <= 0) { flag_add[ire] = 0; continue; }
                    if (flag_add[ire] == -1 && flag_dead && flag_dead[ct]) {
                        if (ct == p) flag_dead[p][ip] = 1;
                        else if (ct == ttype && sav_it[ttype] >= 0) flag_dead[ct][sav_it[ttype]] = 1;
                    }
                }
            } else { /* :942-1000 charge exchange */
                for (int iby = 0; iby < n_by; iby++) {
                    int bt = ci[2 + n_re + iby];
                    if (c->mass[bt] <= 0) continue;
                    int ind_ce;
                    double *B;
                    if (bt == p) { ind_ce = 1; B = P; }
                    else if (sav_it[ttype] >= 0) { ind_ce = 2; B = vxp[bt] + 6 * sav_it[ttype]; }
                    else continue;
                    ind_ce = ind_ce + 1;
                    if (ind_ce == 3) ind_ce = 1;
                    B[3] = vx[ind_ce - 1]; B[4] = vy[ind_ce - 1]; B[5] = vz[ind_ce - 1];
                }
            }
        }
    }
    for (int p = 0; p < c->ntype; p++) { /* :184 */
        np_tot[p] += np_add[p];
        if (t) t->n_add[p] += np_add[p];
    }
    return 0;
}

int o_collisions(o_cfg *c, const o_xs *xs, double **vxp, int64_t *np_tot, const int64_t *cap,
                 int8_t **flag_dead, int32_t *iseed, o_mcc_tally *t) {
    return o_collisions_dsmc(c, xs, vxp, np_tot, cap, flag_dead, iseed, t, NULL);
}

/* ------------------------------------------------------------------------------------ */
/* OpenMP CPU-baseline form of one species' mover + deposit (main.f90:1024-1089): the
 * array is cut into per-thread slabs, each thread moves and compacts its slab and deposits
 * into a private grid; slabs are then closed up and the grids reduced in thread order. */
void o_push_deposit_omp(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                        const int32_t *bcnd, const double *kq, double *vxp, int64_t *np_tot,
                        int8_t *flag_dead, double *npg, int nthreads) {
    int T = nthreads < 1 ? 1 : nthreads;
    const int64_t n = *np_tot;
    const int64_t nn = (int64_t)(c->nx + 3) * (c->ny + 3);
    int64_t *start = (int64_t *)calloc((size_t)T + 1, sizeof(int64_t));
    int64_t *cnt = (int64_t *)calloc((size_t)T, sizeof(int64_t));
    double *priv = (double *)calloc((size_t)T * nn, sizeof(double));
    for (int t = 0; t <= T; t++) start[t] = n * t / T;
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; t++) {
        int64_t m = start[t + 1] - start[t];
        o_part_mover(c, ptype, Ei, Bi, bcnd, vxp + 6 * start[t], &m,
                     flag_dead ? flag_dead + start[t] : NULL, NULL);
        cnt[t] = m;
        o_charge_deposition(c, ptype, vxp + 6 * start[t], m, kq, priv + (int64_t)t * nn);
    }
    int64_t w = cnt[0];
    for (int t = 1; t < T; t++) {
        memmove(vxp + 6 * w, vxp + 6 * start[t], sizeof(double) * 6 * (size_t)cnt[t]);
        w += cnt[t];
    }
    *np_tot = w;
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t k = 0; k < nn; k++) {
        double s = npg[k];
        for (int t = 0; t < T; t++) s += priv[(int64_t)t * nn + k];
        npg[k] = s;
    }
    free(start); free(cnt); free(priv);
}
