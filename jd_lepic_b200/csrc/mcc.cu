// mcc.cu -- null-collision Monte Carlo collisions (collisions.f90:1-207, collision_OMP
// :209-1040) for neutral targets, every ns_coll steps.
//
// The reference draws Nc = N*Pmax particles with replacement from one Park-Miller stream.
// Here every slot is a candidate with probability Pmax = nu_max*ns_coll*dt, independently (a
// Bernoulli trial per slot, drawn as geometric gaps between candidates from Philox4x32-10
// keyed by seed, step, species and slot chunk), so the expected number of candidates and the
// per-particle collision probability sum(nu)*ns_coll*dt are the same, and every result is
// reproducible run to run.  A candidate then follows collision_OMP exactly:
// Maxwellian target velocity (load_gauss), centre-of-mass kinematics, cross section by
// interval search on the union energy grid with linear interpolation, nu/nu_max per reaction,
// one uniform against the cumulative sum, and the reaction outcome (energy- and momentum-
// conserving equal-angle scattering, the fixed-split ionization option, charge exchange).
// The cumulative sum runs over the reactions in ascending nu, as the reference's indexx
// orders them (that order matters once sum(nu/nu_max) exceeds 1).
//
// Products go to a per-species list (unordered atomics) with a unique key parent*8+index;
// a second kernel sorts each list by key and appends it after the occupied slots, so the
// particle order after a collision step is deterministic.
//
// Roofline: the selection pass draws one uniform per candidate (twice: count, then write)
// and reads nothing (it writes the candidate list); only candidates (N*Pmax, about 0.3 % of
// particles) read and write their 20 B record, one candidate per thread.
#include <algorithm>
#include "rho.cuh"

#define MCC_THREADS 256
#define MCC_MAX_REACTIONS 16  // reactions per incident species (checked at context creation)

struct MccP {
    int sp, ntype;
    unsigned int *ss_map;   // ss2D counts (null: not accumulated), see lepic_ctx::ss_map
    long long ss_nn;
    int ss_W;
    int diag;               // collisions' flag_diag: frequencies into ss_diag, no collision
    double *ss_diag;        // ss2D with plt_src = 1, [(2 sp + k) nn + node]
    double nm_vc[LEPIC_MAXSP];   // Nm / Vc per species
    uint32_t *X, *Y;
    float *VX, *VY, *VZ;
    const float *Z;             // the incident species' z (3rd dimension), null without it
    Product *prod[LEPIC_MAXSP];
    int prod_cap[LEPIC_MAXSP];
    DevCounters *cnt;
    double Pmax, nu_max;
    int ncol_sp;
    int cols[MCC_MAX_REACTIONS];
    const double *sig_Er;
    int npt;
    const double *sig;
    const double *Eth;
    const int *col_info;
    double mass[LEPIC_MAXSP], charge[LEPIC_MAXSP], vt0[LEPIC_MAXSP], ndens[LEPIC_MAXSP];
    double qe, pi;
    int flag_ionrep;
    double fEk;
    uint32_t k0, k1, it;
    // tallies: P_loss(3) and cnt_col over the x-regions (collisions.f90:533-543, 896-899, 1025-1033)
    TallyDev *tal;
    double Ek_half[LEPIC_MAXSP];      // 0.5 Nm m
    int S, n_rg, iyl, iyr;
    int ixl[LEPIC_MAXRG], ixr[LEPIC_MAXRG];
    // DSMC with charged targets (collisions.f90:339-418, 524-528): the targets' cell lists of
    // the last sort, their velocities, the claims and the dens_red densities
    int dsmc, nx, ny, tw, th, ntx, W;
    long long nn;
    const int *toff[LEPIC_MAXSP];
    float *TVX[LEPIC_MAXSP], *TVY[LEPIC_MAXSP], *TVZ[LEPIC_MAXSP];
    int *claim[LEPIC_MAXSP];
    const double *np_red;
    const double *nu_max_d;   // the device's nu_max of this step (DSMC), else nu_max above
    double ns_coll_dt;
    // a sort's pending permutation per species (SpeciesBuf::pind), null where there is none:
    // slots and targets are positions of the sorted order, read and written through it
    const int *pind[LEPIC_MAXSP];
};

// the slot of the buffer that holds position j of species s
__device__ __forceinline__ long long mslot(const MccP &P, int s, long long j) {
    return ind_slot(P.pind[s], P.cnt->n_sorted[s], P.cnt->ind_old[s], j);
}

#define TAG_DSMC 0x44534D43u

// collisions.f90:339-403: a target of species tt for an incident in cell (cx, cy), uniform in
// the incident's cell, else in the first non-empty of its x+1, x-1, y+1, y-1 neighbours (inside
// the grid); -1 if none.  u: the draw (slot, step, TAG_DSMC ^ tt).
__device__ __forceinline__ long long pick_target(const MccP &P, int tt, int cx, int cy, uint32_t u) {
    const int ddx[5] = {0, 1, -1, 0, 0}, ddy[5] = {0, 0, 0, 1, -1};
    for (int k = 0; k < 5; k++) {
        const int x = cx + ddx[k], y = cy + ddy[k];
        if (x < 0 || x >= P.nx || y < 0 || y >= P.ny) continue;
        const int key = sort_cell_key(x, y, P.nx, P.ny, P.tw, P.th, P.ntx);
        const long long a = P.toff[tt][key], b = P.toff[tt][key + 1];
        if (b > a) return a + (long long)(u01(u) * (double)(b - a));
    }
    return -1;
}

__device__ __forceinline__ uint32_t dsmc_draw(const MccP &P, long long slot, int tt) {
    return philox4x32_10(U4{(uint32_t)slot, P.it, TAG_DSMC ^ (uint32_t)tt, (uint32_t)P.sp}, P.k0, P.k1).x;
}

// the first x-region holding the cell (ix, iy) (collisions.f90:535-537), -1 if none
__device__ __forceinline__ int region_of(const MccP &P, int ix, int iy) {
    if (iy < P.iyl || iy > P.iyr) return -1;
    for (int r = 0; r < P.n_rg; r++)
        if (ix >= P.ixl[r] && ix <= P.ixr[r]) return r;
    return -1;
}

__device__ __forceinline__ double v2f(float a, float b, float c) {
    return (double)a * a + (double)b * b + (double)c * c;
}

struct Rng {
    U4 ctr;
    uint32_t k0, k1;
    U4 buf;
    int used;
    __device__ double next() {
        if (used == 4) {
            buf = philox4x32_10(ctr, k0, k1);
            ctr.w++;
            used = 0;
        }
        uint32_t v = used == 0 ? buf.x : used == 1 ? buf.y : used == 2 ? buf.z : buf.w;
        used++;
        return u01(v);
    }
};

// load_gauss.f90:16-39
__device__ __forceinline__ void load_gauss(double vt, double r1, double r2, double pi, double *a, double *b) {
    double vp = vt * sqrt(-log(1.0 - r1));
    double th = 2.0 * pi * r2;
    double s, c;
    sincos(th, &s, &c);
    *a = vp * c;
    *b = vp * s;
}

// collisions.f90:485-519: cross section of reaction c at relative energy E (eV); returns
// -1 when E is outside (E_1, E_npt]
__device__ __forceinline__ double sigma_at(const MccP &P, int c, double E) {
    const double *Er = P.sig_Er;
    const int npt = P.npt;
    if (!(E > Er[0]) || E > Er[npt - 1]) return -1.0;
    int lo = 0, hi = npt - 1; // Er[lo] < E <= Er[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (E <= Er[mid]) hi = mid; else lo = mid;
    }
    const double *sg = P.sig + (long long)c * npt;
    double EL = Er[lo], ER = Er[hi], sL = sg[lo], sR = sg[hi];
    return sL + (E - EL) * (sR - sL) / (ER - EL);
}

// plt_src = 1 (collisions.f90:546-600): reaction c of the incident in `slot` (of the buffer) at frequency k2
// (1/s) adds k2 Nm/Vc, with the incident's CIC weights, to the source of every charged byproduct
// other than the incident's and the target's species and to the sink of a charged reactant
// that is not among the byproducts; elastic and excitation reactions (types 1, 3) add nothing.
__device__ void diag_source_sink(const MccP &P, long long slot, int c, int sp, int tt, double k2) {
    const int *ci = P.col_info + c * 10;
    const int n_re = ci[0], n_by = ci[1], rt = ci[2 + n_re + n_by];
    if (rt == 1 || rt == 3) return;
    const uint32_t X = P.X[slot], Y = P.Y[slot], mask = (1u << P.S) - 1u;
    const double inv = 1.0 / (double)(1u << P.S);
    const double px = 1.0 - (double)(X & mask) * inv, py = 1.0 - (double)(Y & mask) * inv;  // (ix h - x)/h
    const double w[4] = {px * py, (1.0 - px) * py, (1.0 - px) * (1.0 - py), px * (1.0 - py)};
    const long long n00 = ((X >> P.S) + 1) + (long long)((Y >> P.S) + 1) * P.ss_W;
    const long long nd[4] = {n00, n00 + 1, n00 + P.ss_W + 1, n00 + P.ss_W};
    bool inc_kept = false, tgt_kept = false;
    for (int ib = 0; ib < n_by; ib++) {
        const int bt = ci[2 + n_re + ib];
        if (P.charge[bt] != 0.0 && bt != sp && bt != tt) {
            double *m = P.ss_diag + (size_t)(2 * bt) * P.ss_nn;
            const double k1 = P.nm_vc[bt] * k2;
            for (int q = 0; q < 4; q++) atomicAdd(m + nd[q], w[q] * k1);
        }
        if (bt == sp) inc_kept = true;
        if (bt == tt) tgt_kept = true;
    }
    for (int i_re = 0; i_re < 2; i_re++) {
        const int bt = i_re == 0 ? sp : tt;
        if ((i_re == 0 ? inc_kept : tgt_kept) || P.charge[bt] == 0.0) continue;
        double *m = P.ss_diag + (size_t)(2 * bt + 1) * P.ss_nn;
        const double k1 = P.nm_vc[bt] * k2;
        for (int q = 0; q < 4; q++) atomicAdd(m + nd[q], w[q] * k1);
    }
}

__device__ void collide_one(const MccP &P, long long slot, double nu_max, unsigned int *n_cand_local) {
    const long long st = mslot(P, P.sp, slot);   // where the incident's record is
    float fvx = P.VX[st];
    if (isnan(fvx)) return;
    (*n_cand_local)++;
    const int sp = P.sp;
    Rng R;
    R.ctr = U4{(uint32_t)slot, P.it, (uint32_t)sp | 0x4D430000u, (uint32_t)P.diag};  // the diagnostic pass: own stream
    R.k0 = P.k0; R.k1 = P.k1; R.used = 4;
    const double vx1 = fvx, vy1 = P.VY[st], vz1 = P.VZ[st];
    const double mp = fabs(P.mass[sp]);
    int rg = -1;
    if (P.n_rg > 0) rg = region_of(P, (int)(P.X[st] >> P.S) + 1, (int)(P.Y[st] >> P.S) + 1);
    // per target species: drawn velocity and CM quantities (collision_OMP :336-482)
    double tvx[LEPIC_MAXSP], tvy[LEPIC_MAXSP], tvz[LEPIC_MAXSP], mu[LEPIC_MAXSP], vr[LEPIC_MAXSP];
    double vcx[LEPIC_MAXSP], vcy[LEPIC_MAXSP], vcz[LEPIC_MAXSP];
    long long tslot[LEPIC_MAXSP];   // the DSMC target's record of a charged target species (-1: none)
    double np_t[LEPIC_MAXSP];
#pragma unroll
    for (int t = 0; t < LEPIC_MAXSP; t++) tslot[t] = -1;
    unsigned drawn = 0;
    int cx = 0, cy = 0;
    if (P.dsmc) { cx = (int)(P.X[st] >> P.S); cy = (int)(P.Y[st] >> P.S); }
    double nu[MCC_MAX_REACTIONS];
    double sum_nu = 0.0;
    for (int q = 0; q < P.ncol_sp; q++) {
        const int c = P.cols[q];
        const int *ci = P.col_info + c * 10;
        const int n_re = ci[0];
        const int tt = ci[2 + n_re - 1];
        nu[q] = 0.0;
        const bool charged = P.charge[tt] != 0.0;
        if (charged && (!P.dsmc || tt == sp)) continue; // like-particle DSMC is not handled
        if (!(drawn & (1u << tt))) {
            double a, b, z, dummy;
            if (!charged) {
                load_gauss(P.vt0[tt], R.next(), R.next(), P.pi, &a, &b);
                load_gauss(P.vt0[tt], R.next(), R.next(), P.pi, &z, &dummy);
                tslot[tt] = -1;
                np_t[tt] = P.ndens[tt];
            } else {
                // the target particle (:339-403) if this candidate holds its claim, and the
                // target density at the incident's cell (:524-528)
                long long t = pick_target(P, tt, cx, cy, dsmc_draw(P, slot, tt));   // a position
                const long long ts = t >= 0 ? mslot(P, tt, t) : -1;                  // its record
                if (t >= 0 && ((!P.diag && P.claim[tt][t] != (int)slot) || isnan(P.TVX[tt][ts]))) t = -1;
                tslot[tt] = t >= 0 ? ts : -1;
                a = b = z = 0.0;
                if (t >= 0) { a = P.TVX[tt][ts]; b = P.TVY[tt][ts]; z = P.TVZ[tt][ts]; }
                const long long m = (cx + 1) + (long long)(cy + 1) * P.W + tt * P.nn;
                np_t[tt] = 0.25 * (P.np_red[m] + P.np_red[m + 1] + P.np_red[m + P.W] + P.np_red[m + P.W + 1]);
            }
            tvx[tt] = a; tvy[tt] = b; tvz[tt] = z;
            const double mt = fabs(P.mass[tt]);
            mu[tt] = mp * mt / (mp + mt);
            vr[tt] = sqrt((vx1 - a) * (vx1 - a) + (vy1 - b) * (vy1 - b) + (vz1 - z) * (vz1 - z));
            const double sm = mp + mt;
            vcx[tt] = (mp * vx1 + mt * a) / sm;
            vcy[tt] = (mp * vy1 + mt * b) / sm;
            vcz[tt] = (mp * vz1 + mt * z) / sm;
            drawn |= 1u << tt;
        }
        if (charged && tslot[tt] < 0) continue;  // no target for this species (:389-398)
        const double Ekr = (0.5 * mu[tt] * (vr[tt] * vr[tt])) / P.qe;
        if (Ekr > P.sig_Er[P.npt - 1]) atomicAdd(&P.cnt->n_overflow, 1ull);
        const double s = sigma_at(P, c, Ekr);
        if (s < 0.0) continue;
        nu[q] = np_t[tt] * s * vr[tt] / nu_max; // :522-532
        sum_nu = sum_nu + nu[q];
        if (rg >= 0) { // :535-543
            atomicAdd(&P.tal->cnt_col[0][c][rg], nu[q] * nu_max);
            atomicAdd(&P.tal->cnt_col[1][c][rg], 1.0);
        }
        if (P.diag) diag_source_sink(P, st, c, sp, tt, nu[q] * nu_max);
    }
    if (P.diag) return;   // collisions.f90:649: flag_diag makes every event a null collision
    // :619 indexx: reactions ordered by ascending nu (straight insertion, stable); the order
    // decides the outcome when sum(nu) > 1, i.e. when nu_max was capped (main.f90:494-495)
    int order[MCC_MAX_REACTIONS];
    for (int q = 0; q < P.ncol_sp; q++) {
        int k = q;
        while (k > 0 && nu[order[k - 1]] > nu[q]) { order[k] = order[k - 1]; k--; }
        order[k] = q;
    }
    const double r = R.next(); // :624-647
    if (!(r <= sum_nu)) return;
    int qsel = -1;
    double cum = 0.0;
    for (int k = 0; k < P.ncol_sp; k++) {
        cum = cum + nu[order[k]];
        if (r <= cum) { qsel = order[k]; break; }
    }
    if (qsel < 0) return;
    const int c = P.cols[qsel];
    const int *ci = P.col_info + c * 10;
    const int n_re = ci[0], n_by = ci[1], rt = ci[2 + n_re + n_by];
    const int tt = ci[2 + n_re - 1];
    atomicAdd(&P.cnt->n_coll[c], 1ull);
    if (rg >= 0) atomicAdd(&P.tal->cnt_col[2][c][rg], P.tal->inv_np_rg[sp][rg]); // :1026-1033
    const uint32_t X = P.X[st], Y = P.Y[st];
    const double v2in = v2f(fvx, (float)vy1, (float)vz1);
    if (rt == 4) { // charge exchange :942-1000: the incident ion takes the neutral's velocity
        for (int ib = 0; ib < n_by; ib++) {
            int bt = ci[2 + n_re + ib];
            if (P.mass[bt] <= 0.0) continue;
            if (bt == sp) {
                const float a = (float)tvx[tt], b = (float)tvy[tt], cz = (float)tvz[tt];
                P.VX[st] = a; P.VY[st] = b; P.VZ[st] = cz;
                atomicAdd(&P.tal->P3[sp], P.Ek_half[sp] * (v2f(a, b, cz) - v2in)); // :980-983
            } else if (bt == tt && P.charge[tt] != 0.0 && tslot[tt] >= 0) {
                // a charged target takes the incident's velocity (:955-978)
                const long long t = tslot[tt];
                const double v2t = v2f(P.TVX[tt][t], P.TVY[tt][t], P.TVZ[tt][t]);
                P.TVX[tt][t] = fvx; P.TVY[tt][t] = (float)vy1; P.TVZ[tt][t] = (float)vz1;
                atomicAdd(&P.tal->P3[tt], P.Ek_half[tt] * (v2in - v2t));
            }
        }
        return;
    }
    const double Eth = P.Eth[c];
    double Ee = 0.5 * mu[tt] * (vr[tt] * vr[tt]) - Eth * P.qe; // :683
    int opt_scat = 1;
    double Ek_b[16];
    double sum_mass = 0.0, th = 0.0, th_add = 0.0, sin_ph = 0.0, cos_ph = 0.0;
    for (int q = 0; q < 16; q++) Ek_b[q] = 0.0;
    bool ion_rep = false;
    if (rt == 2 && P.flag_ionrep >= 1 && n_by == 3) { // :689-727
        int cnt_ele = 0, flag_ion = 0;
        for (int ib = 0; ib < n_by; ib++) {
            int bt = ci[2 + n_re + ib];
            if (bt == 0) {
                cnt_ele++;
                if (cnt_ele == 1) Ek_b[ib] = P.fEk;
                if (cnt_ele == 2) Ek_b[ib] = 1.0 - P.fEk;
            }
            if (bt != 0 && P.charge[bt] != 0.0) flag_ion = 1;
        }
        ion_rep = true;
        if (cnt_ele == 2 && flag_ion == 1) {
            opt_scat = 2;
            Ee = 0.5 * P.mass[0] * (vx1 * vx1 + vy1 * vy1 + vz1 * vz1) - Eth * P.qe;
            if (Ee < 0.0) Ee = 0.0;
        }
    }
    if (!ion_rep) { // :728-750 (the SCATTER rotation's output is not used by the reference)
        for (int ib = 0; ib < n_by; ib++) sum_mass = sum_mass + 1.0 / fabs(P.mass[ci[2 + n_re + ib]]);
        double r0 = R.next(), r1 = R.next();
        th_add = 2.0 * P.pi / (double)n_by;
        th = acos(1.0 - 2.0 * r0);
        sincos(2.0 * P.pi * r1, &sin_ph, &cos_ph);
    }
    if (Ee < 0.0) return;
    bool incident_kept = false;
    for (int ib = 0; ib < n_by; ib++) { // :767-902
        const int bt = ci[2 + n_re + ib];
        if (P.mass[bt] <= 0.0) continue;
        bool to_incident = false, to_target = false;
        if (ib == 0 && bt == sp) to_incident = true;
        if (rt == 1 || rt == 3) {
            if (bt == sp) to_incident = true;
            else if (bt == tt && P.charge[tt] != 0.0 && tslot[tt] >= 0) to_target = true;  // :794-797
            else continue;
        }
        double vbx = 0.0, vby = 0.0, vbz = 0.0;
        if (opt_scat == 1) {
            double s, cth;
            sincos(th, &s, &cth);
            th = th + th_add;
            const double ex = cth, ey = s * sin_ph, ez = s * cos_ph;
            const double mb = fabs(P.mass[bt]);
            const double vp = sqrt(2.0 * (Ee / sum_mass) / (mb * mb));
            vbx = vcx[tt] + vp * ex;
            vby = vcy[tt] + vp * ey;
            vbz = vcz[tt] + vp * ez;
        } else if (bt == 0) {
            double r0 = R.next(), r1 = R.next();
            double cth = 1.0 - 2.0 * r0, sth = 2.0 * sqrt(r0 * (1.0 - r0));
            double s, cph;
            sincos(2.0 * P.pi * r1, &s, &cph);
            const double vp = sqrt(2.0 * (Ee * Ek_b[ib] / fabs(P.mass[bt])));
            vbx = vp * cth; vby = vp * sth * s; vbz = vp * sth * cph;
        } else {
            double z, dummy;
            load_gauss(P.vt0[bt], R.next(), R.next(), P.pi, &vbx, &vby);
            load_gauss(P.vt0[bt], R.next(), R.next(), P.pi, &z, &dummy);
            vbz = z;
        }
        if (to_target) {
            const long long t = tslot[tt];
            const double v2t = v2f(P.TVX[tt][t], P.TVY[tt][t], P.TVZ[tt][t]);
            atomicAdd(&P.tal->P3[tt], P.Ek_half[tt] * (v2f((float)vbx, (float)vby, (float)vbz) - v2t));
            P.TVX[tt][t] = (float)vbx; P.TVY[tt][t] = (float)vby; P.TVZ[tt][t] = (float)vbz;
            continue;
        }
        // P_loss(3) += 0.5 Nm m (v_new^2 - v_old^2), v_old = 0 for a created particle (:821-828, :896-899)
        atomicAdd(&P.tal->P3[bt], P.Ek_half[bt] * (v2f((float)vbx, (float)vby, (float)vbz) - (to_incident ? v2in : 0.0)));
        if (to_incident) {
            incident_kept = true;
            P.VX[st] = (float)vbx; P.VY[st] = (float)vby; P.VZ[st] = (float)vbz;
        } else {
            if (P.ss_map)   // collisions.f90:809: a created particle at the incident's (ix, iy)
                atomicAdd(P.ss_map + (size_t)(2 * bt) * P.ss_nn + ((X >> P.S) + 1) + (long long)((Y >> P.S) + 1) * P.ss_W, 1u);
            unsigned int k = atomicAdd(&P.cnt->prod_count[bt], 1u);
            if ((int)k < P.prod_cap[bt]) {
                Product pr;
                pr.key = (unsigned long long)slot * 8ull + (unsigned long long)ib;
                pr.X = X; pr.Y = Y;
                pr.vx = (float)vbx; pr.vy = (float)vby; pr.vz = (float)vbz;
                pr.z = P.Z ? P.Z[st] : 0.0f;   // collisions.f90:813: the incident's z
                P.prod[bt][k] = pr;
            } else {
                set_err(P.cnt, LERR_CAPACITY, 200);
            }
        }
    }
    // reactants :908-935: a positive-mass incident that is not byproduct 1 is removed
    for (int ire = 0; ire < n_re; ire++) {
        const int ct = ci[2 + ire];
        if (P.mass[ct] <= 0.0) continue;
        if (ct == sp && !incident_kept && ire == 0) {
            atomicAdd(&P.tal->P3[sp], -P.Ek_half[sp] * v2in);  // removal in the mover (part_expmover.f90:91-95)
            P.VX[st] = __int_as_float(HOLE_NAN);
            if (P.ss_map)   // collisions.f90:931: the removed particle, at the incident's (ix, iy)
                atomicAdd(P.ss_map + (size_t)(2 * sp + 1) * P.ss_nn + ((P.X[st] >> P.S) + 1) +
                              (long long)((P.Y[st] >> P.S) + 1) * P.ss_W, 1u);
            atomicAdd(&P.cnt->n_dead[sp], 1ull);
            atomicAdd((unsigned long long *)&P.cnt->n_alive[sp], (unsigned long long)-1ll);
        }
        if (ire == 1 && ct == tt && P.charge[tt] != 0.0 && tslot[tt] >= 0 && rt != 1 && rt != 3) {
            const long long t = tslot[tt];  // a charged target that is not a byproduct dies (:921-930)
            atomicAdd(&P.tal->P3[tt], -P.Ek_half[tt] * v2f(P.TVX[tt][t], P.TVY[tt][t], P.TVZ[tt][t]));
            P.TVX[tt][t] = __int_as_float(HOLE_NAN);
            if (P.ss_map)
                atomicAdd(P.ss_map + (size_t)(2 * tt + 1) * P.ss_nn + ((P.X[st] >> P.S) + 1) +
                              (long long)((P.Y[st] >> P.S) + 1) * P.ss_W, 1u);
            atomicAdd(&P.cnt->n_dead[tt], 1ull);
            atomicAdd((unsigned long long *)&P.cnt->n_alive[tt], (unsigned long long)-1ll);
        }
    }
}

// the collision probability of this step: the host's (neutral targets) or the device's
// nu_max (charged targets: it depends on the densities, collisions.f90:98-117)
__device__ __forceinline__ double step_nu_max(const MccP &P) { return P.dsmc ? P.nu_max_d[P.sp] : P.nu_max; }

// Selection: every slot is a candidate with probability Pmax, independently of the others (a
// Bernoulli trial per slot), drawn as the geometric gaps between candidates: a thread walks a
// chunk of SEL_CHUNK slots, each gap floor(log u / log(1 - Pmax)) slots long, so that the
// random numbers number the candidates (Pmax is ~0.3 %) instead of the slots.  The uniforms
// come from Philox4x32-10 keyed by (chunk, draw, step, species); P(gap >= k) = (1 - Pmax)^k
// to the 2^-32 grain of u.  The walk runs twice, counting and then writing, so that each warp
// takes its place in the list with one atomic.  The list's order does not matter: every draw
// of a collision is keyed by its slot, a DSMC target goes to the smallest claiming slot, and
// products are sorted before they are appended.
#define SEL_CHUNK 4096

__device__ __forceinline__ int select_walk(const MccP &P, long long ch, long long lo, long long hi, double lq,
                                           bool all, int *out) {
    long long pos = lo - 1;
    int cnt = 0;
    U4 r{0u, 0u, 0u, 0u};
    for (uint32_t k = 0;; k++) {
        if ((k & 3u) == 0u)
            r = philox4x32_10(U4{(uint32_t)ch, k >> 2, P.it, (uint32_t)P.sp | 0x53470000u}, P.k0, P.k1);
        const uint32_t v = (k & 3u) == 0u ? r.x : (k & 3u) == 1u ? r.y : (k & 3u) == 2u ? r.z : r.w;
        const double g = all ? 0.0 : floor(log(u01(v)) / lq);
        if (g >= (double)(hi - 1 - pos)) break;   // the next candidate lies beyond the chunk
        pos += (long long)g + 1;
        if (out) out[cnt] = (int)pos;
        cnt++;
    }
    return cnt;
}

__global__ void __launch_bounds__(MCC_THREADS) k_mcc_select(MccP P, int *cand) {
    const long long n = P.cnt->n_slots[P.sp];
    const double Pmax = P.dsmc ? step_nu_max(P) * P.ns_coll_dt : P.Pmax;
    const bool any = Pmax > 0.0, all = Pmax >= 1.0;
    const double lq = any && !all ? log1p(-Pmax) : -1.0;
    const unsigned lane = threadIdx.x & 31;
    const long long nchunk = (n + SEL_CHUNK - 1) / SEL_CHUNK;
    for (long long c0 = blockIdx.x * (long long)blockDim.x; c0 < nchunk; c0 += (long long)gridDim.x * blockDim.x) {
        const long long ch = c0 + threadIdx.x;   // every lane takes the same trip count
        const long long lo = ch * SEL_CHUNK, hi = min(lo + SEL_CHUNK, n);
        const bool mine = ch < nchunk && any;
        const int c = mine ? select_walk(P, ch, lo, hi, lq, all, nullptr) : 0;
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if ((int)lane >= o) incl += t;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        unsigned wbase = 0;
        if (lane == 31 && total) wbase = atomicAdd(&P.cnt->n_cand_list, (unsigned)total);
        wbase = __shfl_sync(0xffffffffu, wbase, 31);
        if (mine && c) select_walk(P, ch, lo, hi, lq, all, cand + (long long)wbase + incl - c);
    }
}

// The collisions of the listed candidates, one per thread: a candidate runs the whole of
// collision_OMP (target draw, interval search, scattering), which on a warp of slots where
// one in ~300 is a candidate would run with one lane active.
__global__ void __launch_bounds__(MCC_THREADS) k_mcc(MccP P, const int *cand) {
    const long long m = P.cnt->n_cand_list;
    const double nu_max = step_nu_max(P);
    unsigned int ncand = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
        collide_one(P, cand[i], nu_max, &ncand);
    for (int o = 16; o > 0; o >>= 1) ncand += __shfl_xor_sync(0xffffffffu, ncand, o);
    if ((threadIdx.x & 31) == 0 && ncand) atomicAdd(&P.cnt->n_cand[P.sp], (unsigned long long)ncand);
}

// collisions(..., flag_diag = 1) of collisions.f90:268-299: every particle of the species
// through the collision frequencies, no collision performed
__global__ void __launch_bounds__(MCC_THREADS) k_mcc_diag(MccP P) {
    const long long n = P.cnt->n_slots[P.sp];
    const double nu_max = step_nu_max(P);
    unsigned int unused = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        collide_one(P, i, nu_max, &unused);
}

// DSMC claims: every candidate of this step picks its charged targets as collide_one will and
// claims them with the smallest incident slot, so that a target takes part in one collision
// of the step (the winner is independent of the order the threads run in).
__global__ void __launch_bounds__(MCC_THREADS) k_mcc_claim(MccP P, const int *cand) {
    const long long m = P.cnt->n_cand_list;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        const long long slot = cand[i];
        const long long st = mslot(P, P.sp, slot);
        if (isnan(P.VX[st])) continue;
        const int cx = (int)(P.X[st] >> P.S), cy = (int)(P.Y[st] >> P.S);
        unsigned done = 0;
        for (int k = 0; k < P.ncol_sp; k++) {
            const int *ci = P.col_info + P.cols[k] * 10;
            const int tt = ci[2 + ci[0] - 1];
            if (P.charge[tt] == 0.0 || tt == P.sp || (done & (1u << tt))) continue;
            done |= 1u << tt;
            const long long t = pick_target(P, tt, cx, cy, dsmc_draw(P, slot, tt));
            if (t >= 0) atomicMin(P.claim[tt] + t, (int)slot);
        }
    }
}

// nu_max of every species from the densities of this step (collisions.f90:98-123)
struct NuMaxP {
    int ntype, p_ncol[LEPIC_MAXSP];
    int cols[LEPIC_MAXSP][MCC_MAX_REACTIONS], tt[LEPIC_MAXSP][MCC_MAX_REACTIONS];
    double np_mx_neutral[LEPIC_MAXSP], charge[LEPIC_MAXSP], nu_uplim[LEPIC_MAXSP], ns_coll_dt;
    const double *sigv_mx, *np_mx_charged;
    double *nu_max;
    DevCounters *cnt;
};
__global__ void k_nu_max(NuMaxP P) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int s = 0; s < P.ntype; s++) {
        double nu = 0.0;
        for (int q = 0; q < P.p_ncol[s]; q++) {
            const int t = P.tt[s][q];
            const double n = P.charge[t] != 0.0 ? P.np_mx_charged[t] : P.np_mx_neutral[t];
            nu = nu + n * P.sigv_mx[s * LEPIC_MAXCOL + P.cols[s][q]];
        }
        nu = fmin(nu, P.nu_uplim[s]);
        P.nu_max[s] = nu;
        if (nu * P.ns_coll_dt > 1.0) set_err(P.cnt, LERR_RANGE, 210);  // :119-123
    }
}

// Ordered append of one species' products after its occupied slots (single CTA).
__global__ void k_mcc_commit(int sp, Product *prod, int prod_cap, unsigned long long *sortbuf,
                             uint32_t *X, uint32_t *Y, float *VX, float *VY, float *VZ, float *Z, long long cap,
                             DevCounters *cnt, int mcc, int ind) {
    __shared__ unsigned long long sm[4096];
    int n = (int)min(cnt->prod_count[sp], (unsigned int)prod_cap);
    if (n == 0) return;
    unsigned long long *a = n <= 4096 ? sm : sortbuf;
    for (int q = threadIdx.x; q < n; q += blockDim.x) a[q] = (prod[q].key << 24) | (unsigned long long)q;
    __syncthreads();
    bitonic_sort(a, n, threadIdx.x, blockDim.x, BlockSync());
    // positions n_slots.. of the sorted order; with a pending permutation their records go after
    // the slots the buffer held before the sort
    const long long pos = cnt->n_slots[sp];
    const long long base = ind ? cnt->ind_old[sp] + (pos - cnt->n_sorted[sp]) : pos;
    int m = n;
    if (base + m > cap) {
        m = (int)max(cap - base, 0ll);
        if (threadIdx.x == 0) set_err(cnt, LERR_CAPACITY, 201);
    }
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
        const Product &p = prod[(int)(a[q] & 0xFFFFFFull)];
        long long s = base + q;
        X[s] = p.X; Y[s] = p.Y; VX[s] = p.vx; VY[s] = p.vy; VZ[s] = p.vz;
        if (Z) Z[s] = p.z;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        cnt->n_slots[sp] = pos + m;
        cnt->n_alive[sp] += m;
        if (mcc) cnt->n_add[sp] += (unsigned long long)m;
        cnt->prod_count[sp] = 0;
    }
}

// np_tot_rg (collisions.f90:143-154): the particles of a species in each x-region from the
// density, k * sum of np over the region's nodes, k = dx dy zmax / Nm; one CTA per (species,
// region), a fixed-order sum.  Stores 1 / np_tot_rg (0 for an empty region).
__global__ void k_region_np(RhoParams R, int n_rg, int iyl, int iyr, const int *ixl, const int *ixr,
                            const double *kfac, TallyDev *tal) {
    __shared__ double red[256];
    const int s = blockIdx.x / LEPIC_MAXRG, r = blockIdx.x % LEPIC_MAXRG;
    if (r >= n_rg || s >= R.ntype) return;
    const int w = ixr[r] - ixl[r] + 1, h = iyr - iyl + 1;
    double acc = 0.0;
    for (long long t = threadIdx.x; t < (long long)w * h; t += blockDim.x)
        acc += np_val(R, s, ixl[r] + (int)(t % w), iyl + (int)(t / w));
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double np = kfac[s] * red[0];
        tal->inv_np_rg[s][r] = np > 0.0 ? 1.0 / np : 0.0;
    }
}

int mcc_collide(lepic_ctx *c, int it, bool diag) {
    if (!c->has_xs) return LEPIC_OK;
    if (c->n_rg > 0) {
        RhoParams R = rho_params(c);
        double kfac[LEPIC_MAXSP] = {0};
        for (int s = 0; s < c->cfg.ntype; s++) kfac[s] = c->cfg.dx * c->cfg.dy * c->cfg.zmax / c->cfg.Nm[s];
        LCUDA(cudaMemcpyAsync(c->rg_scratch, c->ixl_rg, sizeof(int) * LEPIC_MAXRG, cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaMemcpyAsync(c->rg_scratch + LEPIC_MAXRG, c->ixr_rg, sizeof(int) * LEPIC_MAXRG, cudaMemcpyHostToDevice,
                              c->stream));
        LCUDA(cudaMemcpyAsync(c->rg_kfac, kfac, sizeof(double) * LEPIC_MAXSP, cudaMemcpyHostToDevice, c->stream));
        k_region_np<<<LEPIC_MAXSP * LEPIC_MAXRG, 256, 0, c->stream>>>(R, c->n_rg, c->iyl_rg, c->iyr_rg, c->rg_scratch,
                                                                     c->rg_scratch + LEPIC_MAXRG, c->rg_kfac, c->tally);
        LCUDA(cudaGetLastError());
    }
    const lepic_config &g = c->cfg;
    if (!c->dsmc) {
        for (int s = 0; s < g.ntype; s++) {
            if (c->p_ncol[s] == 0 || g.mass[s] <= 0.0) continue;
            double Pmax = c->nu_max[s] * (double)g.ns_coll * g.dt;
            if (Pmax > 1.0) { c->last_err = "collision probability Pmax > 1"; return LEPIC_ERANGE; }
        }
    } else {
        // charged targets: dens_red (main.f90:970) for the densities and their maxima, then
        // nu_max on the device (collisions.f90:98-123)
        int r = field_dens_red(c);
        if (r != LEPIC_OK) return r;
        NuMaxP N;
        memset(&N, 0, sizeof(N));
        N.ntype = g.ntype;
        for (int s = 0; s < g.ntype; s++) {
            N.p_ncol[s] = g.mass[s] > 0.0 ? c->p_ncol[s] : 0;
            for (int q = 0; q < c->p_ncol[s]; q++) {
                const int ic = c->hsig_list[s * LEPIC_MAXCOL + q];
                N.cols[s][q] = ic;
                N.tt[s][q] = c->hcol_tt[ic];
            }
            N.nu_uplim[s] = g.nu_uplim[s];
        }
        for (int t = 0; t < g.nsp; t++) { N.np_mx_neutral[t] = g.np_mx[t]; N.charge[t] = g.charge[t]; }
        N.ns_coll_dt = (double)g.ns_coll * g.dt;
        N.sigv_mx = c->sigv_mx_d;
        N.np_mx_charged = c->np_mx;
        N.nu_max = c->nu_max_d;
        N.cnt = c->dcnt;
        k_nu_max<<<1, 32, 0, c->stream>>>(N);
        LCUDA(cudaGetLastError());
    }
    for (int s = 0; s < g.ntype; s++) {
        if (c->p_ncol[s] == 0 || g.mass[s] <= 0.0 || (!c->dsmc && c->nu_max[s] <= 0.0)) continue;
        SpeciesBuf &B = c->sp[s];
        MccP P;
        memset(&P, 0, sizeof(P));
        bool claims = false;   // a charged target species of this incident gets DSMC claims
        P.sp = s; P.ntype = g.ntype;
        P.ss_map = diag ? nullptr : ss_counts(c); P.ss_nn = c->nn; P.ss_W = g.nx + 3;
        P.diag = diag ? 1 : 0; P.ss_diag = c->ss_diag;
        for (int t = 0; t < g.ntype; t++) P.nm_vc[t] = g.Nm[t] / (g.dx * g.dy * g.zmax);
        P.X = B.X[B.cur]; P.Y = B.Y[B.cur]; P.VX = B.VX[B.cur]; P.VY = B.VY[B.cur]; P.VZ = B.VZ[B.cur];
        P.Z = B.Z[B.cur];
        for (int t = 0; t < g.ntype; t++) P.pind[t] = c->sp[t].ind ? c->sp[t].pind : nullptr;
        for (int t = 0; t < g.ntype; t++) { P.prod[t] = c->sp[t].prod; P.prod_cap[t] = c->sp[t].prod_cap; }
        P.cnt = c->dcnt;
        P.nu_max = c->nu_max[s];
        P.Pmax = c->nu_max[s] * (double)g.ns_coll * g.dt;
        P.ncol_sp = c->p_ncol[s];
        for (int q = 0; q < c->p_ncol[s]; q++) P.cols[q] = c->hsig_list[s * LEPIC_MAXCOL + q];
        P.sig_Er = c->sig_Er; P.npt = c->npt; P.sig = c->sig; P.Eth = c->Eth; P.col_info = c->col_info;
        for (int t = 0; t < g.nsp; t++) {
            P.mass[t] = g.mass[t]; P.charge[t] = g.charge[t]; P.vt0[t] = g.vt0[t]; P.ndens[t] = g.np_mx[t];
        }
        P.qe = g.qe;
        P.pi = 4.0 * atan(1.0);
        P.flag_ionrep = c->flag_ionrep;
        P.fEk = c->fEk;
        P.k0 = (uint32_t)g.seed;
        P.k1 = (uint32_t)(g.seed >> 32) ^ 0xA5A5F00Du;
        P.it = (uint32_t)it;
        P.tal = c->tally;
        for (int t = 0; t < g.ntype; t++) P.Ek_half[t] = 0.5 * g.Nm[t] * g.mass[t];
        P.S = c->S;
        P.n_rg = c->n_rg; P.iyl = c->iyl_rg; P.iyr = c->iyr_rg;
        for (int r = 0; r < LEPIC_MAXRG; r++) { P.ixl[r] = c->ixl_rg[r]; P.ixr[r] = c->ixr_rg[r]; }
        if (c->dsmc) {
            P.dsmc = 1;
            P.nx = g.nx; P.ny = g.ny; P.tw = c->tw; P.th = c->th; P.ntx = c->ntx; P.W = g.nx + 3; P.nn = c->nn;
            for (int t = 0; t < g.ntype; t++) {
                SpeciesBuf &T = c->sp[t];
                P.toff[t] = T.cell_off;
                P.TVX[t] = T.VX[T.cur]; P.TVY[t] = T.VY[T.cur]; P.TVZ[t] = T.VZ[T.cur];
                P.claim[t] = T.claim;
            }
            P.np_red = c->np_red;
            P.nu_max_d = c->nu_max_d;
            P.ns_coll_dt = (double)g.ns_coll * g.dt;
            for (int q = 0; q < c->p_ncol[s]; q++) {
                const int t = c->hcol_tt[c->hsig_list[s * LEPIC_MAXCOL + q]];
                if (t < g.ntype && g.charge[t] != 0.0 && t != s && c->sp[t].claim) {
                    LCUDA(cudaMemsetAsync(c->sp[t].claim, 0x7f, sizeof(int) * c->sp[t].cap, c->stream));
                    claims = true;
                }
            }
        }
        if (diag) {
            k_mcc_diag<<<c->num_sms * 8, MCC_THREADS, 0, c->stream>>>(P);
            LCUDA(cudaGetLastError());
            continue;
        }
        // candidates (the sort's key buffer holds the list: one int per slot at most)
        LCUDA(cudaMemsetAsync(&c->dcnt->n_cand_list, 0, sizeof(unsigned int), c->stream));
        k_mcc_select<<<c->num_sms * 8, MCC_THREADS, 0, c->stream>>>(P, c->keys);
        LCUDA(cudaGetLastError());
        if (c->dsmc && claims) {
            k_mcc_claim<<<c->num_sms * 8, MCC_THREADS, 0, c->stream>>>(P, c->keys);
            LCUDA(cudaGetLastError());
        }
        k_mcc<<<c->num_sms * 8, MCC_THREADS, 0, c->stream>>>(P, c->keys);
        LCUDA(cudaGetLastError());
    }
    if (diag) return LEPIC_OK;
    for (int t = 0; t < g.ntype; t++) {
        int r = commit_products(c, t, true);
        if (r != LEPIC_OK) return r;
    }
    return LEPIC_OK;
}

int commit_products(lepic_ctx *c, int sp, bool mcc) {
    SpeciesBuf &B = c->sp[sp];
    k_mcc_commit<<<1, 1024, 0, c->stream>>>(sp, B.prod, B.prod_cap, c->prod_sort, B.X[B.cur], B.Y[B.cur],
                                            B.VX[B.cur], B.VY[B.cur], B.VZ[B.cur], B.Z[B.cur], B.cap, c->dcnt,
                                            mcc ? 1 : 0, B.ind ? 1 : 0);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}
