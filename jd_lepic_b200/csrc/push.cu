// push.cu -- part_mover (part_expmover.f90:1-517) fused with charge_deposition (:520-610).
//
// One pass over the particle stream per species and step: read 20 B, write 20 B.
//   gather   CIC of E (float2 per node, L1/L2-cached) and B at the old position
//   push     Boris (magnetised) or leap-frog, FP32
//   move     x += dt*v on uint32 fixed-point positions; the sub-unit remainder is rounded
//            stochastically (hash of slot, step, axis) so slow particles move unbiased
//   walls    FLOOR cell -> check_outofbounds -> "all four corners are walls" byte
//   deposit  integer CIC weights (exact products of the fixed-point offsets, scaled to
//            2^44) accumulated in a shared-memory uint64 window around the CTA's sort tile
//            (plus a halo for particles that drifted since the sort); anything outside the
//            window goes straight to the global uint64 grid.  Integer sums are associative,
//            so the density is bit-reproducible whatever the atomic order.  A thread keeps a
//            run of particles in one cell as its moments (count, sum fx, sum fy, sum fx fy)
//            where those give the weights exactly, and adds each run once.
// Work is dispensed dynamically: the sort's per-tile items first, then fixed-size chunks of
// the unsorted tail (particles created by collisions since the sort); each CTA prefetches its
// next iteration of the stream into L2 with bulk copies.
//
// Roofline: 40 B per particle-step of algorithmic HBM traffic (X,Y,VX,VY,VZ read+write).
#include <algorithm>
#include "lepic_internal.cuh"

#define PUSH_THREADS 128
#define PUSH_CHUNK 16384

struct PushP {
    int nx, ny, S, W;
    uint32_t *X, *Y;
    float *VX, *VY, *VZ;
    // a sort's pending permutation (IND): position j is read from record
    // ind_slot(pind, n_sorted, ind_old, j) of these arrays and written to X..VZ above at j
    const uint32_t *Xi, *Yi;
    const float *VXi, *VYi, *VZi;
    const int *pind;
    const float4 *E;           // node pairs: (Ex, Ey)[n], (Ex, Ey)[n+1]
    const float4 *B;
    float Bcx, Bcy, Bcz;
    float tcx, tcy, tcz;       // constant field (BMODE 1): t = k1 B and s = k2 B of the Boris
    float scx, scy, scz;       // rotation, k2 = 2 k1 / (1 + k1^2 |B|^2)
    const uint8_t *cellwall;   // cell flags at [ix + iy W] (1: all four corners are walls)
    unsigned long long *acc;
    unsigned int *ss_sink;     // this species' ss2D sink counts (null: not accumulated)
    const WorkItem *items;
    DevCounters *cnt;
    int sp;
    float k1;                  // dt*q/(2m)
    float cdx, cdy;            // dt * 2^S / dx
    float inv2S;               // 2^-S
    int pbc, spec, nmn, negion_nmn;
    uint32_t step_key, step_key2;
    int tw, th, ntx, M, WX, WY, win;
    unsigned WX1, WY1;         // WX - 1, WY - 1
    int mom_up, mom_sup;       // LEPIC_DEP_SHIFT - 2S and LEPIC_DEP_SHIFT - S (moments deposit)
    long long xlim, ylim;      // nx<<S, ny<<S
    // the 3rd dimension (walls.cu): z per slot, its length, the end plates' potential and
    // phi for the electrons' test, the ions' loss factor hz 2 dt / zmax and the uB map
    float *Z;                  // null: no 3rd-dimension model
    int zneg, za1, zsize;
    float zmax, dtf, nu_fac;
    double phi0, m_over_2qe, nmq;
    const double *phi;
    const float *uB;
    TallyDev *tal;
    uint32_t zk0, zk1, it;
    // dielectric walls: the charge a wall loss leaves on its label's rows (null: none)
    double *dq;
    const int32_t *bcnd;
    int32_t dtype[LEPIC_MAXLABEL];
    // refluxing at x = 0 (opt_inj = +-4 with the Neumann option) and secondary emission by
    // positive ions on one wall label: the push only records the event (k_reflux and
    // k_sec_emit below do the draws after the species' push)
    int reflux, sec_label;
    WallEvent *rf_ev, *sec_ev;
    unsigned int *ev_count;    // [0] reflux events, [1] emission events
    int ev_cap;
};

#define TAG_SECN 0x5345434Eu      // secondary emission: the number of electrons
#define TAG_SECV 0x53454356u      // secondary emission: one electron's velocity
#define TAG_RFX 0x52465831u       // refluxing: flux attempt
#define TAG_RFX2 0x52465832u      // refluxing: the position draw of an attempt
#define REFLUX_MAX_ATTEMPTS 4096

#define PUSH_G 4    // consecutive slots per thread: one 16-byte vector per array

// CIC weights of one particle: exact integer products of the fixed-point offsets, scaled to
// 2^LEPIC_DEP_SHIFT, for (ix,iy) (ix+1,iy) (ix+1,iy+1) (ix,iy+1)
__device__ __forceinline__ void cic_weights_s(int S, uint32_t X, uint32_t Y, uint64_t *w) {
    const uint32_t mask = (1u << S) - 1u;
    const uint32_t A = 1u << S;
    const uint32_t fx = X & mask, fy = Y & mask, ax = A - fx, ay = A - fy;
    w[0] = (uint64_t)ax * ay; w[1] = (uint64_t)fx * ay; w[2] = (uint64_t)fx * fy; w[3] = (uint64_t)ax * fy;
    const int sh = 2 * S - LEPIC_DEP_SHIFT;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (sh > 0) w[k] = (w[k] + (1ull << (sh - 1))) >> sh;
        else if (sh < 0) w[k] <<= -sh;
    }
}
__device__ __forceinline__ void cic_weights(const PushP &P, uint32_t X, uint32_t Y, uint64_t *w) {
    cic_weights_s(P.S, X, Y, w);
}

// one particle's weights added to the global accumulators of its cell's four nodes
__device__ __forceinline__ void deposit_global(unsigned long long *acc, int S, int W, uint32_t X, uint32_t Y) {
    uint64_t w[4];
    cic_weights_s(S, X, Y, w);
    unsigned long long *q = acc + ((X >> S) + 1) + (long long)((Y >> S) + 1) * W;
    atomicAdd(q, (unsigned long long)w[0]);
    atomicAdd(q + 1, (unsigned long long)w[1]);
    atomicAdd(q + W + 1, (unsigned long long)w[2]);
    atomicAdd(q + W, (unsigned long long)w[3]);
}

// the four accumulators of cell (ix, iy): the CTA's shared-memory window when the cell's four
// nodes lie in it (window-relative cell 0 <= lx < WX - 1, 0 <= ly < WY - 1; an item without a
// window has its origin far away), else the global grid
__device__ __forceinline__ void add_cell(const PushP &P, unsigned long long *win, int ox, int oy,
                                         int ix, int iy, const uint64_t *w) {
    const int lx = ix - ox, ly = iy - oy;
    unsigned long long *q;
    int row;
    if ((unsigned)lx < P.WX1 && (unsigned)ly < P.WY1) {
        q = win + lx + ly * P.WX;
        row = P.WX;
    } else {
        q = P.acc + ix + (long long)iy * P.W;
        row = P.W;
    }
    atomicAdd(q, (unsigned long long)w[0]);
    atomicAdd(q + 1, (unsigned long long)w[1]);
    atomicAdd(q + row + 1, (unsigned long long)w[2]);
    atomicAdd(q + row, (unsigned long long)w[3]);
}

// A run's moments added to cell (ix, iy) as node weights: n particles with offsets fx, fy
// summed as sx = sum fx, sy = sum fy, sxy = sum fx fy give sum (A-fx)(A-fy), sum fx (A-fy),
// sum fx fy, sum (A-fx) fy (A = 2^S).  Used when 2S <= LEPIC_DEP_SHIFT: every product is then
// exact and only shifted up, so the run's weights equal the sum of its particles' cic_weights
// bit for bit, for two 32-bit adds, one 32x32 product and one 64-bit add per particle.  The
// shift up by 2^(LEPIC_DEP_SHIFT - 2S) is applied to the moments before the differences (a
// shift distributes over sums modulo 2^64); n 2^(2S) shifted up is n 2^LEPIC_DEP_SHIFT.  Each
// weight is formed just before its atomic, so that few 64-bit values are live at once.
__device__ __forceinline__ void add_run(const PushP &P, unsigned long long *win, int ox, int oy, int ix, int iy,
                                        uint32_t n, uint32_t sx, uint32_t sy, uint64_t sxy) {
    const int lx = ix - ox, ly = iy - oy;
    unsigned long long *q;
    int row;
    if ((unsigned)lx < P.WX1 && (unsigned)ly < P.WY1) {
        q = win + lx + ly * P.WX;
        row = P.WX;
    } else {
        q = P.acc + ix + (long long)iy * P.W;
        row = P.W;
    }
    const uint64_t c2 = sxy << P.mom_up;
    atomicAdd(q + row + 1, (unsigned long long)c2);
    const uint64_t ax = (uint64_t)sx << P.mom_sup;
    atomicAdd(q + 1, (unsigned long long)(ax - c2));
    const uint64_t ay = (uint64_t)sy << P.mom_sup;
    atomicAdd(q + row, (unsigned long long)(ay - c2));
    atomicAdd(q, (unsigned long long)(((uint64_t)n << LEPIC_DEP_SHIFT) - ax - ay + c2));
}

// part_mover for one particle in registers; returns false for a hole or a particle lost in
// this step (its VX becomes NaN: the slot is a hole).  BMODE: 0 no B, 1 constant, 2 map;
// GEN: the periodic / specular / Neumann boundary options (off in the common deck).
template <int BMODE, bool GEN>
__device__ __forceinline__ bool move_regs(const PushP &P, int i, uint32_t &X, uint32_t &Y, float &vx, float &vy,
                                          float &vz, DevCounters *cnt, unsigned int &lost, int &ixo, int &iyo) {
    if (isnan(vx)) return false; // hole
    const uint32_t mask = (1u << P.S) - 1u;
    const float inv2S = P.inv2S;
    // gather at the old position: ix = INT(x/h)+1, px = (ix*h - x)/h
    const int cx = (int)(X >> P.S), cy = (int)(Y >> P.S);
    const float fx = (float)(X & mask) * inv2S, fy = (float)(Y & mask) * inv2S;
    const int n00 = (cx + 1) + (cy + 1) * P.W;
    const float4 r0 = __ldg(P.E + n00), r1 = __ldg(P.E + n00 + P.W);   // nodes n00, +1 and +W, +W+1
    // the wall byte of the current cell, fetched with the field (independent of the move)
    const bool wall_now = !GEN && __ldg(P.cellwall + n00) != 0;
    // bilinear in lerp form: along x on the rows iy and iy+1, then along y (the CIC weights
    // (1-fx)(1-fy), fx(1-fy), fx fy, (1-fx) fy of the four nodes, in six operations per component)
    const float ax = fmaf(fx, r0.z - r0.x, r0.x), bx = fmaf(fx, r1.z - r1.x, r1.x);
    const float ay = fmaf(fx, r0.w - r0.y, r0.y), by = fmaf(fx, r1.w - r1.y, r1.y);
    const float Ex = fmaf(fy, bx - ax, ax);
    const float Ey = fmaf(fy, by - ay, ay);
    const float k1 = P.k1;
    bool mag = false;
    float Bx = 0.f, By = 0.f, Bz = 0.f;
    if (BMODE == 1) {
        mag = true; Bx = P.Bcx; By = P.Bcy; Bz = P.Bcz;
    } else if (BMODE == 2) {
        const float4 b00 = __ldg(P.B + n00);
        if (b00.w > 1.e-5f) {
            const float4 b10 = __ldg(P.B + n00 + 1), b11 = __ldg(P.B + n00 + P.W + 1);
            const float4 b01 = __ldg(P.B + n00 + P.W);
            const float px = 1.0f - fx, py = 1.0f - fy;
            const float k00 = px * py, k10 = fx * py, k11 = fx * fy, k01 = px * fy;
            Bx = k00 * b00.x + k10 * b10.x + k11 * b11.x + k01 * b01.x;
            By = k00 * b00.y + k10 * b10.y + k11 * b11.y + k01 * b01.y;
            Bz = k00 * b00.z + k10 * b10.z + k11 * b11.z + k01 * b01.z;
            mag = true;
        }
    }
    float ux0 = vx, uy0 = vy, uz0 = vz;
    if (mag) { // Boris, part_expmover.f90:187-206, with t = k1 B and s = k2 B
        float tx, ty, tz, sx, sy, sz;
        if (BMODE == 1) {   // constant field: t and s computed once per launch
            tx = P.tcx; ty = P.tcy; tz = P.tcz;
            sx = P.scx; sy = P.scy; sz = P.scz;
        } else {
            const float Bt2 = Bx * Bx + By * By + Bz * Bz;
            const float k2 = k1 * (2.0f / (1.0f + k1 * k1 * Bt2));
            tx = k1 * Bx; ty = k1 * By; tz = k1 * Bz;
            sx = k2 * Bx; sy = k2 * By; sz = k2 * Bz;
        }
        const float v1x = fmaf(k1, Ex, ux0), v1y = fmaf(k1, Ey, uy0), v1z = uz0;
        // v3 = v1 + v1 x t;  u = v1 + v3 x s + k1 E
        const float v3x = fmaf(v1y, tz, fmaf(-v1z, ty, v1x));
        const float v3y = fmaf(v1z, tx, fmaf(-v1x, tz, v1y));
        const float v3z = fmaf(v1x, ty, fmaf(-v1y, tx, v1z));
        ux0 = fmaf(v3y, sz, fmaf(-v3z, sy, fmaf(k1, Ex, v1x)));
        uy0 = fmaf(v3z, sx, fmaf(-v3x, sz, fmaf(k1, Ey, v1y)));
        uz0 = fmaf(v3x, sy, fmaf(-v3y, sx, v1z));
    } else { // leap-frog, :210-211
        ux0 = ux0 + 2.0f * k1 * Ex;
        uy0 = uy0 + 2.0f * k1 * Ey;
    }
    // a speed above 3e8 m/s or a non-finite velocity (a non-finite field) is an error: the
    // particle is removed (a NaN component makes the comparison false)
    if (!(ux0 * ux0 + uy0 * uy0 + uz0 * uz0 <= 9.0e16f)) {
        set_err(cnt, LERR_RANGE, 101);
        lost++;
        vx = __int_as_float(HOLE_NAN);
        return false;
    }
    // move (:216-217) in fixed-point units: the displacement rounded stochastically,
    // floor(d + u) with u uniform on [0, 1) in steps of 2^-23, which rounds up with probability
    // frac(d) and so moves slow particles unbiased.  u comes from a multiplicative hash of the
    // slot and a per-step key, one per axis: its low 23 bits (an odd multiplier permutes the
    // residues mod 2^23) as the mantissa of 1 + u, so floor(d + 1 + u) - 1 needs no conversion
    const uint32_t hx = ((uint32_t)i ^ P.step_key) * 0x9E3779B1u;
    const uint32_t hy = ((uint32_t)i ^ P.step_key2) * 0x85EBCA77u;
    const float ux = __uint_as_float((hx & 0x007FFFFFu) | 0x3F800000u);
    const float uy = __uint_as_float((hy & 0x007FFFFFu) | 0x3F800000u);
    const int dX = (int)((uint32_t)__float2int_rd(fmaf(ux0, P.cdx, ux)) - 1u);
    const int dY = (int)((uint32_t)__float2int_rd(fmaf(uy0, P.cdy, uy)) - 1u);
    if (!GEN) {
        // a particle that stays in its cell (the common case) and whose cell is not a wall cell
        // is neither lost nor out of range (a wrap of the 32-bit sum always changes the cell)
        const uint32_t Xs = X + (uint32_t)dX, Ys = Y + (uint32_t)dY;
        if (!wall_now && (Xs >> P.S) == (uint32_t)cx && (Ys >> P.S) == (uint32_t)cy) {
            X = Xs; Y = Ys;
            vx = ux0; vy = uy0; vz = uz0;
            ixo = cx + 1; iyo = cy + 1;
            return true;
        }
    }
    long long Xn = (long long)X + (long long)dX;
    long long Yn = (long long)Y + (long long)dY;
    if (GEN && P.pbc) { // :222-241
        const long long Ym = P.ylim;
        long long k4 = Yn / Ym; // INT: truncation toward zero
        if (Yn >= Ym) {
            if (P.spec == 0) Yn = Yn - k4 * Ym;
            else { Yn = (k4 + 1) * Ym - Yn; uy0 = -uy0; }
        }
        if (Yn <= 0) {
            if (P.spec == 0) Yn = (1 - k4) * Ym + Yn;
            else { Yn = k4 * Ym - Yn; uy0 = -uy0; }
            if (Yn >= Ym) Yn = 0; // y = ymax exactly is kept as y = 0
        }
    }
    // FLOOR cell + check_outofbounds + four-corner wall test (:244-258)
    int ixn = (int)(Xn >> P.S) + 1, iyn = (int)(Yn >> P.S) + 1;
    ixn = min(max(ixn, 0), P.nx + 1);
    iyn = min(max(iyn, 0), P.ny + 1);
    bool is_lost = P.cellwall[ixn + iyn * P.W] != 0;
    if (GEN && !is_lost && P.negion_nmn && Xn < 0) is_lost = true; // :261-266
    if (is_lost) {
        lost++;
        if (P.ss_sink) {   // ss2D sink at the node nearest the loss point (part_expmover.f90:327-332)
            const long long hf = 1ll << (P.S - 1);
            const int ixw = min(max((int)((Xn + hf) >> P.S) + 1, 0), P.nx + 1);
            const int iyw = min(max((int)((Yn + hf) >> P.S) + 1, 0), P.ny + 1);
            atomicAdd(P.ss_sink + ixw + (long long)iyw * P.W, 1u);
        }
        if (GEN && P.dq && P.cellwall[ixn + iyn * P.W] != 0) {
            // dielectric charging (part_expmover.f90:340-350): Nm q split by the loss point's y
            // between the rows iy and iy+1 of the loss cell's label, when that label or the
            // one above is a dielectric
            const int lab = min(max(P.bcnd[ixn + iyn * P.W], 0), LEPIC_MAXLABEL - 1);
            const int up = min(max(P.bcnd[ixn + (iyn + 1) * P.W], 0), LEPIC_MAXLABEL - 1);
            if (max(P.dtype[lab], P.dtype[up]) == 1) {
                const double py = (double)iyn - (double)Yn * (double)P.inv2S;   // (iy h - y)/h
                double *row = P.dq + (long long)lab * (P.ny + 3);
                atomicAdd(row + iyn, P.nmq * py);
                atomicAdd(row + iyn + 1, P.nmq * (1.0 - py));
            }
        }
        if (GEN && P.sec_label && P.cellwall[ixn + iyn * P.W] != 0 && P.bcnd[ixn + iyn * P.W] == P.sec_label) {
            // secondary emission: the event, drawn by k_sec_emit after this push
            const unsigned int e = atomicAdd(P.ev_count + 1, 1u);
            if (e < (unsigned int)P.ev_cap)
                P.sec_ev[e] = WallEvent{i, (int)min(max(Yn, 0ll), P.ylim - 1), ux0, uy0, P.Z ? P.Z[i] + P.dtf * uz0 : 0.0f};
            else set_err(cnt, LERR_CAPACITY, 102);
        }
        // the slot becomes a hole that keeps its loss for the tallies (lepic_internal.cuh,
        // loss_hole_tally): X = the loss cell's node, Y = the new vx, VY, VZ = the new vy, vz,
        // VX = a NaN whose payload marks a fresh wall loss (1) or another loss (2)
        const bool wall = !GEN || P.cellwall[ixn + iyn * P.W] != 0;
        X = (uint32_t)(ixn + iyn * P.W);
        Y = __float_as_uint(ux0);
        vy = uy0; vz = uz0;
        vx = __int_as_float(wall ? LOSS_NAN_WALL : LOSS_NAN_OTHER);
        return false;
    }
    if (GEN && P.nmn && Xn <= 0) { // :454-459 specular reflection, or :445-470 refluxing
        if (P.reflux) {
            // the event (slot, x <= 0, the velocity before) for k_reflux, which draws the new
            // state, writes it and deposits it: the particle is stored as it is and not deposited
            const unsigned int e = atomicAdd(P.ev_count, 1u);
            if (e < (unsigned int)P.ev_cap) {
                P.rf_ev[e] = WallEvent{i, (int)max(Xn, -2147483647ll), ux0, uy0, uz0};
                X = 0u;
                Y = (uint32_t)min(max(Yn, 0ll), P.ylim - 1);
                vx = ux0; vy = uy0; vz = uz0;
                return false;
            }
            set_err(cnt, LERR_CAPACITY, 103);
        }
        Xn = -Xn; ux0 = -ux0;
    }
    if (Xn < 0 || Xn >= P.xlim || Yn < 0 || Yn >= P.ylim) {
        set_err(cnt, LERR_RANGE, 100);
        Xn = min(max(Xn, 0ll), P.xlim - 1);
        Yn = min(max(Yn, 0ll), P.ylim - 1);
    }
    X = (uint32_t)Xn;
    Y = (uint32_t)Yn;
    vx = ux0; vy = uy0; vz = uz0;
    ixo = (int)(X >> P.S) + 1;
    iyo = (int)(Y >> P.S) + 1;
    return true;
}

// The 3rd virtual dimension (part_expmover.f90:216-219, 269-309, 400-421) for a particle that
// the wall test kept, at its new cell (ix, iy): z moves with the new vz; electrons and negative
// ions leaving [0, zmax] are lost if 0.5 m vz^2 / qe >= phi(ix,iy) - phi0, else reflected; a
// positive ion is lost with probability hz 2 uB / zmax dt.  A lost particle's slot becomes a
// hole holding an igrid-0 loss record; P_loss(1) also takes Nm q phi at the loss point.
__device__ __forceinline__ bool zstep(const PushP &P, int i, uint32_t &X, uint32_t &Y, float &vx, float &vy,
                                      float &vz, int ix, int iy, unsigned int &lost) {
    float z = P.Z[i] + P.dtf * vz;   // :219
    bool gone = false;
    if (P.zneg) {
        if (z <= 0.0f || z >= P.zmax) {                                   // :276-292
            const double Eki = P.m_over_2qe * (double)vz * (double)vz;
            if (Eki >= P.phi[ix + (long long)iy * P.W] - P.phi0) gone = true;
            else { vz = -vz; z = z <= 0.0f ? 0.02f * P.zmax : 0.98f * P.zmax; }
        }
    } else {                                                              // :294-307
        const int ixc = P.zsize == 1 ? ix : (int)(X >> P.S) / P.zsize + 1;
        const int iyc = P.zsize == 1 ? iy : (int)(Y >> P.S) / P.zsize + 1;
        const float ub = P.uB[(ixc - 1) + (long long)(iyc - 1) * (P.za1 + 1)];
        const uint32_t u = philox4x32_10(U4{(uint32_t)i, P.it, 0x5A4C4F53u, (uint32_t)P.sp}, P.zk0, P.zk1).x;
        if (u01(u) <= (double)(P.nu_fac * ub)) gone = true;
    }
    P.Z[i] = z;
    if (!gone) return true;
    // Nm q phi at the loss point, the bilinear phi of the cell (:400-421)
    const uint32_t mask = (1u << P.S) - 1u;
    const double px = 1.0 - (double)(X & mask) * (double)P.inv2S, py = 1.0 - (double)(Y & mask) * (double)P.inv2S;
    const long long n00 = ix + (long long)iy * P.W;
    const double phip = px * py * P.phi[n00] + (1.0 - px) * py * P.phi[n00 + 1] +
                        (1.0 - px) * (1.0 - py) * P.phi[n00 + P.W + 1] + px * (1.0 - py) * P.phi[n00 + P.W];
    atomicAdd(&P.tal->P1z[P.sp], P.nmq * phip);
    lost++;
    X = (uint32_t)n00;
    Y = __float_as_uint(vx);
    vx = __int_as_float(LOSS_NAN_OTHER);
    return false;
}

// Each thread takes PUSH_G consecutive slots per iteration (one 16-byte vector load and store
// per array): after the sort consecutive particles mostly share a cell, so the deposit
// accumulates runs of equal cells in registers and adds each run to the accumulators once.
// A work item's range is rounded down to multiples of 8 slots at both ends, so consecutive items
// still tile the slot array exactly; particles a rounded range takes from a neighbouring
// tile reach the global grid when they fall outside the window.
template <int BMODE, bool GEN, bool MOVE, bool MOM, bool IND>
__global__ void __launch_bounds__(PUSH_THREADS, 8) k_push_deposit(PushP P) {
    extern __shared__ unsigned long long win[];
    __shared__ int s_tile, s_start, s_end;
    __shared__ unsigned int s_lost;
    DevCounters *cnt = P.cnt;
    const long long n_slots = cnt->n_slots[P.sp], n_sorted = cnt->n_sorted[P.sp];
    const long long ind_old = IND ? cnt->ind_old[P.sp] : 0;
    const int n_items = cnt->n_items[P.sp];
    const long long tail0 = n_sorted & ~7ll;
    for (;;) {
        if (threadIdx.x == 0) {
            unsigned int w = atomicAdd(&cnt->work_next[P.sp], 1u);
            if ((int)w < n_items) {
                WorkItem it = P.items[w];
                s_tile = it.tile; s_start = it.start & ~7; s_end = it.end & ~7;
            } else {
                long long st = tail0 + (long long)(w - n_items) * PUSH_CHUNK;
                if (st >= n_slots) { s_tile = -2; s_start = s_end = 0; }
                else { s_tile = -1; s_start = (int)st; s_end = (int)min(st + PUSH_CHUNK, n_slots); }
            }
            s_lost = 0;
        }
        __syncthreads();
        const int tile = s_tile;
        if (tile == -2) break;
        const bool use_win = P.win && tile >= 0;
        int ox = 1 << 30, oy = 1 << 30;   // no window: every cell is outside it
        if (use_win) {
            int tx = tile % P.ntx, ty = tile / P.ntx;
            ox = tx * P.tw + 1 - P.M;
            oy = ty * P.th + 1 - P.M;
            for (int q = threadIdx.x; q < P.WX * P.WY; q += blockDim.x) win[q] = 0ull;
        }
        __syncthreads();
        unsigned int lost = 0;
        const int end = s_end;
        for (int base = s_start; base < end; base += PUSH_G * PUSH_THREADS) { // uniform trip count
            const int g = base + PUSH_G * threadIdx.x;
            const bool grp_ok = g < end;
            // the CTA's next iteration of the five arrays into L2 with bulk (TMA) prefetches, so
            // its vector loads meet L2 instead of HBM latency (push 3.76 -> 3.57 ms per step on
            // the 2048^2 bench; staging the stream in shared memory through mbarriers measured
            // 3.83, per-thread prefetches 3.58)
            if (MOVE && threadIdx.x == 0) {
                const int bn = base + PUSH_G * PUSH_THREADS;
                if (bn < end) {
                    const uint32_t nb = (uint32_t)((min(PUSH_G * PUSH_THREADS, end - bn) + 7) & ~7) * 4u;
                    if (!IND) {
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.X + bn), "r"(nb) : "memory");
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.Y + bn), "r"(nb) : "memory");
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.VX + bn), "r"(nb) : "memory");
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.VY + bn), "r"(nb) : "memory");
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.VZ + bn), "r"(nb) : "memory");
                    } else if (bn < n_sorted) {
                        // the permutation of the next iteration, and the records from where it starts
                        // (the permutation is close to a shift inside a tile)
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.pind + bn), "r"(nb) : "memory");
                        const long long s0 = (long long)P.pind[bn] & ~3ll;
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.Xi + s0), "r"(nb) : "memory");
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.Yi + s0), "r"(nb) : "memory");
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.VXi + s0), "r"(nb) : "memory");
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.VYi + s0), "r"(nb) : "memory");
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(P.VZi + s0), "r"(nb) : "memory");
                    }
                }
            }
            uint32_t X[PUSH_G], Y[PUSH_G];
            float vx[PUSH_G], vy[PUSH_G], vz[PUSH_G];
            if (grp_ok && IND) {
                // position j of the sorted order from its record in the input buffer
                int sl[PUSH_G];
                if (g + PUSH_G <= n_sorted) {
                    const int4 pm = *reinterpret_cast<const int4 *>(P.pind + g);
                    sl[0] = pm.x; sl[1] = pm.y; sl[2] = pm.z; sl[3] = pm.w;
                } else {
#pragma unroll
                    for (int p = 0; p < PUSH_G; p++) sl[p] = (int)ind_slot(P.pind, n_sorted, ind_old, (long long)(g + p));
                }
#pragma unroll
                for (int p = 0; p < PUSH_G; p++) {
                    if (g + p < end) {
                        const int s = sl[p];
                        X[p] = __ldg(P.Xi + s); Y[p] = __ldg(P.Yi + s);
                        vx[p] = __ldg(P.VXi + s); vy[p] = __ldg(P.VYi + s); vz[p] = __ldg(P.VZi + s);
                    } else {
                        X[p] = 0u; Y[p] = 0u; vx[p] = __int_as_float(HOLE_NAN); vy[p] = 0.0f; vz[p] = 0.0f;
                    }
                }
            } else if (grp_ok) {   // storage is whole groups of 8: the last, partial group is masked below
                const uint4 x0 = *reinterpret_cast<const uint4 *>(P.X + g);
                const uint4 y0 = *reinterpret_cast<const uint4 *>(P.Y + g);
                const float4 a0 = *reinterpret_cast<const float4 *>(P.VX + g);
                const float4 b0 = *reinterpret_cast<const float4 *>(P.VY + g);
                const float4 c0 = *reinterpret_cast<const float4 *>(P.VZ + g);
                X[0] = x0.x; X[1] = x0.y; X[2] = x0.z; X[3] = x0.w;
                Y[0] = y0.x; Y[1] = y0.y; Y[2] = y0.z; Y[3] = y0.w;
                vx[0] = a0.x; vx[1] = a0.y; vx[2] = a0.z; vx[3] = a0.w;
                vy[0] = b0.x; vy[1] = b0.y; vy[2] = b0.z; vy[3] = b0.w;
                vz[0] = c0.x; vz[1] = c0.y; vz[2] = c0.z; vz[3] = c0.w;
            }
            int rkey = -1, rix = 0, riy = 0;   // the current run of equal cells
            uint64_t rw[4] = {0, 0, 0, 0};     // its weights, or (MOM) its moments n, sx, sy, sxy
            const uint32_t fmask = (1u << P.S) - 1u;
            if (grp_ok) {
#pragma unroll
                for (int p = 0; p < PUSH_G; p++) {
                    const int i = g + p;
                    if (i >= end) break;
                    bool alive;
                    int ix, iy;   // the deposit cell INT(x/h)+1 (x >= 0)
                    if (MOVE) {
                        alive = move_regs<BMODE, GEN>(P, i, X[p], Y[p], vx[p], vy[p], vz[p], cnt, lost, ix, iy);
                        if (GEN && alive && P.Z) alive = zstep(P, i, X[p], Y[p], vx[p], vy[p], vz[p], ix, iy, lost);
                    } else {
                        alive = !isnan(vx[p]);
                        ix = (int)(X[p] >> P.S) + 1;
                        iy = (int)(Y[p] >> P.S) + 1;
                    }
                    if (!alive) continue;
                    const int key = ix + iy * P.W;
                    if (MOM) {
                        const uint32_t fx = X[p] & fmask, fy = Y[p] & fmask;
                        const uint64_t fxy = (uint64_t)fx * fy;
                        if (key != rkey) {
                            if (rkey >= 0)
                                add_run(P, win, ox, oy, rix, riy, (uint32_t)rw[0], (uint32_t)rw[1], (uint32_t)rw[2], rw[3]);
                            rkey = key; rix = ix; riy = iy;
                            rw[0] = 1; rw[1] = fx; rw[2] = fy; rw[3] = fxy;
                        } else {
                            rw[0] += 1; rw[1] += fx; rw[2] += fy; rw[3] += fxy;
                        }
                        continue;
                    }
                    uint64_t w[4];
                    cic_weights(P, X[p], Y[p], w);
                    if (key != rkey) {
                        if (rkey >= 0) add_cell(P, win, ox, oy, rix, riy, rw);
                        rkey = key; rix = ix; riy = iy;
                        rw[0] = w[0]; rw[1] = w[1]; rw[2] = w[2]; rw[3] = w[3];
                    } else {
                        rw[0] += w[0]; rw[1] += w[1]; rw[2] += w[2]; rw[3] += w[3];
                    }
                }
                if (MOVE) {
                    *reinterpret_cast<uint4 *>(P.X + g) = make_uint4(X[0], X[1], X[2], X[3]);
                    *reinterpret_cast<uint4 *>(P.Y + g) = make_uint4(Y[0], Y[1], Y[2], Y[3]);
                    *reinterpret_cast<float4 *>(P.VX + g) = make_float4(vx[0], vx[1], vx[2], vx[3]);
                    *reinterpret_cast<float4 *>(P.VY + g) = make_float4(vy[0], vy[1], vy[2], vy[3]);
                    *reinterpret_cast<float4 *>(P.VZ + g) = make_float4(vz[0], vz[1], vz[2], vz[3]);
                }
            }
            // every lane adds its last run itself: lanes whose runs share a cell (the usual case
            // after the sort) meet at the same shared-memory words, and the serialised atomics
            // cost less issue than any warp-level combination of the runs (a group-masked warp
            // reduction measured 16 % slower on the whole push, a segmented shuffle scan 4 %)
            if (rkey >= 0) {
                if (MOM) {
                    add_run(P, win, ox, oy, rix, riy, (uint32_t)rw[0], (uint32_t)rw[1], (uint32_t)rw[2], rw[3]);
                } else {
                    add_cell(P, win, ox, oy, rix, riy, rw);
                }
            }
        }
        // lost-particle count: one atomic per warp, then per CTA
        for (int o = 16; o > 0; o >>= 1) lost += __shfl_xor_sync(0xffffffffu, lost, o);
        if ((threadIdx.x & 31) == 0 && lost) atomicAdd(&s_lost, lost);
        __syncthreads();
        if (use_win) {
            for (int q = threadIdx.x; q < P.WX * P.WY; q += blockDim.x) {
                unsigned long long v = win[q];
                if (v) {
                    int lx = q % P.WX, ly = q / P.WX;
                    atomicAdd(P.acc + (ox + lx) + (long long)(oy + ly) * P.W, v);
                }
            }
        }
        if (threadIdx.x == 0 && s_lost) {
            atomicAdd(&cnt->n_lost[P.sp], (unsigned long long)s_lost);
            atomicAdd((unsigned long long *)&cnt->n_alive[P.sp], (unsigned long long)(-(long long)s_lost));
        }
        __syncthreads();
    }
}

// the kernel's dynamic shared-memory limit, set once per device (this also loads the kernel)
template <int BMODE, bool GEN, bool MOVE, bool MOM, bool IND>
static int set_push_attr(lepic_ctx *c) {
    static bool attr_set[64] = {false};
    if (!attr_set[c->dev & 63]) {
        LCUDA(cudaFuncSetAttribute(k_push_deposit<BMODE, GEN, MOVE, MOM, IND>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        attr_set[c->dev & 63] = true;
    }
    return LEPIC_OK;
}

template <int BMODE, bool GEN, bool MOVE, bool MOM, bool IND>
static int launch_one(lepic_ctx *c, PushP &P, size_t smem) {
    const int ra = set_push_attr<BMODE, GEN, MOVE, MOM, IND>(c);
    if (ra != LEPIC_OK) return ra;
    int occ = 0;
    LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_push_deposit<BMODE, GEN, MOVE, MOM, IND>,
                                                        PUSH_THREADS, smem));
    k_push_deposit<BMODE, GEN, MOVE, MOM, IND><<<c->num_sms * std::max(1, occ), PUSH_THREADS, smem, c->stream>>>(P);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

// ind: the fast mover reading through a pending permutation (only without the general mover)
template <int BMODE, bool MOM>
static int launch_m(lepic_ctx *c, PushP &P, size_t smem, bool gen, bool move, bool ind) {
    if (!move) return launch_one<BMODE, false, false, MOM, false>(c, P, smem);
    if (gen) return launch_one<BMODE, true, true, MOM, false>(c, P, smem);
    return ind ? launch_one<BMODE, false, true, MOM, true>(c, P, smem) : launch_one<BMODE, false, true, MOM, false>(c, P, smem);
}

// The mover that reads through a pending permutation, configured (and so loaded) ahead of its
// first launch: the first sort of a species that may leave its permutation pending calls this,
// so that the first push after a deferred sort pays no kernel loading.
template <int BMODE>
static int preload_ind_b(lepic_ctx *c) {
    return 2 * c->S <= LEPIC_DEP_SHIFT ? set_push_attr<BMODE, false, true, true, true>(c)
                                       : set_push_attr<BMODE, false, true, false, true>(c);
}
int push_preload_ind(lepic_ctx *c, int s) {
    const lepic_config &g = c->cfg;
    int bmode = g.flag_B;
    if (g.flag_B_pos == 1 && g.charge[s] > 0.0) bmode = 0; // as push_deposit
    if (bmode == 1) return preload_ind_b<1>(c);
    if (bmode == 2) return preload_ind_b<2>(c);
    return preload_ind_b<0>(c);
}

// moments deposit where the weights are exact (2S <= LEPIC_DEP_SHIFT, grids of 1024 and up)
template <int BMODE>
static int launch_b(lepic_ctx *c, PushP &P, size_t smem, bool gen, bool move, bool ind) {
    return 2 * P.S <= LEPIC_DEP_SHIFT ? launch_m<BMODE, true>(c, P, smem, gen, move, ind)
                                      : launch_m<BMODE, false>(c, P, smem, gen, move, ind);
}

// Refluxing (part_expmover.f90:445-470), one thread per event of this species' push: vx from
// the shifted-Maxwellian flux about vb cos(th_B) by acceptance-rejection against fmax
// (shifted_maxwellian_flux, part_injection.f90:239-265), (vy, vz) from load_gauss with
// vy += vb sin(th_B), x = vx r dt; an attempt whose x falls outside [0, xmax] is drawn again.
// The draws come from the counter stream keyed by (slot, attempt, species, step).  P_loss(1)
// takes 0.5 Nm m v^2 before, P_loss(4) after; the particle is written and deposited.  With the
// 3rd dimension its z moves by dt vz (its end-plate test is not taken in this step).  If no
// attempt is kept the particle is reflected as without refluxing and the call reports ERANGE.
struct RefluxP {
    const WallEvent *ev;
    const unsigned int *count;
    int cap, sp, S, W;
    uint32_t *X;
    const uint32_t *Y;
    float *VX, *VY, *VZ, *Z;
    unsigned long long *acc;
    TallyDev *tal;
    DevCounters *cnt;
    double vbx, vby, vt, fmax, dt, xmax, sx, ekf;
    float dtf;
    long long xlim;
    uint32_t k0, k1, it;
};

__global__ void k_reflux(RefluxP R) {
    const int n = (int)min(*R.count, (unsigned int)R.cap);
    const double vm = fmax(0.0, R.vbx - 4.0 * R.vt), vp = R.vbx + 4.0 * R.vt;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const WallEvent E = R.ev[e];
        const int i = E.slot;
        double ux = E.u, uy = E.v, uz = E.w;
        long long Xn = -(long long)E.a;       // the specular reflection, if no attempt is kept
        bool got = false;
        for (uint32_t a = 0; a < REFLUX_MAX_ATTEMPTS && !got; a++) {
            const uint32_t c1 = (a << 3) | (uint32_t)R.sp;
            const U4 f = philox4x32_10(U4{(uint32_t)i, c1, TAG_RFX, R.it}, R.k0, R.k1);
            const double v = vm + u01(f.x) * (vp - vm);
            const double fv = v * exp(-(v - R.vbx) * (v - R.vbx) / (R.vt * R.vt));
            if (u01(f.y) > fv / R.fmax) continue;
            double vy, vz;
            gauss_pair(R.vt, f.z, f.w, &vy, &vz);
            vy += R.vby;
            const U4 g = philox4x32_10(U4{(uint32_t)i, c1, TAG_RFX2, R.it}, R.k0, R.k1);
            const double x = v * (u01(g.x) * R.dt);
            if (x < 0.0 || x > R.xmax) continue;
            atomicAdd(&R.tal->P1r[R.sp], R.ekf * (ux * ux + uy * uy + uz * uz));
            atomicAdd(&R.tal->P4r[R.sp], R.ekf * (v * v + vy * vy + vz * vz));
            Xn = min((long long)(x * R.sx), R.xlim - 1);   // truncation: the cell is INT(x/h)
            ux = v; uy = vy; uz = vz;
            got = true;
        }
        if (!got) {
            set_err(R.cnt, LERR_RANGE, 104);
            Xn = min(Xn, R.xlim - 1);
            ux = -ux;
        }
        const uint32_t X = (uint32_t)Xn;
        R.X[i] = X;
        R.VX[i] = (float)ux; R.VY[i] = (float)uy; R.VZ[i] = (float)uz;
        if (R.Z) R.Z[i] = R.Z[i] + R.dtf * E.w;
        deposit_global(R.acc, R.S, R.W, X, R.Y[i]);   // the deposit the push left out
    }
}

// Secondary emission (part_expmover.f90:354-392), one thread per event of a positive ion
// species' push: INT(gam) electrons, one more with probability gam - INT(gam), at
// (xg_sec, y, z) of the loss point with vx = -SIGN(1, vx_ion) vt sqrt(-ln(1-r)) and (vy, vz)
// from load_gauss at the emission temperature; each adds 0.5 Nm m (vx^2 + vz^2 + vz^2) to the
// electrons' P_loss(4) (the reference's sum: vz taken twice, vy not).  The draws come from the
// counter stream keyed by (slot, step, species, electron); the electrons wait in the electrons'
// product list (key slot * 8 + k) for the ordered append after the push and are deposited now:
// they are in this step's density, as in the reference, where the deposition follows the movers.
struct SecP {
    const WallEvent *ev;
    const unsigned int *count;
    int cap, sp, S, W;
    double gam, vt, ekf0;
    uint32_t X;
    Product *prod;
    unsigned int *prod_count;
    int prod_cap;
    unsigned long long *acc0;
    TallyDev *tal;
    DevCounters *cnt;
    uint32_t k0, k1, it;
};

__global__ void k_sec_emit(SecP Q) {
    const int n = (int)min(*Q.count, (unsigned int)Q.cap);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const WallEvent E = Q.ev[e];
        const int i = E.slot;
        const U4 r = philox4x32_10(U4{(uint32_t)i, Q.it, TAG_SECN, (uint32_t)Q.sp}, Q.k0, Q.k1);
        int m = (int)Q.gam;
        if (u01(r.x) <= Q.gam - (double)m) m++;
        if (m == 0) continue;
        const unsigned int base = atomicAdd(Q.prod_count, (unsigned int)m);
        const uint32_t Y = (uint32_t)E.a;
        const double sgn = E.u >= 0.0f ? 1.0 : -1.0;
        for (int k = 0; k < m; k++) {
            const U4 v = philox4x32_10(U4{(uint32_t)i, Q.it, TAG_SECV, ((uint32_t)Q.sp << 8) | (uint32_t)k}, Q.k0, Q.k1);
            const double vx = -sgn * Q.vt * sqrt(-log(1.0 - u01(v.x)));
            double vy, vz;
            gauss_pair(Q.vt, v.y, v.z, &vy, &vz);
            if (base + k >= (unsigned int)Q.prod_cap) { set_err(Q.cnt, LERR_CAPACITY, 105); continue; }
            atomicAdd(&Q.tal->P4r[0], Q.ekf0 * (vx * vx + vz * vz + vz * vz));
            Product pr;
            pr.key = (unsigned long long)i * 8ull + (unsigned long long)k;
            pr.X = Q.X; pr.Y = Y;
            pr.vx = (float)vx; pr.vy = (float)vy; pr.vz = (float)vz;
            pr.z = E.w;
            Q.prod[base + k] = pr;
            deposit_global(Q.acc0, Q.S, Q.W, Q.X, Y);
        }
    }
}

// the event lists of the push, allocated when a wall model first needs them
static int wall_events(lepic_ctx *c) {
    if (c->ev_count) return LEPIC_OK;
    long long cap = 65536;
    for (int s = 0; s < c->cfg.ntype; s++) cap = std::max(cap, c->sp[s].cap / 64);
    cap = std::min(cap, (long long)1 << 26);
    if (cudaMalloc((void **)&c->rf_ev, sizeof(WallEvent) * cap) != cudaSuccess ||
        cudaMalloc((void **)&c->sec_ev, sizeof(WallEvent) * cap) != cudaSuccess ||
        cudaMalloc((void **)&c->ev_count, 2 * sizeof(unsigned int)) != cudaSuccess) {
        c->last_err = "wall events: cudaMalloc failed";
        return LEPIC_ENOMEM;
    }
    c->ev_cap = (int)cap;
    return LEPIC_OK;
}

int push_deposit(lepic_ctx *c, int it, bool move) {
    const lepic_config &g = c->cfg;
    for (int s = 0; s < g.ntype; s++)
        LCUDA(cudaMemsetAsync(c->sp[s].acc, 0, sizeof(unsigned long long) * c->nn, c->stream));
    LCUDA(cudaMemsetAsync(c->dcnt->work_next, 0, sizeof(c->dcnt->work_next), c->stream));
    const double amu = 1.66053886e-27;
    bool any_sec = false;
    for (int s = 0; s < g.ntype; s++) {
        SpeciesBuf &B = c->sp[s];
        PushP P;
        memset(&P, 0, sizeof(P));
        P.nx = g.nx; P.ny = g.ny; P.S = c->S; P.W = g.nx + 3;
        // a pending permutation: the fast mover reads through it and writes the sorted order into
        // the other buffer; anything else moves the records first
        if (B.ind && (!move || push_needs_general(c, s))) {
            const int r = materialize_species(c, s);
            if (r != LEPIC_OK) return r;
        }
        const bool ind = B.ind;
        P.X = B.X[B.cur]; P.Y = B.Y[B.cur]; P.VX = B.VX[B.cur]; P.VY = B.VY[B.cur]; P.VZ = B.VZ[B.cur];
        if (ind) {
            P.Xi = P.X; P.Yi = P.Y; P.VXi = P.VX; P.VYi = P.VY; P.VZi = P.VZ;
            P.pind = B.pind;
            const int o = 1 - B.cur;
            P.X = B.X[o]; P.Y = B.Y[o]; P.VX = B.VX[o]; P.VY = B.VY[o]; P.VZ = B.VZ[o];
        }
        P.E = c->Ef; P.B = c->Bf;
        int bmode = g.flag_B;
        if (g.flag_B_pos == 1 && g.charge[s] > 0.0) bmode = 0; // :185
        P.Bcx = (float)g.Bc[0]; P.Bcy = (float)g.Bc[1]; P.Bcz = (float)g.Bc[2];
        {
            const float k1f = (float)(g.dt * g.charge[s] / (2.0 * g.mass[s]));
            const float Bt2 = P.Bcx * P.Bcx + P.Bcy * P.Bcy + P.Bcz * P.Bcz;
            const float k2 = k1f * (2.0f / (1.0f + k1f * k1f * Bt2));
            P.tcx = k1f * P.Bcx; P.tcy = k1f * P.Bcy; P.tcz = k1f * P.Bcz;
            P.scx = k2 * P.Bcx; P.scy = k2 * P.Bcy; P.scz = k2 * P.Bcz;
        }
        P.cellwall = c->cellwall_w;
        P.acc = B.acc;
        P.ss_sink = ss_counts(c) ? ss_counts(c) + (size_t)(2 * s + 1) * c->nn : nullptr;
        P.items = B.items;
        P.cnt = c->dcnt;
        P.sp = s;
        P.k1 = (float)(g.dt * g.charge[s] / (2.0 * g.mass[s]));
        P.cdx = (float)(g.dt * (double)(1u << c->S) / g.dx);
        P.cdy = (float)(g.dt * (double)(1u << c->S) / g.dy);
        P.inv2S = 1.0f / (float)(1u << c->S);
        P.mom_up = LEPIC_DEP_SHIFT - 2 * c->S;
        P.mom_sup = LEPIC_DEP_SHIFT - c->S;
        P.pbc = g.flag_pbc; P.spec = g.flag_spec; P.nmn = g.flag_nmn;
        P.negion_nmn = (g.charge[s] < 0 && g.mass[s] >= amu && g.flag_nmn == 1) ? 1 : 0;
        P.step_key = (uint32_t)(g.seed * 0x2545F491ull) ^ ((uint32_t)it * 0x27D4EB2Fu) ^ ((uint32_t)s * 0x165667B1u);
        P.step_key2 = (uint32_t)(g.seed * 0x94D049BBull) ^ ((uint32_t)it * 0xC2B2AE3Du) ^ ((uint32_t)s * 0x9E3779B9u);
        P.tw = c->tw; P.th = c->th; P.ntx = c->ntx;
        P.M = 3;
        P.WX = c->tw + 1 + 2 * P.M;
        P.WY = c->th + 1 + 2 * P.M;
        P.WX1 = (unsigned)(P.WX - 1);
        P.WY1 = (unsigned)(P.WY - 1);
        size_t smem = sizeof(unsigned long long) * (size_t)P.WX * P.WY;
        P.win = smem <= 64 * 1024 ? 1 : 0;
        if (!P.win) smem = 0;
        P.xlim = (long long)g.nx << c->S;
        P.ylim = (long long)g.ny << c->S;
        P.nmq = g.Nm[s] * g.charge[s];
        P.bcnd = c->bcnd;
        P.tal = c->tally;
        P.zk0 = (uint32_t)g.seed; P.zk1 = (uint32_t)(g.seed >> 32) ^ 0x5A10C5u;
        P.it = (uint32_t)it;
        if (c->dq) {
            P.dq = c->dq;
            for (int l = 0; l < LEPIC_MAXLABEL; l++) P.dtype[l] = c->dtype[l];
        }
        // refluxing and secondary emission: the push records events, drawn after it
        RefluxP R;
        memset(&R, 0, sizeof(R));
        SecP Q;
        memset(&Q, 0, sizeof(Q));
        {
            double vb, fm, vt, sn, cs;
            if (move && sources_reflux(c, s, &vb, &fm, &vt, &sn, &cs)) {
                P.reflux = 1;
                R.vbx = vb * cs; R.vby = vb * sn; R.vt = vt; R.fmax = fm;
                R.dt = g.dt; R.xmax = g.nx * g.dx; R.sx = (double)(1u << c->S) / g.dx;
                R.ekf = 0.5 * g.Nm[s] * g.mass[s];
            }
        }
        if (move && c->sec_label > 0 && c->sec_gam > 0.0 && g.charge[s] > 0.0) {
            P.sec_label = c->sec_label;
            Q.gam = c->sec_gam;
            Q.vt = std::sqrt(2.0 * g.qe * std::fabs(c->sec_THm) / std::fabs(g.mass[0]));
            Q.ekf0 = 0.5 * g.Nm[0] * g.mass[0];
            Q.X = (uint32_t)std::min<long long>((long long)(c->sec_xg / g.dx * (double)(1u << c->S)),
                                                ((long long)g.nx << c->S) - 1);
            any_sec = true;
        }
        if (P.reflux || P.sec_label) {
            int r = wall_events(c);
            if (r != LEPIC_OK) return r;
            LCUDA(cudaMemsetAsync(c->ev_count, 0, 2 * sizeof(unsigned int), c->stream));
            P.rf_ev = c->rf_ev; P.sec_ev = c->sec_ev; P.ev_count = c->ev_count; P.ev_cap = c->ev_cap;
        }
        if (c->zloss && B.Z[0]) {
            P.Z = B.Z[B.cur];
            P.zneg = g.charge[s] < 0.0 ? 1 : 0;
            P.za1 = c->za1; P.zsize = c->zsize_na;
            P.zmax = (float)g.zmax;
            P.dtf = (float)g.dt;
            P.nu_fac = (float)(c->hz * 2.0 / g.zmax * g.dt);
            P.phi0 = c->phi0_end;
            P.m_over_2qe = 0.5 * g.mass[s] / g.qe;
            P.phi = c->phi;
            P.uB = c->uB + (size_t)s * (c->za1 + 1) * (c->za2 + 1);
        }
        // the boundary options, the 3rd dimension and the wall models take the general mover
        const bool gen = P.pbc || P.nmn || P.negion_nmn || P.Z || P.dq || P.reflux || P.sec_label;
        int r;
        if (bmode == 1) r = launch_b<1>(c, P, smem, gen, move, ind);
        else if (bmode == 2) r = launch_b<2>(c, P, smem, gen, move, ind);
        else r = launch_b<0>(c, P, smem, gen, move, ind);
        if (r != LEPIC_OK) return r;
        if (ind) {   // the sorted order now sits in the other buffer
            B.cur = 1 - B.cur;
            B.ind = false;
        }
        const int eg = c->num_sms * 2;
        if (P.reflux) {
            R.ev = c->rf_ev; R.count = c->ev_count; R.cap = c->ev_cap; R.sp = s; R.S = c->S; R.W = P.W;
            R.X = P.X; R.Y = P.Y; R.VX = P.VX; R.VY = P.VY; R.VZ = P.VZ; R.Z = P.Z; R.acc = B.acc;
            R.tal = c->tally; R.cnt = c->dcnt; R.dtf = (float)g.dt; R.xlim = P.xlim;
            R.k0 = P.zk0; R.k1 = P.zk1; R.it = P.it;
            k_reflux<<<eg, 128, 0, c->stream>>>(R);
            LCUDA(cudaGetLastError());
        }
        if (P.sec_label) {
            SpeciesBuf &E = c->sp[0];
            Q.ev = c->sec_ev; Q.count = c->ev_count + 1; Q.cap = c->ev_cap; Q.sp = s; Q.S = c->S; Q.W = P.W;
            Q.prod = E.prod; Q.prod_count = &c->dcnt->prod_count[0]; Q.prod_cap = E.prod_cap; Q.acc0 = E.acc;
            Q.tal = c->tally; Q.cnt = c->dcnt; Q.k0 = P.zk0; Q.k1 = P.zk1; Q.it = P.it;
            k_sec_emit<<<eg, 128, 0, c->stream>>>(Q);
            LCUDA(cudaGetLastError());
        }
    }
    // the secondary electrons of this push, appended in the order of their ions' slots
    if (any_sec) return commit_products(c, 0, false);
    return LEPIC_OK;
}

bool push_needs_general(const lepic_ctx *c, int s) {
    const lepic_config &g = c->cfg;
    double vb, fm, vt, sn, cs;
    return g.flag_pbc || g.flag_nmn || (c->zloss && c->sp[s].Z[0]) || c->dq ||
           sources_reflux(c, s, &vb, &fm, &vt, &sn, &cs) || (c->sec_label > 0 && c->sec_gam > 0.0 && g.charge[s] > 0.0);
}
