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
//            so the density is bit-reproducible whatever the atomic order.
// Work is dispensed dynamically: the sort's per-tile items first, then fixed-size chunks of
// the unsorted tail (particles created by collisions since the sort).
//
// Roofline: 40 B per particle-step of algorithmic HBM traffic (X,Y,VX,VY,VZ read+write).
#include <algorithm>
#include "lepic_internal.cuh"

#define PUSH_THREADS 256
#define PUSH_CHUNK 2048

struct PushP {
    int nx, ny, S, W;
    uint32_t *X, *Y;
    float *VX, *VY, *VZ;
    const float2 *E;
    const float4 *B;
    float Bcx, Bcy, Bcz;
    const uint8_t *cellwall;
    unsigned long long *acc;
    const WorkItem *items;
    DevCounters *cnt;
    int sp;
    float k1;                  // dt*q/(2m)
    float cdx, cdy;            // dt * 2^S / dx
    int pbc, spec, nmn, negion_nmn;
    uint32_t step_key;
    int tw, th, ntx, M, WX, WY, win;
    long long xlim, ylim;      // nx<<S, ny<<S
};

// CIC deposit of one particle per lane, aggregated per cell inside the warp: lanes whose
// particles share a cell (the usual case after the sort) sum their four integer weights with
// two exact 32-bit warp reductions each (22-bit halves: 32 lanes x 2^22 < 2^32), and one lane
// issues the four atomics.  Must be called by all 32 lanes of the warp.
__device__ __forceinline__ void deposit_warp(const PushP &P, unsigned long long *win, int ox, int oy,
                                             bool use_win, bool have, uint32_t X, uint32_t Y) {
    const int ix = (int)(X >> P.S) + 1, iy = (int)(Y >> P.S) + 1; // INT(x/h)+1, x >= 0
    const int key = have ? ix + iy * P.W : -1;
    const unsigned grp = __match_any_sync(0xffffffffu, key);
    if (key < 0) return;
    const uint32_t mask = (1u << P.S) - 1u;
    const uint32_t A = 1u << P.S;
    const uint32_t fx = X & mask, fy = Y & mask, ax = A - fx, ay = A - fy;
    // (ix,iy) (ix+1,iy) (ix+1,iy+1) (ix,iy+1): 32x32 -> 64-bit products
    uint64_t w[4] = {(uint64_t)ax * ay, (uint64_t)fx * ay, (uint64_t)fx * fy, (uint64_t)ax * fy};
    const int sh = 2 * P.S - LEPIC_DEP_SHIFT;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (sh > 0) w[k] = (w[k] + (1ull << (sh - 1))) >> sh;
        else if (sh < 0) w[k] <<= -sh;
    }
    if (__popc(grp) > 1) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const unsigned lo = __reduce_add_sync(grp, (unsigned)(w[k] & 0x3FFFFFull));
            const unsigned hi = __reduce_add_sync(grp, (unsigned)(w[k] >> 22));
            w[k] = ((uint64_t)hi << 22) + lo;
        }
        if ((int)(threadIdx.x & 31) != __ffs(grp) - 1) return;
    }
    const int lx = ix - ox, ly = iy - oy;
    unsigned long long *q;
    int row;
    if (use_win && lx >= 0 && lx + 1 < P.WX && ly >= 0 && ly + 1 < P.WY) {
        q = win + lx + ly * P.WX;
        row = P.WX;
    } else {
        q = P.acc + ix + (long long)iy * P.W;
        row = P.W;
    }
    if (w[0]) atomicAdd(q, (unsigned long long)w[0]);
    if (w[1]) atomicAdd(q + 1, (unsigned long long)w[1]);
    if (w[2]) atomicAdd(q + row + 1, (unsigned long long)w[2]);
    if (w[3]) atomicAdd(q + row, (unsigned long long)w[3]);
}

struct Part {
    uint32_t X, Y;
    float vx, vy, vz;
};

__device__ __forceinline__ void load_part(const PushP &P, int i, bool ok, Part &p) {
    if (ok) {
        p.vx = P.VX[i]; p.X = P.X[i]; p.Y = P.Y[i]; p.vy = P.VY[i]; p.vz = P.VZ[i];
    } else {
        p.vx = __int_as_float(0x7fc00000); p.X = 0; p.Y = 0; p.vy = 0.f; p.vz = 0.f;
    }
}

// part_mover for one particle already in registers; returns false for a hole or a particle
// lost in this step (the slot then becomes a hole).  BMODE: 0 no B, 1 constant, 2 map;
// GEN: the periodic / specular / Neumann boundary options (off in the common deck).
template <int BMODE, bool GEN>
__device__ __forceinline__ bool move_one(const PushP &P, int i, Part &p, DevCounters *cnt, unsigned int &lost) {
    if (isnan(p.vx)) return false; // hole
    const uint32_t mask = (1u << P.S) - 1u;
    const float inv2S = 1.0f / (float)(1u << P.S);
    uint32_t X = p.X, Y = p.Y;
    float vx = p.vx, vy = p.vy, vz = p.vz;
    // gather at the old position: ix = INT(x/h)+1, px = (ix*h - x)/h
    const int cx = (int)(X >> P.S), cy = (int)(Y >> P.S);
    const float fx = (float)(X & mask) * inv2S, fy = (float)(Y & mask) * inv2S;
    const float px = 1.0f - fx, py = 1.0f - fy;
    const float k00 = px * py, k10 = fx * py, k11 = fx * fy, k01 = px * fy;
    const int n00 = (cx + 1) + (cy + 1) * P.W;
    const float2 e00 = __ldg(P.E + n00), e10 = __ldg(P.E + n00 + 1);
    const float2 e11 = __ldg(P.E + n00 + P.W + 1), e01 = __ldg(P.E + n00 + P.W);
    const float Ex = k00 * e00.x + k10 * e10.x + k11 * e11.x + k01 * e01.x;
    const float Ey = k00 * e00.y + k10 * e10.y + k11 * e11.y + k01 * e01.y;
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
            Bx = k00 * b00.x + k10 * b10.x + k11 * b11.x + k01 * b01.x;
            By = k00 * b00.y + k10 * b10.y + k11 * b11.y + k01 * b01.y;
            Bz = k00 * b00.z + k10 * b10.z + k11 * b11.z + k01 * b01.z;
            mag = true;
        }
    }
    if (mag) { // Boris, part_expmover.f90:187-206
        const float Bt2 = Bx * Bx + By * By + Bz * Bz;
        const float k2 = k1 * (2.0f / (1.0f + k1 * k1 * Bt2));
        const float v1x = vx + k1 * Ex, v1y = vy + k1 * Ey, v1z = vz;
        const float v3x = v1x + k1 * (v1y * Bz - v1z * By);
        const float v3y = v1y + k1 * (v1z * Bx - v1x * Bz);
        const float v3z = v1z + k1 * (v1x * By - v1y * Bx);
        vx = v1x + k2 * (v3y * Bz - v3z * By) + k1 * Ex;
        vy = v1y + k2 * (v3z * Bx - v3x * Bz) + k1 * Ey;
        vz = v1z + k2 * (v3x * By - v3y * Bx);
    } else { // leap-frog, :210-211
        vx = vx + 2.0f * k1 * Ex;
        vy = vy + 2.0f * k1 * Ey;
    }
    // a non-finite velocity (a non-finite field) is an error: the particle is removed
    if (!(fabsf(vx) <= 3.0e8f && fabsf(vy) <= 3.0e8f && fabsf(vz) <= 3.0e8f)) {
        set_err(cnt, LERR_RANGE, 101);
        lost++;
        P.VX[i] = __int_as_float(0x7fc00000);
        return false;
    }
    // move (:216-217): integer part plus an unbiased stochastic rounding of the fractional part
    // of the displacement (16-bit uniforms from one integer hash of slot and step)
    uint32_t h = (uint32_t)i * 0x9E3779B1u ^ P.step_key;
    h = (h ^ (h >> 16)) * 0x7FEB352Du;
    h ^= h >> 15;
    const float ux = (float)(h & 0xFFFFu) * (1.0f / 65536.0f);
    const float uy = (float)(h >> 16) * (1.0f / 65536.0f);
    const float ddx = vx * P.cdx, ddy = vy * P.cdy;
    const float fdx = floorf(ddx), fdy = floorf(ddy);
    long long Xn = (long long)X + (long long)((int)fdx + ((ux < ddx - fdx) ? 1 : 0));
    long long Yn = (long long)Y + (long long)((int)fdy + ((uy < ddy - fdy) ? 1 : 0));
    if (GEN && P.pbc) { // :222-241
        const long long Ym = P.ylim;
        long long k4 = Yn / Ym; // INT: truncation toward zero
        if (Yn >= Ym) {
            if (P.spec == 0) Yn = Yn - k4 * Ym;
            else { Yn = (k4 + 1) * Ym - Yn; vy = -vy; }
        }
        if (Yn <= 0) {
            if (P.spec == 0) Yn = (1 - k4) * Ym + Yn;
            else { Yn = k4 * Ym - Yn; vy = -vy; }
            if (Yn >= Ym) Yn = 0; // y = ymax exactly is kept as y = 0
        }
    }
    // FLOOR cell + check_outofbounds + four-corner wall test (:244-258)
    int ixn = (int)(Xn >> P.S) + 1, iyn = (int)(Yn >> P.S) + 1;
    ixn = min(max(ixn, 0), P.nx + 1);
    iyn = min(max(iyn, 0), P.ny + 1);
    bool is_lost = P.cellwall[ixn + iyn * (P.nx + 2)] != 0;
    if (GEN && !is_lost && P.negion_nmn && Xn < 0) is_lost = true; // :261-266
    if (is_lost) {
        lost++;
        P.VX[i] = __int_as_float(0x7fc00000); // the slot becomes a hole
        return false;
    }
    if (GEN && P.nmn && Xn <= 0) { Xn = -Xn; vx = -vx; } // :454-459
    if (Xn < 0 || Xn >= P.xlim || Yn < 0 || Yn >= P.ylim) {
        set_err(cnt, LERR_RANGE, 100);
        Xn = min(max(Xn, 0ll), P.xlim - 1);
        Yn = min(max(Yn, 0ll), P.ylim - 1);
    }
    X = (uint32_t)Xn;
    Y = (uint32_t)Yn;
    P.X[i] = X; P.Y[i] = Y;
    P.VX[i] = vx; P.VY[i] = vy; P.VZ[i] = vz;
    p.X = X;
    p.Y = Y;
    return true;
}

// Two particles per thread per iteration (two independent load -> push -> store chains in
// flight), then the two warp-aggregated deposits.
template <int BMODE, bool GEN, bool MOVE>
__global__ void __launch_bounds__(PUSH_THREADS) k_push_deposit(PushP P) {
    extern __shared__ unsigned long long win[];
    __shared__ int s_tile, s_start, s_end;
    __shared__ unsigned int s_lost;
    DevCounters *cnt = P.cnt;
    const long long n_slots = cnt->n_slots[P.sp], n_sorted = cnt->n_sorted[P.sp];
    const int n_items = cnt->n_items[P.sp];
    for (;;) {
        if (threadIdx.x == 0) {
            unsigned int w = atomicAdd(&cnt->work_next[P.sp], 1u);
            if ((int)w < n_items) {
                WorkItem it = P.items[w];
                s_tile = it.tile; s_start = it.start; s_end = it.end;
            } else {
                long long st = n_sorted + (long long)(w - n_items) * PUSH_CHUNK;
                if (st >= n_slots) { s_tile = -2; s_start = s_end = 0; }
                else { s_tile = -1; s_start = (int)st; s_end = (int)min(st + PUSH_CHUNK, n_slots); }
            }
            s_lost = 0;
        }
        __syncthreads();
        const int tile = s_tile;
        if (tile == -2) break;
        const bool use_win = P.win && tile >= 0;
        int ox = 0, oy = 0;
        if (use_win) {
            int tx = tile % P.ntx, ty = tile / P.ntx;
            ox = tx * P.tw + 1 - P.M;
            oy = ty * P.th + 1 - P.M;
            for (int q = threadIdx.x; q < P.WX * P.WY; q += blockDim.x) win[q] = 0ull;
        }
        __syncthreads();
        unsigned int lost = 0;
        const int end = s_end;
        for (int base = s_start; base < end; base += 2 * PUSH_THREADS) { // uniform trip count
            const int i0 = base + threadIdx.x, i1 = i0 + PUSH_THREADS;
            Part p0, p1;
            load_part(P, i0, i0 < end, p0);
            load_part(P, i1, i1 < end, p1);
            bool h0, h1;
            if (MOVE) {
                h0 = move_one<BMODE, GEN>(P, i0, p0, cnt, lost);
                h1 = move_one<BMODE, GEN>(P, i1, p1, cnt, lost);
            } else {
                h0 = !isnan(p0.vx);
                h1 = !isnan(p1.vx);
            }
            deposit_warp(P, win, ox, oy, use_win, h0, p0.X, p0.Y);
            deposit_warp(P, win, ox, oy, use_win, h1, p1.X, p1.Y);
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

template <int BMODE, bool GEN, bool MOVE>
static int launch_one(lepic_ctx *c, PushP &P, size_t smem) {
    static bool attr_set[64] = {false};
    if (!attr_set[c->dev & 63]) {
        LCUDA(cudaFuncSetAttribute(k_push_deposit<BMODE, GEN, MOVE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   64 * 1024));
        attr_set[c->dev & 63] = true;
    }
    int occ = 0;
    LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_push_deposit<BMODE, GEN, MOVE>, PUSH_THREADS, smem));
    k_push_deposit<BMODE, GEN, MOVE><<<c->num_sms * std::max(1, occ), PUSH_THREADS, smem, c->stream>>>(P);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

template <int BMODE>
static int launch_b(lepic_ctx *c, PushP &P, size_t smem, bool gen, bool move) {
    if (!move) return launch_one<BMODE, false, false>(c, P, smem);
    return gen ? launch_one<BMODE, true, true>(c, P, smem) : launch_one<BMODE, false, true>(c, P, smem);
}

int push_deposit(lepic_ctx *c, int it, bool move) {
    const lepic_config &g = c->cfg;
    for (int s = 0; s < g.ntype; s++)
        LCUDA(cudaMemsetAsync(c->sp[s].acc, 0, sizeof(unsigned long long) * c->nn, c->stream));
    LCUDA(cudaMemsetAsync(c->dcnt->work_next, 0, sizeof(c->dcnt->work_next), c->stream));
    const double amu = 1.66053886e-27;
    for (int s = 0; s < g.ntype; s++) {
        SpeciesBuf &B = c->sp[s];
        PushP P;
        memset(&P, 0, sizeof(P));
        P.nx = g.nx; P.ny = g.ny; P.S = c->S; P.W = g.nx + 3;
        P.X = B.X[B.cur]; P.Y = B.Y[B.cur]; P.VX = B.VX[B.cur]; P.VY = B.VY[B.cur]; P.VZ = B.VZ[B.cur];
        P.E = c->Ef; P.B = c->Bf;
        int bmode = g.flag_B;
        if (g.flag_B_pos == 1 && g.charge[s] > 0.0) bmode = 0; // :185
        P.Bcx = (float)g.Bc[0]; P.Bcy = (float)g.Bc[1]; P.Bcz = (float)g.Bc[2];
        P.cellwall = c->cellwall;
        P.acc = B.acc;
        P.items = B.items;
        P.cnt = c->dcnt;
        P.sp = s;
        P.k1 = (float)(g.dt * g.charge[s] / (2.0 * g.mass[s]));
        P.cdx = (float)(g.dt * (double)(1u << c->S) / g.dx);
        P.cdy = (float)(g.dt * (double)(1u << c->S) / g.dy);
        P.pbc = g.flag_pbc; P.spec = g.flag_spec; P.nmn = g.flag_nmn;
        P.negion_nmn = (g.charge[s] < 0 && g.mass[s] >= amu && g.flag_nmn == 1) ? 1 : 0;
        P.step_key = (uint32_t)(g.seed * 0x2545F491ull) ^ ((uint32_t)it * 0x27D4EB2Fu) ^ ((uint32_t)s * 0x165667B1u);
        P.tw = c->tw; P.th = c->th; P.ntx = c->ntx;
        P.M = 3;
        P.WX = c->tw + 1 + 2 * P.M;
        P.WY = c->th + 1 + 2 * P.M;
        size_t smem = sizeof(unsigned long long) * (size_t)P.WX * P.WY;
        P.win = smem <= 64 * 1024 ? 1 : 0;
        if (!P.win) smem = 0;
        P.xlim = (long long)g.nx << c->S;
        P.ylim = (long long)g.ny << c->S;
        const bool gen = P.pbc || P.nmn || P.negion_nmn;
        int r;
        if (bmode == 1) r = launch_b<1>(c, P, smem, gen, move);
        else if (bmode == 2) r = launch_b<2>(c, P, smem, gen, move);
        else r = launch_b<0>(c, P, smem, gen, move);
        if (r != LEPIC_OK) return r;
    }
    return LEPIC_OK;
}
