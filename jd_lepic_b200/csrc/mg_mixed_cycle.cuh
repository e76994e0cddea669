// mg_mixed_cycle.cuh -- the device side of the preconditioned CG Poisson solve (mg_mixed.cu),
// written once for the V-cycle's real type R: mg_mixed.cu includes it in namespace mx32 with
// R = float (the mixed-precision solver, mode 1) and in namespace mx64 with R = double (the same
// algorithm with an FP64 cycle, mode 4: the comparison that separates the precision from the
// algorithm).  Everything that decides the answer (u, r, p, Ap, dot products) is FP64 in both.
// No include guard on purpose: it is included twice, into two namespaces.
struct MXL {
    int nx, ny;
    R aw, an, ac;         // the cycle's stencil of this level (in R)
    double awd, and_, acd;    // FP64 stencil (finest level only)
    R *e, *r;
    R *e2;                // tiled cycle: the pre-smoothed e between the down and up passes
    const int8_t *bc;
    double *u, *b;
};

struct MXP {
    MXL L[LEPIC_MAXLEV];
    int ng, Ls;
    R omega;
    int nu1, nu2, nuc, max_iter;
    double eps, alpha;
    int pbc, nmn;
    double *r64, *p64, *ap64;  // finest-level CG vectors, (nx+3)(ny+3)
    double *partials;
    DevCounters *cnt;
    unsigned bar_extra;        // lepic_options::barrier_extra
    int soff_e[LEPIC_MAXLEV], soff_r[LEPIC_MAXLEV], soff_b[LEPIC_MAXLEV]; // shared-memory copies
    int smem_bytes;
    int tiled;       // 1: the big levels smooth in shared-memory tiles (temporal blocking)
    int tile_cap;    // nodes a tile region may hold
    int tx[LEPIC_MAXLEV], ty[LEPIC_MAXLEV];   // tile size per level
    // exact solve of level Ls (instead of CTA 0's cycle through levels Ls..ng-1): e = M r over
    // the level's cn unknowns, M the inverse of its operator (FP32, cn x cn)
    const R *cinv;
    const int *cidx;           // node index of each unknown, then its r index
    int cn;
};

template <class Team>
__device__ void sweep32(const Team &T, const MXL &L, int color, R omega) {
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    const R aw = L.aw, ae = L.aw, an = L.an, as = L.an, ac = L.ac;
    const R inv_ac = R(1.0) / ac;
    const int hw = nx / 2 + 1;
    for (Walk2 w(T.rank(), T.size(), hw, ny + 1); w.ok(); w.next()) {
        const int j = w.j + 1;
        const int i = ((((j + 1 + color) & 1) != 0) ? 1 : 2) + 2 * w.k;
        if (i > nx + 1) continue;
        const int n = i + j * W;
        const int bc = L.bc[n];
        if (bc > 0) continue;
        const R rij = L.r[(i - 1) + (j - 1) * (nx + 1)];
        R *e = L.e;
        R s;
        if (bc == -2) {
            s = rij - an * e[n + W] - as * e[n - W] - R(2.0) * ae * e[n + 1];
        } else {
            if (bc == 0 && j == ny + 1) continue;
            s = rij - aw * e[n - 1] - an * e[n + W] - as * e[n - W] - ae * e[n + 1];
        }
        e[n] = (R(1.0) - omega) * e[n] + omega * s * inv_ac;
    }
}

template <class Team>
__device__ void pbc32(const Team &T, const MXL &L) {
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    for (int i = (int)T.rank(); i <= nx + 2; i += (int)T.size()) {
        if (L.bc[i + 1 * W] <= 0) L.e[i] = L.e[i + ny * W];
        if (L.bc[i + (ny + 1) * W] <= 0) L.e[i + (ny + 1) * W] = L.e[i + W];
    }
}

// nsweep red-black sweeps; `reverse` runs black-red (the adjoint order, used after the
// coarse-grid correction so that the V-cycle is a symmetric preconditioner)
template <class Team>
__device__ bool smooth32(const Team &T, const MXP &P, const MXL &L, int nsweep, bool reverse) {
    for (int k = 0; k < nsweep; k++)
        for (int cc = 0; cc < 2; cc++) {
            const int color = reverse ? 1 - cc : cc;
            sweep32(T, L, color, P.omega);
            if (!T.sync()) return false;
            if (P.pbc) {
                pbc32(T, L);
                if (!T.sync()) return false;
            }
        }
    return true;
}

__device__ __forceinline__ R getres32(const MXL &L, int ir, int jr, int flag) {
    const int W = L.nx + 3;
    R aw = L.aw, ae = L.aw;
    const R an = L.an, as = L.an, ac = L.ac;
    const int n = ir + jr * W;
    const R *e = L.e;
    R uw;
    if (ir == 1 && flag == 1) { uw = R(0.0); aw = R(0.0); ae = R(2.0) * ae; }
    else uw = e[n - 1];
    return L.r[(ir - 1) + (jr - 1) * (L.nx + 1)] -
           (aw * uw + ae * e[n + 1] + an * e[n + W] + as * e[n - W] + ac * e[n]);
}

__device__ __forceinline__ R rpbc32(const MXL &F, int x, int nmn) {
    const int W = F.nx + 3, ny = F.ny;
    bool set;
    if (x & 1) set = F.bc[x + (ny + 1) * W] <= 0;
    else set = (x - 1 >= 1 && F.bc[x - 1 + (ny + 1) * W] <= 0) ||
               (x + 1 <= F.nx + 1 && F.bc[x + 1 + (ny + 1) * W] <= 0);
    return set ? getres32(F, x, ny, nmn) : R(0.0);
}

// mg.f90:335-444 applied to the correction equation
template <class Team>
__device__ void restrict32(const Team &T, const MXL &F, const MXL &C, int pbc, int nmn) {
    const int nx = F.nx, ny = F.ny, W = nx + 3, nx2 = C.nx, ny2 = C.ny, W2 = nx2 + 3;
    for (Walk2 w(T.rank(), T.size(), nx2 + 1, ny2 + 1); w.ok(); w.next()) {
        const int t = w.flat();
        const int i = w.k + 1, j = w.j + 1;
        int ir = 2 * i - 1, jr = 2 * j - 1;
        R out = R(0.0);
        if (C.bc[i + j * W2] <= 0) {
            const int8_t *bc = F.bc;
#define FB(a, b) bc[(a) + (b) * W]
            R r1 = 0, r2 = 0, r3 = 0, r4 = 0, r5 = 0, r6 = 0, r7 = 0, r8 = 0;
            R r9 = getres32(F, ir, jr, nmn);
            if (ir != nx + 1 && jr != ny + 1 && FB(ir + 1, jr + 1) <= 0) r1 = getres32(F, ir + 1, jr + 1, nmn);
            if (ir != nx + 1 && FB(ir + 1, jr) <= 0) r2 = getres32(F, ir + 1, jr, nmn);
            if (FB(ir + 1, jr - 1) <= 0) {
                if (ir != nx + 1 && jr != 1) r3 = getres32(F, ir + 1, jr - 1, nmn);
                else if (jr == 1 && pbc) r3 = rpbc32(F, ir + 1, nmn);
            }
            if (FB(ir, jr - 1) <= 0) {
                if (jr != 1) r4 = getres32(F, ir, jr - 1, nmn);
                else if (pbc) r4 = rpbc32(F, ir, nmn);
            }
            if (FB(ir - 1, jr - 1) <= 0 && ir != 1) {
                if (jr != 1) r5 = getres32(F, ir - 1, jr - 1, nmn);
                else if (pbc) r5 = rpbc32(F, ir - 1, nmn);
            }
            if (FB(ir - 1, jr) <= 0 && ir != 1) r6 = getres32(F, ir - 1, jr, nmn);
            if (FB(ir - 1, jr + 1) <= 0 && ir != 1 && jr != ny + 1) r7 = getres32(F, ir - 1, jr + 1, nmn);
            if (FB(ir, jr + 1) <= 0 && jr != ny + 1) r8 = getres32(F, ir, jr + 1, nmn);
#undef FB
            out = (R(4.0) * r9 + R(2.0) * (r2 + r4 + r6 + r8) + r1 + r3 + r5 + r7) * R(0.0625);
        }
        C.r[t] = out;
    }
    const int tot2 = W2 * (ny2 + 3);
    for (int t = (int)T.rank(); t < tot2; t += (int)T.size()) C.e[t] = R(0.0);
}

template <class Team>
__device__ void prolong32(const Team &T, const MXL &C, const MXL &F) {
    const int W = F.nx + 3, nx2 = C.nx, ny2 = C.ny, W2 = nx2 + 3;
    for (Walk2 w(T.rank(), T.size(), nx2 + 1, ny2 + 1); w.ok(); w.next()) {
        const int i = w.k + 1, j = w.j + 1;
        const R *e = C.e;
        R r1 = e[i + j * W2], r2 = e[i + (j - 1) * W2];
        R r3 = e[i - 1 + (j - 1) * W2], r4 = e[i - 1 + j * W2];
        const int n = (2 * i - 1) + (2 * j - 1) * W;
        R *u = F.e;
        const int8_t *bc = F.bc;
        if (bc[n] <= 0) u[n] += r1;
        if (bc[n - W] <= 0) u[n - W] += R(0.5) * (r1 + r2);
        if (bc[n - W - 1] <= 0) u[n - W - 1] += R(0.25) * (r1 + r2 + r3 + r4);
        if (bc[n - 1] <= 0) u[n - 1] += R(0.5) * (r1 + r4);
    }
}


// ---------------------------------------------------------------------------------------
// Temporal blocking of the big levels.  A CTA takes a TX x TY tile of updatable nodes, loads
// e, r and the mask of the tile plus a halo of H nodes into shared memory, and runs all K
// half-sweeps of a smoothing stage there: half-sweep h updates the nodes at least h + 1 nodes
// inside the (unclamped) region, so after K half-sweeps the tile itself holds exactly the
// values the grid-wide sweeps would produce (every node sees the same operations in the same
// colour order).  Down: smoothing then the restriction of the coarse nodes whose fine centre
// lies in the tile (H = K + 2).  Up: the prolongation of the region, then smoothing (H = K).
// One grid barrier per level and direction instead of one per half-sweep.  Tiles read their
// halo from one buffer and write their result to the other (e -> e2 down, e2 -> e up), so a
// tile never sees a neighbour's finished values.
#define MX_TX 64     // the largest tile (the host chooses each level's tile, up to 64 x 64)
#define MX_TY 64

struct Region {
    int i0, j0, i1, j1;      // tile interior [i0, i1) x [j0, j1) (updatable nodes)
    int ri0, rj0, RW, RH;    // region origin and size (clamped to the node array)
    int RP;                  // row pitch in shared memory: RW rounded up to a multiple of 4
    int H;
    R *e, *r;
    int8_t *b;
    R *ce;               // the coarse nodes the region's prolongation reads
    __device__ __forceinline__ int at(int i, int j) const { return (i - ri0) + (j - rj0) * RP; }
};

__device__ __forceinline__ Region make_region(const MXL &L, int tile, int TX, int TY, int H, unsigned char *smem,
                                              int cap) {
    Region g;
    const int nx = L.nx, ny = L.ny;
    const int ntx = (nx + 1 + TX - 1) / TX;
    const int ti = tile % ntx, tj = tile / ntx;
    g.i0 = 1 + ti * TX;
    g.j0 = 1 + tj * TY;
    g.i1 = min(g.i0 + TX, nx + 2);
    g.j1 = min(g.j0 + TY, ny + 2);
    g.H = H;
    g.ri0 = max(g.i0 - H, 0);
    g.rj0 = max(g.j0 - H, 0);
    g.RW = min(g.i1 + H, nx + 3) - g.ri0;
    g.RH = min(g.j1 + H, ny + 3) - g.rj0;
    g.RP = (g.RW + 3) & ~3;
    g.e = (R *)smem;
    g.r = g.e + cap;
    g.b = (int8_t *)(g.r + cap);
    g.ce = (R *)((int8_t *)g.b + cap);   // cap is a multiple of 16 (the host rounds it)
    return g;
}

#define MX_BATCH 4   // mask bytes per thread whose loads are all issued before their stores

// one element global -> shared by an asynchronous copy (no register staging); completed by
// cp_async_wait before the CTA barrier that publishes the region
__device__ __forceinline__ void cp_async_elem(R *dst, const R *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (sizeof(R) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// e (from e_src, or zeros when e_src is null), mask and (at updatable nodes) r of the region
// into shared memory: e and r by asynchronous copies, all issued before the mask's loads; the
// caller waits (cp_async_wait) before its barrier.  The mask moves in 32-bit words: a shared
// row starts on a word (the pitch is a multiple of 4), the global row anywhere, so each word
// is two aligned global words and a funnel shift (the masks are allocated 16 bytes longer for
// the words past a row's end).
__device__ __forceinline__ void region_load(const MXL &L, const R *e_src, const Region &g) {
    const int W = L.nx + 3;
    for (Walk2 w(threadIdx.x, blockDim.x, g.RW, g.RH); w.ok(); w.next()) {
        const int i = g.ri0 + w.k, j = g.rj0 + w.j;
        const int q = w.k + w.j * g.RP;
        if (e_src) cp_async_elem(g.e + q, e_src + i + j * W);
        else g.e[q] = R(0.0);
        if (i >= 1 && i <= L.nx + 1 && j >= 1 && j <= L.ny + 1) cp_async_elem(g.r + q, L.r + (i - 1) + (j - 1) * (L.nx + 1));
        else g.r[q] = R(0.0);
    }
    const int wpr = g.RP >> 2;
    const uint32_t *bw = reinterpret_cast<const uint32_t *>(L.bc);
    uint32_t *sb = reinterpret_cast<uint32_t *>(g.b);
    Walk2 w(threadIdx.x, blockDim.x, wpr, g.RH);
    while (w.ok()) {   // two words per thread in flight
        const int q0 = w.k + w.j * wpr;
        const int gs0 = g.ri0 + (g.rj0 + w.j) * W + 4 * w.k;   // the word's first byte
        w.next();
        const bool two = w.ok();
        const int q1 = two ? w.k + w.j * wpr : q0;
        const int gs1 = two ? g.ri0 + (g.rj0 + w.j) * W + 4 * w.k : gs0;
        if (two) w.next();
        const uint32_t a0 = __ldg(bw + (gs0 >> 2)), b0 = __ldg(bw + (gs0 >> 2) + 1);
        const uint32_t a1 = __ldg(bw + (gs1 >> 2)), b1 = __ldg(bw + (gs1 >> 2) + 1);
        sb[q0] = __funnelshift_r(a0, b0, (gs0 & 3) * 8);
        sb[q1] = __funnelshift_r(a1, b1, (gs1 & 3) * 8);
    }
}

// the coarse nodes (ci0.., cj0..) the prolongation of the region reads, into g.ce, by
// asynchronous copies (the caller waits)
__device__ __forceinline__ void coarse_load(const MXL &C, const Region &g, int ci0, int cj0, int CW, int CH) {
    const int W2 = C.nx + 3;
    for (Walk2 w(threadIdx.x, blockDim.x, CW, CH); w.ok(); w.next())
        cp_async_elem(g.ce + w.flat(), C.e + (ci0 + w.k) + (cj0 + w.j) * W2);
}

// the tile (and, for a tile on the border, the ghost nodes beside it) from shared memory to
// e_dst: the tiles together write every node of the level exactly once
__device__ __forceinline__ void region_store(const MXL &L, const Region &g, R *e_dst) {
    const int W = L.nx + 3;
    const int wi0 = g.i0 == 1 ? 0 : g.i0, wj0 = g.j0 == 1 ? 0 : g.j0;
    const int wi1 = g.i1 == L.nx + 2 ? L.nx + 3 : g.i1, wj1 = g.j1 == L.ny + 2 ? L.ny + 3 : g.j1;
    for (Walk2 w(threadIdx.x, blockDim.x, wi1 - wi0, wj1 - wj0); w.ok(); w.next()) {
        const int i = wi0 + w.k, j = wj0 + w.j;
        e_dst[i + j * W] = g.e[g.at(i, j)];
    }
}

// half-sweep h of colour `color` on the region (the same update as sweep32)
__device__ __forceinline__ void region_half_sweep(const MXL &L, const Region &g, int h, int color, R omega) {
    const int nx = L.nx, ny = L.ny;
    const R aw = L.aw, ae = L.aw, an = L.an, as = L.an, ac = L.ac;
    const R inv_ac = R(1.0) / ac;
    // nodes at least h + 1 inside the unclamped region, within the updatable range
    const int lo_i = max(g.i0 - g.H + h + 1, 1), hi_i = min(g.i1 + g.H - h - 1, nx + 2);
    const int lo_j = max(g.j0 - g.H + h + 1, 1), hi_j = min(g.j1 + g.H - h - 1, ny + 2);
    if (lo_i >= hi_i || lo_j >= hi_j) return;
    const int hw = (hi_i - lo_i + 1) / 2 + 1;
    const int RW = g.RP;   // the row pitch
    for (Walk2 w(threadIdx.x, blockDim.x, hw, hi_j - lo_j); w.ok(); w.next()) {
        const int j = lo_j + w.j;
        int i = lo_i + 2 * w.k;
        if (((i + j + 1 + color) & 1) != 0) i++;   // colour 0: i + j odd; colour 1: i + j even
        if (i >= hi_i) continue;
        const int q = g.at(i, j);
        const int bc = g.b[q];
        if (bc > 0) continue;
        R s;
        if (bc == -2) {
            s = g.r[q] - an * g.e[q + RW] - as * g.e[q - RW] - R(2.0) * ae * g.e[q + 1];
        } else {
            if (bc == 0 && j == ny + 1) continue;
            s = g.r[q] - aw * g.e[q - 1] - an * g.e[q + RW] - as * g.e[q - RW] - ae * g.e[q + 1];
        }
        g.e[q] = (R(1.0) - omega) * g.e[q] + omega * s * inv_ac;
    }
}

// getres32 on the region (no Neumann column: the CG path has no Neumann or periodic decks)
__device__ __forceinline__ R region_res(const MXL &L, const Region &g, int i, int j) {
    const R aw = L.aw, ae = L.aw, an = L.an, as = L.an, ac = L.ac;
    const int q = g.at(i, j), RW = g.RP;
    return g.r[q] - (aw * g.e[q - 1] + ae * g.e[q + 1] + an * g.e[q + RW] + as * g.e[q - RW] + ac * g.e[q]);
}

// smoothing + restriction of level l into level l + 1 (C.r), tile by tile; the coarse e is
// not zeroed: the next level's pass starts from zeros itself
__device__ void tiled_down(const BigTeam &, const MXP &P, int l) {
    extern __shared__ __align__(16) unsigned char mx_smem[];
    const MXL &F = P.L[l], &C = P.L[l + 1];
    const int nx = F.nx, ny = F.ny, nx2 = C.nx, W2 = nx2 + 3;
    const int K = 2 * P.nu1, H = K + 2;
    const int TX = P.tx[l], TY = P.ty[l];
    const int ntiles = ((nx + 1 + TX - 1) / TX) * ((ny + 1 + TY - 1) / TY);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const Region g = make_region(F, tile, TX, TY, H, mx_smem, P.tile_cap);
        region_load(F, nullptr, g);   // every level of the cycle starts from e = 0
        cp_async_wait();
        __syncthreads();
        for (int h = 0; h < K; h++) {
            region_half_sweep(F, g, h, h & 1, P.omega);
            __syncthreads();
        }
        // coarse nodes whose fine centre (2i-1, 2j-1) lies in the tile
        const int ic0 = (g.i0 + 2) / 2, ic1 = g.i1 / 2 + 1, jc0 = (g.j0 + 2) / 2, jc1 = g.j1 / 2 + 1;
        for (Walk2 w(threadIdx.x, blockDim.x, ic1 - ic0, jc1 - jc0); w.ok(); w.next()) {
            const int i = ic0 + w.k, j = jc0 + w.j;
            const int ir = 2 * i - 1, jr = 2 * j - 1;
            R out = R(0.0);
            if (C.bc[i + j * W2] <= 0) {
#define RB(x_, y_) g.b[g.at(x_, y_)]
                R r1 = 0, r2 = 0, r3 = 0, r4 = 0, r5 = 0, r6 = 0, r7 = 0, r8 = 0;
                const R r9 = region_res(F, g, ir, jr);
                if (ir != nx + 1 && jr != ny + 1 && RB(ir + 1, jr + 1) <= 0) r1 = region_res(F, g, ir + 1, jr + 1);
                if (ir != nx + 1 && RB(ir + 1, jr) <= 0) r2 = region_res(F, g, ir + 1, jr);
                if (RB(ir + 1, jr - 1) <= 0 && ir != nx + 1 && jr != 1) r3 = region_res(F, g, ir + 1, jr - 1);
                if (RB(ir, jr - 1) <= 0 && jr != 1) r4 = region_res(F, g, ir, jr - 1);
                if (RB(ir - 1, jr - 1) <= 0 && ir != 1 && jr != 1) r5 = region_res(F, g, ir - 1, jr - 1);
                if (RB(ir - 1, jr) <= 0 && ir != 1) r6 = region_res(F, g, ir - 1, jr);
                if (RB(ir - 1, jr + 1) <= 0 && ir != 1 && jr != ny + 1) r7 = region_res(F, g, ir - 1, jr + 1);
                if (RB(ir, jr + 1) <= 0 && jr != ny + 1) r8 = region_res(F, g, ir, jr + 1);
#undef RB
                out = (R(4.0) * r9 + R(2.0) * (r2 + r4 + r6 + r8) + r1 + r3 + r5 + r7) * R(0.0625);
            }
            C.r[(i - 1) + (j - 1) * (nx2 + 1)] = out;
        }
        // the smoothed tile into the partner buffer: neighbouring tiles still read F.e as halo
        region_store(F, g, F.e2);
        __syncthreads();
    }
}

// prolongation of level l + 1 into level l + smoothing, tile by tile
__device__ void tiled_up(const BigTeam &, const MXP &P, int l) {
    extern __shared__ __align__(16) unsigned char mx_smem[];
    const MXL &F = P.L[l], &C = P.L[l + 1];
    const int nx = F.nx, ny = F.ny;
    const int K = 2 * P.nu2, H = K;
    const int TX = P.tx[l], TY = P.ty[l];
    const int ntiles = ((nx + 1 + TX - 1) / TX) * ((ny + 1 + TY - 1) / TY);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const Region g = make_region(F, tile, TX, TY, H, mx_smem, P.tile_cap);
        region_load(F, F.e2, g);
        const int ci0 = g.ri0 / 2, cj0 = g.rj0 / 2;
        const int ci1 = min((g.ri0 + g.RW + 1) / 2, C.nx + 2), cj1 = min((g.rj0 + g.RH + 1) / 2, C.ny + 2);
        const int CW = ci1 - ci0 + 1, CH = cj1 - cj0 + 1;
        coarse_load(C, g, ci0, cj0, CW, CH);
        cp_async_wait();
        __syncthreads();
        // prolong32 written per fine node: each fine node (i, j), 0 <= i <= nx+1, 0 <= j <= ny+1,
        // takes the correction of the one coarse node prolong32 assigns it, in the same order
        for (Walk2 w(threadIdx.x, blockDim.x, g.RW, g.RH); w.ok(); w.next()) {
            const int i = g.ri0 + w.k, j = g.rj0 + w.j;
            if (i > nx + 1 || j > ny + 1) continue;
            const int q = w.k + w.j * g.RP;
            if (g.b[q] > 0) continue;
            const int i2 = (i + 2) / 2, j2 = (j + 2) / 2;    // the coarse node whose stencil holds (i, j)
            const R *e = g.ce + (i2 - ci0) + (j2 - cj0) * CW;
            const R r1 = e[0];
            const bool io = (i & 1) != 0, jo = (j & 1) != 0;
            if (io && jo) {
                g.e[q] += r1;
            } else if (io) {
                const R r2 = e[-CW];
                g.e[q] += R(0.5) * (r1 + r2);
            } else if (jo) {
                const R r4 = e[-1];
                g.e[q] += R(0.5) * (r1 + r4);
            } else {
                const R r2 = e[-CW], r3 = e[-1 - CW], r4 = e[-1];
                g.e[q] += R(0.25) * (r1 + r2 + r3 + r4);
            }
        }
        __syncthreads();
        for (int h = 0; h < K; h++) {
            region_half_sweep(F, g, h, 1 - (h & 1), P.omega);
            __syncthreads();
        }
        // the tile (with the ghost nodes the prolongation touched) back into F.e
        region_store(F, g, F.e);
        __syncthreads();
    }
}

// The coarse part of the cycle (levels >= Ls) on CTA 0, with every coarse level's e, r and
// mask held in shared memory: the restricted r of level Ls comes in from global memory, the
// correction e of level Ls goes back out, everything in between stays on chip.
__device__ __forceinline__ MXL smem_level(const MXP &P, unsigned char *base, int l) {
    MXL S = P.L[l];
    S.e = (R *)(base + P.soff_e[l]);
    S.r = (R *)(base + P.soff_r[l]);
    S.bc = (const int8_t *)(base + P.soff_b[l]);
    return S;
}

__device__ void small_cycle(const MXP &P) {
    extern __shared__ __align__(16) unsigned char mx_smem[];
    SmallTeam T;
    const int ng = P.ng, Ls = P.Ls;
    for (int l = Ls; l < ng; l++) {
        const int nn = (P.L[l].nx + 3) * (P.L[l].ny + 3);
        int8_t *bcs = (int8_t *)(mx_smem + P.soff_b[l]);
        const int8_t *bcg = P.L[l].bc;
        for (int t = threadIdx.x; t < nn; t += blockDim.x) bcs[t] = bcg[t];
    }
    {
        const MXL S = smem_level(P, mx_smem, Ls);
        const int nr = (S.nx + 1) * (S.ny + 1);
        const int nn = (S.nx + 3) * (S.ny + 3);
        const R *rg = P.L[Ls].r;
        for (int t = threadIdx.x; t < nr; t += blockDim.x) S.r[t] = rg[t];
        for (int t = threadIdx.x; t < nn; t += blockDim.x) S.e[t] = R(0.0);
    }
    __syncthreads();
    for (int l = Ls; l <= ng - 2; l++) {
        const MXL F = smem_level(P, mx_smem, l);
        smooth32(T, P, F, P.nu1, false);
        restrict32(T, F, smem_level(P, mx_smem, l + 1), P.pbc, P.nmn);
        __syncthreads();
    }
    {
        const MXL S = smem_level(P, mx_smem, ng - 1);
        smooth32(T, P, S, P.nuc, false);
        smooth32(T, P, S, P.nuc, true);
    }
    for (int l = ng - 2; l >= Ls; l--) {
        const MXL F = smem_level(P, mx_smem, l);
        prolong32(T, smem_level(P, mx_smem, l + 1), F);
        __syncthreads();
        smooth32(T, P, F, P.nu2, true);
    }
    const MXL S = smem_level(P, mx_smem, Ls);
    const int nn = (S.nx + 3) * (S.ny + 3);
    R *eg = P.L[Ls].e;
    for (int t = threadIdx.x; t < nn; t += blockDim.x) eg[t] = S.e[t];
    __syncthreads();
}

// level Ls solved exactly: e = M r, one row of M per warp across the whole grid (a fixed
// summation order per row, whatever the launch); e is zero at every other node of the level
__device__ void coarse_direct(const MXP &P) {
    const MXL &L = P.L[P.Ls];
    const int nn = (L.nx + 3) * (L.ny + 3);
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
    const int n = P.cn;
    const int *ridx = P.cidx + n;
    for (int k = gw; k < n; k += nw) {
        const R *row = P.cinv + (size_t)k * n;
        R a = R(0.0);
        for (int j = lane; j < n; j += 32) a = rfma(row[j], L.r[ridx[j]], a);
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) L.e[P.cidx[k]] = a;
    }
    const int W = L.nx + 3;
    for (int t = (int)(blockIdx.x * (long long)blockDim.x + threadIdx.x); t < nn; t += (int)(gridDim.x * blockDim.x)) {
        const int i = t % W, j = t / W;
        if (i == 0 || j == 0 || i == L.nx + 2 || j == L.ny + 2 || L.bc[t] > 0) L.e[t] = R(0.0);
    }
}

// one symmetric V-cycle on A e = r32 of level 0, from e = 0 (the caller zeroes e)
__device__ bool vcycle32(const MXP &P) {
    BigTeam B{P.cnt, P.partials, P.bar_extra};
    const int ng = P.ng, Ls = P.Ls;
    if (P.tiled) { // Ls <= ng - 1: the small cycle takes the coarse levels
        for (int l = 0; l < Ls; l++) {
            tiled_down(B, P, l);
            if (!B.sync()) return false;
        }
        if (P.cn) coarse_direct(P);
        else if (blockIdx.x == 0) small_cycle(P);
        if (!B.sync()) return false;
        for (int l = Ls - 1; l >= 0; l--) {
            tiled_up(B, P, l);
            if (!B.sync()) return false;
        }
        return true;
    }
    for (int l = 0; l < Ls && l <= ng - 2; l++) {
        if (!smooth32(B, P, P.L[l], P.nu1, false)) return false;
        restrict32(B, P.L[l], P.L[l + 1], P.pbc, P.nmn);
        if (!B.sync()) return false;
    }
    int top;
    if (Ls <= ng - 1) {
        if (P.cn) coarse_direct(P);
        else if (blockIdx.x == 0) small_cycle(P);
        if (!B.sync()) return false;
        top = Ls;
    } else {
        if (!smooth32(B, P, P.L[ng - 1], P.nuc, false)) return false;
        if (!smooth32(B, P, P.L[ng - 1], P.nuc, true)) return false;
        top = ng - 1;
    }
    for (int l = top - 1; l >= 0; l--) {
        prolong32(B, P.L[l + 1], P.L[l]);
        if (!B.sync()) return false;
        if (!smooth32(B, P, P.L[l], P.nu2, true)) return false;
    }
    return true;
}


// The FP64 passes walk FB nodes per thread at a time and issue all their loads before any
// arithmetic: a thread holds ~40 nodes of the 2049^2 level, and one node at a time leaves
// each pass waiting on ~40 memory latencies in a row.  The sums keep the walk order.  The
// five-point passes take two nodes at a time (the kernel's 80 registers), the others four.
#define FB 4
#define FB5 2

// the next FB interior positions of the walk: flat index t over (nx+1)(ny+1), node index n
// over (nx+3)(ny+3); v = false past the end (n = t = 0, read but never written)
template <int NB>
__device__ __forceinline__ void walk_batch(Walk2 &w, int W, int *t, int *n, bool *v) {
#pragma unroll
    for (int u = 0; u < NB; u++) {
        v[u] = w.ok();
        t[u] = v[u] ? w.flat() : 0;
        n[u] = v[u] ? (w.k + 1) + (w.j + 1) * W : 0;
        if (v[u]) w.next();
    }
}

// r = b - A u at unknowns (bcnd <= 0), zero elsewhere; r32 = (R) r; e = 0 (all nodes);
// returns ||r||^2 over bcnd == -1 nodes and the reference's L1 sum.  With B0 the same walk also
// forms ||b0||^2 over bcnd == -1 nodes, b0 = b minus the wall terms of A u (the norm the
// stopping test scales by), and the three sums share one grid barrier.  Without WRITE only the
// sums are formed (the convergence check: r, r32 and e stay as they are).
template <bool B0, bool WRITE = true>
__device__ bool true_residual(const BigTeam &B, const MXP &P, double *rr, double *l1, double *bb = nullptr) {
    const MXL &L = P.L[0];
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    const double aw = L.awd, an = L.and_, ac = L.acd;
    double a = 0.0, s1 = 0.0, s0 = 0.0;
    Walk2 w(B.rank(), B.size(), nx + 1, ny + 1);
    while (w.ok()) {
        int t[FB5], n[FB5];
        bool v[FB5];
        walk_batch<FB5>(w, W, t, n, v);
        int bc[FB5], bw[FB5], be[FB5], bs[FB5], bn[FB5];
        double bb_[FB5], uc[FB5], uw[FB5], ue[FB5], us[FB5], un[FB5];
        const double *u = L.u;
#pragma unroll
        for (int k = 0; k < FB5; k++) {
            const int m = n[k];
            const int mw = v[k] ? m - 1 : m + 1, ms = v[k] ? m - W : m;
            bc[k] = v[k] ? L.bc[m] : 1;
            bb_[k] = L.b[t[k]];
            uc[k] = u[m]; uw[k] = u[mw]; ue[k] = u[m + 1];
            us[k] = v[k] ? u[ms] : 0.0; un[k] = u[m + W];
            if (B0) { bw[k] = L.bc[mw]; be[k] = L.bc[m + 1]; bs[k] = L.bc[ms]; bn[k] = L.bc[m + W]; }
        }
#pragma unroll
        for (int k = 0; k < FB5; k++) {
            if (!v[k]) continue;
            double r = 0.0;
            if (bc[k] <= 0) {
                r = bb_[k] - (aw * uw[k] + an * un[k] + an * us[k] + aw * ue[k] + ac * uc[k]);
                if (bc[k] == -1) { a += r * r; s1 += fabs(r); }
            }
            if (B0 && bc[k] == -1) {
                const double d = bb_[k] - ((bw[k] > 0 ? aw * uw[k] : 0.0) + (bn[k] > 0 ? an * un[k] : 0.0) +
                                           (bs[k] > 0 ? an * us[k] : 0.0) + (be[k] > 0 ? aw * ue[k] : 0.0));
                s0 += d * d;
            }
            if (WRITE) {
                P.r64[n[k]] = r;
                L.r[t[k]] = (R)r;
            }
        }
    }
    if (WRITE) {
        for (Walk2 w2(B.rank(), B.size(), W, ny + 3); w2.ok(); w2.next()) {
            const int t = w2.flat();
            L.e[t] = R(0.0);
            if (w2.k == 0 || w2.j == 0 || w2.k == nx + 2 || w2.j == ny + 2) P.r64[t] = 0.0;
        }
    }
    if (B0) {
        double out[3];
        if (!team_sums<3>(B, {a, s1, s0}, out)) return false;
        *rr = out[0]; *l1 = out[1]; *bb = out[2];
    } else {
        double out[2];
        if (!team_sums<2>(B, {a, s1}, out)) return false;
        *rr = out[0]; *l1 = out[1];
    }
    return true;
}

// z = e (FP32 cycle output): returns r.z
__device__ bool dot_rz(const BigTeam &B, const MXP &P, double *rz) {
    const MXL &L = P.L[0];
    const int nn = (L.nx + 3) * (L.ny + 3);
    const int st = (int)B.size();
    double a = 0.0;
    for (int t0 = (int)B.rank(); t0 < nn; t0 += FB * st) {
        int bc[FB];
        double r[FB];
        R e[FB];
#pragma unroll
        for (int k = 0; k < FB; k++) {
            const int t = t0 + k * st;
            const bool v = t < nn;
            bc[k] = v ? L.bc[t] : 1;
            r[k] = v ? P.r64[t] : 0.0;
            e[k] = v ? L.e[t] : R(0.0);
        }
#pragma unroll
        for (int k = 0; k < FB; k++)
            if (bc[k] <= 0) a += r[k] * (double)e[k];
    }
    return team_sum(B, a, rz);
}

// p = z + beta p and q = A p in one pass: A p_new = A z + beta A p_old, so q = A z + beta q
// needs z's neighbours but not p's, and no barrier separates the p update from the stencil
// (z = e at unknowns, 0 on walls and ghosts; p and q are 0 on walls).  Returns p.q.
__device__ bool update_pq(const BigTeam &B, const MXP &P, double beta, bool first, double *pq) {
    const MXL &L = P.L[0];
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    const double aw = L.awd, an = L.and_, ac = L.acd;
    double a = 0.0;
    Walk2 w(B.rank(), B.size(), nx + 1, ny + 1);
    while (w.ok()) {
        int t[FB5], n[FB5];
        bool v[FB5];
        walk_batch<FB5>(w, W, t, n, v);
        const int8_t *bc = L.bc;
        const R *e = L.e;
        int b0[FB5], bw[FB5], be[FB5], bs[FB5], bn[FB5];
        R z0[FB5], zw[FB5], ze[FB5], zs[FB5], zn[FB5];
        double p0[FB5], q0[FB5];
#pragma unroll
        for (int k = 0; k < FB5; k++) {
            const int m = n[k];
            const int ms = v[k] ? m - W : m;
            b0[k] = v[k] ? bc[m] : 1;
            bw[k] = bc[m - 1 + (v[k] ? 0 : 1)]; be[k] = bc[m + 1]; bs[k] = bc[ms]; bn[k] = bc[m + W];
            z0[k] = e[m]; zw[k] = e[m - 1 + (v[k] ? 0 : 1)]; ze[k] = e[m + 1]; zs[k] = e[ms]; zn[k] = e[m + W];
            p0[k] = P.p64[m];
            q0[k] = P.ap64[m];
        }
#pragma unroll
        for (int k = 0; k < FB5; k++) {
            if (!v[k]) continue;
            const int m = n[k];
            if (b0[k] > 0) {
                P.p64[m] = 0.0;
                P.ap64[m] = 0.0;
                continue;
            }
            const double z = (double)z0[k];
            const double dzw = bw[k] <= 0 ? (double)zw[k] : 0.0, dze = be[k] <= 0 ? (double)ze[k] : 0.0;
            const double dzs = bs[k] <= 0 ? (double)zs[k] : 0.0, dzn = bn[k] <= 0 ? (double)zn[k] : 0.0;
            const double Az = aw * dzw + an * dzn + an * dzs + aw * dze + ac * z;
            const double p = first ? z : z + beta * p0[k];
            const double q = first ? Az : Az + beta * q0[k];
            P.p64[m] = p;
            P.ap64[m] = q;
            a += p * q;
        }
    }
    return team_sum(B, a, pq);
}

// u += alpha p; r -= alpha Ap; r32 = r; e = 0; returns ||r||^2 over bcnd == -1 nodes
__device__ bool update_ur(const BigTeam &B, const MXP &P, double alpha, double *rr) {
    const MXL &L = P.L[0];
    const int nx = L.nx, ny = L.ny, W = nx + 3;
    double a = 0.0;
    Walk2 w(B.rank(), B.size(), nx + 1, ny + 1);
    while (w.ok()) {
        int t[FB], n[FB];
        bool v[FB];
        walk_batch<FB>(w, W, t, n, v);
        int bc[FB];
        double uu[FB], pp[FB], r0[FB], ap[FB];
#pragma unroll
        for (int k = 0; k < FB; k++) {
            bc[k] = v[k] ? L.bc[n[k]] : 1;
            uu[k] = L.u[n[k]]; pp[k] = P.p64[n[k]]; r0[k] = P.r64[n[k]]; ap[k] = P.ap64[n[k]];
        }
#pragma unroll
        for (int k = 0; k < FB; k++) {
            if (bc[k] > 0) continue;
            L.u[n[k]] = uu[k] + alpha * pp[k];
            const double r = r0[k] - alpha * ap[k];
            P.r64[n[k]] = r;
            L.r[t[k]] = (R)r;
            if (bc[k] == -1) a += r * r;
        }
    }
    if (!P.tiled) { // the grid-wide cycle starts from the zeroed e; the tiled one loads zeros itself
        const int nn = W * (ny + 3);
        for (int t = (int)B.rank(); t < nn; t += (int)B.size()) L.e[t] = R(0.0);
    }
    return team_sum(B, a, rr);
}

__global__ void __launch_bounds__(MG_THREADS, 3) k_mg_mixed(MXP P) {
    BigTeam B{P.cnt, P.partials, P.bar_extra};
    double bb = 0.0, rr = 0.0, l1 = 0.0, rz = 0.0, pap = 0.0;
    if (!true_residual<true>(B, P, &rr, &l1, &bb)) return;
    const double b0 = sqrt(bb), tol = P.eps * b0;
    int it = 0, restarts = 0;
    bool conv = sqrt(rr) <= tol;
    bool first = true;
    while (!conv && it < P.max_iter) {
        if (!vcycle32(P)) return;            // z = M^-1 r in L[0].e
        double rz_new;
        if (!dot_rz(B, P, &rz_new)) return;
        if (!update_pq(B, P, first ? 0.0 : rz_new / rz, first, &pap)) return;
        rz = rz_new;
        first = false;
        // A (eps0 * Laplacian, diagonal -4a) and the V-cycle are both negative definite, so
        // r.z and p.Ap are both negative and the step length is positive
        const double alpha = rz / pap;
        if (!(alpha > 0.0) || !isfinite(alpha)) break; // no descent: stop and report
        if (!update_ur(B, P, alpha, &rr)) return;
        it++;
        if (sqrt(rr) <= tol) {               // confirm on the true residual (its sums only)
            if (!true_residual<false, false>(B, P, &rr, &l1)) return;
            conv = sqrt(rr) <= tol;
            if (!conv) {                     // restart from the true residual
                if (!true_residual<false>(B, P, &rr, &l1)) return;
                first = true;
                restarts++;
            }
        }
    }
    if (!conv) {
        if (!true_residual<false, false>(B, P, &rr, &l1)) return;
        conv = sqrt(rr) <= tol;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.cnt->mg_cycles = it;
        P.cnt->mg_sweeps_fine = it * (P.nu1 + P.nu2);
        P.cnt->mg_res_l1 = l1 / P.alpha;
        P.cnt->mg_ktot = (double)restarts;
        P.cnt->mg_res_l2 = sqrt(rr);
        P.cnt->mg_b_l2 = b0;
        if (!conv) set_err(P.cnt, LERR_NOTCONV, 600);
    }
}

