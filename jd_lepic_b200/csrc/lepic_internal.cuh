// lepic_internal.cuh -- shared definitions of the sm_100a implementation.
//
// HBM layout (one context, one GPU):
//   particles  per charged species, structure of arrays, two copies (sort ping-pong):
//              X, Y  uint32 fixed point in cell units: cell = X >> S, offset = X & (2^S-1)
//              VX, VY, VZ float.  A free slot ("hole") has VX = NaN.  20 B per particle.
//   grids      node arrays (nx+3)*(ny+3), x fastest (the reference's Fortran order):
//              phi double, E double2 (FP64 result) + float2 (gather copy), B float4,
//              deposit accumulators uint64 per species (fixed point 2^-44), bcnd int32 and
//              an int8 copy, per-cell "all four corners are walls" bytes for the loss test.
//   multigrid  per level u, b (double) and the FP32 e, r of the mixed-precision cycle.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include "../../include/lepic_gpu.h"

#define LEPIC_DEP_SHIFT 44          // deposit fixed point: weight * 2^44
#define LEPIC_MAXLEV 16

// device error bits (DevCounters::err)
#define LERR_CAPACITY 1
#define LERR_TIMEOUT 2
#define LERR_RANGE 4
#define LERR_DIVERGED 8
#define LERR_NOTCONV 16

struct WorkItem {           // one CTA's share of the push: particles [start, end) of a tile
    int tile;               // sort tile (-1: no shared-memory window, global atomics)
    int start, end, pad;
};

struct Product {            // a particle created by a collision, before its ordered append
    unsigned long long key; // parent slot * 8 + byproduct index (unique, orders the append)
    uint32_t X, Y;
    float vx, vy, vz;
    float z;                // the parent's z (collisions.f90:813; 0 without the 3rd dimension)
};

// A wall event the push records for a follow-up kernel (push.cu): refluxing (a = the fixed-point
// x <= 0 the move reached, (u, v, w) = the velocity before) or secondary emission (a = the
// fixed-point y of the ion's loss point, u = the ion's vx, w = its z there).
struct WallEvent {
    int slot;
    int a;
    float u, v, w;
};

struct DevCounters {
    long long n_slots[LEPIC_MAXSP];    // occupied slots (sorted region + appended tail)
    long long n_sorted[LEPIC_MAXSP];   // end of the region the work list covers
    long long n_alive[LEPIC_MAXSP];
    unsigned long long n_lost[LEPIC_MAXSP], n_dead[LEPIC_MAXSP];
    unsigned long long n_cand[LEPIC_MAXSP], n_add[LEPIC_MAXSP];
    unsigned long long n_coll[LEPIC_MAXCOL];
    unsigned long long n_overflow;
    unsigned int work_next[LEPIC_MAXSP];  // push work-item dispenser
    int n_items[LEPIC_MAXSP];
    unsigned int prod_count[LEPIC_MAXSP]; // products waiting for the ordered append
    int n_big;                            // sort: segments too long for one warp
    unsigned int scatter_next;            // sort: the scatter's work-unit dispenser
    long long ind_old[LEPIC_MAXSP];       // sort: the slots occupied before it (pending permutation)
    unsigned int n_cand_list;             // collisions: candidates of the species being treated
    int err;
    int err_where;
    // multigrid results
    int mg_cycles, mg_sweeps_fine;
    double mg_res_l1, mg_ktot, mg_res_l2, mg_b_l2;
    unsigned long long bar_arrived;       // grid barrier of the cooperative kernels: arrivals
                                          // since the launch (zeroed before each launch)
    int abort_flag;                       // set to end every wait of a cooperative kernel
};

// Loss, power and collision tallies (part_mover's p_mac and P_loss(1), collisions' P_loss(3)
// and cnt_col), cumulative since the context was created or the tallies were reset.
struct TallyDev {
    unsigned long long n_loss[LEPIC_MAXSP][LEPIC_MAXLABEL];
    double v2_loss[LEPIC_MAXSP][LEPIC_MAXLABEL];     // sum of v^2 [m^2/s^2]
    double P3[LEPIC_MAXSP];                           // collisions' energy change [J]
    double cnt_col[3][LEPIC_MAXCOL][LEPIC_MAXRG];
    double P1z[LEPIC_MAXSP];                          // P_loss(1)'s Nm q phi of 3rd-dimension losses [J]
    double P1r[LEPIC_MAXSP];                          // P_loss(1): refluxed particles' energy before [J]
    double P4r[LEPIC_MAXSP];                          // P_loss(4): refluxed and secondary particles' energy [J]
    double inv_np_rg[LEPIC_MAXSP][LEPIC_MAXRG];       // 1/np_tot_rg of the current collision step
};

// A particle lost in the push leaves a hole that keeps its loss until the sort or a tally read
// takes it (part_expmover.f90:314-427): VX = a NaN with payload LOSS_NAN_WALL (a wall loss,
// igrid = bcnd of the loss cell) or LOSS_NAN_OTHER (igrid 0), X = the loss cell's node index,
// Y = the bits of the new vx, VY, VZ = the new vy, vz.  Any other hole is the plain NaN.
#define LOSS_NAN_WALL 0x7fc00001
#define LOSS_NAN_OTHER 0x7fc00002
#define HOLE_NAN 0x7fc00000

// adds a fresh loss hole to p_mac (count and v^2 per label); returns true if it was one
__device__ __forceinline__ bool loss_hole_tally(TallyDev *T, int sp, const int32_t *bcnd, float vx, uint32_t X,
                                                uint32_t Y, float vy, float vz) {
    const int bits = __float_as_int(vx);
    if (bits != LOSS_NAN_WALL && bits != LOSS_NAN_OTHER) return false;
    const int lab = bits == LOSS_NAN_WALL ? min(max(bcnd[X], 0), LEPIC_MAXLABEL - 1) : 0;
    const float ux = __uint_as_float(Y);
    atomicAdd(&T->n_loss[sp][lab], 1ull);
    atomicAdd(&T->v2_loss[sp][lab], (double)ux * ux + (double)vy * vy + (double)vz * vz);
    return true;
}

struct MGLevel {
    int nx, ny;
    double hx, hy;
    double *u;       // (nx+3)(ny+3)
    double *b;       // (nx+1)(ny+1)
    int8_t *bc;      // (nx+3)(ny+3), bcnd clamped to [-4, 1]
    float *e32;      // mixed precision correction (nx+3)(ny+3)
    float *e32b;     // the pre-smoothed correction of the tiled V-cycle (ping-pong partner)
    float *r32;      // mixed precision right-hand side (nx+1)(ny+1)
    double *e64, *e64b, *r64;  // the same three in FP64 for the FP64-cycle comparison (mode 4),
                               // allocated at its first use
};

struct SpeciesBuf {
    int *cell_off = nullptr;   // per-key start offsets of the last sort (DSMC target lists)
    int *claim = nullptr;      // DSMC: the incident slot that holds each target slot
    uint32_t *X[2], *Y[2];
    float *VX[2], *VY[2], *VZ[2];
    float *Z[2] = {nullptr, nullptr};   // z [m], kept only with the 3rd-dimension model (hz >= 0)
    int cur;
    long long cap;
    unsigned long long *acc;   // deposit accumulator, one node grid
    WorkItem *items;
    int max_items;
    Product *prod;             // product list
    int prod_cap;
    // A sort inside lepic_gpu_step may leave its permutation pending instead of moving the
    // records: position j of the sorted order is then slot pind[j] of buffer cur for
    // j < n_sorted, and slot ind_old + (j - n_sorted) for the products appended since (ind_old =
    // the slots occupied before the sort).  The collisions and the push read and write through
    // it; the push writes the sorted order into the other buffer and ends the pending state.
    int *pind = nullptr;
    bool ind = false;
    // the slots are in the order of a sort (false after a put, a load or a restart): only then
    // is a sort's permutation close to the identity, so that the push can read through it
    // without scattered loads; the first sort after a load moves the records itself
    bool ordered = false;
};

// the slot of buffer cur that holds position j of a species' sorted order (see SpeciesBuf)
__device__ __forceinline__ long long ind_slot(const int *pind, long long n_sorted, long long ind_old, long long j) {
    return pind ? (j < n_sorted ? (long long)pind[j] : ind_old + (j - n_sorted)) : j;
}

struct lepic_ctx {
    lepic_config cfg;
    lepic_options opt;         // solver settings (lepic_gpu_set_options), defaults at create
    int dev = 0, num_sms = 0;
    cudaStream_t stream = nullptr;
    // downloads overlapped with the following work (lepic_gpu_iterative_solver_async,
    // lepic_gpu_get_grid_async): a device snapshot of the grid, copied to the host on cstream
    cudaStream_t cstream = nullptr;
    cudaEvent_t ev_snap = nullptr;
    cudaEvent_t ev_down = nullptr, ev_up = nullptr;   // after the last download / upload into phi
    void *snap = nullptr;
    size_t snap_bytes = 0;
    int down_pending = 0, up_pending = 0;
    int S = 0;                 // fractional bits of the fixed-point positions
    long long nn = 0;          // nodes (nx+3)(ny+3)
    int tw = 0, th = 0, ntx = 0, nty = 0, ntiles = 0;
    long long nkeys = 0;       // ntiles * tw * th
    // static grids
    int32_t *bcnd = nullptr;
    int8_t *bc8 = nullptr;
    uint8_t *cellwall = nullptr;   // (nx+2)(ny+2) cells, 1 = all corners are walls
    uint8_t *cellwall_w = nullptr; // the same flags at [ix + iy (nx+3)], the node index of the cell's corner
    double *kq = nullptr;
    float4 *Bf = nullptr;
    // dynamic grids
    double *phi = nullptr, *rhs = nullptr;
    double2 *Ed = nullptr;       // the current FP64 field: one half of Ed_base (nn each)
    double2 *Ed_base = nullptr;  // 2 nn: the field and the pass buffer of calc_Efield
    float4 *Ef = nullptr;         // gather copy in node pairs: (Ex, Ey)[n], (Ex, Ey)[n+1]
    double *npd = nullptr;        // FP64 np grids (ntype), filled on demand
    double *np_red = nullptr;
    double *np_mx = nullptr;
    SpeciesBuf sp[LEPIC_MAXSP];
    // sort scratch
    int *keys = nullptr, *perm = nullptr, *counts = nullptr, *offsets = nullptr;
    int *cursor = nullptr, *blocksums = nullptr, *bigseg = nullptr;
    long long scratch_cap = 0;
    // multigrid
    MGLevel lev[LEPIC_MAXLEV];
    int nlev = 0;
    double *partials = nullptr;
    int mg_grid = 0, mg_grid_mixed = 0, mg_grid_mixed64 = 0;
    double *cg_r = nullptr, *cg_p = nullptr, *cg_ap = nullptr;  // finest-level CG vectors
    // exact solve of the mixed cycle's on-chip top level: the inverse of that level's operator
    // (FP32, cn x cn, symmetric) and, per unknown, its node and right-hand-side indices
    float *mx_cinv = nullptr;
    double *mx_cinv64 = nullptr;    // the same inverse in FP64 (mode 4's cycle)
    int *mx_cidx = nullptr;         // [2 cn]: node index, then r index
    int mx_cn = 0, mx_clev = -1;
    // warm start of the mixed solve: 1 extrapolates 2 phi_(n-1) - phi_(n-2) from the inputs of
    // the last two solves (phi_hist holds the previous input, have_hist says it is valid)
    int warm_xtrap = 0, have_hist = 0;
    double *phi_hist = nullptr;
    // collisions
    bool has_xs = false;
    bool dsmc = false;             // a reaction has a charged target (collisions.f90:339-418)
    double *sigv_mx_d = nullptr;   // [ptype*LEPIC_MAXCOL + icol]
    double *nu_max_d = nullptr;    // per species, formed on the device each collision step
    int hcol_tt[LEPIC_MAXCOL] = {0};  // target species of each reaction
    int npt = 0, ncol = 0;
    double *sig_Er = nullptr, *sig = nullptr, *Eth = nullptr;
    int *col_info = nullptr;
    int hsig_list[LEPIC_MAXSP * LEPIC_MAXCOL] = {0};
    unsigned long long *prod_sort = nullptr;
    int p_ncol[LEPIC_MAXSP] = {0};
    double nu_max[LEPIC_MAXSP] = {0};
    int flag_ionrep = 0;
    double fEk = 0;
    // learned warm start (cnn.cu), created on first use
    void *learn = nullptr;
    double phi_scale = 1.0;        // max |phi| of the initial potential (network input scale)
    long long n_unknown = 0;       // nodes with bcnd <= 0
    // the 3rd virtual dimension of the 2.5D model (part_expmover.f90:269-309), when hz >= 0:
    // z kept per particle (SpeciesBuf::Z), electrons and negative ions lost through the end
    // plates when their z-energy exceeds phi - phi0 (else reflected), positive ions lost at the
    // rate hz 2 uB / zmax with uB the Bohm speed on the averaging grid
    int zloss = 0;
    double hz = 0.0, phi0_end = 0.0;
    int za1 = 0, za2 = 0, zsize_na = 1;   // the uB grid: na = n / size_na, (na1+1)(na2+1) nodes
    float *uB = nullptr;                  // [ptype][(na1+1)(na2+1)], m/s
    // dielectric walls (part_expmover.f90:340-350, main.f90:756-809): per wall label its type
    // (1: dielectric), the capacitance Ca [F/m^2], and the charge collected per label and row
    // since the last update, dq[label][0..ny+2] (null: no dielectrics)
    int32_t dtype[LEPIC_MAXLABEL] = {0};
    // secondary emission by positive ions (lepic_gpu_set_secondary): label, coefficient,
    // the emitting grid's x [m] and the electrons' temperature [eV]
    int sec_label = 0;
    double sec_gam = 0.0, sec_xg = 0.0, sec_THm = 0.0;
    // the push's wall events (refluxing, emission) and their counts, allocated when first needed
    WallEvent *rf_ev = nullptr, *sec_ev = nullptr;
    unsigned int *ev_count = nullptr;
    int ev_cap = 0;
    double Ca = 0.0;
    double *dq = nullptr;
    // particle sources (sources.cu), created by lepic_gpu_set_sources
    void *src = nullptr;
    // averaging diagnostics (diag.cu), created by lepic_gpu_set_avg
    void *avg = nullptr;
    // ss2D with plt_src = 0: per species a source and a sink count per node, [(2 sp + k) nn
    // + node], k = 0 source, 1 sink; accumulated between averaging samples while averaging is
    // configured (null otherwise)
    unsigned int *ss_map = nullptr;
    // plt_src (read_input.f90:113-117): 0 counts made/removed macroparticles in ss_map; 1 fills
    // ss_diag (FP64, same layout) at each averaging sample from the collision frequencies
    int plt_src = 0;
    double *ss_diag = nullptr;
    // counters
    DevCounters *dcnt = nullptr;
    TallyDev *tally = nullptr;
    // x-regions of the collision tallies (main.f90:316-328), node indices
    int n_rg = 0, iyl_rg = 0, iyr_rg = 0;
    int ixl_rg[LEPIC_MAXRG] = {0}, ixr_rg[LEPIC_MAXRG] = {0};
    int *rg_scratch = nullptr;     // device copy of ixl_rg, ixr_rg
    double *rg_kfac = nullptr;     // dx dy zmax / Nm per species
    DevCounters *hcnt = nullptr;  // pinned mirror
    std::string last_err;
};

// ---------------------------------------------------------------------------------------
// Counter-based RNG: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), written from the
// published round function: two 32x32->64 multiplies per round, Weyl key schedule.
struct U4 { uint32_t x, y, z, w; };
__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}
__device__ __forceinline__ double u01(uint32_t v) { return ((double)v + 0.5) * 2.3283064365386963e-10; }

// load_gauss.f90:16-39 from two counter draws: vp = vt sqrt(-ln(1-r1)), th = 2 pi r2
__device__ __forceinline__ void gauss_pair(double vt, uint32_t a, uint32_t b, double *x, double *y) {
    const double pi = 3.141592653589793;
    const double vp = vt * sqrt(-log(1.0 - u01(a)));
    double s, co;
    sincos(2.0 * pi * u01(b), &s, &co);
    *x = vp * co;
    *y = vp * s;
}

// 32-bit integer mix (MurmurHash3 finaliser), used for the stochastic rounding of moves.
__device__ __forceinline__ uint32_t mix32(uint32_t h) {
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
    return h;
}

__device__ __forceinline__ void set_err(DevCounters *c, int bit, int where) {
    atomicOr(&c->err, bit);
    atomicCAS(&c->err_where, 0, where);
}

// Bounded software grid barrier for cooperative launches.  Every wait gives up after a
// clock budget (about 2 s) and then raises LERR_TIMEOUT; any raised error ends all waits.
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_volatile_i32(const int *p) {
    int v;
    asm volatile("ld.volatile.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
// Each CTA adds one arrival to a counter that only grows during the launch (zeroed before it):
// the arrivals of barrier k are the values k nblocks .. (k + 1) nblocks - 1 (no CTA arrives at
// barrier k + 1 before barrier k is complete), so a CTA reads its barrier from the value its
// atomic returns and waits until the counter reaches the end of that barrier.  With no reset
// between barriers one atomic and one acquire poll are on the critical path (1.8 us per
// barrier over 444 CTAs on B200, against 2.8 us for a count-and-generation barrier, measured
// by a standalone probe).
__device__ __forceinline__ bool grid_barrier(DevCounters *c, unsigned int nblocks) {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        const unsigned long long nb = nblocks;
        const unsigned long long target = (atomicAdd(&c->bar_arrived, 1ull) / nb + 1) * nb;
        long long t0 = clock64();
        while (ld_acquire_u64(&c->bar_arrived) < target) {
            if (ld_volatile_i32(&c->abort_flag) != 0) { ok = 0; break; }
            if (clock64() - t0 > 4000000000LL) {
                set_err(c, LERR_TIMEOUT, 900);
                atomicExch(&c->abort_flag, 1);
                ok = 0;
                break;
            }
        }
        __threadfence();
        if (ld_volatile_i32(&c->abort_flag) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// bitonic sort (all comparators ascending, "flip" form): valid for any n with the missing
// tail of the power of two treated as +infinity.  sync() separates the stages.
template <class T, class Sync>
__device__ void bitonic_sort(T *a, int n, int rank, int size, Sync sync) {
    int P = 1;
    while (P < n) P <<= 1;
    for (int blk = 2; blk <= P; blk <<= 1) {
        for (int t = rank; t < P / 2; t += size) {
            int half = blk >> 1;
            int pos = (t / half) * blk + (t % half);
            int partner = (pos / blk) * blk + blk - 1 - (pos % blk);
            if (partner < n) {
                T x = a[pos], y = a[partner];
                if (x > y) { a[pos] = y; a[partner] = x; }
            }
        }
        sync();
        for (int stride = blk >> 2; stride >= 1; stride >>= 1) {
            for (int t = rank; t < P / 2; t += size) {
                int pos = (t / stride) * 2 * stride + (t % stride);
                int partner = pos + stride;
                if (partner < n) {
                    T x = a[pos], y = a[partner];
                    if (x > y) { a[pos] = y; a[partner] = x; }
                }
            }
            sync();
        }
    }
}

// the sort key of cell (cx, cy): tile-major, then row-major inside the tile (sort.cu)
__device__ __forceinline__ int sort_cell_key(int cx, int cy, int nx, int ny, int tw, int th, int ntx) {
    cx = min(max(cx, 0), nx - 1);
    cy = min(max(cy, 0), ny - 1);
    const int tx = cx / tw, ty = cy / th;
    const int lx = cx - tx * tw, ly = cy - ty * th;
    return ((ty * ntx + tx) * th + ly) * tw + lx;
}

struct WarpSync { __device__ void operator()() const { __syncwarp(); } };
struct BlockSync { __device__ void operator()() const { __syncthreads(); } };

// ---------------------------------------------------------------------------------------
// Host-side launchers, one translation unit each.
int field_calc_rhs(lepic_ctx *c);
int field_dens_red(lepic_ctx *c);
int field_calc_efield(lepic_ctx *c);
int field_np_grid(lepic_ctx *c, int ptype, double *d_out);
int mg_solve(lepic_ctx *c, double eps, int mode);
int mg_init(lepic_ctx *c);
int mg_residual_stats(lepic_ctx *c);
// the Bohm speed map of the 3rd-dimension model from an averaging sample (walls.cu)
int zloss_after_avg(lepic_ctx *c, const double *data, int na1, int na2, int size_na, int cnt);
// refluxing at x = 0 (sources.cu): true when the sources' opt_inj is +-4 and the Neumann option
// is on; then the species' shifted-flux parameters (part_injection.f90:34-47, :267-290)
bool sources_reflux(const lepic_ctx *c, int sp, double *vb, double *fmax, double *vt, double *sin_thB,
                    double *cos_thB);
// the ordered append of a species' waiting products (mcc.cu); mcc: count them as collision
// products (n_add)
int commit_products(lepic_ctx *c, int sp, bool mcc);
// the dielectric walls' potential from the charge they collected (walls.cu, main.f90:756-809)
int dielectric_update(lepic_ctx *c);
// xtrap: the warm start may extrapolate; fp64: the V-cycle in FP64 (mode 4) instead of FP32
int mg_mixed_solve(lepic_ctx *c, double eps, bool xtrap, bool fp64 = false);
int push_deposit(lepic_ctx *c, int it, bool move);
int sort_species(lepic_ctx *c, int ptype, bool defer = false);
// moves the records of a pending permutation (the gather a deferred sort left out)
int materialize_species(lepic_ctx *c, int ptype);
int materialize_all(lepic_ctx *c);
int push_preload_ind(lepic_ctx *c, int s);
// the context's stream waits for a staged upload into phi still in flight (api.cu): every
// reader and writer of phi calls it
int wait_upload(lepic_ctx *c);
// true when the push of species s takes the general mover (boundary options, wall models,
// the 3rd dimension); such a species' sort is not deferred
bool push_needs_general(const lepic_ctx *c, int s);
int particles_load(lepic_ctx *c, const lepic_load_spec *spec);
int particles_put(lepic_ctx *c, int ptype, const double *vxp, long long n);
int particles_get(lepic_ctx *c, int ptype, double *vxp, long long cap, long long *n_out);
int sources_before_push(lepic_ctx *c, int it);
int sources_after_push(lepic_ctx *c, int it);
void sources_free(lepic_ctx *c);
int avg_step(lepic_ctx *c, int it);
int mcc_collide(lepic_ctx *c, int it, bool diag = false);
// the ss2D counts the kernels add to (null unless averaging is set up with plt_src = 0)
static inline unsigned int *ss_counts(const lepic_ctx *c) { return c->plt_src == 0 ? c->ss_map : nullptr; }
void avg_free(lepic_ctx *c);

#define LCUDA(call)                                                                     \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess) {                                                        \
            c->last_err = std::string(#call) + ": " + cudaGetErrorString(_e);           \
            return LEPIC_ECUDA;                                                         \
        }                                                                               \
    } while (0)

static inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }
