// sort.cu -- part_sorting (sorting.f90:92-251): counting sort of one species by cell.
//
// The reference (one thread) produces a STABLE order: particles grouped by cell index
// ic = (ix-1) + nx*(iy-1) + 1, original order kept inside a cell.  Here:
//   1. keys + histogram        (warp-aggregated atomics on the per-key counts)
//   2. exclusive scan           (three-phase, fixed order)
//   3. scatter of slot indices  (atomics; each warp takes one old tile's slots, or a chunk of the
//                               appended tail, in slot order, so a key comes out of order only
//                               where it receives particles from another tile or the tail)
//   4. per-key segment sort of the slot indices (bitonic, ascending; segments already in
//      order are skipped) -> stable again
//   5. gather of the 5 SoA fields into the other buffer, holes dropped
//   6. push work list: per tile, chunks of CHUNK particles
// so the result is bit-identical to the reference's, independent of thread timing.
// The key is the reference's cell index when tile_w = nx, tile_h = 1; other tile shapes
// order cells tile by tile (the push kernel then stages a compact node window per tile).
//
// Roofline (per particle per sort): read X,Y (8 B) twice, keys 4+4 B, perm 4+4+4 B, the
// 20 B record read + written once: ~72 B, amortised over the nsort = 10 step cadence.
#include <algorithm>
#include <climits>
#include "lepic_internal.cuh"

#define SORT_THREADS 256
#define PUSH_CHUNK 16384
#define SEG_WARP_MAX 256
#define SEG_BLOCK_MAX 8192
#define SEG_CHECK_STEPS 4

struct KeyP {
    int S, nx, ny, tw, th, ntx;
    int twl, thl;   // log2 of tw and th when both are powers of two, else -1
};
// sort_cell_key, with shifts in place of the two divisions for power-of-two tiles (the same key)
__device__ __forceinline__ int cell_key(const KeyP &K, uint32_t X, uint32_t Y) {
    if (K.twl >= 0) {
        const int cx = min(max((int)(X >> K.S), 0), K.nx - 1), cy = min(max((int)(Y >> K.S), 0), K.ny - 1);
        const int tx = cx >> K.twl, ty = cy >> K.thl;
        return (((ty * K.ntx + tx) << K.thl) + (cy & (K.th - 1))) * K.tw + (cx & (K.tw - 1));
    }
    return sort_cell_key((int)(X >> K.S), (int)(Y >> K.S), K.nx, K.ny, K.tw, K.th, K.ntx);
}

// the key pass also takes the loss holes of the pushes since the last sort into the tallies
// (the sort drops the holes).  Four consecutive slots per thread: one 16-byte load per array
// (storage is whole groups of 8 slots), so each thread has its loads in flight together;
// equal keys of a warp add their count with one atomic.
__global__ void k_keys_hist(KeyP K, const uint32_t *X, const uint32_t *Y, const float *VX, const float *VY,
                            const float *VZ, const int32_t *bcnd, TallyDev *tal, const DevCounters *cnt, int sp,
                            int *keys, int *counts) {
    const long long n = cnt->n_slots[sp];
    const long long ng = (n + 3) / 4;
    for (long long g0 = blockIdx.x * (long long)blockDim.x; g0 < ng; g0 += (long long)gridDim.x * blockDim.x) {
        const long long g = g0 + threadIdx.x;
        int key[4] = {-1, -1, -1, -1};
        if (g < ng) {
            const long long i = 4 * g;
            const uint4 x = *reinterpret_cast<const uint4 *>(X + i);
            const uint4 y = *reinterpret_cast<const uint4 *>(Y + i);
            const float4 v = *reinterpret_cast<const float4 *>(VX + i);
            const uint32_t xs[4] = {x.x, x.y, x.z, x.w}, ys[4] = {y.x, y.y, y.z, y.w};
            const float vs[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int p = 0; p < 4; p++) {
                if (i + p >= n) break;
                if (!isnan(vs[p])) key[p] = cell_key(K, xs[p], ys[p]);
                else loss_hole_tally(tal, sp, bcnd, vs[p], xs[p], ys[p], VY[i + p], VZ[i + p]);
            }
            if (i + 4 <= n) {
                *reinterpret_cast<int4 *>(keys + i) = make_int4(key[0], key[1], key[2], key[3]);
            } else {
                for (int p = 0; p < 4 && i + p < n; p++) keys[i + p] = key[p];
            }
        }
        const unsigned lane = threadIdx.x & 31;
#pragma unroll
        for (int p = 0; p < 4; p++) {
            const unsigned m = __match_any_sync(0xffffffffu, key[p]);
            if (key[p] >= 0 && lane == (unsigned)(__ffs(m) - 1)) atomicAdd(&counts[key[p]], __popc(m));
        }
    }
}

// three-phase exclusive scan of counts[0..n) into offsets[0..n], offsets[n] = total
#define SCAN_ITEMS 2048
__global__ void k_scan_blocks(const int *counts, long long n, int *blocksums) {
    __shared__ int s[SORT_THREADS];
    long long base = (long long)blockIdx.x * SCAN_ITEMS;
    int a = 0;
    for (int k = threadIdx.x; k < SCAN_ITEMS; k += blockDim.x) {
        long long i = base + k;
        if (i < n) a += counts[i];
    }
    s[threadIdx.x] = a;
    __syncthreads();
    for (int w = SORT_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) blocksums[blockIdx.x] = s[0];
}
__global__ void k_scan_top(int *blocksums, int nb) { // single block, in place, exclusive
    __shared__ int s[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        int i = base + threadIdx.x;
        int v = (i < nb) ? blocksums[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            int t = ((int)threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        int incl = s[threadIdx.x];
        if (i < nb) blocksums[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += incl;
        __syncthreads();
    }
}
__global__ void k_scan_final(const int *counts, long long n, const int *blocksums, int *offsets) {
    __shared__ int s[SORT_THREADS];
    __shared__ int carry;
    long long base = (long long)blockIdx.x * SCAN_ITEMS;
    if (threadIdx.x == 0) carry = blocksums[blockIdx.x];
    __syncthreads();
    for (int k0 = 0; k0 < SCAN_ITEMS; k0 += blockDim.x) {
        long long i = base + k0 + threadIdx.x;
        int v = (i < n) ? counts[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < SORT_THREADS; o <<= 1) {
            int t = ((int)threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        int incl = s[threadIdx.x];
        if (i < n) offsets[i] = carry + incl - v;
        if (i == n - 1) offsets[n] = carry + incl;
        __syncthreads();
        if (threadIdx.x == SORT_THREADS - 1) carry += incl;
        __syncthreads();
    }
}

// Each warp scatters one work unit in slot order: a work item of the previous sort (the slots of
// one old tile, or a part of it) or a SCATTER_CHUNK-slot chunk of the tail appended since.  A
// particle that changed cell inside its old tile is met by the same warp in slot order as the
// particles of its new cell, so its position comes out in stable order; only a cell that
// receives particles from another work unit (a neighbouring tile, the tail) can come out of
// order, and the segment sort below checks every segment and sorts those.  (Fixed 1024-slot
// chunks cut every tile into pieces, so a particle moving to the next row of cells reached
// another chunk and nearly every electron cell needed the segment sort.)  Units are dispensed
// dynamically: the items' sizes follow the density.
#define SCATTER_CHUNK 1024
#define SCATTER_STEPS 8
__global__ void k_scatter(const int *keys, const WorkItem *items, DevCounters *cnt, int sp, int *cursor, int *perm) {
    const long long n = cnt->n_slots[sp];
    const long long ns = min(cnt->n_sorted[sp], n);
    const int ni = cnt->n_items[sp];
    const long long units = ni + (n - ns + SCATTER_CHUNK - 1) / SCATTER_CHUNK;
    const unsigned lane = threadIdx.x & 31;
    for (;;) {
        long long u = 0;
        if (lane == 0) u = (long long)atomicAdd(&cnt->scatter_next, 1u);
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= units) break;
        long long c0, c1;
        if (u < ni) {
            const WorkItem w = items[u];
            c0 = w.start;
            c1 = min((long long)w.end, ns);
        } else {
            c0 = ns + (u - ni) * SCATTER_CHUNK;
            c1 = min(c0 + SCATTER_CHUNK, n);
        }
        // SCATTER_STEPS 32-slot steps at a time: their atomics are in flight together (issued in
        // step order, so a key that runs across steps still receives ascending positions), and the
        // next iteration's keys are loaded before this one's atomics
        int nk[SCATTER_STEPS];
#pragma unroll
        for (int v = 0; v < SCATTER_STEPS; v++) {
            const long long i = c0 + 32 * v + lane;
            nk[v] = (i < c1) ? keys[i] : -1;
        }
        for (long long i0 = c0; i0 < c1; i0 += SCATTER_STEPS * 32) {
            int key[SCATTER_STEPS], base[SCATTER_STEPS];
            unsigned m[SCATTER_STEPS];
#pragma unroll
            for (int v = 0; v < SCATTER_STEPS; v++) {
                key[v] = nk[v];
                const long long i = i0 + SCATTER_STEPS * 32 + 32 * v + lane;
                nk[v] = (i < c1) ? keys[i] : -1;
            }
#pragma unroll
            for (int v = 0; v < SCATTER_STEPS; v++) {
                m[v] = __match_any_sync(0xffffffffu, key[v]);
                base[v] = 0;
                if (key[v] >= 0 && (int)lane == __ffs(m[v]) - 1) base[v] = atomicAdd(&cursor[key[v]], __popc(m[v]));
            }
#pragma unroll
            for (int v = 0; v < SCATTER_STEPS; v++) {
                const int b = __shfl_sync(m[v], base[v], __ffs(m[v]) - 1);
                if (key[v] >= 0) perm[b + __popc(m[v] & ((1u << lane) - 1u))] = (int)(i0 + 32 * v + lane);
            }
        }
    }
}

// ascending bitonic sort of 64 values held two per lane (index lane and lane + 32), padded with
// INT_MAX; the compare-exchange partner of index i at stride j is i ^ j: a shuffle for j < 32,
// the lane's other register for j = 32
__device__ __forceinline__ void warp_sort64(int &v0, int &v1, int lane) {
#pragma unroll
    for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j == 32) {
                const int lo = min(v0, v1), hi = max(v0, v1);
                v0 = lo;
                v1 = hi;
            } else {
                const int p0 = __shfl_xor_sync(0xffffffffu, v0, j);
                const int p1 = __shfl_xor_sync(0xffffffffu, v1, j);
                const bool lower = (lane & j) == 0;
                const bool asc0 = (lane & k) == 0, asc1 = ((lane + 32) & k) == 0;
                v0 = (lower == asc0) ? min(v0, p0) : max(v0, p0);
                v1 = (lower == asc1) ? min(v1, p1) : max(v1, p1);
            }
        }
    }
}

// A warp takes 32 consecutive segments: one coalesced load of their bounds, then one pass over
// their slot lists in 32-wide steps that marks each segment holding a descending adjacent pair
// (the segment of a position is found by a binary search over the 32 bounds held in the lanes);
// only the marked segments are sorted: up to 64 slots in registers, up to SEG_WARP_MAX in the
// warp's shared memory, longer ones listed for k_segsort_big.  (One segment per warp, each with
// its own dependent loads of bounds and slots, was latency-bound on the segments in order.)
__global__ void k_segsort_warp(const int *offsets, long long nkeys, int *perm, int *bigseg,
                               DevCounters *cnt) {
    __shared__ int buf[SORT_THREADS / 32][SEG_WARP_MAX];
    const unsigned full = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long ngroups = (nkeys + 31) / 32;
    for (long long gi = gw; gi < ngroups; gi += nw) {
        const long long k = gi * 32 + lane;
        const int s0 = offsets[k < nkeys ? k : nkeys];
        const int s1 = offsets[k < nkeys ? k + 1 : nkeys];
        const int S0 = __shfl_sync(full, s0, 0), S1 = __shfl_sync(full, s1, 31);
        unsigned dirty = 0;
        for (int q0 = S0; q0 < S1 - 1; q0 += 32 * SEG_CHECK_STEPS) {   // the pairs (q, q+1)
            int a[SEG_CHECK_STEPS], b[SEG_CHECK_STEPS];
#pragma unroll
            for (int u = 0; u < SEG_CHECK_STEPS; u++) {   // every step's loads in flight together
                const int q = q0 + 32 * u + lane;
                a[u] = 0; b[u] = 0;
                if (q < S1 - 1) { a[u] = perm[q]; b[u] = perm[q + 1]; }
            }
            unsigned mark = 0;
#pragma unroll
            for (int u = 0; u < SEG_CHECK_STEPS; u++) {
                const int q = q0 + 32 * u + lane;
                int lo = 0;                                // the last lane whose segment starts at or before q
#pragma unroll
                for (int st = 16; st > 0; st >>= 1) {
                    const int sv = __shfl_sync(full, s0, lo + st);
                    if (sv <= q) lo += st;
                }
                const int e = __shfl_sync(full, s1, lo);
                if (q < S1 - 1 && a[u] > b[u] && q + 1 < e) mark |= 1u << lo;
            }
            dirty |= __reduce_or_sync(full, mark);
        }
        while (dirty) {
            const int l = __ffs(dirty) - 1;
            dirty &= dirty - 1;
            const int t0 = __shfl_sync(full, s0, l), n = __shfl_sync(full, s1, l) - t0;
            if (n <= 64) {   // in registers
                int v0 = lane < n ? perm[t0 + lane] : INT_MAX;
                int v1 = lane + 32 < n ? perm[t0 + lane + 32] : INT_MAX;
                warp_sort64(v0, v1, lane);
                if (lane < n) perm[t0 + lane] = v0;
                if (lane + 32 < n) perm[t0 + lane + 32] = v1;
            } else if (n <= SEG_WARP_MAX) {
                int *a = buf[warp];
                for (int q = lane; q < n; q += 32) a[q] = perm[t0 + q];
                __syncwarp();
                bitonic_sort(a, n, lane, 32, WarpSync());
                for (int q = lane; q < n; q += 32) perm[t0 + q] = a[q];
                __syncwarp();
            } else if (lane == 0) {
                const int slot = atomicAdd(&cnt->n_big, 1);
                bigseg[slot] = (int)(gi * 32 + l);
            }
        }
    }
}

__global__ void k_segsort_big(const int *offsets, int *perm, const int *bigseg, const DevCounters *cnt) {
    __shared__ int a[SEG_BLOCK_MAX];
    const int nbig = cnt->n_big;
    for (int s = blockIdx.x; s < nbig; s += gridDim.x) {
        int k = bigseg[s];
        int s0 = offsets[k], n = offsets[k + 1] - s0;
        if (n <= SEG_BLOCK_MAX) {
            for (int q = threadIdx.x; q < n; q += blockDim.x) a[q] = perm[s0 + q];
            __syncthreads();
            bitonic_sort(a, n, threadIdx.x, blockDim.x, BlockSync());
            for (int q = threadIdx.x; q < n; q += blockDim.x) perm[s0 + q] = a[q];
        } else {
            bitonic_sort(perm + s0, n, threadIdx.x, blockDim.x, BlockSync());
        }
        __syncthreads();
    }
}

// four consecutive outputs per thread: one 16-byte permutation load, twenty independent
// gathers, 16-byte stores (the slot arrays are allocated in whole groups of 8)
__global__ void k_gather(const int *perm, const int *offsets, long long nkeys, const uint32_t *X,
                         const uint32_t *Y, const float *VX, const float *VY, const float *VZ,
                         uint32_t *X2, uint32_t *Y2, float *VX2, float *VY2, float *VZ2, const float *Z,
                         float *Z2) {
    const long long n = offsets[nkeys];
    const long long ng = (n + 3) / 4;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ng;
         g += (long long)gridDim.x * blockDim.x) {
        const long long j = 4 * g;
        if (j + 4 <= n) {
            const int4 p = *reinterpret_cast<const int4 *>(perm + j);
            const uint4 x = make_uint4(X[p.x], X[p.y], X[p.z], X[p.w]);
            const uint4 y = make_uint4(Y[p.x], Y[p.y], Y[p.z], Y[p.w]);
            const float4 a = make_float4(VX[p.x], VX[p.y], VX[p.z], VX[p.w]);
            const float4 b = make_float4(VY[p.x], VY[p.y], VY[p.z], VY[p.w]);
            const float4 c = make_float4(VZ[p.x], VZ[p.y], VZ[p.z], VZ[p.w]);
            *reinterpret_cast<uint4 *>(X2 + j) = x;
            *reinterpret_cast<uint4 *>(Y2 + j) = y;
            *reinterpret_cast<float4 *>(VX2 + j) = a;
            *reinterpret_cast<float4 *>(VY2 + j) = b;
            *reinterpret_cast<float4 *>(VZ2 + j) = c;
            if (Z) *reinterpret_cast<float4 *>(Z2 + j) = make_float4(Z[p.x], Z[p.y], Z[p.z], Z[p.w]);
        } else {
            for (long long q = j; q < n; q++) {
                const int i = perm[q];
                X2[q] = X[i]; Y2[q] = Y[i]; VX2[q] = VX[i]; VY2[q] = VY[i]; VZ2[q] = VZ[i];
                if (Z) Z2[q] = Z[i];
            }
        }
    }
}

// per tile: ceil(count / CHUNK) work items; single block, fixed order
__global__ void k_items(const int *offsets, int ntiles, int keys_per_tile, WorkItem *items,
                        int max_items, DevCounters *cnt, int sp, long long nkeys) {
    __shared__ int s[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ntiles; base += 1024) {
        int t = base + threadIdx.x;
        int st = 0, en = 0, ni = 0;
        if (t < ntiles) {
            st = offsets[(long long)t * keys_per_tile];
            en = offsets[(long long)(t + 1) * keys_per_tile];
            ni = (en - st + PUSH_CHUNK - 1) / PUSH_CHUNK;
        }
        s[threadIdx.x] = ni;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            int v = ((int)threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += v;
            __syncthreads();
        }
        int first = carry + s[threadIdx.x] - ni;
        for (int q = 0; q < ni; q++) {
            int idx = first + q;
            if (idx < max_items) {
                WorkItem w;
                w.tile = t;
                w.start = st + q * PUSH_CHUNK;
                w.end = min(en, st + (q + 1) * PUSH_CHUNK);
                w.pad = 0;
                items[idx] = w;
            }
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry += s[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        int nitems = carry;
        if (nitems > max_items) { set_err(cnt, LERR_CAPACITY, 300); nitems = max_items; }
        long long total = offsets[nkeys];
        cnt->ind_old[sp] = cnt->n_slots[sp];
        cnt->n_items[sp] = nitems;
        cnt->n_slots[sp] = total;
        cnt->n_sorted[sp] = total;
        cnt->n_alive[sp] = total;
    }
}

int sort_species(lepic_ctx *c, int sp, bool defer) {
    SpeciesBuf &B = c->sp[sp];
    const int cur = B.cur, nxt = 1 - cur;
    auto log2_or = [](int v) { int l = 0; while ((1 << l) < v) l++; return (1 << l) == v ? l : -1; };
    KeyP K{c->S, c->cfg.nx, c->cfg.ny, c->tw, c->th, c->ntx, log2_or(c->tw), log2_or(c->th)};
    if (K.twl < 0 || K.thl < 0) K.twl = K.thl = -1;
    if (B.ind) {   // a permutation still pending: move its records first
        int r = materialize_species(c, sp);
        if (r != LEPIC_OK) return r;
        return sort_species(c, sp, defer);
    }
    if (defer && B.Z[0]) defer = false;   // the push that ends the pending state does not carry z
    if (!B.ordered) defer = false;         // a random order: the gather streams, the push would not
    if ((defer || c->opt.sort_defer == 1) && !B.pind) {
        // at the species' first sort, deferred or not (after a load the first one is not): the
        // permutation's buffer and the mover that reads through it are ready before the time
        // loop, whose first deferred sort would otherwise allocate (a device-wide wait while
        // the driver maps and clears 4 B per slot) and whose next push would load a kernel
        if (cudaMalloc((void **)&B.pind, sizeof(int) * (size_t)std::max(B.cap, 8ll)) != cudaSuccess) {
            c->last_err = "sort: cudaMalloc of the pending permutation failed";
            return LEPIC_ENOMEM;
        }
        const int r = push_preload_ind(c, sp);
        if (r != LEPIC_OK) return r;
    }
    int *perm = defer ? B.pind : c->perm;
    const long long nk = c->nkeys;
    int grid = c->num_sms * 8;
    LCUDA(cudaMemsetAsync(c->counts, 0, sizeof(int) * (nk + 1), c->stream));
    LCUDA(cudaMemsetAsync(&c->dcnt->n_big, 0, sizeof(int), c->stream));
    LCUDA(cudaMemsetAsync(&c->dcnt->scatter_next, 0, sizeof(unsigned int), c->stream));
    k_keys_hist<<<grid, SORT_THREADS, 0, c->stream>>>(K, B.X[cur], B.Y[cur], B.VX[cur], B.VY[cur], B.VZ[cur],
                                                        c->bcnd, c->tally, c->dcnt, sp, c->keys, c->counts);
    int nb = div_up(nk, SCAN_ITEMS);
    k_scan_blocks<<<nb, SORT_THREADS, 0, c->stream>>>(c->counts, nk, c->blocksums);
    k_scan_top<<<1, 1024, 0, c->stream>>>(c->blocksums, nb);
    k_scan_final<<<nb, SORT_THREADS, 0, c->stream>>>(c->counts, nk, c->blocksums, c->offsets);
    LCUDA(cudaMemcpyAsync(c->cursor, c->offsets, sizeof(int) * nk, cudaMemcpyDeviceToDevice, c->stream));
    k_scatter<<<grid, SORT_THREADS, 0, c->stream>>>(c->keys, B.items, c->dcnt, sp, c->cursor, perm);
    k_segsort_warp<<<grid, SORT_THREADS, 0, c->stream>>>(c->offsets, nk, perm, c->bigseg, c->dcnt);
    k_segsort_big<<<c->num_sms, 512, 0, c->stream>>>(c->offsets, perm, c->bigseg, c->dcnt);
    if (!defer)
        k_gather<<<grid, SORT_THREADS, 0, c->stream>>>(perm, c->offsets, nk, B.X[cur], B.Y[cur], B.VX[cur],
                                                       B.VY[cur], B.VZ[cur], B.X[nxt], B.Y[nxt], B.VX[nxt],
                                                       B.VY[nxt], B.VZ[nxt], B.Z[cur], B.Z[nxt]);
    k_items<<<1, 1024, 0, c->stream>>>(c->offsets, c->ntiles, c->tw * c->th, B.items, B.max_items,
                                       c->dcnt, sp, nk);
    LCUDA(cudaGetLastError());
    // the cell lists of this order (sorting.f90's Plist) for the DSMC target search
    if (B.cell_off)
        LCUDA(cudaMemcpyAsync(B.cell_off, c->offsets, sizeof(int) * (nk + 1), cudaMemcpyDeviceToDevice, c->stream));
    if (defer) B.ind = true;   // the records stay in buffer cur until the push
    else B.cur = nxt;
    B.ordered = true;
    return LEPIC_OK;
}

// the gather of a pending permutation over every position of the sorted order, the products
// appended since included; holes are carried as they are (the next sort drops them)
__global__ void k_gather_ind(const int *pind, const DevCounters *cnt, int sp, const uint32_t *X, const uint32_t *Y,
                             const float *VX, const float *VY, const float *VZ, uint32_t *X2, uint32_t *Y2,
                             float *VX2, float *VY2, float *VZ2) {
    const long long n = cnt->n_slots[sp], ns = cnt->n_sorted[sp], old = cnt->ind_old[sp];
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const long long i = ind_slot(pind, ns, old, j);
        X2[j] = X[i]; Y2[j] = Y[i]; VX2[j] = VX[i]; VY2[j] = VY[i]; VZ2[j] = VZ[i];
    }
}

int materialize_species(lepic_ctx *c, int sp) {
    SpeciesBuf &B = c->sp[sp];
    if (!B.ind) return LEPIC_OK;
    const int cur = B.cur, nxt = 1 - cur;
    k_gather_ind<<<c->num_sms * 8, SORT_THREADS, 0, c->stream>>>(B.pind, c->dcnt, sp, B.X[cur], B.Y[cur], B.VX[cur],
                                                                  B.VY[cur], B.VZ[cur], B.X[nxt], B.Y[nxt],
                                                                  B.VX[nxt], B.VY[nxt], B.VZ[nxt]);
    LCUDA(cudaGetLastError());
    B.cur = nxt;
    B.ind = false;
    return LEPIC_OK;
}

int materialize_all(lepic_ctx *c) {
    for (int s = 0; s < c->cfg.ntype; s++) {
        const int r = materialize_species(c, s);
        if (r != LEPIC_OK) return r;
    }
    return LEPIC_OK;
}
