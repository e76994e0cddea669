// backup.cu -- the particle backup of main.f90:1102-1139 and its reader restart.f90:48-149,
// streamed between the device's structure-of-arrays particles and the reference's file.
//
// File: Fortran unformatted sequential records (4-byte little-endian length markers before
// and after each record), as the reference's compilers write them:
//   (time, gtype, Pabs_cor)                      real(8), integer(4), real(8)
//   np_tot(1:ntype, 1:nproc)                     integer(4)
//   vxp(1:6, 1:np_tot(ptype,iproc)) per iproc, ptype (iproc outer)   real(8)
// A record longer than 2^31 - 9 bytes is split into subrecords: the leading marker of every
// subrecord but the last is negative, the trailing marker of every subrecord but the first
// (the convention of the Intel and GNU Fortran runtimes).
//
// Device side: live particles are packed in slot order (holes skipped) into FP64 vxp(6, n)
// chunks -- a count of live particles per 1024-slot block, its prefix sum on the host, one
// packing kernel per chunk -- copied to pinned host buffers (two, alternating, so that the
// next chunk is packed and copied while the host writes the previous one).  z is not kept on
// the device and is written as 0.  Reading unpacks FP64 chunks into the fixed-point and FP32
// arrays after the occupied slots, then deposits every species (restart_OMP).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "lepic_internal.cuh"

#define BK_BLOCK 1024                 // slots per counting block
#define BK_CHUNK (1ll << 22)          // slots per packing chunk (a multiple of BK_BLOCK)
static const long long kMaxSub = 2147483639ll;  // the runtimes' largest subrecord

// live particles per BK_BLOCK slots
__global__ void k_live_counts(const float *VX, long long n, int *counts) {
    __shared__ int s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * BK_BLOCK;
    int c = 0;
    for (int t = threadIdx.x; t < BK_BLOCK; t += blockDim.x) {
        const long long i = base + t;
        if (i < n && !isnan(VX[i])) c++;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s, c);
    __syncthreads();
    if (threadIdx.x == 0) counts[blockIdx.x] = s;
}

// packs the live particles of blocks [b0, b0 + nb) into out (vxp(6, .) from offset
// off[b] - off[b0] of block b), in slot order
__global__ void __launch_bounds__(BK_BLOCK) k_pack(const uint32_t *X, const uint32_t *Y, const float *VX,
                                                  const float *VY, const float *VZ, const float *Z, long long n,
                                                  long long b0, const long long *off, double ux, double uy,
                                                  double *out) {
    __shared__ int wsum[BK_BLOCK / 32];
    const long long b = b0 + blockIdx.x;
    const long long i = b * BK_BLOCK + threadIdx.x;
    const float vx = i < n ? VX[i] : __int_as_float(HOLE_NAN);
    const bool live = !isnan(vx);
    const unsigned m = __ballot_sync(0xffffffffu, live);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wsum[w] = __popc(m);
    __syncthreads();
    int pre = 0;
    for (int k = 0; k < w; k++) pre += wsum[k];
    if (!live) return;
    const long long o = off[b] - off[b0] + pre + __popc(m & ((1u << lane) - 1u));
    double *p = out + 6 * o;
    p[0] = (double)X[i] * ux;   // as lepic_gpu_get_particles
    p[1] = (double)Y[i] * uy;
    p[2] = Z ? (double)Z[i] : 0.0;   // z: the 3rd dimension's, else 0
    p[3] = vx;
    p[4] = VY[i];
    p[5] = VZ[i];
}

// unpacks n FP64 particles into the slots from dst (as lepic_gpu_put_particles); a particle
// outside the box raises LERR_RANGE and becomes a hole
__global__ void k_unpack(const double *in, long long n, long long dst, double sx, double sy, long long xl,
                         long long yl, uint32_t *X, uint32_t *Y, float *VX, float *VY, float *VZ, float *Z,
                         DevCounters *cnt) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const double *p = in + 6 * k;
        const long long xi = llrint(p[0] * sx), yi = llrint(p[1] * sy);
        const long long s = dst + k;
        if (!(xi >= 0 && xi < xl && yi >= 0 && yi < yl) || !(p[3] == p[3])) {
            set_err(cnt, LERR_RANGE, 800);
            X[s] = 0; Y[s] = 0; VX[s] = __int_as_float(HOLE_NAN); VY[s] = 0.f; VZ[s] = 0.f;
            continue;
        }
        X[s] = (uint32_t)xi; Y[s] = (uint32_t)yi;
        VX[s] = (float)p[3]; VY[s] = (float)p[4]; VZ[s] = (float)p[5];
        if (Z) Z[s] = (float)p[2];
    }
}

// ---------------------------------------------------------------------------------------
// Fortran sequential records with subrecords
struct RecWriter {
    FILE *f = nullptr;
    long long left = 0, sub_left = 0;   // bytes of the record / of the current subrecord
    bool first = true, ok = true;
    long long max_sub = kMaxSub;
    void marker(long long v) {
        const int32_t m = (int32_t)v;
        ok = ok && fwrite(&m, 4, 1, f) == 1;
    }
    void begin(long long len) {
        left = len;
        first = true;
        if (len == 0) {  // an empty record: both markers at once
            marker(0);
            marker(0);
            sub_left = 0;
            return;
        }
        open_sub();
    }
    void open_sub() {
        sub_left = std::min(left, max_sub);
        marker(sub_left < left ? -sub_left : sub_left);   // negative: more subrecords follow
    }
    void write(const void *p, long long nbytes) {
        const char *c = (const char *)p;
        while (nbytes > 0 && ok) {
            const long long k = std::min(nbytes, sub_left);
            ok = ok && fwrite(c, 1, (size_t)k, f) == (size_t)k;
            c += k; nbytes -= k; sub_left -= k;
            if (sub_left == 0) close_sub();
        }
    }
    void close_sub() {
        const long long len = std::min(left, max_sub);
        marker(first ? len : -len);                       // negative: continues a subrecord
        left -= len;
        first = false;
        if (left > 0) open_sub();
    }
    void end() {
        if (left == 0 && sub_left == 0) return;
        ok = false;  // wrote fewer bytes than announced
    }
};

struct RecReader {
    FILE *f = nullptr;
    long long sub_left = 0;
    bool last = true, ok = true;
    bool marker(int32_t *m) { return fread(m, 4, 1, f) == 1; }
    // starts a record: sub_left is the first subrecord's length, last whether it is the only one
    bool begin() {
        int32_t m;
        if (!marker(&m)) return ok = false;
        sub_left = std::llabs((long long)m);
        last = m >= 0;
        return true;
    }
    // reads nbytes of the record's data, across subrecords
    bool read(void *p, long long nbytes) {
        char *c = (char *)p;
        while (nbytes > 0) {
            if (sub_left == 0) {
                if (last) return ok = false;  // past the end of the record
                int32_t t, h;
                if (!marker(&t) || !marker(&h)) return ok = false;
                sub_left = std::llabs((long long)h);
                last = h >= 0;
            }
            const long long k = std::min(nbytes, sub_left);
            if (fread(c, 1, (size_t)k, f) != (size_t)k) return ok = false;
            c += k; nbytes -= k; sub_left -= k;
        }
        return true;
    }
    // the record must end here
    bool end() {
        if (sub_left != 0 || !last) return ok = false;
        int32_t t;
        return ok = ok && marker(&t);
    }
};

// a smaller subrecord limit (lepic_options::fortran_max_subrecord) exercises the
// multi-subrecord layout with small files
static long long max_subrecord(const lepic_ctx *c) {
    const long long v = c->opt.fortran_max_subrecord;
    return (v >= 8 && v <= kMaxSub) ? v : kMaxSub;
}

// ---------------------------------------------------------------------------------------
extern "C" int lepic_gpu_write_backup(lepic_ctx *c, const char *path, double time, int32_t gtype, double Pabs_cor) {
    if (!c || !path) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    int r = lepic_gpu_sync(c);
    if (r != LEPIC_OK) return r;
    const lepic_config &g = c->cfg;
    // live particles per species and block
    std::vector<std::vector<long long>> offs(g.ntype);
    std::vector<int32_t> np_tot(g.ntype);
    long long max_blocks = 1;
    for (int s = 0; s < g.ntype; s++) max_blocks = std::max<long long>(max_blocks, div_up(c->hcnt->n_slots[s], BK_BLOCK));
    int *d_counts = nullptr;
    long long *d_off = nullptr;
    double *d_out = nullptr;
    double *h_buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    FILE *f = nullptr;
    auto cleanup = [&]() {
        if (d_counts) cudaFree(d_counts);
        if (d_off) cudaFree(d_off);
        if (d_out) cudaFree(d_out);
        for (int k = 0; k < 2; k++) {
            if (h_buf[k]) cudaFreeHost(h_buf[k]);
            if (ev[k]) cudaEventDestroy(ev[k]);
        }
        if (f) fclose(f);
    };
#define BK_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t _e = (call);                                                                   \
        if (_e != cudaSuccess) {                                                                   \
            c->last_err = std::string(#call) + ": " + cudaGetErrorString(_e);                     \
            cleanup();                                                                             \
            return LEPIC_ECUDA;                                                                    \
        }                                                                                          \
    } while (0)
    BK_CUDA(cudaMalloc((void **)&d_counts, sizeof(int) * max_blocks));
    BK_CUDA(cudaMalloc((void **)&d_off, sizeof(long long) * (max_blocks + 1)));
    BK_CUDA(cudaMalloc((void **)&d_out, sizeof(double) * 6 * BK_CHUNK));
    for (int k = 0; k < 2; k++) {
        BK_CUDA(cudaMallocHost((void **)&h_buf[k], sizeof(double) * 6 * BK_CHUNK));
        BK_CUDA(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
    }
    for (int s = 0; s < g.ntype; s++) {
        const long long n = c->hcnt->n_slots[s];
        const long long nb = div_up(n, BK_BLOCK);
        SpeciesBuf &B = c->sp[s];
        std::vector<int> cnt(nb);
        if (nb > 0) {
            k_live_counts<<<(unsigned)nb, 256, 0, c->stream>>>(B.VX[B.cur], n, d_counts);
            BK_CUDA(cudaGetLastError());
            BK_CUDA(cudaMemcpyAsync(cnt.data(), d_counts, sizeof(int) * nb, cudaMemcpyDeviceToHost, c->stream));
            BK_CUDA(cudaStreamSynchronize(c->stream));
        }
        offs[s].assign(nb + 1, 0);
        for (long long b = 0; b < nb; b++) offs[s][b + 1] = offs[s][b] + cnt[b];
        if (offs[s][nb] > 2147483647ll) { c->last_err = "np_tot beyond integer(4)"; cleanup(); return LEPIC_ECAPACITY; }
        np_tot[s] = (int32_t)offs[s][nb];
    }
    f = fopen(path, "wb");
    if (!f) { c->last_err = std::string("cannot open ") + path; cleanup(); return LEPIC_EINVAL; }
    RecWriter w;
    w.f = f;
    w.max_sub = max_subrecord(c);
    w.begin(8 + 4 + 8);
    w.write(&time, 8); w.write(&gtype, 4); w.write(&Pabs_cor, 8);
    w.end();
    w.begin(4ll * g.ntype);
    w.write(np_tot.data(), 4ll * g.ntype);
    w.end();
    const double ux = g.dx * std::ldexp(1.0, -c->S), uy = g.dy * std::ldexp(1.0, -c->S);
    for (int s = 0; s < g.ntype && w.ok; s++) {
        SpeciesBuf &B = c->sp[s];
        const long long n = c->hcnt->n_slots[s];
        const long long nb = (long long)offs[s].size() - 1;
        w.begin(48ll * np_tot[s]);
        if (nb > 0) BK_CUDA(cudaMemcpyAsync(d_off, offs[s].data(), sizeof(long long) * (nb + 1), cudaMemcpyHostToDevice,
                                            c->stream));
        const long long blocks_per_chunk = BK_CHUNK / BK_BLOCK;
        long long pend_bytes[2] = {0, 0};
        int pend = -1;   // buffer waiting to be written
        int k = 0;
        for (long long b0 = 0; b0 < nb; b0 += blocks_per_chunk, k ^= 1) {
            const long long bn = std::min(blocks_per_chunk, nb - b0);
            const long long cnt = offs[s][b0 + bn] - offs[s][b0];
            k_pack<<<(unsigned)bn, BK_BLOCK, 0, c->stream>>>(B.X[B.cur], B.Y[B.cur], B.VX[B.cur], B.VY[B.cur],
                                                             B.VZ[B.cur], B.Z[B.cur], n, b0, d_off, ux, uy,
                                                             d_out);
            BK_CUDA(cudaGetLastError());
            if (pend == k) {  // the buffer this chunk goes to is still being written: finish it
                w.write(h_buf[k], pend_bytes[k]);
                pend = -1;
            }
            BK_CUDA(cudaMemcpyAsync(h_buf[k], d_out, sizeof(double) * 6 * cnt, cudaMemcpyDeviceToHost, c->stream));
            BK_CUDA(cudaEventRecord(ev[k], c->stream));
            if (pend == (k ^ 1)) {  // write the previous chunk while this one is copied
                w.write(h_buf[k ^ 1], pend_bytes[k ^ 1]);
                pend = -1;
            }
            BK_CUDA(cudaEventSynchronize(ev[k]));
            pend_bytes[k] = 48 * cnt;
            pend = k;
        }
        if (pend >= 0) w.write(h_buf[pend], pend_bytes[pend]);
        w.end();
    }
    const bool ok = w.ok;
    if (fclose(f) != 0 || !ok) {
        f = nullptr;
        c->last_err = std::string("write failed: ") + path;
        cleanup();
        return LEPIC_EINVAL;
    }
    f = nullptr;
    cleanup();
    return LEPIC_OK;
#undef BK_CUDA
}

extern "C" int lepic_gpu_read_backup(lepic_ctx *c, const char *path, double *time, int32_t *gtype, double *Pabs_cor) {
    if (!c || !path) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    int r = lepic_gpu_sync(c);
    if (r != LEPIC_OK) return r;
    const lepic_config &g = c->cfg;
    FILE *f = fopen(path, "rb");
    if (!f) { c->last_err = std::string("cannot open ") + path; return LEPIC_EINVAL; }
    RecReader rd;
    rd.f = f;
    double t = 0.0, pc = 0.0;
    int32_t gt = 0;
    bool ok = rd.begin() && rd.read(&t, 8) && rd.read(&gt, 4) && rd.read(&pc, 8) && rd.end();
    // np_tot(1:ntype, 1:nproc): nproc from the record length (single subrecord)
    std::vector<int32_t> np;
    if (ok) {
        ok = rd.begin() && rd.last && rd.sub_left % (4ll * g.ntype) == 0;
        if (ok) {
            np.resize((size_t)(rd.sub_left / 4));
            ok = rd.read(np.data(), rd.sub_left) && rd.end();
        }
    }
    if (!ok) { fclose(f); c->last_err = "backup header unreadable"; return LEPIC_EINVAL; }
    const int nproc = (int)(np.size() / g.ntype);
    std::vector<long long> want(g.ntype, 0), alive0(g.ntype);
    for (int s = 0; s < g.ntype; s++) alive0[s] = c->hcnt->n_alive[s];
    for (int p = 0; p < nproc; p++)
        for (int s = 0; s < g.ntype; s++) {
            if (np[(size_t)p * g.ntype + s] < 0) ok = false;
            want[s] += np[(size_t)p * g.ntype + s];
        }
    for (int s = 0; s < g.ntype && ok; s++)
        if (c->hcnt->n_slots[s] + want[s] > c->sp[s].cap) {
            fclose(f);
            c->last_err = "backup exceeds the particle capacity (restart.f90:117-121)";
            return LEPIC_ECAPACITY;
        }
    double *d_in = nullptr, *h_in = nullptr;
    if (cudaMalloc((void **)&d_in, sizeof(double) * 6 * BK_CHUNK) != cudaSuccess ||
        cudaMallocHost((void **)&h_in, sizeof(double) * 6 * BK_CHUNK) != cudaSuccess) {
        if (d_in) cudaFree(d_in);
        fclose(f);
        c->last_err = "read_backup: allocation failed";
        return LEPIC_ENOMEM;
    }
    const double sx = (double)(1u << c->S) / g.dx, sy = (double)(1u << c->S) / g.dy;
    const long long xl = (long long)g.nx << c->S, yl = (long long)g.ny << c->S;
    for (int p = 0; p < nproc && ok; p++)
        for (int s = 0; s < g.ntype && ok; s++) {
            const long long n = np[(size_t)p * g.ntype + s];
            SpeciesBuf &B = c->sp[s];
            const long long base = c->hcnt->n_slots[s];
            ok = rd.begin();
            for (long long k0 = 0; k0 < n && ok; k0 += BK_CHUNK) {
                const long long m = std::min(BK_CHUNK, n - k0);
                ok = rd.read(h_in, 48 * m);
                if (!ok) break;
                if (cudaMemcpyAsync(d_in, h_in, 48 * m, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) { ok = false; break; }
                k_unpack<<<(unsigned)std::min<long long>(div_up(m, 256), (long long)c->num_sms * 8), 256, 0, c->stream>>>(
                    d_in, m, base + k0, sx, sy, xl, yl, B.X[B.cur], B.Y[B.cur], B.VX[B.cur], B.VY[B.cur], B.VZ[B.cur],
                    B.Z[B.cur], c->dcnt);
                if (cudaStreamSynchronize(c->stream) != cudaSuccess) { ok = false; break; }
            }
            ok = ok && rd.end();
            c->hcnt->n_slots[s] = base + n;   // host mirror until the counters are written below
        }
    cudaFree(d_in);
    cudaFreeHost(h_in);
    fclose(f);
    if (!ok) { c->last_err = std::string("backup unreadable: ") + path; return LEPIC_EINVAL; }
    for (int s = 0; s < g.ntype; s++) {
        long long v = c->hcnt->n_slots[s], a = alive0[s] + want[s], zero = 0;
        LCUDA(cudaMemcpy(&c->dcnt->n_slots[s], &v, sizeof(v), cudaMemcpyHostToDevice));
        LCUDA(cudaMemcpy(&c->dcnt->n_alive[s], &a, sizeof(a), cudaMemcpyHostToDevice));
        LCUDA(cudaMemcpy(&c->dcnt->n_sorted[s], &zero, sizeof(zero), cudaMemcpyHostToDevice));
        int zi = 0;
        LCUDA(cudaMemcpy(&c->dcnt->n_items[s], &zi, sizeof(int), cudaMemcpyHostToDevice));
        c->sp[s].ordered = false;
    }
    if (time) *time = t;
    if (gtype) *gtype = gt;
    if (Pabs_cor) *Pabs_cor = pc;
    r = lepic_gpu_sync(c);
    if (r != LEPIC_OK) return r;
    return lepic_gpu_charge_deposition(c);  // restart_OMP: np of the loaded particles
}

// ---------------------------------------------------------------------------------------
// restart.f90:115-129: |np_dup| - 1 copies of every slot appended after the occupied slots
// (copy i of slot k at i * n + k).  A copied hole stays a plain hole (a loss record is tallied
// once, from the original).
__global__ void k_duplicate(long long n, int copies, uint32_t *X, uint32_t *Y, float *VX, float *VY, float *VZ,
                            float *Z) {
    const long long tot = n * (long long)copies;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const long long k = t % n, d = n + t;
        const float vx = VX[k];
        X[d] = X[k]; Y[d] = Y[k];
        VX[d] = isnan(vx) ? __int_as_float(HOLE_NAN) : vx;
        VY[d] = VY[k]; VZ[d] = VZ[k];
        if (Z) Z[d] = Z[k];
    }
}

extern "C" int lepic_gpu_duplicate_particles(lepic_ctx *c, int32_t np_dup) {
    if (!c) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    const int dup = np_dup < 0 ? -np_dup : np_dup;
    if (dup <= 1) return LEPIC_OK;
    int r = lepic_gpu_sync(c);
    if (r != LEPIC_OK) return r;
    const lepic_config &g = c->cfg;
    for (int s = 0; s < g.ntype; s++)   // restart.f90:117-121
        if ((long long)dup * c->hcnt->n_slots[s] > c->sp[s].cap) {
            c->last_err = "|np_dup| * np_tot exceeds the particle capacity (restart.f90:117-121)";
            return LEPIC_ECAPACITY;
        }
    for (int s = 0; s < g.ntype; s++) {
        SpeciesBuf &B = c->sp[s];
        const long long n = c->hcnt->n_slots[s];
        if (n > 0) {
            const long long tot = n * (dup - 1);
            k_duplicate<<<(unsigned)std::min<long long>(div_up(tot, 256), (long long)c->num_sms * 16), 256, 0,
                          c->stream>>>(n, dup - 1, B.X[B.cur], B.Y[B.cur], B.VX[B.cur], B.VY[B.cur], B.VZ[B.cur],
                                       B.Z[B.cur]);
            LCUDA(cudaGetLastError());
        }
        const long long slots = n * dup, alive = c->hcnt->n_alive[s] * dup;
        LCUDA(cudaMemcpyAsync(&c->dcnt->n_slots[s], &slots, sizeof(slots), cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaMemcpyAsync(&c->dcnt->n_alive[s], &alive, sizeof(alive), cudaMemcpyHostToDevice, c->stream));
        LCUDA(cudaStreamSynchronize(c->stream));   // the host values above are locals
    }
    r = lepic_gpu_sync(c);
    if (r != LEPIC_OK) return r;
    return lepic_gpu_charge_deposition(c);  // restart_OMP: np of every particle
}
