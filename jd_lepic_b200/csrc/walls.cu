// walls.cu -- the boundary models of the mover beyond its plain walls: dielectric walls and
// secondary emission (below; the push does the per-particle part) and
// the 3rd virtual dimension of the 2.5D model (hz >= 0 in the deck,
// read_input.f90:158-162; part_expmover.f90:216-219, 269-309, 400-421): its set-up and its Bohm
// speed map.  The losses themselves happen in the push (push.cu, the general mover).
//
//   electrons and negative ions: z moves with vz; at z <= 0 or z >= zmax a particle whose
//     z-energy 0.5 m vz^2 / qe reaches phi(ix,iy) - phi0 is lost through the end plate, any
//     other is reflected (vz -> -vz, z -> 0.02 zmax or 0.98 zmax)
//   positive ions: lost with probability hz 2 uB(ix_c,iy_c) / zmax * dt per step, uB the Bohm
//     speed sqrt(qe Te / m) on the averaging grid, Te the averaged electron temperature
//     (main.f90:950-960); the draw is a counter-based stream keyed by (seed, step, species, slot)
// A loss of this kind has no wall label (p_mac's igrid 0) and adds Nm q phi at the loss point to
// P_loss(1) besides its kinetic energy (part_expmover.f90:400-421).
#include <algorithm>
#include <cstring>
#include <vector>
#include "lepic_internal.cuh"

struct Dtype { int32_t v[LEPIC_MAXLABEL]; };   // the wall labels' types, passed by value

__global__ void k_zinit(float *Z, long long n, double zmax, uint32_t k0, uint32_t k1, uint32_t sp) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const U4 q = philox4x32_10(U4{(uint32_t)i, sp, 0x5A494E49u, (uint32_t)(i >> 32)}, k0, k1);
        Z[i] = (float)(u01(q.x) * zmax);
    }
}

// main.f90:950-960: uB(ix,iy,ptype) = sqrt(qe Te / m(ptype)), Te = data_pavg(2,ix,iy,1)/cnt_avg,
// for the ions (ptype >= 2)
__global__ void k_ub_from_avg(const double *data, int nodes, int cnt, double qe, double m, float *uB) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nodes; t += gridDim.x * blockDim.x) {
        const double Te = data[7 * t + 1] / (double)cnt;   // column 2 of species 1 (electrons)
        uB[t] = (float)sqrt(qe * fmax(Te, 0.0) / m);
    }
}

int zloss_after_avg(lepic_ctx *c, const double *data, int na1, int na2, int size_na, int cnt) {
    if (!c->zloss || !c->uB || size_na != c->zsize_na || na1 != c->za1 || na2 != c->za2 || cnt <= 0)
        return LEPIC_OK;
    const int nodes = (na1 + 1) * (na2 + 1);
    for (int s = 1; s < c->cfg.ntype; s++) {
        k_ub_from_avg<<<std::max(1, std::min(div_up(nodes, 256), c->num_sms * 4)), 256, 0, c->stream>>>(
            data, nodes, cnt, c->cfg.qe, std::fabs(c->cfg.mass[s]), c->uB + (size_t)s * nodes);
        LCUDA(cudaGetLastError());
    }
    return LEPIC_OK;
}

extern "C" int lepic_gpu_set_zloss(lepic_ctx *c, const lepic_zloss_config *z) {
    if (!c || !z) return LEPIC_EINVAL;
    if (const int rm = materialize_all(c)) return rm;   // records of a pending sort moved first
    const lepic_config &g = c->cfg;
    if (z->hz < 0.0) {   // the reference's "no losses in the 3rd dimension" (read_input.f90:162)
        c->zloss = 0;
        return LEPIC_OK;
    }
    if (z->size_na < 1 || g.nx % z->size_na || g.ny % z->size_na || !(g.zmax > 0.0)) {
        c->last_err = "set_zloss: size_na must divide nx and ny, zmax must be positive";
        return LEPIC_EINVAL;
    }
    int r = lepic_gpu_sync(c);
    if (r != LEPIC_OK) return r;
    const uint32_t k0 = (uint32_t)g.seed, k1 = (uint32_t)(g.seed >> 32) ^ 0x5A5A1234u;
    for (int s = 0; s < g.ntype; s++) {
        SpeciesBuf &B = c->sp[s];
        if (!B.Z[0]) {
            const size_t cap8 = (size_t)((B.cap + 7) / 8) * 8;
            for (int k = 0; k < 2; k++) {
                if (cudaMalloc((void **)&B.Z[k], sizeof(float) * cap8) != cudaSuccess) {
                    c->last_err = "set_zloss: cudaMalloc failed";
                    return LEPIC_ENOMEM;
                }
                LCUDA(cudaMemsetAsync(B.Z[k], 0, sizeof(float) * cap8, c->stream));
            }
            const long long n = c->hcnt->n_slots[s];   // the particles already there: z = rnd zmax
            if (n > 0) {
                k_zinit<<<(unsigned)std::min<long long>(div_up(n, 256), (long long)c->num_sms * 8), 256, 0, c->stream>>>(
                    B.Z[B.cur], n, g.zmax, k0, k1, (uint32_t)s);
                LCUDA(cudaGetLastError());
            }
        }
    }
    const int na1 = g.nx / z->size_na, na2 = g.ny / z->size_na;
    if (!c->uB || na1 != c->za1 || na2 != c->za2) {
        if (c->uB) cudaFree(c->uB);
        c->uB = nullptr;
        const size_t nb = sizeof(float) * (size_t)(na1 + 1) * (na2 + 1) * g.ntype;
        if (cudaMalloc((void **)&c->uB, nb) != cudaSuccess) {
            c->last_err = "set_zloss: cudaMalloc failed";
            return LEPIC_ENOMEM;
        }
        LCUDA(cudaMemsetAsync(c->uB, 0, nb, c->stream));
    }
    c->za1 = na1; c->za2 = na2; c->zsize_na = z->size_na;
    c->hz = z->hz;
    c->phi0_end = z->phi0;
    c->zloss = 1;
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

extern "C" int lepic_gpu_set_bohm_speed(lepic_ctx *c, const double *uB) {
    if (!c || !uB || !c->zloss || !c->uB) return LEPIC_EINVAL;
    const size_t n = (size_t)(c->za1 + 1) * (c->za2 + 1) * c->cfg.ntype;
    std::vector<float> f(n);
    for (size_t k = 0; k < n; k++) f[k] = (float)uB[k];
    LCUDA(cudaMemcpyAsync(c->uB, f.data(), sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

// ---------------------------------------------------------------------------------------
// Dielectric walls (generate_boundary.f90:149-152: a vertical wall drawn as dielectric;
// part_expmover.f90:340-350; main.f90:756-809).  A wall loss on a dielectric label leaves its
// charge Nm q on the label's rows iy and iy+1 of the loss cell (split by the loss point's y; the
// push adds it to dq).  Once per step, before the Poisson solve, every wall node of a dielectric
// label on the rows iyl..iyr (2..ny, all rows with the periodic option) takes
// phi += kd(iy) dq(label, iy) / (Ca dy), kd = 2 on the half cells iy = 1 and ny+1, and dq
// starts again from zero.
__global__ void k_dielectric(double *phi, const int32_t *bcnd, const double *dq, Dtype dt, double Ca, double dy,
                             int nx, int ny, int iyl, int iyr) {
    const int W = nx + 3, rows = iyr - iyl + 1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)W * rows;
         t += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(t % W), iy = iyl + (int)(t / W);
        const int lab = bcnd[ix + (long long)iy * W];
        if (lab < 1) continue;
        const int l = min(lab, LEPIC_MAXLABEL - 1);
        if (dt.v[l] != 1) continue;
        const double kd = (iy == 1 || iy == ny + 1) ? 2.0 : 1.0;
        phi[ix + (long long)iy * W] += kd * dq[(long long)l * (ny + 3) + iy] / (Ca * dy);
    }
}

int dielectric_update(lepic_ctx *c) {
    if (const int r = wait_upload(c)) return r;   // a staged upload into phi
    const lepic_config &g = c->cfg;
    Dtype dt;
    for (int l = 0; l < LEPIC_MAXLABEL; l++) dt.v[l] = c->dtype[l];
    const int iyl = g.flag_pbc ? 0 : 2, iyr = g.flag_pbc ? g.ny + 2 : g.ny;
    const long long work = (long long)(g.nx + 3) * (iyr - iyl + 1);
    if (work > 0) {
        k_dielectric<<<(unsigned)std::min<long long>(div_up(work, 256), (long long)c->num_sms * 4), 256, 0, c->stream>>>(
            c->phi, c->bcnd, c->dq, dt, c->Ca, g.dy, g.nx, g.ny, iyl, iyr);
        LCUDA(cudaGetLastError());
    }
    LCUDA(cudaMemsetAsync(c->dq, 0, sizeof(double) * LEPIC_MAXLABEL * (g.ny + 3), c->stream));
    return LEPIC_OK;
}

extern "C" int lepic_gpu_set_dielectrics(lepic_ctx *c, const int32_t *dtype, double Ca) {
    if (!c || !dtype) return LEPIC_EINVAL;
    bool any = false;
    for (int l = 0; l < LEPIC_MAXLABEL; l++) {
        if (dtype[l] != 0 && dtype[l] != 1) { c->last_err = "set_dielectrics: dtype must be 0 or 1"; return LEPIC_EINVAL; }
        any = any || dtype[l] == 1;
    }
    if (any && !(Ca > 0.0)) { c->last_err = "set_dielectrics: Ca must be positive"; return LEPIC_EINVAL; }
    int r = lepic_gpu_sync(c);
    if (r != LEPIC_OK) return r;
    if (!any) {
        if (c->dq) cudaFree(c->dq);
        c->dq = nullptr;
        return LEPIC_OK;
    }
    const size_t nb = sizeof(double) * LEPIC_MAXLABEL * (c->cfg.ny + 3);
    if (!c->dq) {
        if (cudaMalloc((void **)&c->dq, nb) != cudaSuccess) { c->last_err = "set_dielectrics: cudaMalloc failed"; return LEPIC_ENOMEM; }
        LCUDA(cudaMemsetAsync(c->dq, 0, nb, c->stream));
    }
    for (int l = 0; l < LEPIC_MAXLABEL; l++) c->dtype[l] = dtype[l];
    c->Ca = Ca;
    LCUDA(cudaStreamSynchronize(c->stream));
    return LEPIC_OK;
}

extern "C" int lepic_gpu_dielectric_update(lepic_ctx *c) {
    if (!c || !c->dq) return LEPIC_EINVAL;
    return dielectric_update(c);
}

extern "C" int lepic_gpu_get_dielectric_charge(lepic_ctx *c, double *dq) {
    if (!c || !dq || !c->dq) return LEPIC_EINVAL;
    LCUDA(cudaMemcpyAsync(dq, c->dq, sizeof(double) * LEPIC_MAXLABEL * (c->cfg.ny + 3), cudaMemcpyDeviceToHost,
                          c->stream));
    return lepic_gpu_sync(c);
}

extern "C" int lepic_gpu_set_dielectric_charge(lepic_ctx *c, const double *dq) {
    if (!c || !dq || !c->dq) return LEPIC_EINVAL;
    LCUDA(cudaMemcpyAsync(c->dq, dq, sizeof(double) * LEPIC_MAXLABEL * (c->cfg.ny + 3), cudaMemcpyHostToDevice,
                          c->stream));
    return lepic_gpu_sync(c);
}

extern "C" int lepic_gpu_set_secondary(lepic_ctx *c, const lepic_secondary_config *sec) {
    if (!c || !sec) return LEPIC_EINVAL;
    const lepic_config &g = c->cfg;
    if (!(sec->gam_sec >= 0.0 && sec->gam_sec < 8.0)) { c->last_err = "set_secondary: 0 <= gam_sec < 8"; return LEPIC_EINVAL; }
    if (sec->gam_sec > 0.0) {
        if (sec->igrid_sec < 1) { c->last_err = "set_secondary: igrid_sec must be a wall label >= 1"; return LEPIC_EINVAL; }
        if (!(sec->xg_sec >= 0.0 && sec->xg_sec <= g.nx * g.dx)) { c->last_err = "set_secondary: xg_sec outside the box"; return LEPIC_EINVAL; }
        if (!(sec->THm > 0.0)) { c->last_err = "set_secondary: THm must be positive"; return LEPIC_EINVAL; }
        if (g.charge[0] >= 0.0) { c->last_err = "set_secondary: species 0 must be the electron"; return LEPIC_EINVAL; }
    }
    int r = lepic_gpu_sync(c);
    if (r != LEPIC_OK) return r;
    c->sec_gam = sec->gam_sec;
    c->sec_label = sec->gam_sec > 0.0 ? sec->igrid_sec : 0;
    c->sec_xg = sec->xg_sec;
    c->sec_THm = sec->THm;
    return LEPIC_OK;
}
