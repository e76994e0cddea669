// field.cu -- charge density to Poisson right-hand side, density reduction, electric field.
// Compiled with -fmad=false: every FP64 product and sum is rounded as written, so the
// field values equal the CPU restatement's bit for bit.
//
// Roofline: all three are HBM/L2 streams over the (nx+3)(ny+3) node grid:
//   calc_rhs  reads ntype*8 B (uint64 accumulators) + 1 B mask + 8 B kq, writes 8 B / node
//   efield    reads 8 B phi (5-point, cached) + 1 B mask, writes 16 B (FP64) + 8 B (FP32)
#include <algorithm>
#include "rho.cuh"

// calc_rho.f90:37-77: rhs(ix,iy) = -sum_ptype charge(ptype)*np(ix,iy,ptype)
// one node per thread: the column from the thread, the row from blockIdx.y (no division)
__global__ void k_calc_rhs(RhoParams P, double *rhs) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > P.nx) return;
    for (int j = blockIdx.y; j <= P.ny; j += gridDim.y) {   // gridDim.y <= 65535
        const int ix = k + 1, iy = j + 1;
        double r = 0.0;
        for (int s = 0; s < P.ntype; s++) r = r - P.charge[s] * np_val(P, s, ix, iy);
        rhs[k + (long long)j * (P.nx + 1)] = r;
    }
}

// calc_rho.f90:134-199: np_red = np (one rank), np_mx = max over bcnd == -1 nodes.
// The maximum of non-negative doubles is taken on their bit patterns (order-free).
__global__ void k_dens_red(RhoParams P, double *np_red, unsigned long long *np_mx) {
    const long long nn = (long long)(P.nx + 3) * (P.ny + 3);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
         t += (long long)gridDim.x * blockDim.x) {
        int ix = (int)(t % (P.nx + 3)), iy = (int)(t / (P.nx + 3));
        bool in = ix >= 1 && ix <= P.nx + 1 && iy >= 1 && iy <= P.ny + 1;
        for (int s = 0; s < P.ntype; s++) {
            double v = in ? np_val(P, s, ix, iy) : 0.0;
            np_red[s * nn + t] = v;
            if (in && P.bc[t] == -1 && v > 0.0) atomicMax(&np_mx[s], (unsigned long long)__double_as_longlong(v));
        }
    }
}

__global__ void k_np_grid(RhoParams P, int s, double *out) {
    const long long nn = (long long)(P.nx + 3) * (P.ny + 3);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
         t += (long long)gridDim.x * blockDim.x) {
        int ix = (int)(t % (P.nx + 3)), iy = (int)(t / (P.nx + 3));
        bool in = ix >= 1 && ix <= P.nx + 1 && iy >= 1 && iy <= P.ny + 1;
        out[t] = in ? np_val(P, s, ix, iy) : np_raw(P, s, ix, iy);
    }
}

int field_calc_rhs(lepic_ctx *c) {
    RhoParams P = rho_params(c);
    const dim3 grid(div_up(c->cfg.nx + 1, 256), std::min(c->cfg.ny + 1, 65535));
    k_calc_rhs<<<grid, 256, 0, c->stream>>>(P, c->rhs);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

int field_dens_red(lepic_ctx *c) {
    RhoParams P = rho_params(c);
    LCUDA(cudaMemsetAsync(c->np_mx, 0, sizeof(double) * LEPIC_MAXSP, c->stream));
    int grid = (int)std::min<long long>(div_up(c->nn, 256), (long long)c->num_sms * 16);
    k_dens_red<<<grid, 256, 0, c->stream>>>(P, c->np_red, (unsigned long long *)c->np_mx);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

int field_np_grid(lepic_ctx *c, int ptype, double *d_out) {
    RhoParams P = rho_params(c);
    int grid = (int)std::min<long long>(div_up(c->nn, 256), (long long)c->num_sms * 16);
    k_np_grid<<<grid, 256, 0, c->stream>>>(P, ptype, d_out);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}

// ---------------------------------------------------------------------------------------
// Efield.f90:1-128.
// Pass 1 (:19-34): central differences at nodes with bcnd <= 0, into the scratch field E;
// every other node (walls, ghosts) takes the current field's value, which the reference's
// in/out Ei holds there when the wall pass reads it.
__global__ void k_efield_interior(int nx, int ny, double h1, double h2, const double *phi,
                                  const int8_t *bc, const double2 *Ecur, double2 *E) {
    const int W = nx + 3;
    const long long nn = (long long)(nx + 3) * (ny + 3);
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn;
         n += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(n % W), iy = (int)(n / W);
        if (ix >= 1 && ix <= nx + 1 && iy >= 1 && iy <= ny + 1 && bc[n] <= 0) {
            double2 e;
            e.x = -(phi[n + 1] - phi[n - 1]) / (2.0 * h1);
            e.y = -(phi[n + W] - phi[n - W]) / (2.0 * h2);
            E[n] = e;
        } else {
            E[n] = Ecur[n];
        }
    }
}
// Pass 2, periodic rows (:68-82) when part == 0, then the Neumann column (:52-63) when
// part == 1; one thread per column / row.  The reference visits row 1 first, so its periodic
// copies read column 1 before the Neumann step zeroes Ex there: two launches keep that order.
__global__ void k_efield_nmn_pbc(int nx, int ny, double h2, const double *phi, const int8_t *bc,
                                 double2 *E, int part) {
    const int W = nx + 3;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (part == 1 && t >= 1 && t <= ny + 1) { // Neumann: any node of row iy with bcnd == -2
        int iy = t;
        for (int ix = 1; ix <= nx + 1; ix++) {
            if (bc[ix + iy * W] != -2) continue;
            E[1 + iy * W].x = 0.0;
            if (iy > 1 && iy < ny + 1)
                E[1 + iy * W].y = -(phi[1 + (iy + 1) * W] - phi[1 + (iy - 1) * W]) / (2.0 * h2);
        }
    }
    if (part == 0 && t >= 1 && t <= nx + 1) { // periodic: node (ix, 1)
        int ix = t;
        int b = bc[ix + 1 * W];
        if (b == 0 || b == -2) {
            E[ix + 1 * W].y = -(phi[ix + 2 * W] - phi[ix + ny * W]) / (2.0 * h2);
            E[ix + 0 * W].y = E[ix + ny * W].y;
            E[ix + (ny + 1) * W].y = E[ix + 1 * W].y;
            E[ix + (ny + 2) * W].y = E[ix + 2 * W].y;
            E[ix + 0 * W].x = E[ix + ny * W].x;
            E[ix + (ny + 2) * W].x = E[ix + 2 * W].x;
        }
    }
}
// Pass 2, walls (:87-118): zero, then linear extrapolation from the interior side.  Reads the
// pass-1 field and writes a second buffer, so every wall node sees the same input.
__global__ void k_efield_walls(int nx, int ny, const int8_t *bc, const double2 *Ein, double2 *Eout,
                               float4 *Ef) {
    const int W = nx + 3;
    const long long nn = (long long)(nx + 3) * (ny + 3);
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn;
         n += (long long)gridDim.x * blockDim.x) {
        int ix = (int)(n % W), iy = (int)(n / W);
        double2 e = Ein[n];
        if (ix >= 1 && ix <= nx + 1 && iy >= 1 && iy <= ny + 1 && bc[n] >= 1) {
            e.x = 0.0;
            e.y = 0.0;
            // the +-2 neighbours exist only inside the ghost frame (0..n+2)
            if (bc[n + 1] <= 0) e.x = 2.0 * Ein[n + 1].x - (ix + 2 <= nx + 2 ? Ein[n + 2].x : 0.0);
            if (bc[n - 1] <= 0) e.x = 2.0 * Ein[n - 1].x - (ix >= 2 ? Ein[n - 2].x : 0.0);
            if (bc[n + W] <= 0) e.y = 2.0 * Ein[n + W].y - (iy + 2 <= ny + 2 ? Ein[n + 2 * W].y : 0.0);
            if (bc[n - W] <= 0) e.y = 2.0 * Ein[n - W].y - (iy >= 2 ? Ein[n - 2 * W].y : 0.0);
        }
        Eout[n] = e;
        // FP32 gather copy in node pairs: node n is the first half of pair n and the second
        // half of pair n - 1, so the push reads two adjacent nodes with one 16-byte load
        const float2 f = make_float2((float)e.x, (float)e.y);
        float2 *half = reinterpret_cast<float2 *>(Ef);
        half[2 * n] = f;
        if (n > 0) half[2 * n - 1] = f;
    }
}

// Both passes in one for decks without the periodic and Neumann options: a wall node takes the
// pass-1 values of its neighbours recomputed from phi (the same operations, so the same bits),
// and the result goes to the other half of the field buffer, so that every node reads the
// previous field where pass 1 would have copied it.
__device__ __forceinline__ double2 efield_pass1(int nx, int ny, double h1, double h2, const double *phi,
                                                const int8_t *bc, const double2 *Ecur, int mx, int my, int W) {
    const int m = mx + my * W;
    if (mx >= 1 && mx <= nx + 1 && my >= 1 && my <= ny + 1 && bc[m] <= 0) {
        double2 e;
        e.x = -(phi[m + 1] - phi[m - 1]) / (2.0 * h1);
        e.y = -(phi[m + W] - phi[m - W]) / (2.0 * h2);
        return e;
    }
    return Ecur[m];
}
// one node per thread: the column from the thread, the row from blockIdx.y (no division)
__global__ void k_efield_fused(int nx, int ny, double h1, double h2, const double *phi, const int8_t *bc,
                               const double2 *Ecur, double2 *Eout, float4 *Ef) {
    const int W = nx + 3;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    if (ix >= W) return;
    for (int iy = blockIdx.y; iy < ny + 3; iy += gridDim.y) {   // gridDim.y <= 65535
    const int n = ix + iy * W;
    double2 e;
    if (ix >= 1 && ix <= nx + 1 && iy >= 1 && iy <= ny + 1 && bc[n] >= 1) {   // pass 2 at a wall
        e.x = 0.0;
        e.y = 0.0;
        if (bc[n + 1] <= 0)
            e.x = 2.0 * efield_pass1(nx, ny, h1, h2, phi, bc, Ecur, ix + 1, iy, W).x -
                  (ix + 2 <= nx + 2 ? efield_pass1(nx, ny, h1, h2, phi, bc, Ecur, ix + 2, iy, W).x : 0.0);
        if (bc[n - 1] <= 0)
            e.x = 2.0 * efield_pass1(nx, ny, h1, h2, phi, bc, Ecur, ix - 1, iy, W).x -
                  (ix >= 2 ? efield_pass1(nx, ny, h1, h2, phi, bc, Ecur, ix - 2, iy, W).x : 0.0);
        if (bc[n + W] <= 0)
            e.y = 2.0 * efield_pass1(nx, ny, h1, h2, phi, bc, Ecur, ix, iy + 1, W).y -
                  (iy + 2 <= ny + 2 ? efield_pass1(nx, ny, h1, h2, phi, bc, Ecur, ix, iy + 2, W).y : 0.0);
        if (bc[n - W] <= 0)
            e.y = 2.0 * efield_pass1(nx, ny, h1, h2, phi, bc, Ecur, ix, iy - 1, W).y -
                  (iy >= 2 ? efield_pass1(nx, ny, h1, h2, phi, bc, Ecur, ix, iy - 2, W).y : 0.0);
    } else {
        e = efield_pass1(nx, ny, h1, h2, phi, bc, Ecur, ix, iy, W);
    }
    Eout[n] = e;
    const float2 f = make_float2((float)e.x, (float)e.y);
    float2 *half = reinterpret_cast<float2 *>(Ef);
    half[2 * (long long)n] = f;
    if (n > 0) half[2 * (long long)n - 1] = f;
    }
}

int field_calc_efield(lepic_ctx *c) {
    if (const int r = wait_upload(c)) return r;   // a staged upload into phi
    const int nx = c->cfg.nx, ny = c->cfg.ny;
    int grid = (int)std::min<long long>(div_up(c->nn, 256), (long long)c->num_sms * 16);
    if (!c->cfg.flag_pbc && !c->cfg.flag_nmn) {
        double2 *other = c->Ed == c->Ed_base ? c->Ed_base + c->nn : c->Ed_base;
        const dim3 g2(div_up(nx + 3, 256), std::min(ny + 3, 65535));
        k_efield_fused<<<g2, 256, 0, c->stream>>>(nx, ny, c->cfg.dx, c->cfg.dy, c->phi, c->bc8, c->Ed, other, c->Ef);
        LCUDA(cudaGetLastError());
        c->Ed = other;
        return LEPIC_OK;
    }
    // E (FP64) lives in the current half; the other half holds pass 1, which the wall pass reads
    double2 *E0 = c->Ed == c->Ed_base ? c->Ed_base + c->nn : c->Ed_base, *E1 = c->Ed;
    k_efield_interior<<<grid, 256, 0, c->stream>>>(nx, ny, c->cfg.dx, c->cfg.dy, c->phi, c->bc8, E1, E0);
    if (c->cfg.flag_pbc || c->cfg.flag_nmn) // the passes test the labels, as Efield.f90:43-82 does
        for (int part = 0; part < 2; part++)
            k_efield_nmn_pbc<<<div_up(std::max(nx, ny) + 2, 256), 256, 0, c->stream>>>(nx, ny, c->cfg.dy,
                                                                                       c->phi, c->bc8, E0, part);
    int grid2 = (int)std::min<long long>(div_up(c->nn, 256), (long long)c->num_sms * 16);
    k_efield_walls<<<grid2, 256, 0, c->stream>>>(nx, ny, c->bc8, E0, E1, c->Ef);
    LCUDA(cudaGetLastError());
    return LEPIC_OK;
}
