/*
 * cnn_oracle.c -- CPU restatement of the learned Poisson warm-start network (forward,
 * energy-norm loss, backward).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU network kernels.  Only tests/ load it.
 *
 * The network has no counterpart in the reference (its Poisson solve starts from the previous
 * step's potential, iterative_solver.f90:1-69); this file states the network exactly as the
 * GPU implements it, so that the tensor-core kernels can be checked value by value:
 *
 *   input x: 2 channels (scaled residual of the previous potential, scaled potential)
 *   encoder  level l = 0..3 at resolution H/2^l, channels C = 16, 32, 64, 64:
 *            e_la = relu(conv(in_l)),  e_l = relu(conv(e_la)),
 *            in_0 = x,  in_l = pool(e_{l-1})  (2x2 average)
 *   decoder  for l = 2, 1, 0:  u_l = up(d_{l+1}) (nearest, d_3 = e_3),
 *            d_la = relu(conv(u_l)) with C_l output channels,  d_l = d_la + e_l
 *   output   out = conv(d_0) to 1 channel (+ bias, no activation)
 *   conv     3x3, zero padding, weights W[cout][cin][3][3] (ky, kx), bias b[cout]
 *
 * In "emulation" mode every tensor the GPU stores in BF16 is rounded to BF16 (round to nearest
 * even) at the same point as on the GPU, weights are rounded to BF16 and biases to FP32;
 * accumulations are exact (double).  With emulation off the same code is a plain
 * double-precision network, used for finite-difference checks of the backward pass.
 *
 * Loss (the energy norm of the error, the quantity conjugate gradients minimise):
 *   e = (out - t) * m,  L = (1/(N H W)) sum over horizontal and vertical neighbour pairs
 *                            inside each image of (e_p - e_q)^2.
 *
 * Parameter vector: for each conv in the order e0a e0b e1a e1b e2a e2b e3a e3b d2 d1 d0 out,
 * W (cout*cin*9 values) then b (cout values).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CN_LAYERS 12

static const int cn_cin[CN_LAYERS] = {2, 16, 16, 32, 32, 64, 64, 64, 64, 64, 32, 16};
static const int cn_cout[CN_LAYERS] = {16, 16, 32, 32, 64, 64, 64, 64, 64, 32, 16, 1};

static int g_emu = 1;

static double R(double v) {
    if (!g_emu) return v;
    float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (double)f; /* inf / nan pass */
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&f, &u, 4);
    return (double)f;
}

int o_cnn_nparams(void) {
    int n = 0;
    for (int l = 0; l < CN_LAYERS; l++) n += cn_cout[l] * cn_cin[l] * 9 + cn_cout[l];
    return n;
}

static void offsets(int *ow, int *ob) {
    int n = 0;
    for (int l = 0; l < CN_LAYERS; l++) {
        ow[l] = n;
        n += cn_cout[l] * cn_cin[l] * 9;
        ob[l] = n;
        n += cn_cout[l];
    }
}

typedef struct { int N, H, W, C; double *v; } T4;

static T4 t_new(int N, int H, int W, int C) {
    T4 t = {N, H, W, C, (double *)calloc((size_t)N * H * W * C, sizeof(double))};
    return t;
}
static void t_free(T4 *t) { free(t->v); t->v = NULL; }
#define AT(t, n, y, x, c) (t).v[((((size_t)(n) * (t).H + (y)) * (t).W + (x)) * (t).C + (c))]

/* acc[n][y][x][co] = sum_{ci,ky,kx} in[n][y+ky-1][x+kx-1][ci] * W[co][ci][ky][kx] (zero pad) */
static void conv_acc(const T4 *in, const double *w, int cout, T4 *acc) {
    const int N = in->N, H = in->H, W = in->W, cin = in->C;
    for (int n = 0; n < N; n++)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
                for (int co = 0; co < cout; co++) {
                    double s = 0.0;
                    for (int ky = 0; ky < 3; ky++) {
                        const int yy = y + ky - 1;
                        if (yy < 0 || yy >= H) continue;
                        for (int kx = 0; kx < 3; kx++) {
                            const int xx = x + kx - 1;
                            if (xx < 0 || xx >= W) continue;
                            const double *ip = &AT(*in, n, yy, xx, 0);
                            const double *wp = w + ((size_t)co * cin) * 9 + ky * 3 + kx;
                            for (int ci = 0; ci < cin; ci++) s += ip[ci] * wp[(size_t)ci * 9];
                        }
                    }
                    AT(*acc, n, y, x, co) = s;
                }
}

/* transposed conv: gin[n][y][x][ci] = sum_{co,ky,kx} g[n][y-ky+1][x-kx+1][co] * W[co][ci][ky][kx] */
static void conv_t(const T4 *g, const double *w, int cin, T4 *gin) {
    const int N = g->N, H = g->H, W = g->W, cout = g->C;
    for (int n = 0; n < N; n++)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
                for (int ci = 0; ci < cin; ci++) {
                    double s = 0.0;
                    for (int ky = 0; ky < 3; ky++) {
                        const int yy = y - ky + 1;
                        if (yy < 0 || yy >= H) continue;
                        for (int kx = 0; kx < 3; kx++) {
                            const int xx = x - kx + 1;
                            if (xx < 0 || xx >= W) continue;
                            const double *gp = &AT(*g, n, yy, xx, 0);
                            for (int co = 0; co < cout; co++)
                                s += gp[co] * w[((size_t)co * cin + ci) * 9 + ky * 3 + kx];
                        }
                    }
                    AT(*gin, n, y, x, ci) = s;
                }
}

/* dW[co][ci][ky][kx] += sum_p g[p][co] * in[p + (ky-1, kx-1)][ci];  db[co] += sum_p g[p][co] */
static void conv_dw(const T4 *in, const T4 *g, double *dw, double *db) {
    const int N = in->N, H = in->H, W = in->W, cin = in->C, cout = g->C;
    for (int n = 0; n < N; n++)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
                for (int co = 0; co < cout; co++) {
                    const double gv = AT(*g, n, y, x, co);
                    if (gv == 0.0) continue;
                    db[co] += gv;
                    for (int ky = 0; ky < 3; ky++) {
                        const int yy = y + ky - 1;
                        if (yy < 0 || yy >= H) continue;
                        for (int kx = 0; kx < 3; kx++) {
                            const int xx = x + kx - 1;
                            if (xx < 0 || xx >= W) continue;
                            for (int ci = 0; ci < cin; ci++)
                                dw[((size_t)co * cin + ci) * 9 + ky * 3 + kx] += gv * AT(*in, n, yy, xx, ci);
                        }
                    }
                }
}

static T4 pool_avg(const T4 *a) {
    T4 o = t_new(a->N, a->H / 2, a->W / 2, a->C);
    for (int n = 0; n < a->N; n++)
        for (int y = 0; y < o.H; y++)
            for (int x = 0; x < o.W; x++)
                for (int c = 0; c < a->C; c++) {
                    const double s = (AT(*a, n, 2 * y, 2 * x, c) + AT(*a, n, 2 * y, 2 * x + 1, c)) +
                                     (AT(*a, n, 2 * y + 1, 2 * x, c) + AT(*a, n, 2 * y + 1, 2 * x + 1, c));
                    AT(o, n, y, x, c) = R(s * 0.25);
                }
    return o;
}

static T4 up2(const T4 *a) {
    T4 o = t_new(a->N, a->H * 2, a->W * 2, a->C);
    for (int n = 0; n < a->N; n++)
        for (int y = 0; y < o.H; y++)
            for (int x = 0; x < o.W; x++)
                for (int c = 0; c < a->C; c++) AT(o, n, y, x, c) = AT(*a, n, y / 2, x / 2, c);
    return o;
}

/* fwd conv with bias + relu; act = R(relu), sum (optional) = R(relu + skip) */
static void conv_relu(const T4 *in, const double *w, const double *b, int cout, T4 *act, const T4 *skip, T4 *sum) {
    T4 acc = t_new(in->N, in->H, in->W, cout);
    conv_acc(in, w, cout, &acc);
    const size_t np = (size_t)in->N * in->H * in->W;
    for (size_t p = 0; p < np; p++)
        for (int c = 0; c < cout; c++) {
            double z = acc.v[p * cout + c] + b[c];
            z = z > 0.0 ? z : 0.0;
            if (g_emu) z = (double)(float)z;
            act->v[p * cout + c] = R(z);
            if (skip) sum->v[p * cout + c] = R(z + skip->v[p * cout + c]);
        }
    t_free(&acc);
}

typedef struct {
    T4 x, e0a, e0, p1, e1a, e1, p2, e2a, e2, p3, e3a, e3, u2, d2a, d2, u1, d1a, d1, u0, d0a, d0;
    double *out;
} Fwd;

static void forward(const double *prm, Fwd *F, int N, int H, int W) {
    int ow[CN_LAYERS], ob[CN_LAYERS];
    offsets(ow, ob);
#define WL(l) (prm + ow[l])
#define BL(l) (prm + ob[l])
    F->e0a = t_new(N, H, W, 16); F->e0 = t_new(N, H, W, 16);
    conv_relu(&F->x, WL(0), BL(0), 16, &F->e0a, NULL, NULL);
    conv_relu(&F->e0a, WL(1), BL(1), 16, &F->e0, NULL, NULL);
    F->p1 = pool_avg(&F->e0);
    F->e1a = t_new(N, H / 2, W / 2, 32); F->e1 = t_new(N, H / 2, W / 2, 32);
    conv_relu(&F->p1, WL(2), BL(2), 32, &F->e1a, NULL, NULL);
    conv_relu(&F->e1a, WL(3), BL(3), 32, &F->e1, NULL, NULL);
    F->p2 = pool_avg(&F->e1);
    F->e2a = t_new(N, H / 4, W / 4, 64); F->e2 = t_new(N, H / 4, W / 4, 64);
    conv_relu(&F->p2, WL(4), BL(4), 64, &F->e2a, NULL, NULL);
    conv_relu(&F->e2a, WL(5), BL(5), 64, &F->e2, NULL, NULL);
    F->p3 = pool_avg(&F->e2);
    F->e3a = t_new(N, H / 8, W / 8, 64); F->e3 = t_new(N, H / 8, W / 8, 64);
    conv_relu(&F->p3, WL(6), BL(6), 64, &F->e3a, NULL, NULL);
    conv_relu(&F->e3a, WL(7), BL(7), 64, &F->e3, NULL, NULL);
    F->u2 = up2(&F->e3);
    F->d2a = t_new(N, H / 4, W / 4, 64); F->d2 = t_new(N, H / 4, W / 4, 64);
    conv_relu(&F->u2, WL(8), BL(8), 64, &F->d2a, &F->e2, &F->d2);
    F->u1 = up2(&F->d2);
    F->d1a = t_new(N, H / 2, W / 2, 32); F->d1 = t_new(N, H / 2, W / 2, 32);
    conv_relu(&F->u1, WL(9), BL(9), 32, &F->d1a, &F->e1, &F->d1);
    F->u0 = up2(&F->d1);
    F->d0a = t_new(N, H, W, 16); F->d0 = t_new(N, H, W, 16);
    conv_relu(&F->u0, WL(10), BL(10), 16, &F->d0a, &F->e0, &F->d0);
    T4 acc = t_new(N, H, W, 1);
    conv_acc(&F->d0, WL(11), 1, &acc);
    F->out = (double *)malloc(sizeof(double) * (size_t)N * H * W);
    for (size_t p = 0; p < (size_t)N * H * W; p++) {
        double z = acc.v[p] + BL(11)[0];
        F->out[p] = g_emu ? (double)(float)z : z;
    }
    t_free(&acc);
}

static void fwd_free(Fwd *F) {
    T4 *all[] = {&F->x, &F->e0a, &F->e0, &F->p1, &F->e1a, &F->e1, &F->p2, &F->e2a, &F->e2, &F->p3, &F->e3a,
                 &F->e3, &F->u2, &F->d2a, &F->d2, &F->u1, &F->d1a, &F->d1, &F->u0, &F->d0a, &F->d0};
    for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); k++) t_free(all[k]);
    free(F->out);
}

/* g = R(acc) * [mask > 0] (mask optional) */
static void round_mask(T4 *g, const T4 *mask) {
    const size_t n = (size_t)g->N * g->H * g->W * g->C;
    for (size_t k = 0; k < n; k++) {
        double v = R(g->v[k]);
        if (mask && !(mask->v[k] > 0.0)) v = 0.0;
        g->v[k] = v;
    }
}

/* out = R(sum of the 2x2 block of gu) (adjoint of nearest upsampling) */
static T4 pool_sum(const T4 *gu) {
    T4 o = t_new(gu->N, gu->H / 2, gu->W / 2, gu->C);
    for (int n = 0; n < gu->N; n++)
        for (int y = 0; y < o.H; y++)
            for (int x = 0; x < o.W; x++)
                for (int c = 0; c < gu->C; c++) {
                    const double s = (AT(*gu, n, 2 * y, 2 * x, c) + AT(*gu, n, 2 * y, 2 * x + 1, c)) +
                                     (AT(*gu, n, 2 * y + 1, 2 * x, c) + AT(*gu, n, 2 * y + 1, 2 * x + 1, c));
                    AT(o, n, y, x, c) = R(s);
                }
    return o;
}

/* out = R(gskip + 0.25 * up(gp)) * [e > 0] (skip gradient plus the adjoint of average pooling) */
static T4 merge(const T4 *gskip, const T4 *gp, const T4 *e) {
    T4 o = t_new(gskip->N, gskip->H, gskip->W, gskip->C);
    for (int n = 0; n < o.N; n++)
        for (int y = 0; y < o.H; y++)
            for (int x = 0; x < o.W; x++)
                for (int c = 0; c < o.C; c++) {
                    double v = R(AT(*gskip, n, y, x, c) + 0.25 * AT(*gp, n, y / 2, x / 2, c));
                    if (!(AT(*e, n, y, x, c) > 0.0)) v = 0.0;
                    AT(o, n, y, x, c) = v;
                }
    return o;
}

static void apply_mask(T4 *g, const T4 *mask) {
    const size_t n = (size_t)g->N * g->H * g->W * g->C;
    for (size_t k = 0; k < n; k++)
        if (!(mask->v[k] > 0.0)) g->v[k] = 0.0;
}

/* Forward, loss and gradient.  x: N*H*W*2, t and m: N*H*W.  out (N*H*W), grad (nparams) may
 * be NULL.  Returns the loss.  H and W must be multiples of 8. */
double o_cnn_loss_grad(const double *prm_in, const double *x, const double *t, const double *m, int N, int H, int W,
                       int emu, double *out, double *grad) {
    g_emu = emu;
    /* the GPU multiplies BF16 weights and adds FP32 biases */
    const int npar = o_cnn_nparams();
    double *pr = (double *)malloc(sizeof(double) * (size_t)npar);
    int ow[CN_LAYERS], ob[CN_LAYERS];
    offsets(ow, ob);
    for (int l = 0; l < CN_LAYERS; l++) {
        for (int k = ow[l]; k < ob[l]; k++) pr[k] = R(prm_in[k]);
        for (int k = ob[l]; k < ob[l] + cn_cout[l]; k++) pr[k] = emu ? (double)(float)prm_in[k] : prm_in[k];
    }
    const double *prm = pr;
    Fwd F;
    memset(&F, 0, sizeof(F));
    F.x = t_new(N, H, W, 2);
    for (size_t k = 0; k < (size_t)N * H * W * 2; k++) F.x.v[k] = R(x[k]);
    forward(prm, &F, N, H, W);
    const size_t np = (size_t)N * H * W;
    if (out) memcpy(out, F.out, np * sizeof(double));
    /* loss and its gradient */
    double *e = (double *)malloc(np * sizeof(double));
    for (size_t p = 0; p < np; p++) e[p] = (F.out[p] - t[p]) * m[p];
    double L = 0.0;
    T4 G = t_new(N, H, W, 1);
    const double inv = 1.0 / (double)np;
    for (int n = 0; n < N; n++)
        for (int y = 0; y < H; y++)
            for (int xx = 0; xx < W; xx++) {
                const size_t p = ((size_t)n * H + y) * W + xx;
                double g = 0.0;
                if (xx + 1 < W) { const double d = e[p] - e[p + 1]; L += d * d; }
                if (y + 1 < H) { const double d = e[p] - e[p + W]; L += d * d; }
                if (xx > 0) g += e[p] - e[p - 1];
                if (xx + 1 < W) g += e[p] - e[p + 1];
                if (y > 0) g += e[p] - e[p - W];
                if (y + 1 < H) g += e[p] - e[p + W];
                g *= 2.0 * inv * m[p];
                if (emu) g = (double)(float)g;
                G.v[p] = R(g);
            }
    L *= inv;
    free(e);
    if (grad) {
        memset(grad, 0, sizeof(double) * (size_t)npar);
#define DW(l) (grad + ow[l])
#define DB(l) (grad + ob[l])
        /* output conv */
        conv_dw(&F.d0, &G, DW(11), DB(11));
        T4 gd0 = t_new(N, H, W, 16);
        conv_t(&G, WL(11), 16, &gd0);
        round_mask(&gd0, NULL);
        /* decoder level 0: d0 = d0a + e0, d0a = relu(conv(u0)), u0 = up(d1) */
        T4 gd0a = t_new(N, H, W, 16);
        memcpy(gd0a.v, gd0.v, sizeof(double) * np * 16);
        apply_mask(&gd0a, &F.d0a);
        conv_dw(&F.u0, &gd0a, DW(10), DB(10));
        T4 gu0 = t_new(N, H, W, 32);
        conv_t(&gd0a, WL(10), 32, &gu0);
        round_mask(&gu0, NULL);
        T4 gd1 = pool_sum(&gu0);
        /* decoder level 1 */
        T4 gd1a = t_new(N, H / 2, W / 2, 32);
        memcpy(gd1a.v, gd1.v, sizeof(double) * np / 4 * 32);
        apply_mask(&gd1a, &F.d1a);
        conv_dw(&F.u1, &gd1a, DW(9), DB(9));
        T4 gu1 = t_new(N, H / 2, W / 2, 64);
        conv_t(&gd1a, WL(9), 64, &gu1);
        round_mask(&gu1, NULL);
        T4 gd2 = pool_sum(&gu1);
        /* decoder level 2 */
        T4 gd2a = t_new(N, H / 4, W / 4, 64);
        memcpy(gd2a.v, gd2.v, sizeof(double) * np / 16 * 64);
        apply_mask(&gd2a, &F.d2a);
        conv_dw(&F.u2, &gd2a, DW(8), DB(8));
        T4 gu2 = t_new(N, H / 4, W / 4, 64);
        conv_t(&gd2a, WL(8), 64, &gu2);
        round_mask(&gu2, NULL);
        T4 ge3 = pool_sum(&gu2);
        /* encoder level 3 */
        apply_mask(&ge3, &F.e3);
        conv_dw(&F.e3a, &ge3, DW(7), DB(7));
        T4 ge3a = t_new(N, H / 8, W / 8, 64);
        conv_t(&ge3, WL(7), 64, &ge3a);
        round_mask(&ge3a, &F.e3a);
        conv_dw(&F.p3, &ge3a, DW(6), DB(6));
        T4 gp3 = t_new(N, H / 8, W / 8, 64);
        conv_t(&ge3a, WL(6), 64, &gp3);
        round_mask(&gp3, NULL);
        /* encoder level 2 */
        T4 ge2 = merge(&gd2, &gp3, &F.e2);
        conv_dw(&F.e2a, &ge2, DW(5), DB(5));
        T4 ge2a = t_new(N, H / 4, W / 4, 64);
        conv_t(&ge2, WL(5), 64, &ge2a);
        round_mask(&ge2a, &F.e2a);
        conv_dw(&F.p2, &ge2a, DW(4), DB(4));
        T4 gp2 = t_new(N, H / 4, W / 4, 32);
        conv_t(&ge2a, WL(4), 32, &gp2);
        round_mask(&gp2, NULL);
        /* encoder level 1 */
        T4 ge1 = merge(&gd1, &gp2, &F.e1);
        conv_dw(&F.e1a, &ge1, DW(3), DB(3));
        T4 ge1a = t_new(N, H / 2, W / 2, 32);
        conv_t(&ge1, WL(3), 32, &ge1a);
        round_mask(&ge1a, &F.e1a);
        conv_dw(&F.p1, &ge1a, DW(2), DB(2));
        T4 gp1 = t_new(N, H / 2, W / 2, 16);
        conv_t(&ge1a, WL(2), 16, &gp1);
        round_mask(&gp1, NULL);
        /* encoder level 0 */
        T4 ge0 = merge(&gd0, &gp1, &F.e0);
        conv_dw(&F.e0a, &ge0, DW(1), DB(1));
        T4 ge0a = t_new(N, H, W, 16);
        conv_t(&ge0, WL(1), 16, &ge0a);
        round_mask(&ge0a, &F.e0a);
        conv_dw(&F.x, &ge0a, DW(0), DB(0));
        T4 *tmp[] = {&gd0, &gd0a, &gu0, &gd1, &gd1a, &gu1, &gd2, &gd2a, &gu2, &ge3, &ge3a, &gp3,
                     &ge2, &ge2a, &gp2, &ge1, &ge1a, &gp1, &ge0, &ge0a};
        for (size_t k = 0; k < sizeof(tmp) / sizeof(tmp[0]); k++) t_free(tmp[k]);
#undef DW
#undef DB
    }
#undef WL
#undef BL
    t_free(&G);
    fwd_free(&F);
    free(pr);
    return L;
}
