/*
 * lepic_oracle.h -- CPU FP64 restatement of the LePIC per-step PIC-MCC routines.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA path: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.  The product
 * library (jd_lepic_b200) never links, loads or calls it.
 *
 * Parity status: the reference (Fortran 90 + MPI + OpenMP) cannot be compiled in this
 * environment (no Fortran compiler) and ships no tests, golden vectors or fixtures for
 * these routines.  Parity against the reference's own outputs is therefore UNPINNED; the
 * restatement is pinned instead by published known answers (Park-Miller minimal standard
 * sequence) and analytic known-answer tests (Boris gyration, E x B drift, CIC charge
 * conservation, manufactured Poisson solutions, MCC rate n*sigma*v).
 *
 * Conventions (identical to the reference's Fortran memory order):
 *   node arrays  f(0:nx+2, 0:ny+2)  ->  f[i + j*(nx+3)], x index fastest
 *   rhs          b(1:nx+1, 1:ny+1)  ->  b[(i-1) + (j-1)*(nx+1)]
 *   E field      Ei(2, 0:nx+2, 0:ny+2) -> Ei[2*(i + j*(nx+3)) + c]
 *   B field      Bi(4, 0:nx+2, 0:ny+2) -> Bi[4*(i + j*(nx+3)) + c]
 *   particles    vxp(6, np) per species -> vxp[6*k + c], c = x,y,z,vx,vy,vz
 * Species index 0 is the electron, then ions, then neutrals (negative mass), 0-based.
 */
#ifndef LEPIC_ORACLE_H
#define LEPIC_ORACLE_H
#include <stdint.h>

#define O_MAXSP 8
#define O_MAXCOL 64

typedef struct {
    int nx, ny;
    double dx, dy, zmax, xmax, ymax, dt;
    double eps0, qe, pi;
    int flag_pbc, flag_spec, flag_nmn;
    int flag_B;            /* 0: no B, 1: constant B (Bc), 2: B map on the field grid (Bi) */
    int flag_B_pos;        /* 1: positive ions unmagnetised */
    double Bc[3];
    int ntype;             /* charged species (electrons first)                */
    int nsp;               /* charged + neutral species                         */
    double charge[O_MAXSP], mass[O_MAXSP], Nm[O_MAXSP], vt0[O_MAXSP];
    double np_mx[O_MAXSP]; /* neutral densities live at the neutral indices     */
    double nu_uplim[O_MAXSP];
    int ns_coll, nsort;
} o_cfg;

typedef struct {
    int npt;                 /* sig_npt_mx: points of the union energy grid           */
    int ncol;                /* number of reactions                                    */
    const double *sig_Er;    /* [npt]                                                  */
    const double *sig;       /* [icol*npt + ipt]                                       */
    const double *Eth;       /* [icol] threshold energy, eV                            */
    const int32_t *col_info; /* [icol*10 + k], the reference's col_info(icol, k+1) with
                                species entries converted to 0-based indices           */
    const int32_t *p_ncol;   /* [ptype]                                                */
    const int32_t *sig_list; /* [ptype*O_MAXCOL + k] reaction index, 0-based           */
    const double *sigv_mx;   /* [ptype*O_MAXCOL + icol]                                */
    int flag_ionrep;
    double fEk;
} o_xs;

typedef struct {
    int64_t n_lost;       /* wall / boundary losses            */
    int64_t n_dead;       /* removed because flag_dead was set */
    int64_t n_loss[16];   /* p_mac(ptype, np_loss, igrid), igrid = bcnd(ix,iy) of a wall
                             loss (part_expmover.f90:338), 0 for the other losses; labels
                             above 15 in the last                                   */
    double v2_loss[16];   /* sum of the lost particles' v^2 per igrid (P_w / 0.5 Nm m) */
    double P1z;           /* P_loss(1)'s Nm q phi of 3rd-dimension losses (:400-421)      */
} o_push_tally;

/* the 3rd virtual dimension (hz >= 0; part_expmover.f90:269-309): z in vxp[2] moves with vz;
 * c->zmax is its length.  Positive ions draw from the device's counter stream (slot index i of
 * the input array, step it, key k0 k1) against nu_fac * uB, nu_fac = hz 2 dt / zmax in FP32. */
typedef struct {
    double phi0;
    const double *phi;      /* phi(0:nx+2, 0:ny+2)                          */
    const float *uB;        /* this species' uB(na1+1, na2+1)               */
    int na1, size_na;
    float nu_fac;
    uint32_t k0, k1, it;
} o_zloss;

typedef struct {
    int64_t n_cand[O_MAXSP];              /* Nc per species                 */
    int64_t n_coll[O_MAXCOL];             /* real collisions per reaction   */
    int64_t n_add[O_MAXSP];               /* products appended per species  */
    int64_t n_overflow;                   /* Ekr above the table            */
    double nu_max[O_MAXSP];
} o_mcc_tally;

/* ran2.f90:1-15 -- Park-Miller minimal standard generator (Schrage). */
double o_ran2(int32_t *irand);
/* load_gauss.f90:16-39 */
void o_load_gauss(double *vx, double *vy, double vt, const double rnd[2]);

/* part_expmover.f90:1-517 (E gather, Boris/leap-frog, move, y wrap, wall loss,
 * Neumann reflection, flag_dead removal, order-preserving compaction).
 * The 3rd-dimension model, dielectric charging, refluxing and secondary emission are in
 * o_part_mover_z / _zd / _x below; not restated: the phase-space tally. */
void o_part_mover(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                  const int32_t *bcnd, double *vxp, int64_t *np_tot, int8_t *flag_dead,
                  o_push_tally *t);
/* the same with the 3rd-dimension model when zl is not NULL */
void o_part_mover_z(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                    const int32_t *bcnd, double *vxp, int64_t *np_tot, int8_t *flag_dead,
                    o_push_tally *t, const o_zloss *zl);

/* dielectric walls (part_expmover.f90:340-350): dtype[label] for labels 0..15 (larger labels in
 * the last), dq[label * (ny+3) + iy] the collected charge summed over species. */
typedef struct {
    const int32_t *dtype;
    double *dq;
} o_dielec;
/* o_part_mover_z that also adds wall losses on dielectric labels to dl->dq when dl is not NULL */
void o_part_mover_zd(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                     const int32_t *bcnd, double *vxp, int64_t *np_tot, int8_t *flag_dead,
                     o_push_tally *t, const o_zloss *zl, const o_dielec *dl);
/* refluxing (part_expmover.f90:445-470) and secondary emission (:354-392), drawn from the
 * device's counter streams (slot i of the input array, step it, key k0 k1) so that the two agree
 * particle by particle. */
typedef struct {
    int reflux;                 /* opt_inj = +-4 with flag_nmn: re-draw at x <= 0           */
    double vb, fmax, vt, sin_thB, cos_thB;
    int sec_label;              /* emitting wall label of this positive species (0: none)   */
    double gam_sec, vt_sec, xg_sec, Nm0, m0;
    double *sec_out;            /* (x, y, z, vx, vy, vz) per electron, in emission order    */
    int64_t sec_cap, n_sec;
    uint32_t k0, k1, it;
    double P1r, P4r, P4sec;     /* P_loss(1) and (4) of this species' refluxing; (4) of the
                                   electrons from the emission                               */
} o_wallx;
/* o_part_mover_zd with the two branches when wx is not NULL */
void o_part_mover_x(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                    const int32_t *bcnd, double *vxp, int64_t *np_tot, int8_t *flag_dead,
                    o_push_tally *t, const o_zloss *zl, const o_dielec *dl, o_wallx *wx);

/* main.f90:756-809 on one rank: phi += kd dq / (Ca dy) on the dielectric labels' wall nodes,
 * kd = 2 on rows 1 and ny+1, rows 2..ny (0..ny+2 with flag_pbc); dq is zeroed. */
void o_dielectric_update(const o_cfg *c, double *phi, const int32_t *bcnd, const int32_t *dtype,
                         double *dq, double Ca);

/* part_expmover.f90:520-610 -- adds into npg (caller zeroes it). */
void o_charge_deposition(const o_cfg *c, int ptype, const double *vxp, int64_t np_tot,
                         const double *kq, double *npg);

/* calc_rho.f90:1-35 */
void o_np_periodic(const o_cfg *c, double *npg, const int32_t *bcnd);
/* calc_rho.f90:37-77 -- npg holds ntype grids back to back. */
void o_calc_rhs(const o_cfg *c, const double *npg, double *rhs);
/* calc_rho.f90:134-199 -- fills np_red (ntype grids) and c->np_mx[0..ntype-1]. */
void o_dens_red(o_cfg *c, const double *npg, double *np_red, const int32_t *bcnd);

/* Efield.f90:1-128, single-threaded loop order. */
void o_calc_efield(const o_cfg *c, const double *phi, double *Ei, const int32_t *bcnd);

/* iterative_solver.f90:1-69 with mg.f90 / sors.f90 on one rank.
 * Returns 0, or -1 when the reference would abort on divergence. */
typedef struct { int k; double ktot; double res; int sweeps_fine; } o_solve_stats;
int o_iterative_solver(const o_cfg *c, double *u, const double *b, const int32_t *bcnd,
                       int ng, int ncycl, double eps, o_solve_stats *st);
/* One red-black SOR smoothing call (sors.f90:1-435), exposed for tests. */
int o_sor_rb(int nx, int ny, double hx, double hy, double eps0, double *u, const double *b,
             const int32_t *bcnd, double *res, double omega, double eps, int kmg, int dig,
             int flag_pbc);
/* mg.f90 helpers exposed for tests. */
void o_restriction(int nx, int ny, double hx, double hy, double eps0, const double *u,
                   const double *b, const int32_t *bcnd, int32_t *bcnd2h, double *r2h,
                   double *e2h, int flag_pbc, int flag_nmn);
void o_prolongation(int nx, int ny, double *u, const double *e2h, const int32_t *bcnd);

/* sorting.f90:92-251 with nproc = 1 (stable counting sort by cell).  plist has
 * pl_max+1 = nx + nx*ny + 2 entries; scratch holds 6*np_tot doubles. */
void o_part_sorting(const o_cfg *c, double *vxp, int64_t np_tot, int32_t *plist,
                    double *scratch);

/* indexx.f90:1-88 (Numerical Recipes index sort), 0-based output. */
void o_indexx(int n, const double *arr, int *indx);

/* collisions.f90:1-207 + collision_OMP :209-1040 + SCATTER :1042-1070 for neutral
 * targets (null-collision MCC), nproc = 1.  vxp/np_tot/cap/flag_dead are per species.
 * Products are appended at np_tot + np_add.  Returns 0, -1 on Pmax > 1, -2 when a
 * species array would exceed its capacity, -3 on a negative collision energy. */
int o_collisions(o_cfg *c, const o_xs *xs, double **vxp, int64_t *np_tot, const int64_t *cap,
                 int8_t **flag_dead, int32_t *iseed, o_mcc_tally *t);

/* The same with charged targets (DSMC, collisions.f90:339-418, 524-528, 767-797, 908-935,
 * 942-1000): plist[tt] is Plist(0:pl_max) of target species tt's array as o_part_sorting leaves
 * it (NULL: reactions on tt are skipped, as o_collisions does), np_red the dens_red grids
 * (ntype node grids); c->np_mx[tt] must hold dens_red's maximum for nu_max.  A target scatters
 * in elastic and excitation events, takes the incident's velocity in charge exchange and is
 * flagged dead when it is a reactant that is not a byproduct. */
typedef struct {
    const int32_t *plist[O_MAXSP];
    const double *np_red;
} o_dsmc;
int o_collisions_dsmc(o_cfg *c, const o_xs *xs, double **vxp, int64_t *np_tot, const int64_t *cap,
                      int8_t **flag_dead, int32_t *iseed, o_mcc_tally *t, const o_dsmc *d);

/* SCATTER, collisions.f90:1042-1070 */
void o_scatter(double *vx1, double *vy1, double *vz1, double vx, double vy, double vz,
               double costheta, double phi);

/* OpenMP variants used only for the timed CPU baseline: same arithmetic as the serial
 * routines; the particle array is split into contiguous per-thread slabs with private
 * density grids, reduced in thread order, like the reference's per-thread slabs. */
void o_push_deposit_omp(const o_cfg *c, int ptype, const double *Ei, const double *Bi,
                        const int32_t *bcnd, const double *kq, double *vxp, int64_t *np_tot,
                        int8_t *flag_dead, double *npg, int nthreads);
int o_iterative_solver_omp(const o_cfg *c, double *u, const double *b, const int32_t *bcnd,
                           int ng, int ncycl, double eps, o_solve_stats *st, int nthreads);
/* The same V-cycles stopped on ||b - A u||_2 <= eps ||b - A u_D||_2 (bcnd == -1 nodes), the
 * criterion of the device's mixed and L2 solves, for a CPU baseline of the same tolerance. */
int o_iterative_solver_l2_omp(const o_cfg *c, double *u, const double *b, const int32_t *bcnd,
                              int ng, int ncycl, double eps, o_solve_stats *st, int nthreads);

/* ---- particle sources: e_heating.f90, part_injection.f90 ----------------------------------
 * Two forms of each routine.  The plain form restates the reference's draw order from one
 * sequential ran2 stream (the vz_sav / x_sav pairing of consecutive particles included).
 * The _ctr form is the same algorithm fed by the counter-based Philox4x32-10 streams the
 * device path draws from (one counter per slot or injected particle and step), so the
 * device's results can be checked particle by particle; it also rounds the stored state
 * the way the device keeps it (FP32 velocities; fixed-point positions with S fractional
 * bits when S > 0). */
#define O_MAXICP 16
typedef struct {
    int flag_c;                 /* 0 slit, 1 disk (read_input.f90:48-51)               */
    double xl_pow, xr_pow, yl_pow, yr_pow;
    int eheat_type, flag_gpp, n_icp;
    double nudt, Pabs_cor;
    int opt_inj, flag_Tp, flag_diffsrc, tag_neg, nproc_mpi, ns_inj;
    double I_inj, THm;
    double ni0[O_MAXSP];
    double th_B;                /* opt_inj = 4: angle of B to the x axis (main.f90:450-452) */
} o_src;

/* Philox4x32-10 (Salmon et al., SC'11) and the device's (0,1) mapping (v + 0.5) 2^-32 */
void o_philox4x32_10(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]);
double o_u01(uint32_t v);

/* e_heating.f90:1-112 on the electrons vxp(6,n); vt[n_icp]; ran2 sequence. */
void o_eheating(const o_cfg *c, const o_src *s, double *vxp, int64_t n, const double *vt,
                int32_t *iseed, double *P_heat, int64_t *n_heated);
void o_eheating_ctr(const o_cfg *c, const o_src *s, double *vxp, int64_t n, const double *vt,
                    uint64_t seed, int32_t it, double *P_heat, int64_t *n_heated);
/* the heating-region tallies of charge_deposition (part_expmover.f90:583-605) */
void o_heat_tally(const o_cfg *c, const o_src *s, const double *vxp, int64_t n, int64_t *Nh,
                  double *sum_dEk);
/* main.f90:1003-1010 for one band; returns vt (the old value when Nh = 0) */
double o_te_update(const o_cfg *c, int eheat_type, double Pabs, double nu_h, int64_t Nh,
                   double sum_dEk, double vt_old);

/* part_injection.f90:1-237 for one species: N_inj[ntype] holds the losses counted by the
 * mover (|opt_inj| = 2) and receives this call's count; particles are appended to vxp
 * from *np (capacity cap).  Returns 0, or -2 when the capacity would be exceeded. */
int o_part_injection(const o_cfg *c, const o_src *s, int ptype, const int32_t *bcnd,
                     const double *phi, int64_t *N_inj, double *vxp, int64_t *np, int64_t cap,
                     int32_t *iseed, double *P_inj, double *P_src);
/* the device's form over all charged species in order: lost[ntype] are the losses since the
 * last injection; vxp[s] / np[s] / cap[s] per species; count[s] receives N_inj.  Returns 0,
 * -2 on capacity, -3 when a particle finds no free cell in 65536 attempts. */
int o_part_injection_ctr(const o_cfg *c, const o_src *s, const int32_t *bcnd, const double *phi,
                         const int64_t *lost, uint64_t seed, int32_t it, int S, double **vxp,
                         int64_t *np, const int64_t *cap, int64_t *count, double *P_inj,
                         double *P_src);

/* part_flux_emitter (part_flux_emitter.f90:1-217), nproc = 1.  Emits into species
 * sp_fx (flat surface) and sp_b (chamfer, = sp_fx when there is no chamfer species) at the
 * grid plane xg1.  vxp[s] / np[s] / cap[s] per species; count[s] receives the particles
 * emitted.  The _ctr form draws from the device's streams (attempt a, particle j) and
 * stores the device's state (FP32 velocities, fixed-point positions with S bits when
 * S > 0, NaN vx for a particle outside the box after its partial move, counted in *n_out).
 * Returns 0, -2 on capacity, -3 when the attempts run out. */
typedef struct {
    double js, xg1, Lg, Lh;
    int n_holes, ns_Hm, n_icp, nproc_mpi;
    int chamfer;                /* ptype_fx == tag_neg and flag_chmfrd              */
    double chmfrd[4];
    int sp_fx, sp_b;
    double THm;
} o_emit;
int o_part_flux_emitter(const o_cfg *c, const o_emit *e, const int32_t *bcnd, double **vxp,
                        int64_t *np, const int64_t *cap, int32_t *iseed, int64_t *count,
                        double *P_inj);
int o_part_flux_emitter_ctr(const o_cfg *c, const o_emit *e, const int32_t *bcnd, uint64_t seed,
                            int32_t it, int S, double **vxp, int64_t *np, const int64_t *cap,
                            int64_t *count, double *P_inj, int64_t *n_out);

/* part_moments (utils.f90:1-131): p_mts(4, 0:na1+2, 0:na2+2) of one species, index
 * m*ncell + ix + iy*(na1+3), ncell = (na1+3)(na2+3), na = n/size_na; zeroed first. */
void o_part_moments(const o_cfg *c, int size_na, int ptype, const double *vxp, int64_t n, const double *kq,
                    double *p_mts);
/* calc_avg (utils.f90:133-266) for one species: npg its np(0:nx+2, 0:ny+2); accumulates
 * data_pavg(7, na1+1, na2+1, ntype).  ss_src, ss_sink (nullable): the species' ss2D counts on
 * the (nx+3)(ny+3) nodes for the source/sink columns (plt_src = 0). */
void o_calc_avg(const o_cfg *c, int size_na, int ptype, const double *npg, const double *p_mts, double *data_pavg,
                const double *ss_src, const double *ss_sink);

#endif
