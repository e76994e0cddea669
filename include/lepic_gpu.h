/*
 * lepic_gpu.h -- C ABI of the B200 (sm_100a) implementation of the LePIC per-timestep
 * PIC-MCC loop.  Plain pointers and sizes only; every entry point returns LEPIC_OK (0) or a
 * negative LEPIC_E* code and never aborts the caller.
 *
 * The reference is F77-style Fortran with implicit interfaces (all arguments by reference,
 * global state in COMMON blocks).  Each entry point below names the reference routine it
 * replaces.  A Fortran host binds them with ISO_C_BINDING and keeps
 * its decks, tables and call sites; device state stays resident between calls and host
 * arrays are exchanged only where a pointer argument is non-NULL.
 *
 * Array layouts are the reference's Fortran memory order (first index fastest):
 *   node arrays  f(0:nx+2, 0:ny+2)         double / int32, index i + j*(nx+3)
 *   rhs          b(1:nx+1, 1:ny+1)         double, index (i-1) + (j-1)*(nx+1)
 *   E field      Ei(2, 0:nx+2, 0:ny+2)     double, interleaved (Ex, Ey)
 *   B field      Bi(4, 0:nx+2, 0:ny+2)     double, interleaved (Bx, By, Bz, |B|)
 *   particles    vxp(6, n) of one species  double, (x, y, z, vx, vy, vz) per particle
 *
 * Threading: one context is used by one host thread at a time.  All device work of a
 * context is ordered on the context's own CUDA stream (lepic_gpu_stream).  Calls whose
 * output pointers are all NULL only enqueue work; calls with an output pointer (or stats)
 * synchronise that stream before returning.
 */
#ifndef LEPIC_GPU_H
#define LEPIC_GPU_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define LEPIC_OK 0
#define LEPIC_EINVAL (-1)     /* bad argument or configuration                          */
#define LEPIC_ENOMEM (-2)     /* device allocation failed                               */
#define LEPIC_ECUDA (-3)      /* a CUDA runtime call failed                             */
#define LEPIC_ECAPACITY (-4)  /* a particle array or product list would overflow        */
#define LEPIC_EDIVERGED (-5)  /* Poisson residual grew 10x: iterative_solver.f90:42-50  */
#define LEPIC_ETIMEOUT (-6)   /* a bounded device-side wait gave up                     */
#define LEPIC_ERANGE (-7)     /* Pmax > 1 (collisions.f90:119-123) or a bad cell index  */
#define LEPIC_ENOTCONV (-8)   /* ncycl V-cycles (mixed: the CG cap) without reaching eps;
                                 phi holds the last iterate, with which the reference's
                                 iterative_solver.f90:56 goes on: a host may continue       */
#define LEPIC_ENOKERNEL (-9)  /* the library was not built for this GPU                 */

#define LEPIC_MAXSP 8   /* species (charged + neutral)  */
#define LEPIC_MAXCOL 64 /* reactions                    */

/* Poisson solve modes for lepic_gpu_iterative_solver */
#define LEPIC_POISSON_FP64_MG 0   /* the reference's V-cycle (mg.f90) in FP64              */
#define LEPIC_POISSON_MIXED_IR 1  /* FP64 CG preconditioned by an FP32 V-cycle            */
#define LEPIC_POISSON_FP64_MG_L2 2 /* mode 0's V-cycles, stopped on the L2 relative residual */
#define LEPIC_POISSON_LEARNED 3   /* mode 1 started from the learned network's prediction   */
#define LEPIC_POISSON_FP64_PCG 4  /* mode 1 with its V-cycle in FP64: the same algorithm, so that
                                     modes 4 and 1 compare the precision alone                  */

/* Grid selectors for lepic_gpu_get_grid / lepic_gpu_set_grid */
#define LEPIC_GRID_PHI 0      /* phi(0:nx+2,0:ny+2)                     */
#define LEPIC_GRID_RHS 1      /* rhs(1:nx+1,1:ny+1)                     */
#define LEPIC_GRID_EI 2       /* Ei(2,0:nx+2,0:ny+2)                    */
#define LEPIC_GRID_NP 16      /* + ptype: np(0:nx+2,0:ny+2,ptype)       */

typedef struct lepic_ctx lepic_ctx;

/* Scalars the reference keeps in the COMMON blocks part_info_int/dp_1/dp_2/dp_3 and constants (particle_info.h,
 * constants.h), plus the device capacities.  Species 0 is the electron, then ions, then
 * neutrals (negative mass, read_reactions.f90:200-205); indices are 0-based. */
typedef struct lepic_config {
    int32_t nx, ny;          /* cells (n(1), n(2)); nodes 1..n+1 plus ghosts 0 and n+2   */
    double dx, dy, zmax;     /* h(1), h(2) [m]; zmax [m] (1 m when hz < 0)               */
    double dt;               /* [s]                                                      */
    double eps0, qe;         /* qe is the float32-rounded 1.60217646e-19 (main.f90:120) */
    int32_t flag_pbc, flag_spec, flag_nmn;
    int32_t flag_B;          /* 0: none, 1: constant Bc, 2: map Bi on the field grid      */
    int32_t flag_B_pos;      /* 1: positive ions unmagnetised (part_expmover.f90:185)    */
    double Bc[3];
    int32_t ntype;           /* charged species                                          */
    int32_t nsp;             /* charged + neutral species                                */
    double charge[LEPIC_MAXSP], mass[LEPIC_MAXSP], Nm[LEPIC_MAXSP], vt0[LEPIC_MAXSP];
    double np_mx[LEPIC_MAXSP];    /* neutral densities at the neutral indices            */
    double nu_uplim[LEPIC_MAXSP]; /* main.f90:494-495                                    */
    int32_t ns_coll, nsort;       /* main.f90:479-480                                    */
    int32_t ng;                   /* multigrid levels (main.f90:264-277)                 */
    int32_t ncycl;                /* maximum V-cycles (main.f90:261)                     */
    double omega;                 /* SOR factor (iterative_solver.f90:28)                */
    int64_t capacity[LEPIC_MAXSP];/* particle slots per charged species (nmax)           */
    uint64_t seed;                /* counter-based RNG key                               */
    int32_t tile_w, tile_h;       /* sort tile in cells; 0,0 = the reference's row-major
                                     cell order (sorting.f90:151)                        */
} lepic_config;

/* Output of read_reactions/ordering (read_reactions.f90:511-697), species 0-based. */
typedef struct lepic_xs_tables {
    int32_t npt;               /* sig_npt_mx                                             */
    int32_t ncol;              /* reactions                                              */
    const double *sig_Er;      /* [npt]                                                  */
    const double *sig;         /* [icol*npt + ipt]                                       */
    const double *Eth;         /* [icol] threshold [eV]                                  */
    const int32_t *col_info;   /* [icol*10 + k] = col_info(icol, k+1), species 0-based   */
    const int32_t *p_ncol;     /* [ptype]                                                */
    const int32_t *sig_list;   /* [ptype*LEPIC_MAXCOL + k], reaction index 0-based       */
    const double *sigv_mx;     /* [ptype*LEPIC_MAXCOL + icol]                            */
    int32_t flag_ionrep;
    double fEk;
} lepic_xs_tables;

typedef struct lepic_solve_stats {
    int32_t cycles;            /* V-cycles (k)                                           */
    int32_t sweeps_fine;       /* SOR sweeps on the finest level                         */
    double res_l1;             /* the reference's normalised L1 residual                 */
    double res_l2_rel;         /* ||b - A u||_2 / ||b||_2 over interior nodes, FP64      */
    double ktot;               /* equivalent fine-grid SOR sweeps (mg.f90:227-229)       */
} lepic_solve_stats;

typedef struct lepic_push_stats {
    int64_t np_tot[LEPIC_MAXSP];  /* live particles after the call                     */
    int64_t n_lost[LEPIC_MAXSP];  /* cumulative wall losses                             */
    int64_t n_dead[LEPIC_MAXSP];  /* cumulative removals of collision-killed particles  */
    int64_t n_slots[LEPIC_MAXSP]; /* occupied slots (live + holes until the next sort)  */
} lepic_push_stats;

typedef struct lepic_mcc_stats {
    int64_t n_cand[LEPIC_MAXSP];  /* cumulative collision candidates                    */
    int64_t n_coll[LEPIC_MAXCOL]; /* cumulative real collisions per reaction            */
    int64_t n_add[LEPIC_MAXSP];   /* cumulative products appended                       */
    int64_t n_overflow;           /* relative energies above the table's last point     */
    double nu_max[LEPIC_MAXSP];   /* collisions.f90:98-106                              */
} lepic_mcc_stats;

/* Synthetic initial load (the one-time load_part.f90:59-224 on the device).  Every sample
 * places one particle of each charged species at the same position (load_part.f90:141),
 * positions follow the density profile, velocities are Maxwellian at vt0. */
typedef struct lepic_load_spec {
    int64_t n_samples;        /* particles per charged species                          */
    int32_t profile;          /* 0: uniform, 1: n_floor + (n_peak-n_floor)*gaussian      */
    double x_load;            /* samples limited to x < x_load [m] (load_part.f90:104)  */
    double n_peak, n_floor;   /* profile 1 [m^-3]                                        */
    double sigma;             /* profile 1 Gaussian sigma [m], centred in the box       */
    uint64_t seed;
} lepic_load_spec;

/* Version of this ABI. */
int32_t lepic_gpu_abi_version(void);

/* Creates a context on the current CUDA device.  bcnd: node labels (>0 Dirichlet wall,
 * -1 interior, -2 Neumann, 0 periodic, <=-4 dielectric) as generate_boundary.f90 leaves
 * them; phi_init: the wall potentials (generate_boundary.f90:210-216); Bi may be NULL when
 * flag_B != 2; xs may be NULL (collision-less).  Replaces the device-side half of
 * main.f90:192-214 (allocation) and main.f90:334-344 (kq). */
int lepic_gpu_create(const lepic_config *cfg, const int32_t *bcnd, const double *phi_init,
                     const double *Bi, const lepic_xs_tables *xs, lepic_ctx **out);
int lepic_gpu_destroy(lepic_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t). */
void *lepic_gpu_stream(lepic_ctx *ctx);
/* Waits for the context's stream and the asynchronous downloads, and reports any device-side
 * error flag as a code. */
int lepic_gpu_sync(lepic_ctx *ctx);
/* Text of the last error of this context (valid until the next call); with ctx NULL, the
 * reason of the last failed lepic_gpu_create. */
const char *lepic_gpu_last_error(lepic_ctx *ctx);

/* Uploads n particles of one charged species, AoS FP64 as vxp(6,n) (z is not kept).
 * Replaces the particle half of restart.f90:48-149.  Particles must lie in the box. */
int lepic_gpu_put_particles(lepic_ctx *ctx, int32_t ptype, const double *vxp, int64_t n);
/* Downloads the live particles of one species in slot order (holes removed), AoS FP64
 * with z = 0.  The backup writer main.f90:1102-1139 reads this. */
int lepic_gpu_get_particles(lepic_ctx *ctx, int32_t ptype, double *vxp, int64_t cap,
                            int64_t *n_out);
/* The same with the reference's own particle array vxp(6, nmax, ntype, nproc) and
 * np_tot(ntype, nproc) (main.f90:192-214): put concatenates a species' slabs in slab order
 * (replacing its particles); get deals a species' live particles to the nproc slabs in equal
 * parts in slot order, as sorting.f90:92-251 rebalances them (LEPIC_ECAPACITY if a slab would
 * exceed nmax). */
int lepic_gpu_put_particles_slabs(lepic_ctx *ctx, const double *vxp, const int32_t *np_tot, int64_t nmax,
                                  int32_t ntype, int32_t nproc);
int lepic_gpu_get_particles_slabs(lepic_ctx *ctx, double *vxp, int32_t *np_tot, int64_t nmax, int32_t ntype,
                                  int32_t nproc);
/* Synthetic initial load on the device (see lepic_load_spec). */
int lepic_gpu_load_particles(lepic_ctx *ctx, const lepic_load_spec *spec);

/* charge_deposition (part_expmover.f90:520-610) of every charged species into np, after
 * zeroing it (main.f90:1076); used after a load or a restart. */
int lepic_gpu_charge_deposition(lepic_ctx *ctx);
/* np_periodic + calc_rhs (calc_rho.f90:1-77): rhs = -sum charge*np.  rhs_out (nullable)
 * receives rhs(1:nx+1,1:ny+1). */
int lepic_gpu_calc_rhs(lepic_ctx *ctx, double *rhs_out);
/* dens_red (calc_rho.f90:134-199): np_red_out (nullable) receives ntype node grids,
 * np_mx_out (nullable) the ntype interior maxima. */
int lepic_gpu_dens_red(lepic_ctx *ctx, double *np_red_out, double *np_mx_out);
/* iterative_solver (iterative_solver.f90:1-69 -> mg.f90 -> sors.f90) on the device phi.
 * phi_inout (nullable): uploaded first (warm start) and downloaded after.  eps is the
 * reference's normalised L1 tolerance for mode 0 and the FP64 relative L2 tolerance
 * ||b-Au||/||b|| for mode 1.  stats (nullable) forces a sync. */
int lepic_gpu_iterative_solver(lepic_ctx *ctx, double *phi_inout, double eps, int32_t mode,
                               lepic_solve_stats *stats);
/* The same solve with its two copies split and the download overlapped: phi_in (nullable) is
 * uploaded before the solve (after any download into host memory still in flight), and phi_out
 * (nullable, may be the same array) receives the solution asynchronously -- the call returns
 * without waiting, the copy runs beside the kernels enqueued next (E field, push), and phi_out
 * is filled once a call that synchronises the context returns (lepic_gpu_sync, or any call with
 * an output pointer or stats).  The host must not read or write phi_out before that. */
int lepic_gpu_iterative_solver_async(lepic_ctx *ctx, const double *phi_in, double *phi_out, double eps,
                                     int32_t mode);
/* Stages the next solve's phi input now, on the copy stream: the host array is copied into phi
 * after the work enqueued so far (the E field that reads phi) and after the copy stream's earlier
 * copies (a download into the same array), beside the kernels enqueued next (the push); the next
 * call that reads or writes phi waits for it.  It is the phi_in of the next
 * lepic_gpu_iterative_solver[_async] call (which then passes NULL), moved off the critical path:
 * a host that keeps phi on its side every step calls
 *   solve_async(NULL, phi) -> efield -> [sort, collisions] -> stage_solver_input(phi) -> push
 * and every step still copies phi both ways.  phi_in must stay unchanged until a call that
 * synchronises the context returns. */
int lepic_gpu_stage_solver_input(lepic_ctx *ctx, const double *phi_in);
/* Warm start of the mixed-precision solve (mode 1): 0 (default) starts from the input phi, as
 * iterative_solver does with its in/out u; 1 starts from the linear extrapolation
 * 2 phi_(n-1) - phi_(n-2) of the inputs of this and the previous solve, for a time loop in
 * which each solve's input is the previous solution.  The answer meets the same tolerance on
 * the true residual either way; a smooth potential needs fewer iterations (2 instead of 4 on
 * the 2048^2 bench).  lepic_gpu_set_grid(LEPIC_GRID_PHI) and this call forget the history. */
int lepic_gpu_set_warm_start(lepic_ctx *ctx, int32_t mode);
/* calc_Efield (Efield.f90:1-128).  Ei_out (nullable) receives Ei(2,0:nx+2,0:ny+2) FP64. */
int lepic_gpu_calc_efield(lepic_ctx *ctx, double *Ei_out);
/* part_sorting (sorting.f90:92-251) of one species by cell.  plist_out (nullable,
 * nx+nx*ny+2 entries) receives Plist(0:pl_max) when the context uses the reference order. */
int lepic_gpu_part_sorting(lepic_ctx *ctx, int32_t ptype, int32_t *plist_out);
/* collisions (collisions.f90:1-207, collision_OMP, SCATTER) for every species, neutral
 * targets, null-collision MCC with a counter-based RNG keyed by (seed, it, species, slot). */
int lepic_gpu_collisions(lepic_ctx *ctx, int32_t it, lepic_mcc_stats *stats);
/* part_mover (part_expmover.f90:1-517) fused with charge_deposition (:520-610) for every
 * charged species: np is zeroed and rebuilt from the moved particles. */
int lepic_gpu_push_deposit(lepic_ctx *ctx, int32_t it, lepic_push_stats *stats);
/* One PIC step, the in-scope body of main.f90:818-1090: calc_rhs -> iterative_solver ->
 * calc_Efield -> part_sorting (MOD(it,nsort)==1) -> [averages, MOD(it,navg)==1]
 * -> collisions (it>1, MOD(it,ns_coll)==1) -> [eheating, MOD(it,ns_heat)==0] -> push_deposit
 * -> [part_injection, MOD(it,ns_inj)==0] -> [part_flux_emitter, js > 0 and (ns_Hm == 1 or
 * MOD(it,ns_Hm) == 1)]; the averages only after lepic_gpu_set_avg, the source steps only after
 * lepic_gpu_set_sources.  eps / mode as lepic_gpu_iterative_solver. */
int lepic_gpu_step(lepic_ctx *ctx, int32_t it, double eps, int32_t mode);

/* Settings of the solvers and of the cooperative launches.  No counterpart in the reference
 * (whose solver settings are the constants of iterative_solver.f90 and sors.f90); the defaults
 * are the measured best on a B200 and nothing else (no environment variable) changes them.
 * Read the current values with lepic_gpu_get_options, change fields, write them back. */
typedef struct lepic_options {
    int32_t mx_nu1, mx_nu2;      /* FP32 V-cycle: sweeps before / after the coarse correction (2, 2)  */
    int32_t mx_nuc;              /* sweeps each way on the coarsest level (2)                        */
    float mx_omega;              /* over-relaxation of the FP32 sweeps (1.15)                        */
    int32_t mx_onchip_bytes;     /* shared memory for the coarse levels CTA 0 runs alone (20480)     */
    int32_t mx_tiled;            /* 1: fine-level sweeps on shared-memory tiles (default); 0: grid-
                                    wide half-sweeps -- identical results, for checking the tiles   */
    int32_t mx_max_iter;         /* CG iterations before LEPIC_ENOTCONV (200)                        */
    int32_t mx_coarse_direct;    /* 1: the on-chip levels' top level (at most 2048 unknowns) solved
                                    exactly by its precomputed inverse, applied by every CTA
                                    (default); 0: CTA 0 cycles through the on-chip levels         */
    int32_t mg_small_nodes;      /* FP64 V-cycle: levels of at most this many nodes on CTA 0 (4500)  */
    int32_t ctas_per_sm;         /* CTAs per SM of the cooperative solver kernels (3)                */
    int32_t barrier_extra;       /* test hook, 0 in use: the solvers' grid barriers wait for this
                                    many CTAs beyond the launch, so the first wait runs out (after
                                    about 2 s), the kernel ends and the call returns LEPIC_ETIMEOUT */
    int64_t fortran_max_subrecord; /* backup writer: subrecord length limit (2^31 - 9, the Intel and
                                    GNU runtimes' value); smaller values exercise the layout         */
    int32_t sort_defer;          /* 1 (default): a sort leaves its permutation pending and the next
                                    push moves the records as it writes them (one pass over them
                                    fewer; every other call that reads them moves them first);
                                    0: the sort moves them itself -- the same order and results  */
    int32_t pad;
} lepic_options;
int lepic_gpu_get_options(lepic_ctx *ctx, lepic_options *out);
int lepic_gpu_set_options(lepic_ctx *ctx, const lepic_options *in);

/* Copies a device grid (LEPIC_GRID_*) to the host, FP64, in the layouts above. */
int lepic_gpu_get_grid(lepic_ctx *ctx, int32_t which, double *out);
/* The same for LEPIC_GRID_PHI, _RHS and _EI without waiting: the grid as it is after the work
 * enqueued so far is copied beside the work enqueued next; out is filled once a call that
 * synchronises the context returns (as for lepic_gpu_iterative_solver_async's phi_out). */
int lepic_gpu_get_grid_async(lepic_ctx *ctx, int32_t which, double *out);
/* Sets phi (LEPIC_GRID_PHI) or rhs (LEPIC_GRID_RHS) from the host. */
int lepic_gpu_set_grid(lepic_ctx *ctx, int32_t which, const double *in);
/* Live particles per species and the cumulative counters. */
int lepic_gpu_get_push_stats(lepic_ctx *ctx, lepic_push_stats *stats);
int lepic_gpu_get_mcc_stats(lepic_ctx *ctx, lepic_mcc_stats *stats);

/* Device pointer of one species' charge accumulator: (nx+3)*(ny+3) int64 node values, the
 * deposited CIC weights in units of 2^-44 (the np grid before its FP64 scaling).  Summing
 * these integers across ranks (e.g. an NCCL int64 all-reduce after lepic_gpu_push_deposit)
 * is the multi-GPU form of calc_rho.f90:71-74 and is exact. */
int lepic_gpu_deposit_grid(lepic_ctx *ctx, int32_t ptype, void **acc);

/* Charge deposition that allocates no device memory.  No counterpart in the reference: it is
 * for callers that cannot call cudaMalloc -- a host whose device memory is reserved up front
 * and handed out by its own (or another framework's) allocator, or code where the implicit
 * synchronisation of an allocation is not allowed.  The caller passes device pointers it
 * owns: X, Y (n fixed-point positions with `shift` fractional bits, as
 * lepic_gpu_particle_arrays returns them), VX (NaN marks a hole left by a lost particle), kq
 * ((nx+3)*(ny+3) node factors), and np_out ((nx+3)*(ny+3) doubles) which receives
 * np = kq * k1 * sum of CIC weights, k1 = Nm / (dx*dy*zmax) -- the np grid of
 * charge_deposition (part_expmover.f90:520-610), identical to the context path.
 * A hole's X and Y do not hold a position, so VX may be NULL only when every one of the n
 * slots is a live particle (freshly loaded or put, or compacted by lepic_gpu_part_sorting);
 * with VX NULL a hole would be deposited as a particle.  A position outside the box
 * (X >= nx << shift or Y >= ny << shift) is skipped, not deposited and not reported.
 * The temporary uint64 accumulator is a fixed static device array of 2^20 nodes (8 MiB) that
 * every GPU loading the library keeps until exit; larger grids ((nx+3)*(ny+3) > 2^20) are
 * rejected with LEPIC_ECAPACITY.  The first call on a device looks up that array's device
 * address and the SM count, so make it before any stream capture.  All calls on a device
 * share the array and each call clears it first: calls that overlap on the GPU race and must
 * be serialised by the caller.  An error left pending by the caller's earlier CUDA work is
 * returned as LEPIC_ECUDA (and left pending) before anything is enqueued.
 * stream is a cudaStream_t (NULL: the default stream); the call only enqueues work. */
int lepic_gpu_deposit_noalloc(const uint32_t *X, const uint32_t *Y, const float *VX, int64_t n,
                              int32_t nx, int32_t ny, int32_t shift, double k1, const double *kq,
                              double *np_out, void *stream);

/* Raw device pointers of one species' SoA arrays (for in-process tools and tests):
 * X, Y are uint32 fixed point in cell units with `shift` fractional bits, VX/VY/VZ float. */
int lepic_gpu_particle_arrays(lepic_ctx *ctx, int32_t ptype, void **X, void **Y, void **VX,
                              void **VY, void **VZ, int64_t *n_slots, int32_t *shift);

/* ---- particle sources: electron heating and volume injection ---------------------------
 * The rest of the reference's per-step particle region (main.f90:1033-1068) on the device:
 * eheating (e_heating.f90:1-112) before the mover, part_injection (part_injection.f90:1-237)
 * after it, and the heating-region tallies that charge_deposition keeps for the
 * self-consistent electron temperature (part_expmover.f90:583-605, main.f90:984-1011).
 * Random numbers come from counter-based streams keyed by (seed, step, species, slot or
 * injected index), so a run is reproducible whatever the launch shape. */
#define LEPIC_MAXICP 16   /* heating bands along y (n_icp) */

/* The deck values of read_input.f90:43-55 and :80-97 and main.f90:493-500, lengths in
 * metres (after the reference's cm -> m and ABS). */
typedef struct lepic_source_config {
    int32_t flag_c;            /* 0: slit |x-xa| <= dr, yl_pow <= y <= yr_pow; 1: disk
                                  (x-xa)^2 + (y-ymax/2)^2 <= dr^2 (xa, dr from xl/xr_pow)  */
    double xl_pow, xr_pow, yl_pow, yr_pow;
    /* eheating */
    int32_t flag_heat;         /* nu_h >= 0 in the deck                                    */
    int32_t ns_heat;           /* heating every ns_heat steps (MOD(it,ns_heat) == 0)       */
    int32_t eheat_type;        /* 1: velocity replaced by a Maxwellian draw; 2: increment  */
    int32_t flag_gpp;          /* 1: Gaussian power profile, nu = 9 Pabs_cor <nu> e^(-9r^2/dr^2) */
    int32_t n_icp;             /* bands along y (1..LEPIC_MAXICP)                          */
    int32_t te_update;         /* 1: lepic_gpu_step updates vt itself before each heating
                                  from this context's tallies (main.f90:984-1011 on one
                                  rank); 0: the host sets vt (lepic_gpu_set_heating)      */
    double nudt;               /* nu_h * ns_heat * dt (main.f90:493)                       */
    double nu_h;               /* [1/s]                                                    */
    double Pabs[LEPIC_MAXICP]; /* absorbed power per band [W]; Pabs[0] > 0 turns on the
                                  region tallies and the self-consistent temperature       */
    double Pabs_cor;           /* Gaussian-profile correction (main.f90:1305-1306)         */
    double vt[LEPIC_MAXICP];   /* heating thermal speed per band [m/s] (main.f90:1010)     */
    /* part_injection */
    int32_t flag_inj;          /* I_inj >= 0 in the deck                                   */
    int32_t ns_inj;            /* injection every ns_inj steps (MOD(it,ns_inj) == 0)       */
    int32_t opt_inj;           /* +-1: fixed current; +-2: a pair per lost positive ion; +-3:
                                  electron beam along z; +-4: emission from the cathode at
                                  x = 0 with a shifted-Maxwellian flux; < 0: Gaussian loading */
    int32_t flag_Tp;           /* 1: electrons injected at THm (|opt_inj| <= 2)            */
    int32_t flag_diffsrc;      /* 1: tally -Nm q phi at each injected particle (P_loss(1)) */
    int32_t tag_neg;           /* 0-based negative-ion species, -1 if none                 */
    int32_t nproc_mpi;         /* ranks sharing I_inj (one context per rank)               */
    double I_inj;              /* [A]                                                      */
    double THm;                /* [eV]                                                     */
    double ni0[LEPIC_MAXSP];   /* charged-species fractions (read_reactions.f90, main.f90:180) */
    uint64_t seed;             /* key of the heating, injection and emission streams       */
    /* part_flux_emitter (part_flux_emitter.f90:1-217): surface emission from the grid plane
     * x = xg1 of the deck (read_input.f90:142-151, generate_boundary.f90:246-271) */
    double js;                 /* emitted current density [A/m^2] (jne*10); <= 0: off      */
    int32_t ptype_fx;          /* 0-based emitted species                                  */
    int32_t tag_b;             /* 0-based species of the chamfer-emitted particles, -1 none */
    int32_t ns_Hm;             /* emission when ns_Hm == 1 or MOD(it, ns_Hm) == 1          */
    int32_t n_holes;
    double xg1, Lg, Lh;        /* grid plane, grid length, hole half size [m] (Lh rounded
                                  to the cell as generate_boundary.f90:267-270 does)       */
    int32_t flag_chmfrd;       /* chamfered aperture (generate_boundary.f90:110-116)       */
    double chmfrd[4];          /* chmfrd_array: x1, x2, (ymax/2 - y1), (ymax/2 - y2) [m]   */
    double th_B;               /* angle of B to the x axis for opt_inj = 4 (main.f90:450-452) */
} lepic_source_config;

/* Cumulative tallies since the context was created or last reset; the reference's names. */
typedef struct lepic_source_tally {
    double P_heat;                   /* P_loss(2,1): sum 0.5 Nm m (v_new^2 - v_old^2) [J]   */
    int64_t n_heated;                /* heating events                                     */
    int64_t n_heat_calls;            /* eheating calls                                     */
    double P_inj[LEPIC_MAXSP];       /* P_loss(4,ptype): sum 0.5 Nm m v^2 of injected [J]  */
    double P_src[LEPIC_MAXSP];       /* P_loss(1,ptype): sum -Nm q phi (flag_diffsrc) [J]  */
    int64_t n_inj[LEPIC_MAXSP];      /* particles injected                                 */
    int64_t n_inj_last[LEPIC_MAXSP]; /* N_inj of the last injection call                   */
    int32_t n_icp;
    int64_t Nh[LEPIC_MAXICP];        /* electrons in the heating region, per band, at the
                                        last tally (charge_deposition's Nh)                */
    double sum_dEk[LEPIC_MAXICP];    /* their kinetic energy 0.5 Nm m v^2 (eheat_type 1)   */
    double vt[LEPIC_MAXICP];         /* heating thermal speed in use                       */
    int64_t n_emit[LEPIC_MAXSP];     /* particles emitted by part_flux_emitter (cumulative) */
    int64_t n_emit_last[LEPIC_MAXSP];/* ... by its last call                                */
    int64_t n_emit_out;              /* emitted, then outside the box after their first
                                        partial move: counted as wall losses (n_lost)      */
} lepic_source_tally;

/* Sets (or replaces) the source configuration; flag_heat = flag_inj = 0 turns both off.
 * lepic_gpu_step then runs eheating before the push and part_injection after it at their
 * cadences, as main.f90:1033-1068 does. */
int lepic_gpu_set_sources(lepic_ctx *ctx, const lepic_source_config *cfg);
/* The host-side temperature update (main.f90:984-1011, e.g. after an MPI reduction of the
 * tallies): new heating speeds per band (n_icp entries) and the Gaussian-profile factor. */
int lepic_gpu_set_heating(lepic_ctx *ctx, const double *vt, int32_t n_icp, double Pabs_cor);
/* eheating (e_heating.f90:1-112) of the electrons at step it (the caller checks the
 * cadence).  Enqueues only. */
int lepic_gpu_eheating(lepic_ctx *ctx, int32_t it);
/* part_injection (part_injection.f90:1-237) of every charged species at step it, in the
 * species order of main.f90:1057-1064, followed by the deposit of the injected particles
 * into np (they are deposited in the step they are born, main.f90:1069-1085).  The counts
 * are computed on the device (fixed current, or the positive-ion losses since the last
 * injection for |opt_inj| = 2).  Enqueues only. */
int lepic_gpu_part_injection(lepic_ctx *ctx, int32_t it);
/* part_flux_emitter (part_flux_emitter.f90:1-217) at step it (the caller checks the
 * cadence): the emitted particles are appended after the deposit (main.f90:1093-1096), so
 * they enter np with the next push.  Enqueues only. */
int lepic_gpu_flux_emitter(lepic_ctx *ctx, int32_t it);
/* charge_deposition's heating-region tallies (Nh, sum_dEk per band) of the current
 * electrons.  Enqueues only; lepic_gpu_source_tallies reads them. */
int lepic_gpu_heating_tally(lepic_ctx *ctx);
/* Reads the tallies (synchronises); reset != 0 zeroes the cumulative ones afterwards. */
int lepic_gpu_source_tallies(lepic_ctx *ctx, lepic_source_tally *out, int32_t reset);

/* ---- averaging diagnostics ------------------------------------------------------------
 * part_moments (utils.f90:1-131) + calc_avg (utils.f90:133-266) + the potential and field
 * averages (main.f90:935-947) on the device, so the averages need no host transfer until the
 * host writes them.  While averaging is configured the device also keeps ss2D with the
 * reference's default plt_src = 0: per species and node a count of macroparticles made
 * (injection, part_injection.f90:205; emission, part_flux_emitter.f90:175; collision
 * products, collisions.f90:809) and removed (wall losses at the nearest node,
 * part_expmover.f90:327-332; collision removals, collisions.f90:931); each sample adds them
 * times Nm/Vc to data_pavg's source/sink columns (6, 7) and zeroes them (main.f90:929-931). */
/* Allocates (or re-allocates and zeroes) the averages on the coarse grid na = n / size_na
 * (read_input.f90:109-111); navg > 0 makes lepic_gpu_step take one sample when
 * MOD(it,navg) == 1, after the sort (main.f90:906). */
int lepic_gpu_set_avg(lepic_ctx *ctx, int32_t size_na, int32_t navg);
/* One averaging sample now (enqueues only). */
int lepic_gpu_calc_avg(lepic_ctx *ctx);
/* Reads data_pavg(7, na1+1, na2+1, ntype) and phi_avg(3, 0:nx+2, 0:ny+2) (each nullable) and
 * the sample count cnt_avg; reset != 0 zeroes them afterwards (main.f90:1290-1296). */
int lepic_gpu_get_avg(lepic_ctx *ctx, double *data_pavg, double *phi_avg, int32_t *cnt_avg, int32_t reset);
/* Reads the current ss2D(2, 0:nx+2, 0:ny+2, ntype) (one rank; synchronises): the counts with
 * plt_src = 0, the densities of the last sample with plt_src = 1.  Replaces the host's copy of
 * ss2D (main.f90:90, 209, 242, 921-931). */
int lepic_gpu_get_source_maps(lepic_ctx *ctx, double *ss2D);
/* plt_src (read_input.f90:113-117, a negative k_eps0 in the deck): 0 (default) counts made and
 * removed macroparticles; 1 makes each averaging sample (lepic_gpu_calc_avg or the step's
 * sample) first run collisions with flag_diag = 1 (collisions.f90:268-299, 546-600, 649): every
 * particle through the collision frequencies of its reactions, no collision performed, the
 * ionization, dissociation and charge-exchange frequencies times Nm/Vc deposited with CIC
 * weights as source (charged byproducts) and sink (charged reactants that do not survive)
 * densities, which calc_avg adds to data_pavg(6:7, ...) as they are (utils.f90:205-209); the
 * region tallies cnt_col count that pass too, as the reference's do. */
int lepic_gpu_set_source_option(lepic_ctx *ctx, int32_t plt_src);

/* Loss, power and collision tallies, cumulative since the context was created or the last
 * reset: part_mover's p_mac and P_loss(1) (part_expmover.f90:316-427), collisions' P_loss(3)
 * and cnt_col (collisions.f90:533-543, 896-899, 980-983, 1025-1033; the removal of a killed
 * incident, part_expmover.f90:83-96, is counted when it is killed), and the sources' P_loss(2)
 * and P_loss(4) (see lepic_source_tally).  FP64 sums made with device atomics: they agree with
 * an ordered FP64 sum to rounding, not bit for bit. */
#define LEPIC_MAXLABEL 16   /* wall labels kept apart (bcnd values, larger ones in the last) */
#define LEPIC_MAXRG 8       /* x-regions of cnt_col (nm_rg)                               */
typedef struct lepic_tallies {
    int64_t n_loss[LEPIC_MAXSP][LEPIC_MAXLABEL]; /* p_mac(ptype, np_loss, igrid): wall losses by
                                                    the label bcnd(ix,iy) of the loss cell   */
    double P_w[LEPIC_MAXSP][LEPIC_MAXLABEL];     /* p_mac(ptype, P_w, igrid): their 0.5 Nm m v^2 [J] */
    double P_loss[4][LEPIC_MAXSP];               /* P_loss(1..4, ptype) [J]: 1 wall losses (+ the
                                                    injection's -Nm q phi term), 2 heating, 3
                                                    collisions, 4 injection and emission      */
    double cnt_col[3][LEPIC_MAXCOL][LEPIC_MAXRG];/* cnt_col(1..3, icol, i_rg): sum nu over the
                                                    candidates, candidate count, sum 1/np_tot_rg
                                                    over the collisions                       */
    int32_t n_rg;
} lepic_tallies;

/* The x-regions of the collision tallies (read_input.f90:120-128; main.f90:316-328): n_rg
 * ranges [xl_rg, xr_rg] and one [yl_rg, yr_rg], metres.  n_rg = 0: none. */
int lepic_gpu_set_regions(lepic_ctx *ctx, int32_t n_rg, const double *xl_rg, const double *xr_rg,
                          double yl_rg, double yr_rg);
/* Reads the tallies (synchronises); reset != 0 zeroes them and the sources' power tallies
 * afterwards (main.f90:1296-1300). */
int lepic_gpu_get_tallies(lepic_ctx *ctx, lepic_tallies *out, int32_t reset);

/* ---- the 3rd virtual dimension of the 2.5D model (hz >= 0) ------------------------------
 * read_input.f90:158-162 and part_expmover.f90:216-219, 269-309, 400-421: each particle keeps
 * z in [0, zmax] (zmax = lepic_config.zmax, the deck's length in the 3rd dimension); electrons
 * and negative ions reaching z <= 0 or z >= zmax are lost through the end plates when
 * 0.5 m vz^2 / qe >= phi(ix,iy) - phi0, else reflected (vz -> -vz, z -> 0.02 or 0.98 zmax);
 * positive ions are lost with probability hz 2 uB / zmax * dt per step, uB the Bohm speed on the
 * averaging grid (main.f90:950-960: sqrt(qe Te / m) from the averaged electron temperature,
 * formed after each averaging sample of the device, or set by the host).  Such a loss has no
 * wall label (p_mac's igrid 0) and adds Nm q phi at the loss point to P_loss(1).  The
 * particles already loaded get z = rnd zmax; loads, injections and emissions draw z as the
 * reference does, collision products take their parent's z, and put/get, backups and sorts
 * carry it. */
typedef struct lepic_zloss_config {
    double hz;           /* h = ns/<n> of the deck; < 0: no 3rd-dimension losses (the default) */
    double phi0;         /* end-plate potential [V] (read_input.f90:158)                      */
    int32_t size_na;     /* the uB grid: na = n / size_na (read_input.f90:109-111)            */
} lepic_zloss_config;
int lepic_gpu_set_zloss(lepic_ctx *ctx, const lepic_zloss_config *cfg);
/* uB(na1+1, na2+1, ntype) [m/s] in Fortran order (main.f90:197), from the host (e.g. after an
 * MPI reduction of the averages); the device's averaging samples overwrite it. */
int lepic_gpu_set_bohm_speed(lepic_ctx *ctx, const double *uB);

/* ---- dielectric walls (generate_boundary.f90:149-152, part_expmover.f90:340-350,
 * main.f90:756-809) ------------------------------------------------------------------------
 * dtype[label] (LEPIC_MAXLABEL entries, labels above the last in the last): 1 for a wall label
 * drawn as dielectric, else 0; Ca its capacitance [F/m^2].  A wall loss on a dielectric label
 * (or under one) leaves Nm q on the label's rows iy and iy+1 of the loss cell, split by the loss
 * point's y; once per step before the Poisson solve (lepic_gpu_step does it, or call
 * lepic_gpu_dielectric_update) the label's wall nodes of rows 2..ny (every row with the periodic
 * option) take phi += kd dq(label, iy) / (Ca dy), kd = 2 on rows 1 and ny+1, and the charge
 * starts again from zero.  A multi-rank host sums the charges over its ranks first, as
 * main.f90:771-772 does (get, all-reduce, set, then lepic_gpu_dielectric_update before the
 * solve; lepic_gpu_step then finds nothing left to add). */
int lepic_gpu_set_dielectrics(lepic_ctx *ctx, const int32_t *dtype, double Ca);
int lepic_gpu_dielectric_update(lepic_ctx *ctx);
/* the charge collected since the last update, dq(0:ny+2, label) as [label][ny+3] [C] */
int lepic_gpu_get_dielectric_charge(lepic_ctx *ctx, double *dq);
/* replaces it (a multi-rank host: the sum over ranks, main.f90:771-772, before the update) */
int lepic_gpu_set_dielectric_charge(lepic_ctx *ctx, const double *dq);

/* ---- secondary emission (read_input.f90:164-184, generate_boundary.f90:119-122,
 * part_expmover.f90:354-392) -----------------------------------------------------------------
 * A positive ion lost on the wall label igrid_sec emits INT(gam_sec) electrons, one more with
 * probability gam_sec - INT(gam_sec), at (xg_sec, y, z) of its loss point with
 * vx = -SIGN(1, vx_ion) vt sqrt(-ln(1-r)), (vy, vz) Maxwellian, vt = sqrt(2 qe THm / m_e); they
 * are appended to the electrons after the push (in the order of their ions' slots) and are in
 * that step's density.  Each adds 0.5 Nm m (vx^2 + vz^2 + vz^2) to the electrons' P_loss(4),
 * the reference's sum.  The draws come from the counter stream keyed by (seed, step, species,
 * slot, electron).  gam_sec = 0 switches it off; 0 <= gam_sec < 8. */
typedef struct lepic_secondary_config {
    double gam_sec;            /* emission coefficient                                     */
    int32_t igrid_sec;         /* the emitting wall label (ABS of the deck's value), >= 1  */
    int32_t pad;
    double xg_sec;             /* x of the emitting grid [m]                               */
    double THm;                /* the electrons' temperature [eV]                          */
} lepic_secondary_config;
int lepic_gpu_set_secondary(lepic_ctx *ctx, const lepic_secondary_config *sec);

/* ---- particle backup (main.f90:1102-1139, restart.f90:48-149) ---------------------------
 * The reference's particlesNNN.bak: Fortran unformatted sequential records (4-byte length
 * markers; records over 2^31-9 bytes split into subrecords as the Intel and GNU runtimes do):
 * (time, gtype, Pabs_cor), np_tot(1:ntype, 1:nproc), then vxp(6, np_tot) per iproc and ptype,
 * FP64.  Written and read in chunks between the device and pinned host buffers. */
/* Writes the live particles of every charged species (slot order, holes skipped; nproc = 1;
 * z written as 0). */
int lepic_gpu_write_backup(lepic_ctx *ctx, const char *path, double time, int32_t gtype, double Pabs_cor);
/* Reads a backup written with any nproc (a species' blocks are appended in file order, as
 * restart.f90:101-133 does for a different thread count) after the occupied slots, then
 * deposits every species into np (restart_OMP).  time, gtype, Pabs_cor (nullable) receive the
 * header.  LEPIC_ECAPACITY if the particles do not fit (restart.f90:117-121). */
int lepic_gpu_read_backup(lepic_ctx *ctx, const char *path, double *time, int32_t *gtype, double *Pabs_cor);
/* The restart's particle duplication (restart.f90:115-129): with |np_dup| > 1 every species'
 * particles are followed by |np_dup| - 1 copies of themselves, then deposited into np
 * (restart_OMP).  LEPIC_ECAPACITY if |np_dup| times the occupied slots exceeds the capacity
 * (restart.f90:117-121).  The reference's external restart (flag_restart = 2, SAV_DATA) reads
 * several files into one rank: call lepic_gpu_read_backup once per file (each appends), then
 * this. */
int lepic_gpu_duplicate_particles(lepic_ctx *ctx, int32_t np_dup);

/* ---- learned warm start of the Poisson solve (no counterpart in the reference) ----------
 * Mode LEPIC_POISSON_LEARNED of lepic_gpu_iterative_solver: a 4-level convolutional network
 * (3x3 convolutions, channels 16/32/64/64, BF16 tensor-core convolutions with FP32
 * accumulation) maps (residual of the previous potential b - A phi_prev, scaled by its RMS;
 * phi_prev scaled) to a correction of phi; the correction is kept only if it lowers the FP64
 * residual, then mode 1 refines it to the requested residual.  After the solve the network is
 * trained online (Adam) on crops of the pair it just saw: input -> (phi_solved - phi_prev)
 * scaled, with the energy norm of the error as the loss.  Periodic or Neumann decks take
 * mode 1's path for them (the FP64 V-cycle). */
typedef struct {
    int32_t enable_training;  /* 0: inference only                                        */
    int32_t warmup_solves;    /* the first solves train every time ...                    */
    int32_t steps_warmup;     /* ... with this many Adam steps each                       */
    int32_t train_every;      /* afterwards every train_every-th solve trains ...          */
    int32_t steps_after;      /* ... with this many steps                                  */
    int32_t crop;             /* training crop edge (pixels, multiple of 8)               */
    int32_t batch;            /* crops per Adam step (1..8)                               */
    float lr;                 /* Adam learning rate                                       */
    uint64_t seed;            /* weight initialisation and crop positions                 */
} lepic_cnn_config;

typedef struct {
    int64_t solves;           /* learned-mode solves so far                               */
    int64_t train_steps;      /* Adam steps so far                                        */
    int32_t last_accepted;    /* 1 if the last prediction was kept                        */
    double last_res_ratio;    /* ||b - A phi_pred|| / ||b - A phi_prev|| of the last solve */
    double last_loss;         /* loss of the last training step                           */
} lepic_cnn_stats;

int lepic_gpu_cnn_configure(lepic_ctx *ctx, const lepic_cnn_config *cfg);
int lepic_gpu_cnn_stats(lepic_ctx *ctx, lepic_cnn_stats *stats);
/* the context's network (a handle for the lepic_cnn_* calls below; NULL before the first
 * learned solve or configure) */
void *lepic_gpu_cnn_net(lepic_ctx *ctx);

/* The network alone, on the current CUDA device: parameters are FP32, in the order
 * e0a e0b e1a e1b e2a e2b e3a e3b d2 d1 d0 out, each W[cout][cin][3][3] then b[cout]. */
int lepic_cnn_create(void **net, uint64_t seed);
int lepic_cnn_destroy(void *net);
int lepic_cnn_nparams(void);
int lepic_cnn_params(void *net, float *params, int64_t n, int32_t set);
/* forward, loss and gradient for N images of H x W (multiples of 8) of host data:
 * x [N][H][W][2], t and m [N][H][W] (m 0/1; both NULL: forward only); out [N][H][W]. */
int lepic_cnn_loss_grad(void *net, const float *x, const float *t, const float *m, int32_t N,
                        int32_t H, int32_t W, float *out, float *grad, double *loss);
int lepic_cnn_adam_step(void *net, float lr);
const char *lepic_cnn_last_error(void *net);

#ifdef __cplusplus
}
#endif
#endif
