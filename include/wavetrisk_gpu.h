/*
 * wavetrisk_gpu.h -- C-ABI of the B200 implementation of WAVETRISK's
 * data-parallel hot path (TRiSK operators, wavelet transforms and threshold
 * mask, multigrid free-surface solve) on the padded lozenge layout.
 *
 * Every entry point is plain C: pointers, sizes and an int status.  A Fortran
 * host binds them with ISO_C_BINDING (bind(C) interfaces).  All arrays are
 * double precision unless stated otherwise.
 *
 * Layout of one grid level l (n = 2^l nodes per lozenge side, P = n + 4):
 *   node (i, j) of lozenge d, i, j in [-2, n+1]  ->  index (d*P + j+2)*P + i+2,
 *   NN = 10*P*P nodes per level (ghost cells included; the two poles live in
 *   ghost cells of the lozenges that touch them, as in the reference);
 *   edge fields are 3 planes (RT, DG, UP) of NN, triangle fields 2 planes
 *   (LORT, UPLT) of NN; layered fields are [nz][...] with layer k = 1 first.
 */
#ifndef WAVETRISK_GPU_H
#define WAVETRISK_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference aborts instead (src/base_ser.f90:54); every
 * call here returns one of these. */
enum {
  WT_OK = 0,
  WT_ERR_ARG = -1,           /* bad argument or size                                */
  WT_ERR_CUDA = -2,          /* CUDA runtime error (message on stderr)              */
  WT_ERR_ALLOC = -3,         /* device allocation failed                            */
  WT_ERR_NONFINITE = -4,     /* NaN/Inf or collapsed layer found in the state       */
  WT_ERR_NOT_CONVERGED = -5, /* elliptic solve hit its iteration cap                */
  WT_ERR_TIMEOUT = -6,       /* a bounded device wait gave up                       */
  WT_ERR_STATE = -7,         /* call out of order (e.g. solve before setup)         */
  WT_ERR_NO_DEVICE = -8      /* no CUDA device / extension unusable                 */
};

/* ---------------------------------------------------------------- grid ---- */
/* Host-side grid builder.  Restates init_grid / init_coordinates /
 * assign_coord / precompute_geometry (src/init.f90:142-524), refine_patch2
 * (src/refine_patch.f90:106-262), the ghost tables of create_comm /
 * create_comm_pole (src/comm.f90:103-530) and the overlap areas of
 * set_RF_wgts (src/wavelet.f90:1512-1566) for levels min_level-1..max_level,
 * with one domain per lozenge. */
typedef struct wt_grid wt_grid;
typedef struct {
  int n, P;
  int64_t NN, n_halo_node, n_halo_edge;
} wt_level_dims;

int wt_grid_build(int min_level, int max_level, int domain_level, double radius, double omega, wt_grid** out);
void wt_grid_free(wt_grid* g);
int wt_grid_level_dims(const wt_grid* g, int level, wt_level_dims* dims);
int wt_grid_copy(const wt_grid* g, int level, const char* name, void* dst);

/* -------------------------------------------------------------- device ---- */
/* Geometry and ghost tables of one level, host pointers (copied at create). */
typedef struct {
  int level, n, P;
  int64_t NN;
  const double *len, *pedlen;  /* 3*NN  primal / dual edge lengths           */
  const double *part;          /* 6*NN  hexagon area parts (Areas%part)      */
  const double *hex_inv;       /* NN    1/hexagon area                        */
  const double *triarea;       /* 2*NN                                        */
  const double *coriolis;      /* 2*NN  f * dual-triangle area                */
  const double *overl_a;       /* 4*NN  Overl_Area%a (wavelet weights)        */
  const double *topo;          /* NN    topography (negative depth, metres)   */
  const int64_t *halo_node;    /* 2*n_halo_node (dst, src)                    */
  int64_t n_halo_node;
  const int64_t *halo_edge;    /* 3*n_halo_edge (dst, src, sign)              */
  int64_t n_halo_edge;
  const double *iu_wgt;        /* 9*NN  I_u_wgt%enc (outer velocity weights, set_WT_wgts,
                                  src/wavelet.f90:1567-1705); NULL on level_start */
  const double *overl_split;   /* 2*NN  Overl_Area%split; may be NULL          */
  const double *rf_wgt;        /* 3*NN  R_F_wgt%enc (flux-restriction weights, set_RF_wgts,
                                  src/wavelet.f90:1512-1540,1176-1360); NULL on level_start */
} wt_level_desc;

typedef struct {
  int level_start, level_end; /* uniform hierarchy: every node of these levels */
  int nz;                     /* Lagrangian layers                             */
  double grav, ref_density, p_top;
  const wt_level_desc* levels; /* level_end - level_start + 1 entries        */
} wt_grid_desc;

typedef struct wt_handle wt_handle;

/* Replaces: initialize/init_structures upload of geometry (src/main.f90:482-524).
 * Allocates every device array once; later calls allocate nothing. */
int wt_create(const wt_grid_desc* desc, wt_handle** out);
int wt_destroy(wt_handle* h);
int wt_status(wt_handle* h);                 /* sticky device error flags -> status */
int wt_clear_status(wt_handle* h);           /* acknowledge: device flag and sticky status back to WT_OK */
int wt_synchronize(wt_handle* h);

/* Prognostic state on level_end: mass, temp [nz][NN]; velo [nz][3][NN];
 * sol_mean mean_m, mean_t [nz][NN] (src/domain.f90:73 sol, sol_mean). */
int wt_upload_state(wt_handle* h, const double* mass, const double* temp, const double* velo,
                    const double* mean_m, const double* mean_t);
int wt_download_state(wt_handle* h, double* mass, double* temp, double* velo);

/* Replaces trend_ml (src/multi_level.f90:5-47) as the trend_fun of the RK
 * stepper (src/time_integr.f90:7-13): trend of the resident state; the halo
 * copy of update_bdry is applied to the state first, as the reference does. */
int wt_trend(wt_handle* h);
int wt_download_trend(wt_handle* h, double* dmass, double* dtemp, double* dvelo);

/* Replaces dt_step => RK4 (src/time_integr.f90:78-103) with WT_after_step on a
 * uniform grid: nsteps full RK4 steps of length dt on the resident state,
 * launched as one captured CUDA graph per step. */
int wt_rk4_step(wt_handle* h, double dt, int nsteps);

/* Same, through host buffers: uploads the state, steps, downloads it. */
int wt_rk4_step_host(wt_handle* h, double dt, int nsteps, double* mass, double* temp, double* velo);

/* Measurement aid: the same RK4 steps launched kernel by kernel with CUDA
 * events around every launch; ms_per_launch[0..5] = average duration of the
 * ghost copy, column, step1, pentagon fix, flux ghost copy and trend+sub-step
 * kernels.  No reference counterpart (the reference times whole steps). */
int wt_profile_rk4(wt_handle* h, double dt, int nsteps, double* ms_per_launch, int* nkernels);

/* ------------------------------------------------------------ elliptic ---- */
/* Barotropic free-surface solve L(eta) = f with
 *   L(q) = theta1 theta2 dt^2 div(g (|H| phi + eta_old) grad q) - q
 * (elliptic_lo, src/barotropic_2d.f90:187-250; phi = 1, eta_old = 0) on the
 * uniform hierarchy level_start..level_end of the handle.  Fields u (solution,
 * initial guess) and f (right-hand side) are multi-level: the levels' NN-node
 * arrays concatenated from level_start to level_end. */
enum { WT_SOLVER_FMG = 0, WT_SOLVER_SRJ = 1, WT_SOLVER_MIXED_IR = 2, WT_SOLVER_MG64 = 3,
       /* Flexible CG (truncated to one previous direction, area-weighted inner
        * product, FP64 recurrences) on level_end, ir_tol / ir_max as for
        * WT_SOLVER_MIXED_IR: preconditioned by the FP32 V-cycle of the mixed
        * solve followed by the learned network's correction of the residual
        * the V-cycle leaves, with plain FP64 multigrid (the FP64 V-cycle) as
        * the fallback when that fails to contract (FCG_LEARNED); by the FP32
        * V-cycle alone (FCG_MG, the method without the network); or
        * unpreconditioned (FCG).  No reference counterpart. */
       WT_SOLVER_FCG_LEARNED = 4, WT_SOLVER_FCG = 5, WT_SOLVER_FCG_MG = 6 };

typedef struct {
  int method;                 /* WT_SOLVER_*                                         */
  /* src/lin_solve.f90:11-26 module parameters (reference defaults in brackets)     */
  int coarse_iter;            /* [50]  BiCGSTAB iterations on level_start           */
  int max_vcycle;             /* [3]                                                 */
  int pre_iter, down_iter, up_iter, post_iter;   /* [2, 2, 2, 4]                    */
  int max_srj_iter;           /* [200]                                               */
  double fine_tol, coarse_tol;/* [1e-3, 1e-3]                                        */
  /* WT_SOLVER_MIXED_IR: FP64 refinement around FP32 V-cycles (down/up_iter sweeps,
   * coarse_iter Jacobi sweeps on level_start); stop at ir_tol or ir_max.
   * WT_SOLVER_MG64: the same cycle entirely in FP64 (precision-matched baseline). */
  double ir_tol;
  int ir_max;
} wt_solver_opts;

typedef struct {
  double nrm_res_init[16];    /* per level: initial ||f - L u|| / ||f||             */
  double nrm_res_final[16];   /* per level: final normalised residual               */
  int iterations[16];         /* per level: V-cycles / SRJ sweeps / BiCGSTAB its    */
  int outer_iterations;       /* refinement steps (WT_SOLVER_MIXED_IR)              */
  double true_rel_residual;   /* FP64 ||f - L u|| / ||f|| on level_end after solve  */
  double ms;                  /* host wall time of the solve                         */
  int precond_fallback;       /* FCG_LEARNED: iteration at which the V-cycle took
                               * over from the network (0: it never did)             */
  int restarts;               /* FCG: restarts from the true residual               */
} wt_solver_report;

/* Builds the operator tables (replaces the per-call coefficient work of
 * elliptic_lo / elliptic_lo_diag); allocates all solver work arrays once. */
int wt_elliptic_setup(wt_handle* h, double dt, double theta1, double theta2, int domain_level);
int wt_elliptic_upload(wt_handle* h, const double* u, const double* f);   /* either may be NULL */
int wt_elliptic_download(wt_handle* h, double* u, double* f);             /* either may be NULL */
/* f(level) = L(u(level)) on [0, n]^2 of one level (elliptic_lo). */
int wt_elliptic_apply(wt_handle* h, int level);
/* f on coarser levels from f on level_end by successive restriction
 * (forward_scalar_transform, src/wavelet.f90:105-155). */
int wt_elliptic_restrict(wt_handle* h);
/* u on level fine from u on fine-1 (prolong, src/lin_solve.f90:243). */
int wt_elliptic_prolong(wt_handle* h, int fine);
/* l2 (src/lin_solve.f90:433) of u (which = 0) or f (which = 1) on one level. */
int wt_elliptic_l2(wt_handle* h, int level, int which, double* out);
/* Replaces elliptic_solver => FMG | SRJ (src/init.f90:127, src/lin_solve.f90:33,142)
 * on the resident u, f.  Returns WT_ERR_NOT_CONVERGED when the mixed solver
 * stops at ir_max above ir_tol. */
int wt_elliptic_solve(wt_handle* h, const wt_solver_opts* opts, wt_solver_report* rep);

/* V-cycle schedule autotuner: solves the resident problem with `base` and each
 * candidate schedule (down_iter, up_iter, coarse_iter; cand = 3*ncand ints, or
 * NULL for the built-in set: down = up in {1, 2, 3}, coarse in {2, 4, 6, 10,
 * 20}), `repeats` times each from the resident u, and writes the fastest that
 * reaches base->ir_tol into *best (with its best wall time in *best_ms).  For
 * methods that solve on level_end only: WT_SOLVER_MIXED_IR, _MG64,
 * _FCG_LEARNED, _FCG_MG.  u and f are kept.  No reference counterpart (the
 * reference's schedule is fixed by its module parameters). */
int wt_elliptic_autotune(wt_handle* h, const wt_solver_opts* base, const int* cand, int ncand, int repeats,
                         wt_solver_opts* best, double* best_ms);

/* ------------------------------------------------ learned preconditioner ---- */
/* A hexagonal-stencil convolution network (7 taps: a node and its six
 * neighbours; 2 -> 32 -> 32 -> 1 channels) mapping a residual r of level_end,
 * scaled by its rms, to an approximation of the error e with L e = r, trained
 * on the residuals a V-cycle leaves and used to correct them
 * (WT_SOLVER_FCG_LEARNED).  Its inputs are r and r times a depth feature
 * (|H| / 2750 m - 1); it has no biases, and its two hidden layers end in the
 * activation p -> p (p > 0), slope p (p <= 0) (wt_learned_activation; slope 1
 * is the identity), so net(a r) = a net(r) for a > 0.  Its output is 0 at the
 * pole slots (slots of [0, n]^2 outside [0, n)^2).  FP32 master weights, BF16
 * weights and activations in every forward and backward kernel, FP32
 * accumulation; the 32 -> 32 layer runs on the tensor cores (tcgen05).  The
 * nodes are the slots of [0, n]^2 of each lozenge that are their own ghost
 * source, numbered lozenge, row j, column i.  Requires wt_elliptic_setup; no
 * reference counterpart (the reference preconditions nothing). */
typedef struct {
  int n_rhs;       /* seeded N(0,1) right-hand sides, zero mean                   */
  int cycles;      /* residual/error pairs per right-hand side: after each of the
                    * first `cycles` FP64 V-cycles of a solve from 0              */
  int epochs;      /* Adam passes over all pairs, one pair per step              */
  float lr;        /* Adam step, cosine-decayed to lr / 20                       */
  unsigned long long seed;
  int down_iter, up_iter, coarse_iter;   /* the generating V-cycle              */
  int batch_rhs;   /* right-hand sides whose pairs are generated and trained on
                    * together (their `epochs` passes), then replaced by the next
                    * batch's; 0 = all n_rhs at once                            */
} wt_learn_opts;

typedef struct {
  int pairs, steps;
  double loss_first_epoch, loss_last_epoch;  /* mean energy-norm loss (below)      */
  double ms_generate, ms_train;              /* host wall time                   */
} wt_learn_report;

int wt_learned_setup(wt_handle* h, unsigned long long seed);   /* He-initialised weights */
/* Hidden activation slope in (0, 1] (1 = identity; default 1). */
int wt_learned_activation(wt_handle* h, float slope);
/* The 32 -> 32 layer on the tensor cores (1, default) or the CUDA cores (0). */
int wt_learned_tensor_cores(wt_handle* h, int on);
/* Mean device time of each layer of the forward pass over reps launches, on a
 * seeded residual (ms[3]: layer 1 with its input, layer 2, layer 3). */
int wt_learned_layer_times(wt_handle* h, int reps, float* ms);
int wt_learned_num_params(void);
/* FP32 master parameters (wt_learned_num_params floats); get or set may be NULL. */
int wt_learned_params(wt_handle* h, float* get, const float* set);
/* Node count; with slot/tap non-NULL also the node slots (ns) and the taps
 * (7*ns, tap-major, -1 where a tap leaves the node set). */
int wt_learned_layout(wt_handle* h, int* ns, int* slot, int* tap);
/* The network's correction z = rms(r) net(r / rms(r)) on the ns nodes (host arrays). */
int wt_learned_infer(wt_handle* h, const double* r, double* z);
/* Training loss, the error in the energy norm of the solve,
 *   <d, -L d>_A / |A|,  d = net(r/rms(r)) - e/rms(r) (net 0 at the poles),
 * (<,>_A weighted by the cell areas 1/hex_inv, |A| their sum) and the gradient
 * 2 A (-L d) / |A| pushed back through the network to the parameters (host
 * arrays; grad: wt_learned_num_params floats).  The solve's u, f are kept. */
int wt_learned_grad(wt_handle* h, const double* r, const double* e, double* loss, float* grad);
/* Generates residual/error pairs with the FP64 multigrid, those after each
 * V-cycle (u and f of level_end are kept), batch_rhs right-hand sides at a
 * time, and trains the network on each batch with Adam on the GPU. */
int wt_learned_train(wt_handle* h, const wt_learn_opts* o, wt_learn_report* rep);

/* ---------------------------------------------------- vertical remap ---- */
/* remap_vertical_coordinates (src/remap.f90:18-76) for the incompressible
 * case (remap_incompressible, :147-216): every layered level of the handle
 * (level_end; every level of the hierarchy after wt_wavelet_setup) is remapped
 * from its Lagrangian layers to the hybrid grid z_k = a_vert[k] eta + b_vert[k]
 * z_s (a_vert, b_vert: nz + 1 host values, index 0 at the bottom; eta the
 * column's free surface from its layer masses, z_s the topography).  Buoyancy
 * is remapped on each node's column and the three edge velocities on the
 * columns averaged with the node at each edge's far end; the new masses are
 * rho0 dz.  remap_type selects the column reconstruction: WT_REMAP_0
 * (remap0, piecewise constant, :259-285), WT_REMAP_1 (remap1, piecewise linear
 * with interface reconciliation, :287-380), WT_REMAP_2PPM (remap2PPM, :382-495).
 * Porosity 1 (no penalization).  The host decides when to remap
 * (src/main.f90:447-454).  nz <= 64. */
enum { WT_REMAP_0 = 0, WT_REMAP_1 = 1, WT_REMAP_2PPM = 2 };
int wt_remap_vertical(wt_handle* h, int remap_type, const double* a_vert, const double* b_vert);
/* cpt_min_mass (src/main.f90:625-693, with cal_min_mass, incompressible case,
 * A/B hybrid grid, porosity 1): the smallest relative layer mass
 * (mean + perturbation) / (ref_density dz_k) over the layers of every node of
 * every level whose node mask is at least ADJZONE (every node of a handle
 * without masks), dz_k = b_vert[k+1] z_s - b_vert[k] z_s from the b_vert of
 * wt_remap_vertical.  *min_mass = 0 where a layer mass is not positive or not
 * a number (the reference aborts there), 1e16 when no node counts.  The host
 * remaps when it drops below min_mass_remap (0.9 by default,
 * src/main.f90:447-454). */
int wt_min_mass(wt_handle* h, const double* b_vert, double* min_mass);

/* ------------------------------------------------------ no allocation ---- */
/* Weighted l2 norm of one level (the solver's l2, src/lin_solve.f90:433-464)
 * for callers that cannot allocate device memory: a host loop running inside
 * a memory pool it does not control, or a code that must not grow its device
 * footprint after start-up.  No reference counterpart: the reference never
 * allocates device memory at all.
 *   field  : device pointer, NN = 10*(2^level + 4)^2 doubles, padded layout;
 *   nsrc   : device pointer to the level's ghost remap (NN ints), or NULL when
 *            the ghosts of field already hold their copies;
 *   result : device pointer to one double, written asynchronously on stream
 *            (a cudaStream_t, or NULL for the default stream).
 * Allocates nothing: the block partial sums live in a fixed device array of
 * 4096 doubles, so level must be <= 8 (WT_ERR_ARG beyond).  Every call on a
 * device shares that array: calls that overlap on the GPU race.  The first
 * call on each device looks the array's address up (cudaGetSymbolAddress);
 * make that first call before any stream capture. */
int wt_elliptic_l2_noalloc(int level, int domain_level, const int* nsrc, const double* field, double* result,
                           void* stream);

/* ------------------------------------------------------------ wavelets ---- */
/* Multi-level fields of the prognostic variables on the hierarchy
 * [level_start, level_end] of the handle, every layer.  The reference keeps
 * them in sol(v,k) and wav_coeff(v,k) (src/shared.f90) with the masks mask_n,
 * mask_e of each domain (src/domain.f90).  Level level_end's scaling fields are
 * the stepper's state (wt_upload_state/wt_rk4_step). */
enum {
  WT_FIELD_MASS = 0, WT_FIELD_TEMP = 1, WT_FIELD_VELO = 2,   /* scaling: [nz][NN], [nz][NN], [nz][3*NN] doubles */
  WT_WAVE_MASS = 3, WT_WAVE_TEMP = 4, WT_WAVE_VELO = 5,      /* wavelet coefficients, same shapes            */
  WT_MASK_NODE = 6, WT_MASK_EDGE = 7,                        /* int32 [NN], [3*NN]                           */
  /* Work fields of the multi-level trend (allocated on first use, zero):
   * a node scalar (Bernoulli or Exner), the scalar trend dscalar, the
   * horizontal flux h_flux and the velocity trend dvelo of every layer. */
  WT_WORK_SCALAR = 8, WT_WORK_DSCALAR = 9,                   /* [nz][NN] doubles                             */
  WT_WORK_FLUX = 10, WT_WORK_DVELO = 11,                     /* [nz][3*NN] doubles                           */
  /* Layer means sol_mean(S_MASS/S_TEMP, k) of the level, [nz][NN] doubles; on
   * level_end they are the stepper's (wt_upload_state). */
  WT_FIELD_MEAN_MASS = 12, WT_FIELD_MEAN_TEMP = 13
};
/* Mask values (src/shared.f90:58-73). */
enum { WT_MASK_ZERO = 0, WT_MASK_TRSK = 2, WT_MASK_ADJZONE = 8, WT_MASK_RESTRCT = 12, WT_MASK_TOLRNZ = 16,
       WT_MASK_FROZEN = 32 };

/* Allocates the coarse-level scaling fields, the wavelet fields (zero) and the
 * masks (TOLRNZ: every point active) of every level.  Needs iu_wgt on every
 * level above level_start. */
int wt_wavelet_setup(wt_handle* h);
/* Host <-> device copy of one field of one level (host layout as the device's).
 * Downloads of scaling and wavelet fields first give ghosts their copies. */
int wt_upload_field(wt_handle* h, int level, int field, const void* src);
int wt_download_field(wt_handle* h, int level, int field, void* dst);
/* The same for n (level, field) pairs at once (the drop-in boundary's
 * wt_upload_fields / wt_download_fields(h, which, host_ptrs)): the copies are
 * queued back to back on the handle's stream with one synchronisation at the
 * end, and each level's ghost copy runs once per download batch.  Arguments are
 * checked before anything is queued. */
int wt_upload_fields(wt_handle* h, int n, const int* levels, const int* fields, const void* const* src);
int wt_download_fields(wt_handle* h, int n, const int* levels, const int* fields, void* const* dst);
/* forward_wavelet_transform(scaling, wavelet, level_start+1) (src/wavelet.f90:20-98):
 * scalar and velocity wavelets of levels > level_start, coarse scaling by
 * lifting (scalars) and averaging (velocity). */
int wt_forward_wt(wt_handle* h);
/* inverse_wavelet_transform(wavelet, scaling, level_start) (src/wavelet.f90:208-296). */
int wt_inverse_wt(wt_handle* h);
/* The threshold pass of mask_active (src/mask.f90:17-38, mask_tol_vars :102-156):
 * level_end on nodes [0, n], coarser levels on [-1, n+1].  threshold is
 * [3][nz] (mass, Theta, velocity per layer), as threshold(v, k). */
int wt_mask_tol_vars(wt_handle* h, const double* threshold, int level_fill);
/* adapt's mask sequence (src/adapt.f90:14-65) on the dense hierarchy, without
 * the tree surgery that the host keeps: init_masks_zero, mask_active
 * (mask_tol_vars + mask_parent_nodes/edges), mask_adj_same_scale,
 * mask_restrict_same_scale (levels < max_level), mask_adj_finer_scale,
 * complete_masks and mask_trsk (src/mask.f90), with comm_masks between sweeps
 * as the serial build does.  child_required (may be NULL) receives
 * check_child_required (src/refine_patch.f90:289-327) for every parent patch
 * of side patch_size and child quadrant (NE, SE, SW, NW) of levels
 * level_start .. level_end-1, level by level, lozenge-major:
 * sum_l 10 * (n_l / patch_size)^2 * 4 bytes.  Exact when every patch of the
 * hierarchy exists (a fully refined tree). */
int wt_mask_build(wt_handle* h, const double* threshold, int level_fill, int max_level, int patch_size,
                  unsigned char* child_required);

/* ---- The patch tree of a partially refined hierarchy (src/refine_patch.f90).
 * Level l holds 10 * (n_l / patch_size)^2 patches of patch_size^2 owned nodes
 * (PATCH_SIZE, src/patch.f90:6), one byte each, lozenge-major [10][rows][cols].
 * Every level's fields stay allocated; the tree decides which patches exist,
 * and the levels above its level_end hold ZERO masks, which the mask-tested
 * transforms, restrictions and mask sweeps leave out as the reference leaves
 * out levels it has not made.  Once a tree exists, wt_adaptive_step refines it
 * on the device inside its graph (while the tree's level_end is the
 * hierarchy's top). */
/* add_second_level (src/refine_patch.f90:247-268) as init_structures calls it
 * (src/main.f90:482-524): every patch of level_start exists, none above, the
 * tree's level_end is level_start.  patch_size: even, dividing n_level_start. */
int wt_tree_init(wt_handle* h, int patch_size);
/* The tree's level_end (levels above it have no patch). */
int wt_tree_level_end(wt_handle* h, int* level_end);
/* One level's patch bytes: exist (1 = the patch exists) and fresh (1 = made
 * by the last refine); either may be NULL. */
int wt_tree_download(wt_handle* h, int level, unsigned char* exist, unsigned char* fresh);
/* Grid sync after a host-side refine or a restart (load_adapt_mpi,
 * src/io.f90:971): the host's tree replaces the device's: exist holds
 * every level's bytes, level_start first; level_start must be complete. */
int wt_grid_sync(wt_handle* h, const unsigned char* exist, int level_end);
/* adapt (src/adapt.f90:14-65) on the tree: init_masks_zero, mask_active,
 * mask_adj_same_scale and mask_restrict_same_scale up to the tree's
 * level_end; refine() (src/refine_patch.f90:12-49: check_child_required of
 * every existing patch below max_level, a child patch per flagged quadrant,
 * level_end + 1 when one of level level_end + 1 is made); then
 * mask_adj_finer_scale, complete_masks and mask_trsk up to the new level_end,
 * and compress_wavelets.  Returns the new level_end and whether a patch was
 * made (either pointer may be NULL). */
int wt_adapt(wt_handle* h, const double* threshold, int level_fill, int max_level, int* level_end, int* refined);
/* inverse_wavelet_transform after adapt (time_step, src/main.f90:444) on the
 * tree: rebuilds the parents whose children the next step reads (the needed
 * nodes of the masks wt_adapt left) and those of the tree's nodes, as the
 * inverse inside wt_adaptive_step does; the scaling values outside the tree,
 * which no step reads, keep what they held.  Without a tree, or with the
 * needed-node maps off, every parent (wt_inverse_wt). */
int wt_inverse_tree(wt_handle* h);
/* count_active (src/main.f90:137-172) over the patches the last refine made:
 * counts[0] node wavelets (mass and Theta of every layer) with |w| >=
 * threshold(v, k), counts[1] edge wavelets (velocity). */
int wt_count_active(wt_handle* h, const double* threshold, long long* counts);
/* out[0] patches of the level, out[1] of them made by the last refine, out[2]
 * owned nodes outside the tree with a node or edge mask that is not ZERO,
 * out[3] owned nodes in the level's needed-node map (-1 without one).  No
 * reference counterpart (diagnostics). */
int wt_tree_stats(wt_handle* h, int level, long long* out);
/* level_end's state on the existing patches only, as the reference's host
 * holds it (its patch storage, src/domain.f90): for every existing patch of
 * level_end in lozenge-major order, its patch_size^2 owned nodes row by row,
 * layer by layer; mass and temp [n_patches][nz][ps*ps], velo
 * [n_patches][nz][3][ps*ps] doubles.  The download returns the patch count
 * (WT_ERR_ARG, with *n_patches set, when it exceeds capacity); the upload
 * needs the count of the device's current tree. */
int wt_download_tree_state(wt_handle* h, double* mass, double* temp, double* velo, long long capacity,
                           long long* n_patches);
int wt_upload_tree_state(wt_handle* h, const double* mass, const double* temp, const double* velo,
                         long long n_patches);
/* mask_adj_child (src/mask.f90:314-466) of the parents of `level` alone, as
 * init_structures applies it to the root level (src/main.f90:514). */
int wt_mask_adj_child(wt_handle* h, int level);
/* cal_lnorm (src/lnorms.f90:7-58) of the hierarchy's scaling fields over
 * levels level_start..level_end: out[v*nz + k] for v = mass, Theta, velocity;
 * scalars are mean + perturbation over nodes [0, n]^2, velocities over the
 * edges of nodes [0, n)^2, both where mask_n >= ADJZONE.  order: 0 "inf"
 * (max |.|), 1 "1" (mean |.|), 2 "2" (rms), 3 "min"; the mean and rms divide
 * by the count of nodes [-1, n+1]^2 with mask_n >= ADJZONE. */
int wt_lnorm(wt_handle* h, int order, double* out);
/* Tuning.  WT_TUNE_WAVELET_LAYERS (process-wide): layers per thread of the
 * interscale wavelet kernels (1..64; 0 = default: 2 up to 16 layers, 4 above).
 * WT_TUNE_SKIP_INACTIVE (per handle, 1 = default): in the RK stages of the
 * hierarchy (wt_rk4_multi, wt_adaptive_step) the finest level's step1 and
 * trend leave out the nodes whose results cannot reach the state after
 * WT_after_step (no counterpart in the reference, which computes every node of
 * every existing patch; the states and masks are the same either way); 0
 * computes every node. */
/* WT_TUNE_FLUX_PRECISION (per handle, 64 = default): 32 runs the flux
 * stencils of step1 (potential vorticity, mass and Theta fluxes, kinetic
 * energy: src/ops.f90:276-366, 472-522, post_step1 :526-737) of the
 * single-level stepper (wt_trend, wt_rk4_step, wt_rk4_step_host) in FP32 with
 * FP32 results, and keeps FP64 for the column pass, the Bernoulli function's
 * geopotential and pressure parts, the divergence, Qperp, the gradients and
 * the RK accumulation.  The first switch to 32 allocates the FP32 work
 * arrays.  The hierarchy's steps (wt_trend_multi, wt_rk4_multi,
 * wt_adaptive_step, wt_rk4_split_explicit) stay FP64 and return WT_ERR_STATE
 * while it is 32.  No reference counterpart (the reference is FP64 only). */
/* WT_TUNE_TEST_TMA_TIMEOUT (per handle, 0 = default; test only): 1 makes
 * every TMA-staged step1 and trend block declare 16 bytes more than its
 * copies deliver, give up after 20 us and take its wait-timeout path (error
 * flag set, block retires the extra bytes, waits for its own copies, returns),
 * so wt_status reports WT_ERR_TIMEOUT; the state of such a step is not
 * meaningful.  No reference counterpart. */
enum { WT_TUNE_WAVELET_LAYERS = 1, WT_TUNE_SKIP_INACTIVE = 2, WT_TUNE_FLUX_PRECISION = 3,
       WT_TUNE_TEST_TMA_TIMEOUT = 4 };
int wt_tune(wt_handle* h, int param, int value);
/* compress_wavelets (src/adapt.f90:79-103): zero the wavelets of inactive points. */
int wt_compress(wt_handle* h);
/* WT_after_step (src/adapt.f90:192-237): wavelets of the current scaling fields,
 * compression, inverse transform. */
int wt_wt_after_step(wt_handle* h);

/* ------------------------------------------------ compute-or-restrict ---- */
/* The coarse-level restrictions of the multi-level trend (trend_ml,
 * src/multi_level.f90:5-43) from level+1 to `level`, level_start <= level <
 * level_end, every layer, on the work fields.
 * scalar_cpt_restr (src/multi_level.f90:311-345): the node scalar of parents
 * [0, n]^2 with mask_n >= RESTRCT is sub-sampled from the child. */
int wt_restrict_scalar(wt_handle* h, int level);
/* flux_cpt_restr (src/multi_level.f90:394-659): the flux of the edges of
 * parents [0, n)^2 with mask_e >= RESTRCT is the conservative restriction of
 * the child's flux and dscalar (interp_flux with R_F_wgt, part_coarse_flux and
 * coarse_flux with the overlap areas).  Needs rf_wgt and overl_split of
 * level+1. */
int wt_restrict_flux(wt_handle* h, int level);
/* The restriction of u_source_cpt_restr (src/multi_level.f90:365-392): the
 * velocity trend of parent edges whose first child edge has mask_e >= ADJZONE
 * is the sum of the two child edges; the others keep the parent's value. */
int wt_restrict_u_source(wt_handle* h, int level);

/* trend_ml over the whole hierarchy (src/multi_level.f90:5-188), every level
 * present: per level from level_end down to level_start, integrate_pressure_up,
 * step1 and post_step1 on the level's scaling fields and layer means, the
 * compute-or-restrict of Bernoulli, Exner and the mass and Theta fluxes from
 * the level above (below level_end), scalar_trend with mask_n >= TRSK, the
 * velocity source computed or restricted (cpt_or_restr_u_source), and du_grad
 * with mask_n >= TRSK.  Needs wt_wavelet_setup, the masks of every level and
 * the layer means (WT_FIELD_MEAN_*) below level_end. */
int wt_trend_multi(wt_handle* h);
/* RK4 (src/time_integr.f90:78-103) over the hierarchy, nsteps steps of dt:
 * each stage evaluates wt_trend_multi's trend, takes RK_sub_step on every
 * level (src/time_integr.f90:206-225) and runs WT_after_step on the stage
 * state; the masks are held fixed.  The solution is the hierarchy's scaling
 * fields (level_end's is the stepper's state). */
int wt_rk4_multi(wt_handle* h, double dt, int nsteps);
/* The explicit part of one mode-split step, RK4_split (src/time_integr.f90:
 * 360-382) without free_surface_update: RK_split (:444-463) four times, each
 * barotropic_correction of the stage's source state (src/barotropic_2d.f90:
 * 52-116, with total_height :368-412), trend_ml, scalar_star and u_star
 * (:9-50, external pressure gradient grad_eta of each level's free surface
 * weighted by theta1) and WT_after_step.  Uses the free surface of every level
 * (wt_barotropic_upload_level) and the masks as they are. */
int wt_rk4_split_explicit(wt_handle* h, double dt, double theta1);
/* barotropic_correction (src/barotropic_2d.f90:52-116) of the hierarchy's
 * scaling fields from each level's free surface. */
int wt_barotropic_correction_multi(wt_handle* h);
/* free_surface_update (src/time_integr.f90:465-478) on the hierarchy:
 * eta_update (src/barotropic_2d.f90:118-129: rhs_elliptic on every level,
 * the elliptic operator's coefficients g (|H| + eta_old) and its diagonal
 * rebuilt from the current free surface, the solve of opts from that surface
 * on every level), barotropic_correction, u_update and WT_after_step.  The
 * reference's WT_after_step from level_start - 1 also forms wavelets at
 * level_start and restricts the velocity below it; the levels the hierarchy
 * holds come out the same.  Needs wt_wavelet_setup and wt_elliptic_setup with
 * the same dt, theta1 and theta2 (WT_ERR_STATE otherwise); rep as for
 * wt_elliptic_solve, whose status it returns (WT_ERR_NOT_CONVERGED when the
 * solve stopped at its cap; the update is then made with that solution). */
int wt_free_surface_update(wt_handle* h, double dt, double theta1, double theta2, const wt_solver_opts* opts,
                           wt_solver_report* rep);
/* The free surface's part of adapt (src/adapt.f90:79-103 compress_wavelets and
 * the inverse transform after it, src/main.f90:441; the free surface is layer
 * zlevels+1 of sol): its wavelets from the last wt_free_surface_update /
 * wt_rk4_split, compressed under the current masks, then its inverse
 * transform.  Call after wt_mask_build; WT_ERR_STATE before any free-surface
 * update. */
int wt_free_surface_adapt(wt_handle* h);
/* RK4_split (src/time_integr.f90:360-382): when theta2 != 1 the flux
 * divergence of the current state into each level's previous divergence,
 * then wt_rk4_split_explicit and wt_free_surface_update. */
int wt_rk4_split(wt_handle* h, double dt, double theta1, double theta2, const wt_solver_opts* opts,
                 wt_solver_report* rep);
/* The free surface of one level of the hierarchy (NN host doubles). */
int wt_free_surface_download(wt_handle* h, int level, double* eta);
/* nsteps adaptive time steps of the hierarchy (the reference's time_step,
 * src/main.f90:405-444, explicit RK4, fixed thresholds): wt_rk4_multi(dt, 1),
 * adapt's mask sequence with threshold[3][nz] (wt_mask_build without the
 * child flags), wt_compress and wt_inverse_wt, replayed as one CUDA graph. */
int wt_adaptive_step(wt_handle* h, double dt, const double* threshold, int level_fill, int max_level, int nsteps);
/* wt_rk4_multi with CUDA events around its phases (7 entries): ms[p] is the
 * mean duration of one occurrence of phase p and count[p] its occurrences per
 * step: 0 column+step1 of level_end, 1 column+step1 of a coarser level,
 * 2 restrictions into a level, 3 k_trend_ml of level_end (with the fused RK
 * sub-step), 4 the same on a coarser level, 5 unused, 6 WT_after_step. */
int wt_profile_rk4_multi(wt_handle* h, double dt, int nsteps, double* ms, int* count);
/* The trends of one level from the last wt_trend_multi: dmass, dtemp [nz][NN],
 * dvelo [nz][3*NN] host doubles (any may be NULL). */
int wt_download_trend_level(wt_handle* h, int level, double* dmass, double* dtemp, double* dvelo);

/* ---------------------------------------------------------- barotropic ---- */
/* The free-surface pieces of the mode-split step on level_end, around the
 * elliptic solve (eta_update / u_update, src/barotropic_2d.f90:118-149).
 * eta is the free surface sol(S_MASS, zlevels+1); div_old the flux divergence
 * of the previous step, trend(S_TEMP, zlevels+1); both NN doubles. */
int wt_barotropic_upload(wt_handle* h, const double* eta, const double* div_old);  /* either may be NULL */
/* flux_divergence (src/barotropic_2d.f90:326-366: step1 itype 4, the
 * vertically summed mass flux of the resident state, and cal_div) and
 * rhs_elliptic (:151-185): rhs = -eta + dt (theta2 div + (1-theta2) div_old) / rho0. */
int wt_rhs_elliptic(wt_handle* h, double dt, double theta2);
/* The same pieces on every level of the hierarchy (after wt_wavelet_setup;
 * coarser levels use the hierarchy's scaling fields, layer means and masks).
 * wt_barotropic_upload_level sets a level's free surface and previous flux
 * divergence (either may be NULL).  wt_rhs_elliptic_multi: flux_divergence
 * over the hierarchy (src/barotropic_2d.f90:326-366) -- on coarser levels the
 * flux is computed or restricted (cpt_or_restr_flux with the child's
 * divergence) -- and rhs_elliptic on every level.  wt_u_update_multi: grad_eta
 * over the hierarchy with cpt_or_restr_eta (:414-474) and u_update (:131-149)
 * on every level. */
int wt_barotropic_upload_level(wt_handle* h, int level, const double* eta, const double* div_old);
int wt_rhs_elliptic_multi(wt_handle* h, double dt, double theta2);
int wt_u_update_multi(wt_handle* h, double dt, double theta1);
int wt_barotropic_download_level(wt_handle* h, int level, double* div_flux, double* rhs, double* grad);
/* grad_eta (src/barotropic_2d.f90:455-474: step1 itype 3, g grad eta) and
 * u_update (:131-149): velo_k -= theta1 dt grad eta on every layer. */
int wt_u_update(wt_handle* h, double dt, double theta1);
/* step1 with itype 1 (scalar gradient flux), 5 (u pedlen), 6 (surface pressure
 * flux) or 7 (mass flux) on one layer of the resident state
 * (src/ops.f90:198-262, comp_SW :396-455): flux (3*NN host doubles) at the
 * edges of nodes [0, n]^2 and the south/west ghost edges; scalar (NN host
 * doubles) is the node field of itypes 1 and 6 (NULL otherwise).  Uses the
 * barotropic work buffers, so it overwrites the last rhs and grad. */
int wt_step1_flux(wt_handle* h, int itype, int layer, const double* scalar, double* flux);
/* step1 itype 8 (src/ops.f90:256-271, comp_SW :460-471) and post_vort
 * (:1159-1228): the vorticity (circulation / triangle area) of one layer of the
 * resident velocity on the triangles the reference's loop over nodes [0, n]^2
 * writes, pentagon corners included.  vort: 2*NN host doubles (LORT plane,
 * UPLT plane); other triangles 0. */
int wt_step1_vort(wt_handle* h, int layer, double* vort);
/* div_flux (NN), rhs (NN), grad (3*NN); any may be NULL. */
int wt_barotropic_download(wt_handle* h, double* div_flux, double* rhs, double* grad);

/* Raw stream of the handle (cudaStream_t), for event timing by the caller. */
void* wt_stream(wt_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* WAVETRISK_GPU_H */
