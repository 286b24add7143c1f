/*
 * wavetrisk_gpu.h -- C-ABI of the B200 implementation of WAVETRISK's
 * data-parallel hot path (TRiSK operators, wavelet transforms and threshold
 * mask, multigrid free-surface solve) on the padded lozenge layout.
 *
 * Every entry point is plain C: pointers, sizes and an int status.  A Fortran
 * host binds them with ISO_C_BINDING.  All arrays are
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

/* Raw stream of the handle (cudaStream_t), for event timing by the caller. */
void* wt_stream(wt_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* WAVETRISK_GPU_H */
