/*
 * libtdda — C ABI of the B200-native DDA forward/adjoint solve.
 *
 * Each entry point replaces one method of Topo-DDA's pybind11 `DDAModel`
 * (python_bindings/PythonBindings.cpp:16-70); the reference file:line it
 * stands in for is given beside it.  All arrays are plain host pointers unless
 * the name ends in `_device`; complex arrays are interleaved (re, im) doubles
 * in the reference's dipole order: element 3*i + c is component c of dipole i.
 * Every call returns a tdda_status; tdda_last_error() gives the message of the
 * last failure on the calling thread.  A model is not re-entrant: calls on one
 * model must not overlap.
 */
#ifndef TDDA_H_
#define TDDA_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    TDDA_OK = 0,
    TDDA_ERR_BAD_ARG = 1,       /* reference: `throw 1` -> RuntimeError */
    TDDA_ERR_OOM = 2,
    TDDA_ERR_NOT_CONVERGED = 3, /* reported in tdda_solve_info, not returned by solves */
    TDDA_ERR_BREAKDOWN = 4,
    TDDA_ERR_CUDA = 5,
    TDDA_ERR_TIMEOUT = 6,
    TDDA_ERR_UNSUPPORTED = 7,
    TDDA_ERR_STATE = 8
} tdda_status;

typedef enum {
    TDDA_SOLVE_RUNNING = 0,
    TDDA_SOLVE_CONVERGED = 1,   /* ||r||/||E|| <= tol (recursive residual) */
    TDDA_SOLVE_MAXITER = 2,     /* reference prints "does not converge" */
    TDDA_SOLVE_BREAKDOWN = 3,   /* r0 . rl == 0 (src/DDAModel.cpp:952-970) */
    TDDA_SOLVE_NONFINITE = 4,   /* residual became NaN/Inf */
    TDDA_SOLVE_ZERO_RHS = 5,    /* ||E|| == 0: solution is 0 */
    TDDA_SOLVE_STAGNATED = 6,   /* mixed precision: residual stopped decreasing */
    TDDA_SOLVE_TIMEOUT = 7      /* the device-side time limit of the solve ran out */
} tdda_solve_status;

typedef enum { TDDA_PREC_C128 = 0, TDDA_PREC_MIXED = 1 } tdda_precision;

typedef struct tdda_model tdda_model;

/* Constructor arguments of DDAModel (python_bindings/PythonBindings.cpp:19-46),
 * minus the arrays, which tdda_model_create takes separately. */
typedef struct {
    double beta_min, beta_max, ita;   /* legacy filter: projection schedule (src/FilterOption.cpp:5-21) */
    const char *beta_type;
    int use_filter;                   /* the legacy filter (tdda_filter_*), src/DDAModel.cpp:255-264 */
    const char *symmetry_type;        /* "None" or "4fold" (src/DDAModel.cpp:163-173) */
    double symmetry_axis[2];
    int is_periodic;
    const char *objective_name;       /* IntegratedE (the reference factory always builds it) */
    const double *obj_para;
    int n_obj_para;
    int num_x, num_y, num_z, num_total;
    double n_K[3];
    double E0;
    double n_E0[3];
    double lam;
    double material[4];               /* (re, im) of material[0], material[1] */
    double nback;
    int MAXm, MAXn;
    double Lm, Ln;                    /* periods in units of d */
    const char *matrix_method;        /* "FCD" or "LDR" */
    double d;
    double integral_delta;
    int verbose;
    int precision;                    /* tdda_precision */
    /* filterIterations / filterRadii of the constructor: the legacy filter
     * (use_filter != 0) uses filter_radii[0] (src/FilterOption.cpp:12-14) */
    const int32_t *filter_iterations;
    const double *filter_radii;
    int n_filters;
} tdda_params;

typedef struct {
    int iterations;      /* reference ITERATION */
    double error;        /* reference Error: ||r||/||E|| */
    int status;          /* tdda_solve_status */
    int refinements;     /* outer complex128 refinement steps (mixed precision) */
    int inner_iterations;/* total complex64 BiCGSTAB iterations (mixed precision) */
    double true_error;   /* ||E - A P|| / ||E|| recomputed in complex128 (mixed precision) */
} tdda_solve_info;

typedef struct {
    int N, NFpara;
    int nx, ny, nz;
    int Lx, Ly, Lz;
    double K;
    double material[4];  /* after the nback rescale (src/AProductCore.cpp:25-33) */
    long long device_bytes;
    double lattice_ms, tensor_fft_ms;
} tdda_model_info;

const char *tdda_status_string(tdda_status s);
const char *tdda_last_error(void);
int tdda_abi_version(void);

/* DDAModel::DDAModel (src/DDAModel.cpp:79-333; binding PythonBindings.cpp:19-59):
 * geometry int32[3N], input_dielectrics double[3N], si/ci double[ntab]. */
tdda_status tdda_model_create(const tdda_params *p, const int32_t *geometry,
                              const double *input_dielectrics, const double *si,
                              const double *ci, int64_t ntab, tdda_model **out);
/* DDAModel::~DDAModel (src/DDAModel.cpp:335-338) */
void tdda_model_destroy(tdda_model *m);
tdda_status tdda_model_get_info(const tdda_model *m, tdda_model_info *info);

/* DDAModel::solveElectricField (src/DDAModel.cpp:874-885; binding :64).
 * P0: complex[3N] or NULL for zeros. */
tdda_status tdda_solve_electric_field(tdda_model *m, const double *P0, int max_iter, double tol,
                                      tdda_solve_info *info);
/* DDAModel::calculateObjective (src/DDAModel.cpp:870-872; binding :61) */
tdda_status tdda_calculate_objective(tdda_model *m, double *out);
/* DDAModel::calculateGradients (src/DDAModel.cpp:398-469; binding :62): the
 * reference's one-sided finite-difference partials + adjoint solve.  grad: double[NFpara]. */
tdda_status tdda_calculate_gradients(tdda_model *m, double epsilon_partial, double original_obj,
                                     int max_iter, double tol, double *grad, int64_t n);
/* DDAModel::UpdateParameters (src/DDAModel.cpp:747-772; binding :66) */
tdda_status tdda_set_parameters(tdda_model *m, const double *values, int64_t n);
/* DDAModel::get_parameter_copy (src/DDAModel.cpp:1341-1343; binding :67) */
tdda_status tdda_get_parameters(const tdda_model *m, double *out, int64_t n);
/* The dipole -> parameter map of src/DDAModel.cpp:163-247 (geometryPara):
 * map[i] is the free parameter that sets dipole i's density; int32[N]. */
tdda_status tdda_get_parameter_map(const tdda_model *m, int32_t *map, int64_t n);
/* DDAModel::get_dielectrics_copy (src/DDAModel.cpp:1346-1348; binding :68): double[3N] */
tdda_status tdda_get_dielectrics(const tdda_model *m, double *out, int64_t n);
/* DDAModel::get_EResult (src/DDAModel.cpp:1254-1256; binding :69): complex[3N] */
tdda_status tdda_get_electric_field(const tdda_model *m, double *out, int64_t n);
/* DDAModel::get_P (src/DDAModel.cpp:1273-1275): complex[3N] */
tdda_status tdda_get_polarization(const tdda_model *m, double *out, int64_t n);

/* DDAModel::Aproductwithalb (src/DDAModel.cpp:1194-1203) when with_al != 0,
 * AProductCore::Aproduct (src/AProductCore.cpp:461-515) otherwise.
 * x, y: complex[3N] host arrays. */
tdda_status tdda_matvec(tdda_model *m, const double *x, double *y, int with_al);
/* The same product through the complex64 operator of a mixed-precision
 * model (what its inner solves apply); x, y stay complex128 on the host. */
tdda_status tdda_matvec_c64(tdda_model *m, const double *x, double *y, int with_al);

/* Device-resident forms (pointers from cudaMalloc / torch; stream may be NULL).
 * Batched solve of (A + diag(1/alpha)) X_k = B_k for k < nrhs, complex[nrhs][3N]
 * in dipole order; B == NULL uses the model's incident field for every k.
 * Same BiCGSTAB as tdda_solve_electric_field (src/DDAModel.cpp:899-1009). */
tdda_status tdda_solve_batch_device(tdda_model *m, const void *B_dev, void *X_dev, int nrhs,
                                    int x0_zero, int max_iter, double tol, void *stream,
                                    tdda_solve_info *infos);
tdda_status tdda_matvec_device(tdda_model *m, const void *x_dev, void *y_dev, int nrhs,
                               int with_al, void *stream);

/* --- extensions (no single reference counterpart) --------------------------
 * Per-dipole design densities rho[N] in [0, 1] (a 3-D design instead of the
 * reference's z-extruded columns, DDAModel::UpdateParameters
 * src/DDAModel.cpp:747-772); sets 1/alpha per dipole. */
tdda_status tdda_set_densities(tdda_model *m, const double *rho, int64_t n);
/* Exact adjoint gradient of the IntegratedE objective with respect to every
 * dipole's density (the analytic form of calculateGradients,
 * src/DDAModel.cpp:398-578): uses the polarisation of the last solve,
 * runs one adjoint solve, grad: double[N]. */
tdda_status tdda_gradient_densities(tdda_model *m, int max_iter, double tol, double *grad, int64_t n,
                                    tdda_solve_info *info);
/* The reference's legacy design filter, for models created with use_filter
 * (in the reference reachable from C++ only).  tdda_filter_update is
 * DDAModel::UpdateStr (src/DDAModel.cpp:774-838) followed by the
 * polarisability update (UpdateAlpha): the raw parameters take `step`
 * (clamped to [0, 1]), are averaged with the in-plane cone weights of
 * src/DDAModel.cpp:580-712 (radius filter_radii[0], periodic images when
 * is_periodic) and projected by SmoothDensity (src/FilterOption.cpp:48-62) at
 * the beta the schedule gives for (it, max_it) (src/FilterOption.cpp:23-45).
 * tdda_filter_gradients is DDAModel::gradients_filtered
 * (src/DDAModel.cpp:354-396).  tdda_filter_state returns the raw and filtered
 * parameters and the current beta (get_Para_origin / get_Para_filtered /
 * get_beta, src/DDAModel.cpp:1258-1360).  All arrays double[NFpara];
 * TDDA_ERR_STATE without use_filter. */
tdda_status tdda_filter_update(tdda_model *m, const double *step, int64_t n, int it, int max_it);
tdda_status tdda_filter_gradients(tdda_model *m, const double *grad, int64_t n, int it, int max_it, double *out);
tdda_status tdda_filter_state(tdda_model *m, double *raw, double *filtered, int64_t n, double *beta);
/* Device-pointer forms of tdda_set_densities / tdda_gradient_densities /
 * tdda_patch_gradient for callers whose densities and gradients live on the
 * GPU (the torch.autograd path): rho_dev and grad_dev are double[N] device
 * arrays in dipole order; the work is ordered after, and the results are
 * ready on, `stream` (NULL: the legacy default stream).  Setting densities
 * checks them in [0, 1] (one small device-to-host read). */
tdda_status tdda_set_densities_device(tdda_model *m, const double *rho_dev, void *stream);
tdda_status tdda_gradient_densities_device(tdda_model *m, int max_iter, double tol, double *grad_dev, void *stream,
                                           tdda_solve_info *info);
tdda_status tdda_patch_gradient_device(tdda_model *m, int max_iter, double tol, double *grad_dev, void *stream,
                                       tdda_solve_info *info);
/* The design-density chain of the differentiation workload on the device (no
 * reference counterpart; the reference's own in-plane filter and exponential
 * projection are the tdda_filter_* entry points): raw_dev[x][y][z] (z
 * fastest) -> filtered_dev[x][y][z] = radius-R cone filter (periodic in x and
 * y, truncated and renormalised in z; 0 < R <= 6 cells) -> rho_dev (dipole
 * order, x fastest) = tanh projection (beta, eta) clamped to [0, 1].  The
 * backward pass maps dJ/drho (dipole order) to dJ/draw ([x][y][z]) given the
 * forward's filtered field; scratch_dev holds nx*ny*nz doubles.  Work runs on
 * `stream`. */
tdda_status tdda_design_forward_device(int nx, int ny, int nz, double radius, double beta, double eta,
                                       const double *raw_dev, double *filtered_dev, double *rho_dev, void *stream);
tdda_status tdda_design_backward_device(int nx, int ny, int nz, double radius, double beta, double eta,
                                        const double *filtered_dev, const double *grad_rho_dev, double *grad_raw_dev,
                                        double *scratch_dev, void *stream);

/* The topology-optimisation loop on the device (calculation_scripts/
 * TopoOptCalculation.py:165-209), each piece in the model's or the caller's
 * device memory:
 * - free parameters -> per-dipole densities through the model's parameter map
 *   (src/DDAModel.cpp:163-247; feed rho_dev to tdda_set_densities_device);
 * - per-dipole gradient -> per-parameter gradient, each parameter's dipoles
 *   added one at a time in dipole order (the host loop's scatter-add);
 * - a forward solve that starts from the model's current polarisation (the
 *   warm start the host loop makes by passing the previous P back in);
 * - the update: penalty and its gradient (binarizers.py:5-34), the penalised
 *   gradient, Adam (optimizers.py:3-23, bias correction inside the moving
 *   averages), the clipped ascent step, every operation rounded on its own in
 *   the order the host loop evaluates it.  penalty_out / penalty_grad_out
 *   (NFpara doubles, the reference's per-iteration penalty files) and
 *   penalty_mean_out (one double) may be null. */
typedef struct {
    int penalty;                       /* 0 parabolic, 1 gaussian, 2 triangular */
    double sigma, mu;                  /* gaussian */
    double slope;                      /* triangular */
    double coeff, one_minus_coeff;     /* penalty coefficient c of this iteration and 1 - c */
    double step;                       /* step size */
    double beta1, beta2;               /* Adam */
    double one_minus_beta1, one_minus_beta2;
    double bias1, bias2;               /* 1 - beta1^(t+1), 1 - beta2^(t+1) at timestep t */
} tdda_ascent_step;
tdda_status tdda_params_to_densities_device(tdda_model *m, const double *params_dev, double *rho_dev,
                                           void *stream);
tdda_status tdda_densities_to_params_device(tdda_model *m, const double *grad_dev, double *grad_params_dev,
                                           void *stream);
tdda_status tdda_solve_electric_field_warm(tdda_model *m, int max_iter, double tol, tdda_solve_info *info);
tdda_status tdda_ascent_step_device(int64_t n, double *params, double *adam_v, double *adam_s,
                                    const double *grad_obj, const tdda_ascent_step *cfg, double *penalty_out,
                                    double *penalty_grad_out, double *penalty_mean_out, void *stream);
/* Observation-patch objective (no reference counterpart; the nearest is
 * ObjPointEDDAModel, src/ObjDDAModel.cpp:20-100, and the off-structure branch
 * of DDAModel::solve_E, src/DDAModel.cpp:1154-1179): points xyz[3*nobs] in grid
 * units, outside the dipoles.  E_obs = E_inc(r_o) - sum_j G(r_o - r_j) P_j with
 * the model's damped periodic lattice sums; J = mean_o |E_obs|^2. */
tdda_status tdda_set_observation_points(tdda_model *m, const int32_t *xyz, int64_t nobs);
tdda_status tdda_observation_field(tdda_model *m, double *E, int64_t n);   /* complex[3*nobs] */
tdda_status tdda_patch_objective(tdda_model *m, double *out);
/* Exact adjoint gradient of the patch objective w.r.t. every dipole density
 * (one adjoint solve with the same operator): grad double[N]. */
tdda_status tdda_patch_gradient(tdda_model *m, int max_iter, double tol, double *grad, int64_t n,
                                tdda_solve_info *info);
/* Timing of the fused operator on the model's stream (CUDA events):
 * ms_matvec = mean time of one A.x (three kernels) for nrhs right-hand
 * sides, ms_pass[3] = mean time of each pass.  precision: 0 complex128,
 * 1 complex64 (mixed-precision models only). */
tdda_status tdda_profile_matvec(tdda_model *m, int precision, int nrhs, int iters, double *ms_matvec,
                                double *ms_pass);
/* Timing of the GMRES Gram-Schmidt kernels on the model's stream (CUDA events;
 * no reference counterpart, measurement support): on a scratch basis of nv
 * vectors of the model's size (3 * nx*ny*nz elements, complex128 for precision
 * 0, complex64 for 1), ms[0] = mean time of one projection pass (V^H w and
 * ||w||^2: the bulk-copy kernel and its block sums), ms[1] = mean time of one
 * update and normalisation pass.  Allocates and frees the scratch basis. */
tdda_status tdda_profile_gram_schmidt(tdda_model *m, int precision, int nv, int iters, double *ms);
/* No reference counterpart (measurement support): the damped periodic lattice
 * sums -- the interaction tensor's entries before its FFT, as
 * AProductCore::A_dic_generator forms them (src/AProductCore.cpp:335-349) --
 * at the integer offsets lo + (i, j, k), i < nb[0], j < nb[1], k < nb[2],
 * written to the device array out_dev: complex128 [nb0][nb1][nb2][6] (xx, xy,
 * xz, yy, yz, zz).  At most 2^28 offsets. */
tdda_status tdda_lattice_offsets_device(tdda_model *m, const int32_t *lo, const int32_t *nb, void *out_dev,
                                        void *stream);
/* Kernels launched by this library since load (all models). */
long long tdda_kernel_launches(void);
/* Solve precision of later solves: TDDA_PREC_C128, or TDDA_PREC_MIXED when
 * the model was created mixed (its complex64 operator exists). */
tdda_status tdda_set_precision(tdda_model *m, int precision);
/* Diagonal (Jacobi) scaling of later solves: 0 none -- the reference's plain
 * BiCGSTAB, the default for complex128 models; 1 Jacobi -- the scaled system
 * D^-1/2 A D^-1/2 (D = 1/alpha + the zero-offset lattice term) is solved
 * inside a complex128 iterative refinement that stops on the true residual
 * (the default for mixed-precision models). */
tdda_status tdda_set_preconditioner(tdda_model *m, int kind);

/* Device-side time limit of later BiCGSTAB solves, in seconds (0: none; no
 * reference counterpart).  BiCGSTAB iterations run as one CUDA graph launch
 * whose while-node repeats them on the device until every right-hand side is
 * done; the loop ends right-hand sides still running after this long with
 * status TDDA_SOLVE_TIMEOUT, and after max_iter iterations with
 * TDDA_SOLVE_MAXITER, without any host poll. */
tdda_status tdda_set_time_limit(tdda_model *m, double seconds);

/* Solver of later solves (no reference counterpart; the reference always runs
 * BiCGSTAB, src/DDAModel.cpp:899-1009).  kind 0: BiCGSTAB (default; the
 * preconditioner setting above applies).  kind 1: polynomial-preconditioned
 * restarted GMRES inside complex128 iterative refinement, for systems on which
 * BiCGSTAB stalls (structures that fill their periodic cell): each refinement
 * step recomputes the true residual in complex128 and runs an inner solve of
 * GMRES cycles of `restart` steps (2..1024) on the Jacobi-scaled operator times
 * a polynomial of `degree` (1..64; 1 is plain GMRES) in it, built from the
 * harmonic Ritz values of the first residual's Krylov space; a restart keeps
 * the `deflate` (0..restart-1) harmonic Ritz vectors of smallest magnitude
 * (deflated restarting, GMRES-DR).  kind 2: as kind 1, and the inner solve of
 * each refinement step after the first starts from the deflation space the
 * previous one ended with, the new residual orthonormalised against it, instead
 * of from the residual alone (1 <= deflate <= restart - 6).  Inner solves run in complex64 for
 * mixed-precision models.  The solve stops when ||E - A P|| / ||E|| <= tol;
 * max_iter bounds the inner operator applications (tdda_solve_info:
 * iterations = GMRES steps, inner_iterations = operator applications,
 * refinements = refinement steps). */
tdda_status tdda_set_solver(tdda_model *m, int kind, int degree, int restart, int deflate);

/* Allocation-free A.x (+ (1/alpha) o x when with_al != 0) for one vector.
 * No counterpart in the reference.  For callers that must not have device
 * memory allocated during a call -- a serving loop admitting work against a
 * fixed device-memory budget, a host thread with a latency deadline (cudaMalloc
 * and cudaFree may wait for the whole device), an application that plans every
 * device byte up front.  x_dev, y_dev: complex128[3N] device arrays in dipole
 * order; the work runs on `stream`.  The only extra memory is a fixed 32 MiB
 * scratch array in the library image (held by every GPU that loads the library
 * until exit): grids needing more (2 * 3 * nx*ny*nz * 16 B + 3 * nx*Ly*Lz * 16 B)
 * are rejected with TDDA_ERR_BAD_ARG.  The first call on a device (and the first
 * after its context was recreated, e.g. by cudaDeviceReset) looks up the
 * scratch's device address, and under lazy module loading (the CUDA default)
 * the first call on a model may load the operator kernels of its grid, which
 * allocates device memory: make one warm-up call per model before the
 * allocation-free region and before any stream capture begins.  Calls share
 * the scratch: calls that overlap on the GPU race and must be serialised by
 * the caller. */
tdda_status tdda_matvec_device_noalloc(tdda_model *m, const void *x_dev, void *y_dev, int with_al,
                                       void *stream);

/* ---------------------------------------------------------------------------
 * Serving engine (no counterpart in the reference: its path solves one
 * structure at a time in one process).  A server owns one GPU and runs a
 * request loop with continuous batching:
 *   - requests are queued at submit and admitted when a worker slot is free and
 *     their device memory fits hbm_budget_bytes (interaction tensors +
 *     per-worker solve workspaces);
 *   - the FFT'd interaction tensor of each (grid, d, lambda, nback, period,
 *     method) stays resident and is reused by later requests with the same key;
 *     idle tensors are evicted least-recently-used when the budget is short;
 *   - queued requests of the same grid (and precision, tolerance, iteration
 *     limit) are merged with the admitted one into one multi-right-hand-side
 *     solve: each polarisation is a right-hand side with its own
 *     polarisability and its own request's tensor (shared when keys match), up
 *     to max_rhs right-hand sides or fewer where the grid's x pass cannot hold
 *     that many;
 *   - each worker drives its batches on its own CUDA stream, so batches of
 *     different workers overlap on the device; BiCGSTAB iterations are replayed
 *     from CUDA graphs when use_graphs is set.
 * Structures are full boxes num_x*num_y*num_z with per-dipole densities.
 * ------------------------------------------------------------------------- */
#define TDDA_SERVER_MAX_POL 4

typedef struct tdda_server tdda_server;

typedef struct {
    int64_t hbm_budget_bytes; /* admission budget for tensors + workspaces */
    int32_t workers;          /* concurrent batches (host thread + CUDA stream each), 1..64 */
    int32_t max_rhs;          /* right-hand sides merged into one batched solve, 1..16 */
    int32_t use_graphs;       /* replay BiCGSTAB iterations from CUDA graphs */
    int32_t graph_steps;      /* iterations per graph (default 4 when 0) */
} tdda_server_config;

typedef struct {
    int32_t num_x, num_y, num_z;  /* box; dipole i = x + num_x*(y + num_y*z) */
    double d, lam, nback, E0;
    double material[4];           /* background, structure: (re, im) each */
    int32_t MAXm, MAXn;           /* periodic images |m| <= MAXm, |n| <= MAXn */
    double Lm, Ln;                /* periods in units of d */
    int32_t method;               /* 0 FCD, 1 LDR (polarisability: LDR for both) */
    double n_K[3];                /* propagation direction of the plane wave */
    int32_t npol;                 /* polarisations = right-hand sides, 1..TDDA_SERVER_MAX_POL */
    double n_E0[TDDA_SERVER_MAX_POL][3];
    const double *rho;            /* num_x*num_y*num_z densities in [0, 1] (copied at submit) */
    int32_t precision;            /* TDDA_PREC_MIXED or TDDA_PREC_C128 (Jacobi-refined) */
    double tol;                   /* true relative residual per right-hand side */
    int32_t max_iter;
    double *P_out;                /* npol*3N complex, dipole order, or NULL; valid until wait returns */
    double *E_out;                /* npol*3N complex E_int = al P / ((2+eps)/3), or NULL */
} tdda_request;

typedef struct {
    int32_t status;               /* tdda_status of the request */
    tdda_solve_info info[TDDA_SERVER_MAX_POL];
    int32_t batch_rhs;            /* right-hand sides of the batch it ran in */
    int32_t batch_requests;       /* requests of that batch */
    int32_t cache_hit;            /* its tensor was resident */
    int32_t worker;
    double queue_ms;              /* submit -> admitted */
    double build_ms;              /* tensor build (0 on a hit) */
    double solve_ms;              /* batch solve incl. setup and result copies */
    double total_ms;              /* submit -> result ready */
} tdda_request_result;

typedef struct {
    int64_t submitted, completed, failed;
    int64_t cache_hits, cache_misses, evictions;
    int64_t batches, merged_requests;   /* requests that joined another's batch */
    int64_t bytes_in_use, peak_bytes, cached_tensors;
    int32_t max_concurrent;             /* most batches in flight at once */
    int32_t admission_waits;            /* times the queue head waited for memory */
} tdda_server_stats;

/* si, ci: the SiCi tables of tdda_model_create (shared by every FCD request). */
tdda_status tdda_server_create(const tdda_server_config *cfg, const double *si, const double *ci, int64_t ntab,
                               tdda_server **out);
/* Queues a request; returns at once with its ticket.  Requests that can never
 * fit the budget fail at submit with TDDA_ERR_OOM. */
tdda_status tdda_server_submit(tdda_server *s, const tdda_request *req, int64_t *ticket);
/* Waits up to timeout_s (< 0: forever) for a ticket; TDDA_ERR_TIMEOUT if not
 * ready.  A ticket can be waited for once. */
tdda_status tdda_server_wait(tdda_server *s, int64_t ticket, double timeout_s, tdda_request_result *result);
/* Builds every worker's solve workspace for one grid (and precision) now,
 * counted against the budget, so that the first requests of that grid do not
 * pay for allocation.  Call before submitting requests. */
tdda_status tdda_server_reserve(tdda_server *s, int32_t num_x, int32_t num_y, int32_t num_z, int32_t precision);
tdda_status tdda_server_get_stats(tdda_server *s, tdda_server_stats *stats);
/* Finishes queued work, then frees every device buffer. */
void tdda_server_destroy(tdda_server *s);

#ifdef __cplusplus
}
#endif

#endif /* TDDA_H_ */
