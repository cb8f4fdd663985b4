/* uqc.h - C ABI of the B200 implementation of UQCreator's IPM hot path.
 *
 * The hot path is one explicit time step of the intrusive polynomial moment
 * method: per-cell dual Newton closure, reconstruction at quadrature nodes,
 * kinetic numerical flux projected onto the moments, explicit Euler update.
 * Plain pointers and sizes only; every call returns an int status (0 = ok,
 * negative = error) and never exits the process. uqc_last_error() gives the
 * message of the last failed call on a handle.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to UQCreator's code/src). The reference calls exit(EXIT_FAILURE) on every
 * error (closure.cpp:180-192, vectorspace.cpp:166-170, settings.cpp:316-322);
 * here the same conditions return a status.
 *
 * State layouts (per cell, nS states x nT moments):
 *   UQC_LAYOUT_REF          the reference's Matrix(nS, nT): column-major,
 *                           element (s, i) at i * nS + s (matrix.cpp:8,107)
 *   UQC_LAYOUT_STATE_MAJOR  element (s, i) at s * nT + i, the order of the
 *                           reference's gradient vectors (closure.cpp:245)
 * Cells are contiguous, nS * nT doubles each, nT = the finest level's size.
 *
 * Threading: a handle owns a CUDA stream (the one passed at creation, or its
 * own). Calls on one handle must be serialised by the caller; distinct
 * handles may be used concurrently from different threads.
 */
#ifndef UQC_H
#define UQC_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct uqc_solver uqc_solver;

enum uqc_status_code {
    UQC_OK               = 0,
    UQC_ERR_ARGUMENT     = -1, /* bad pointer, size or enum value */
    UQC_ERR_CONFIG       = -2, /* invalid or unsupported TOML configuration */
    UQC_ERR_CUDA         = -3, /* CUDA runtime error (message has the name) */
    UQC_ERR_NOT_CONVERGED = -4, /* at least one cell's Newton failed; see uqc_cell_status */
    UQC_ERR_MEMORY       = -5, /* device allocation failed */
    UQC_ERR_STATE        = -6, /* call out of order (e.g. step before init) */
    UQC_ERR_CAPACITY     = -7  /* request exceeds a fixed capacity */
};

enum uqc_layout { UQC_LAYOUT_REF = 0, UQC_LAYOUT_STATE_MAJOR = 1 };

/* Hessian precision of the Newton closure.
 * UQC_FP64:  all-FP64 (the reference's arithmetic).
 * UQC_MIXED: Hessian assembled, factored and solved in FP32; the gradient,
 *            the convergence and line-search tests, the duals and the moment
 *            update stay FP64, so a converged cell meets the same FP64
 *            tolerance. Cells whose FP32 Newton does not converge (FP32
 *            factor not positive definite, line-search or iteration limit)
 *            continue from their last accepted duals in the FP64 form. */
enum uqc_precision { UQC_FP64 = 0, UQC_MIXED = 1 };

/* Per-cell closure status (uqc_cell_status). */
enum uqc_cell_code {
    UQC_CELL_CONVERGED     = 0,
    UQC_CELL_MAX_ITER      = 1, /* "Newton did not converge" (closure.cpp:191-192) */
    UQC_CELL_LINE_SEARCH   = 2, /* "too many refinement steps" (closure.cpp:180-183) */
    UQC_CELL_NOT_PD        = 3, /* posv info > 0 (vectorspace.cpp:166-170) */
    UQC_CELL_NONFINITE     = 4  /* moments or duals not finite on entry */
};

typedef struct uqc_info {
    int n_cells, n_states, n_total, n_quad, n_levels, dim_xi, n_faces, mesh_dim;
    int n_total_level[16]; /* moments per refinement level */
    int precision;         /* uqc_precision in use */
    int newton_mode;       /* 0 reference SolveClosure, 1 guarded, 2 SolveClosureSafe */
    double t;              /* simulated time */
    long long steps;       /* time steps taken */
    int mixed_form;        /* how UQC_MIXED time steps run the closure: 0 one kernel (FP32 Hessian on
                              CUDA cores), 1 rounds of chord / Hessian / inverse kernels with the Hessian
                              on CUDA cores, 2 the same with the Hessian on the tensor cores; -1 before
                              the device side is set up (option "mixed_hessian") */
    int mixed_rounds;      /* re-factorisation rounds per time step of forms 1 and 2 */
} uqc_info;

typedef struct uqc_step_info {
    double t, dt, residual;   /* after the last step (momentsolver.cpp:134,149-152) */
    int steps;                /* steps taken by this call */
    int failed_cells;         /* cells whose closure did not converge */
    long long newton_iterations; /* summed over cells and steps of this call */
    long long line_search_trials;
    int active_cells;         /* cells that needed Newton iterations in the last step */
    long long fallback_cells; /* UQC_MIXED: cells handed to the FP64 form during this call */
    int running;              /* 1 while the loop condition of momentsolver.cpp:79 holds */
} uqc_step_info;

/* ---- lifecycle and configuration ------------------------------------ */

/* Creates a solver from a UQCreator TOML input file: Settings(toml)
 * (settings.h:103, settings.cpp:22-323) + Problem::Create (problem.cpp:18-42) +
 * Mesh::Create (mesh.cpp:19-32) + Closure::Create (closure.cpp:94-131) +
 * MomentSolver(settings, mesh, problem) (momentsolver.h:139). cuda_stream may be
 * NULL (the handle creates its own stream). On error *out is NULL and the
 * message is copied to err (when err != NULL).
 * Meshes: 1-D uniform ([mesh] numberOfCells, a, b; Mesh1D), SU2 triangle
 * meshes ([mesh] format = "SU2", SU2MeshFile relative to the file's directory,
 * SU2BC = [["marker", "dirichlet" | "noslip" | "swwall"], ...];
 * Mesh2D::LoadSU2MeshFromFile, mesh2d.cpp:5-259; "neumann" and "periodic"
 * are refused with UQC_ERR_CONFIG), or the seeded "tri_jitter" mesh of the
 * [uqc] table. Problems: Burgers1D, Euler1D, Euler2D, ShallowWater1D;
 * closures: BoundedBarrier, LogSin, Euler, Euler2D, ShallowWater and the
 * linear StochasticGalerkin, L2Filter, LassoFilter (with any of the problems'
 * states). ExponentialFilter, ShallowWater2D and PNEquations2D return
 * UQC_ERR_CONFIG with the reason (the reference's code for them is undefined,
 * unfinished or racy). */
int uqc_create_from_file( const char* toml_path, void* cuda_stream, uqc_solver** out, char* err, int err_len );
/* Same, from TOML text in memory; files it names are relative to the working directory. */
int uqc_create_from_string( const char* toml_text, void* cuda_stream, uqc_solver** out, char* err, int err_len );
/* The same settings as a struct, for callers without a TOML file: each field
 * is the key of the reference's input file named beside it (Settings::Init,
 * settings.cpp:22-323) or of the [uqc] table. Strings may be NULL where the
 * key is optional; uqc_config_defaults fills the reference's defaults. The
 * handle is the one uqc_create_from_string makes from the equivalent file. */
typedef struct uqc_config {
    const char* problem;        /* [general] problem: "Burgers1D", "Euler1D", "Euler2D", "ShallowWater1D" */
    const char* restart_file;   /* [general] restartFile (NULL: none) */
    int import_dual_state;      /* [general] importDualState */
    int mesh_dimension;         /* [mesh] dimension: 1 or 2 */
    int n_cells;                /* [mesh] numberOfCells (1-D) */
    double a, b;                /* [mesh] a, b (1-D interval) */
    const char* su2_file;       /* [mesh] SU2MeshFile (format "SU2"; NULL: no SU2 mesh) */
    int n_su2_bc;               /* [mesh] SU2BC: markers and types ("dirichlet", "noslip", "swwall") */
    const char* const* su2_bc_marker;
    const char* const* su2_bc_type;
    int dim_xi;                 /* [problem] distribution: dim_xi Legendre dimensions ... */
    double sigma[4];            /* ... with these widths */
    double cfl;                 /* [problem] CFL */
    double t_end;               /* [problem] tEnd */
    double min_residual;        /* [problem] residual (negative: not set) */
    double gamma;               /* [problem] gamma (Euler; 0: default 1.4) */
    const char* closure;        /* [moment_system] closure: "BoundedBarrier", "LogSin", "Euler", "Euler2D", "ShallowWater",
                                   "StochasticGalerkin", "L2Filter", "LassoFilter" */
    int max_degree;             /* [moment_system] moments = [["maxDegree"|"totalDegree"], [degrees]] */
    int n_levels;               /* refinement levels: degree[0..n_levels-1] */
    int degree[16];
    int quad_points[16];        /* [moment_system] quadPoints = [["tensorizedGrid"], [n per level]] */
    int max_iterations;         /* [moment_system] maxIterations */
    double epsilon;             /* [moment_system] epsilon */
    int n_ic;                   /* [uqc] ic */
    double ic[8];
    double bounds[2];           /* [uqc] bounds (bounded barrier) */
    int nx, ny;                 /* [uqc] mesh = "tri_jitter", mesh_params = [nx, ny, jitter, seed] (nx = 0: not used) */
    double jitter;
    unsigned long long seed;
    int precision;              /* [uqc] precision: uqc_precision */
    int newton_mode;            /* [uqc] newton: 0 reference, 1 guarded, 2 safe */
    int steps;                  /* [uqc] steps (0: to tEnd) */
} uqc_config;
void uqc_config_defaults( uqc_config* cfg );
int uqc_create_from_config( const uqc_config* cfg, void* cuda_stream, uqc_solver** out, char* err, int err_len );
void uqc_destroy( uqc_solver* h );                        /* ~MomentSolver (momentsolver.cpp:32-35) */
const char* uqc_last_error( const uqc_solver* h );
int uqc_get_info( const uqc_solver* h, uqc_info* out );
int uqc_set_precision( uqc_solver* h, int precision );
/* Closure::SetMaxIterations (closure.cpp:341) and the epsilon of settings.cpp:314. */
int uqc_set_newton( uqc_solver* h, int max_iterations, double epsilon, int newton_mode );

/* Launch tuning (no reference counterpart; the autotuner uses it):
 *   "closure_group"  threads per cell in the closure kernel: 32 (a warp per
 *                    cell, several cells per CTA), 64 (two warps per cell,
 *                    up to four cells per CTA) or 256 (a CTA per cell);
 *                    0 = automatic.
 *   "update_warps", "check_warps", "chord_warps"  warps (cells) per CTA of
 *                    the update kernel (default 8), the convergence-check
 *                    kernel (default 16) and the mixed form's chord kernel
 *                    (default 16), each capped by shared memory; 0 = default.
 *   "closure_tiny"   systems of at most 6 duals per cell (states x moments)
 *                    on at most 64 nodes: -1 (default) / 1: the Newton of
 *                    each cell runs in registers on one warp (sums over nodes
 *                    by butterfly reduction, every lane solving the small
 *                    system itself), in both precisions (FP64 arithmetic);
 *                    0: the general closure kernel.
 *   "closure_tables_smem"  1: the closure kernels stage the basis tables in
 *                    shared memory; 0: they read them through the L1 cache
 *                    (more cells per SM); -1 = automatic.
 *   "mixed_chord"    UQC_MIXED, 1 (default): inexact (chord) Newton that
 *                    keeps each cell's FP32 factor in device memory (about
 *                    2 n^2 bytes per cell, n = states x moments) and reuses it
 *                    across iterations and time steps while it contracts;
 *                    0: a new factor at every iteration.
 *   "mixed_chord_inverse"  1 (default): the held factor is kept as its
 *                    packed inverse U^-1 (formed at each re-factorisation), so
 *                    a held-factor direction is two mat-vecs instead of two
 *                    triangular solves; used when its shared memory costs no
 *                    cell per SM (else the triangular solves); 0: never.
 *   "mixed_chord_theta"  re-factor after a step with the held factor that
 *                    reduced ||g|| by less than the factor 1/theta (default: 0.2 in the
 *                    rounds form, 0.1 in the single kernel; the autotuner's choices).
 *   "update_test"    1: the update kernel tests the next step's closure
 *                    convergence per cell and lists only the cells that need
 *                    Newton; 0: a check kernel tests every cell at the start
 *                    of each step; -1 (default): 1 with a single refinement
 *                    level, 0 with several.
 *   "graphs"         1 (default): uqc_run and uqc_step_async launch cached
 *                    CUDA graphs of whole time steps; 0: direct launches.
 *   "host_chunks"    uqc_step_host: chunks of cells the copies and kernels
 *                    of a step are split into (1-32, default 6).
 *   "mixed_max_iterations"  UQC_MIXED: Newton iterations of the FP32 pass
 *                    after which a cell continues in the FP64 form (>= 2;
 *                    0 = the configured maxIterations).
 *   "mixed_hessian"  UQC_MIXED time steps of the 2-D Euler closure (one
 *                    refinement level): -1 (default) rounds with the Hessian
 *                    on the tensor cores where its basis-pair table fits one
 *                    MMA (at most 256 pairs, i.e. total degree <= 5 in two
 *                    uncertainties), else the single kernel; 0 the single-kernel
 *                    form; 1 rounds with the CUDA-core Hessian; 2 rounds with
 *                    the tensor-core Hessian (UQC_ERR_CONFIG where it does
 *                    not fit). Rounds: a chord kernel (a warp per cell, held
 *                    inverse H0^-1 in FP32, FP64 gradients and tests), then
 *                    per round the Hessians and inverses of the cells whose
 *                    held inverse stopped contracting, and the chord kernel
 *                    again; cells left after the last round finish in FP64.
 *   "mixed_rounds"   re-factorisation rounds per step of the forms above (1-3, default 2).
 * Unknown keys return UQC_ERR_ARGUMENT. */
int uqc_set_option( uqc_solver* h, const char* key, double value );

/* Host copies of the tables of Closure::Closure (closure.cpp:16-84):
 * phi[k * nT + i] = phiTilde(k, i), phi_wf = phiTildeWf, xi[k * dimXi + l],
 * w[k]. Any pointer may be NULL. */
int uqc_get_tables( const uqc_solver* h, double* phi, double* phi_wf, double* xi, double* w );
/* Host copies of the mesh geometry (Cell/Line/Triangle, cell.h:52-77):
 * per cell area, max edge, centre (2); per face unit normal (2), scaled
 * normal (2), neighbour id (ghost id = n_cells), boundary flag. */
int uqc_get_geometry( const uqc_solver* h, double* area, double* max_edge, double* center, double* unit_normal,
                      double* scaled_normal, int* neighbor, int* boundary );

/* ---- state ------------------------------------------------------------ */

/* Initial moments and duals on the device: MomentSolver::SetupIC
 * (momentsolver.cpp:535-563) and SetDuals without restart (:463-485); with
 * [general] restartFile = "<prefix>" in the input (settings.cpp:74-79) the
 * moments come from <prefix>_moments (DetermineMoments, :418-433) and, with
 * importDualState = true, the duals from <prefix>_duals (:465-466), else the
 * duals start from DS of the moments. The prefix is relative to the input
 * file's directory. A restart with another number of moments is refused. */
int uqc_init_state( uqc_solver* h );
/* Copies caller-owned host state to the device (u, lambda: n_cells * nS * nT
 * doubles in `layout`; level: n_cells refinement levels or NULL to keep). */
int uqc_upload_state( uqc_solver* h, const double* u, const double* lambda, const unsigned* level, int layout, double t );
int uqc_download_state( uqc_solver* h, double* u, double* lambda, unsigned* level, int layout );
/* MomentSolver::Export (momentsolver.cpp:565-588): writes <prefix>_moments
 * and <prefix>_duals in the reference's format (a line per cell, nS x nT values
 * in state-major order with 15 significant digits, each followed by a comma),
 * the files a restart reads. */
int uqc_export_state( uqc_solver* h, const char* path_prefix );

/* ---- hot path ----------------------------------------------------------- */

/* Batched Closure::SolveClosure (closure.cpp:133-193) on the resident state:
 * every cell's duals solved in place for its current refinement level. */
int uqc_solve_closure( uqc_solver* h, uqc_step_info* info );
/* The same on a subset of the resident cells (cells: n_cells host cell ids,
 * or NULL for all cells), with this call's tolerance and iteration limit
 * (tol > 0 and max_iter > 0 override the configured epsilon and
 * maxIterations of settings.cpp:314; 0 keeps them): the closure loop of
 * momentsolver.cpp:83-89 restricted to the cells a caller lists. */
int uqc_solve_closure_cells( uqc_solver* h, const unsigned* cells, int n_cells, double tol, int max_iter, uqc_step_info* info );
/* Closure status and Newton iterations per cell from the last closure solve. */
int uqc_cell_status( uqc_solver* h, int* status, int* iterations );
/* n_steps time steps: the body of MomentSolver::Solve (momentsolver.cpp:79-152)
 * with ExplicitEuler::Advance (expliciteuler.cpp:8-75). Stops early once
 * t >= tEnd or residual <= minResidual (the loop condition of :79). */
int uqc_step( uqc_solver* h, int n_steps, uqc_step_info* info );
/* MomentSolver::Solve's time loop to the configured tEnd (or t_end > 0). */
int uqc_run( uqc_solver* h, double t_end, uqc_step_info* info );
/* One time step from caller-owned HOST state to host state (the call a
 * GpuMomentSolver adapter that keeps the reference's _u / _lambda on the host
 * makes per step, momentsolver.cpp:79-152): the same result as
 * uqc_upload_state(u_in, lambda_in, level_in, UQC_LAYOUT_STATE_MAJOR, t),
 * uqc_step(h, 1, info) and uqc_download_state(u_out, lambda_out, level_out,
 * UQC_LAYOUT_STATE_MAJOR), with the copies beside the kernels: moments and
 * duals go up in chunks of cells, each chunk's closure (check and Newton)
 * starting as its chunk lands and its duals going down as it ends, beside the
 * later chunks' uploads; the update runs in chunks too, each chunk's moments
 * going down as it ends. Moments, duals, levels, t and dt are those of the
 * three calls bit for bit; the residual sums the same terms in another order.
 * Pinned host memory lets the copies run asynchronously.
 * level_in NULL keeps the resident levels, level_out NULL skips them; the out
 * arrays may be the in arrays. uqc_last_timing: [0] from the first copy to the
 * end of the closure phase, [1] the update. */
int uqc_step_host( uqc_solver* h, const double* u_in, const double* lambda_in, const unsigned* level_in, double t, double* u_out,
                   double* lambda_out, unsigned* level_out, uqc_step_info* info );
/* Mean and variance per cell and state (MomentSolver::WriteMeanAndVar,
 * momentsolver.cpp:302-328): out[j * 2 nS + s] = E, out[j * 2 nS + nS + s] = Var. */
int uqc_mean_var( uqc_solver* h, double* out );
/* The same entry point under the name of the drop-in boundary's plan. */
int uqc_moments_mean_var( uqc_solver* h, double* out );
/* Mesh1D::Export / Mesh2D::Export (mesh1d.cpp:90-220, mesh2d.cpp:399-501):
 * legacy VTK unstructured grid (ASCII) at `path` (".vtk" appended when
 * missing) with the reference's arrays E(.) and Var(.) per state as cell data
 * and averaged to the points; 1-D cells are quads extruded to a tenth of the
 * domain, and <path>ExpectedValue / <path>Variance text columns are written too. */
int uqc_write_vtk( uqc_solver* h, const char* path );

/* Drop-in for Closure::SolveClosure on caller-owned HOST arrays (the call a
 * GpuClosure adapter makes): n cells of (lambda, u) in `layout`, solved for
 * n_total[j] moments (NULL = finest). Copies in, solves, copies lambda back.
 * status[j] gets a uqc_cell_code (may be NULL). */
int uqc_closure_solve_host( uqc_solver* h, int n, double* lambda, const double* u, const unsigned* n_total, int layout,
                            int* status );
/* Same on caller-owned DEVICE arrays in UQC_LAYOUT_STATE_MAJOR, enqueued on
 * the handle's stream; no host synchronisation. */
int uqc_closure_solve_device( uqc_solver* h, int n, double* d_lambda, const double* d_u, const unsigned* d_n_total,
                              int* d_status );

/* For callers that must not allocate GPU memory: the batched FP64 closure of
 * uqc_closure_solve_device, on caller-owned DEVICE arrays, without any
 * cudaMalloc/cudaFree, not even on its first call. No counterpart in the
 * reference (its closure runs on the host).
 *
 * Who needs it: code that runs inside a framework owning all device memory
 * (its own arena or pool, where a stray cudaMalloc would fragment or exceed
 * the budget the framework manages), and latency-critical loops that may not
 * reach the allocator, whose calls can synchronise the device. The handle may
 * be freshly created (its own device state is never touched); its
 * configuration and basis tables come from host memory.
 *
 * Precision: always the FP64 form, whatever the handle's precision (the mixed
 * form keeps a per-cell factor store, which would need an allocation); its
 * results are those of uqc_closure_solve_device on a UQC_FP64 handle.
 *
 * Scratch lives in one statically allocated device array inside this library
 * (UQC_NOALLOC_SCRATCH_BYTES, held on every GPU that loads the library until
 * the process exits): the loop-control block, per-cell iteration counts for at
 * most UQC_NOALLOC_MAX_CELLS cells, and copies of the two basis tables (nQ rows
 * of an odd stride >= nT, plus 8 doubles each) and of the nQ node weights, at
 * most UQC_NOALLOC_MAX_TABLE doubles per table (the second table together with
 * the weights). Larger requests return UQC_ERR_CAPACITY. Every call overwrites the whole
 * array, so calls whose work overlaps on the GPU (different streams, or
 * different host threads, at the same time) race and must be serialised by
 * the caller.
 *
 * d_lambda (in/out), d_u: n cells, UQC_LAYOUT_STATE_MAJOR; d_n_total: moments
 * per cell or NULL (finest level); d_status: n uqc_cell_code values (required);
 * cuda_stream: the stream to enqueue on (NULL = the legacy default stream).
 * Asynchronous: results are valid once the stream has reached this point.
 * The first call on each device (with that device current) looks up the
 * array's device address and sets the kernel's shared-memory limit; make that
 * first call before any stream capture begins. The address is kept for the
 * life of the process: do not call cudaDeviceReset on a device while this
 * library is in use there. */
#define UQC_NOALLOC_MAX_CELLS 65536
#define UQC_NOALLOC_MAX_TABLE 8192
#define UQC_NOALLOC_SCRATCH_BYTES ( 256 + 4 * UQC_NOALLOC_MAX_CELLS + 16 * UQC_NOALLOC_MAX_TABLE )
int uqc_closure_solve_device_noalloc( uqc_solver* h, int n, double* d_lambda, const double* d_u, const unsigned* d_n_total,
                                      int* d_status, void* cuda_stream );

/* ---- asynchronous stepping and serving ----------------------------------
 * No reference counterpart: the reference runs one MomentSolver::Solve per
 * process. These entry points let one process keep many solves resident on
 * the device and interleave their time steps. */

/* Enqueues n_steps time steps and a copy of the loop state on the handle's
 * stream and returns at once. Steps after the loop condition fails do no work. */
int uqc_step_async( uqc_solver* h, int n_steps );
/* 1 when the work of the last uqc_step_async has finished (info filled as by
 * uqc_step, for the steps since the previous query), 0 while it runs. */
int uqc_step_query( uqc_solver* h, uqc_step_info* info );
/* Device memory (bytes) the handle holds once its device side is set up. */
int uqc_device_bytes( const uqc_solver* h, unsigned long long* bytes );

/* Spatial sharding, one process (one handle) per GPU. Replaces the MPI work
 * split of MomentSolver::Solve (code/src/momentsolver.cpp:83-152): there every
 * rank keeps all cells, solves the duals of its round-robin cells
 * (_cellIndexPE, :83-89), broadcasts every cell's duals (MPI_Bcast, :92-95),
 * reduces the moments of its quadrature-node slice onto the owner
 * (MPI_Reduce, :144-146) and takes the step as MPI_Allreduce MIN (:133), the
 * residual as MPI_Allreduce SUM (:152). Here a rank keeps its own block of
 * cells and a one-ring halo; one time step is
 *   uqc_step_phase(h, 0)  closure of the owned cells (their nodal states and
 *                         the rank's smallest CFL step, as double bits, at
 *                         *d_dt_bits);
 *   caller: all-reduce MIN of the 8 bytes at *d_dt_bits (as uint64: positive
 *           doubles order as their bits), and the halo exchange: uqc_halo_pack
 *           gathers the rows the peers need (row_doubles each, peers in
 *           ascending order, send_counts[p] rows to peers[p]); the rows
 *           received from peers[p] (recv_counts[p] of them, in the same peer
 *           order) are written contiguously from *d_halo_rows;
 *   uqc_step_phase(h, 1)  flux and update of the owned cells.
 * All on the handle's stream (uqc_stream), so the caller's collectives go on
 * that stream too. A shard's residual (*d_residual after phase 1, the
 * reference's per-rank sum) is its owned cells' part: the caller all-reduces it
 * (SUM) when it applies the minResidual stopping rule; the device loop
 * condition of a sharded handle tests only tEnd and [uqc] steps. */
typedef struct uqc_shard_info {
    int rank, n_ranks;
    int n_global;       /* cells of the whole mesh */
    int n_owned;        /* local cells 0 .. n_owned-1 are owned (in global order) */
    int n_halo;         /* local cells n_owned .. n_owned+n_halo-1: halo, grouped by owner rank */
    int n_peers;        /* ranks this one exchanges with */
    int n_send;         /* rows sent per step (sum of send_counts) */
    int row_doubles;    /* nodal states per cell: n_states x n_quad */
} uqc_shard_info;
/* Makes the handle rank `rank` of n_ranks: the mesh is split by recursive
 * coordinate bisection of the cell centres and the handle keeps its owned
 * cells and their halo (uqc_info.n_cells = n_owned + n_halo; state arrays of
 * every other call are per local cell). Call before any call that uses the
 * device. A sharded handle refuses uqc_step, uqc_run, uqc_step_async,
 * uqc_export_state, uqc_write_vtk and a restart. */
int uqc_partition( uqc_solver* h, int rank, int n_ranks );
/* The shard plan (host only): info, and when non-null: global_ids[n_owned +
 * n_halo] (global cell id of each local cell), peers / send_counts /
 * recv_counts [n_peers], send_cells[n_send] (local ids, grouped by peer). An
 * unsharded handle reports itself as rank 0 of 1. */
int uqc_get_shard( const uqc_solver* h, uqc_shard_info* info, int* global_ids, int* peers, int* send_counts, int* recv_counts,
                   int* send_cells );
/* Device pointers of the exchange: the first halo row of the nodal states,
 * the step's min dt (uint64 bits) and the residual (double). */
int uqc_shard_buffers( uqc_solver* h, double** d_halo_rows, unsigned long long** d_dt_bits, double** d_residual );
/* Gathers the rows the peers need into d_send (n_send x row_doubles doubles,
 * device memory) on the handle's stream. */
int uqc_halo_pack( uqc_solver* h, double* d_send );
/* Half of a time step on the handle's stream: phase 0 the closure, phase 1
 * the flux and update (info, when non-null, is filled as by uqc_step, which
 * waits for the stream). Also valid on an unsharded handle (phase 0 then
 * phase 1 is one uqc_step without the graph). */
int uqc_step_phase( uqc_solver* h, int phase, uqc_step_info* info );

/* Request server: continuous batching of whole UQ solves (each request is a
 * TOML configuration run to its tEnd). Requests wait in submission order and
 * are admitted, first fit, while their device memory fits the budget and
 * fewer than max_active run; each admitted request owns a stream and its
 * state stays on the device; every progress call advances running requests by
 * slices of steps_per_slice time steps (their kernels overlap on the device),
 * retires finished ones (mean and variance are computed and the device memory
 * freed) and admits waiting ones; the order of admission and slices follows
 * the scheduling policy (uqc_server_set_option). A request's result does not depend on what else runs. Times are ms
 * since the server was created. Not thread safe: one thread drives a server. */
typedef struct uqc_server uqc_server;
enum uqc_request_state { UQC_REQ_QUEUED = 0, UQC_REQ_RUNNING = 1, UQC_REQ_DONE = 2, UQC_REQ_FAILED = 3 };
typedef struct uqc_request_info {
    long long id;
    int state;              /* uqc_request_state */
    int status;             /* uqc_status_code of the solve (UQC_OK when done) */
    int n_cells, n_states;  /* mean_var holds n_cells x 2 n_states doubles */
    int steps;              /* time steps taken */
    double t;               /* simulated time reached */
    long long newton_iterations;
    unsigned long long device_bytes;
    double submit_ms, admit_ms, done_ms;
} uqc_request_info;
int uqc_server_create( unsigned long long device_budget_bytes, int max_active, int steps_per_slice, uqc_server** out );
void uqc_server_destroy( uqc_server* s );
const char* uqc_server_last_error( const uqc_server* s );
/* precision: uqc_precision of the request. May be called from another thread
 * than uqc_server_progress (a request front end): the request's solver is
 * built (mesh, tables; host work only) before the server's lock is taken, so
 * the scheduling loop does not wait for it. The other server calls take the
 * same lock; uqc_server_destroy must not race with any of them. */
int uqc_server_submit( uqc_server* s, const char* toml_text, int precision, long long* id );
/* One scheduling pass; counts after it (any pointer may be NULL). */
int uqc_server_progress( uqc_server* s, int* n_queued, int* n_running, int* n_done );
/* State of a request; mean_var (or NULL) receives E and Var per cell and
 * state (the layout of uqc_mean_var) once it is done. */
int uqc_server_request( const uqc_server* s, long long id, uqc_request_info* info, double* mean_var );
/* Error message of a failed request ("" otherwise; valid until it is released). */
const char* uqc_server_request_error( const uqc_server* s, long long id );
/* Forgets a finished request and its result. */
int uqc_server_release( uqc_server* s, long long id );
/* Scheduling options:
 *   "policy"        0 (default): every running request advances by a slice
 *                   per progress call, admission in submission order; 1:
 *                   shortest remaining time first, for admission and for
 *                   slices, with at most "max_stepping" requests stepping at a
 *                   time (the others stay resident and idle). Remaining time =
 *                   cells x duals x nodes x the steps left ([uqc] steps; 1000
 *                   when only tEnd bounds the run) over the server's measured
 *                   rate, minus "aging" x the request's waiting time.
 *   "max_stepping"  requests with a slice in flight under policy 1 (default 0:
 *                   no limit).
 *   "aging"         ms of remaining time one ms of waiting offsets (default 1). */
int uqc_server_set_option( uqc_server* s, const char* key, double value );

/* ---- introspection ----------------------------------------------------- */

/* Device time (ms) of the kernels of the last uqc_step call, by phase:
 * [0] closure + reconstruction, [1] flux + update, [2] total. */
int uqc_last_timing( uqc_solver* h, float* ms3 );
/* Device pointers of the resident state (for zero-copy callers): u, lambda.
 * Between steps u holds the updated moments (as the reference's u after
 * ExplicitEuler::Advance). A caller that writes through the pointers calls
 * this function again after writing (it makes the next step test every cell
 * for convergence instead of the list the last update prepared). */
int uqc_device_state( uqc_solver* h, double** d_u, double** d_lambda );
/* Inverse Hessians H^-1 of the mixed form's re-factorisation (FP32) for n
 * cells of the resident state (cells: host array of cell ids), with the
 * Hessian assembled on CUDA cores (form 1) or on the tensor cores (form 2);
 * out: n x (nS nT)^2 floats, each cell's H^-1 row-major. Clears the handle's
 * held inverses. 2-D Euler with one refinement level (uqc_info.mixed_form >= 1).
 * No reference counterpart: a diagnostic of the tensor-core Hessian. */
int uqc_debug_mixed_inverse( uqc_solver* h, int n, const int* cells, int form, float* out );
/* Number of kernel launches issued by the last uqc_step / uqc_solve_closure. */
int uqc_last_launch_count( uqc_solver* h );
/* CUDA stream of the handle (cudaStream_t). */
void* uqc_stream( uqc_solver* h );

/* Seeded jittered triangle mesh of the "tri_jitter" workloads (host only):
 * xy[2 (nx+1)(ny+1)], node_boundary[(nx+1)(ny+1)], tri[3 * 2 nx ny]. */
int uqc_mesh_tri_jitter( int nx, int ny, double jitter, unsigned long long seed, double* xy, int* node_boundary, int* tri );

#ifdef __cplusplus
}
#endif
#endif /* UQC_H */
