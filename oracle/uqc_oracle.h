/* FP64 CPU restatement of UQCreator's per-time-step IPM hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the product
 * never links, calls or falls back to it.
 *
 * Parity is pinned: tests compare every function here bit for bit with the
 * reference's own sources built as oracle/_ref (oracle/ref/Makefile) and with
 * the golden vectors in tests/golden made from that build.
 *
 * Layout: per cell, state-major vectors x[s * nT + i] (s < nStates, i < nTotal).
 * Tables: phi[k * nT + i] = phiTilde(k, i), phiWf[k * nT + i].
 */
#ifndef UQC_ORACLE_H
#define UQC_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum { UQCO_BOUNDED_BARRIER = 0, UQCO_EULER2D = 1, UQCO_SHALLOW_WATER = 2 };
enum { UQCO_BURGERS = 0, UQCO_EULER = 1, UQCO_SW = 2 };

typedef struct uqco_config {
    int closure;        /* UQCO_BOUNDED_BARRIER | UQCO_EULER2D | UQCO_SHALLOW_WATER */
    int problem;        /* UQCO_BURGERS | UQCO_EULER | UQCO_SW */
    int dim_xi;         /* uncertain dimensions */
    int max_degree;     /* 1 = "maxDegree" index set, 0 = "totalDegree" */
    int n_levels;       /* refinement levels (moments = [[...],[d0..dL-1]]) */
    int degree[16];     /* polynomial degree per level */
    int n_quad;         /* Gauss nodes per dimension (finest level) */
    double sigma[4];    /* distribution widths per dimension */
    double cfl, epsilon;
    int max_iterations;
    int newton_mode;    /* 0 Closure::SolveClosure, 1 same with non-finite trial
                           steps rejected, 2 Closure::SolveClosureSafe */
    double gamma;       /* Euler */
    double bb_minus, bb_plus; /* bounded barrier bounds */
    double ic[8];       /* problem initial-state parameters */
    int mesh_dim;       /* 1 or 2 */
    int n_cells_1d;     /* 1-D: cells, interval [a, b] */
    double a, b;
    /* level rule: 0 the code's indicator (momentsolver.cpp:271-289), 1 the
     * paper's S_l (Paper1/adaptivity.tex:12-14); bounds (0.004, 0.02 in the
     * code, momentsolver.cpp:104-112); retardation schedule: the highest level
     * is ret_lev[k] once the residual has fallen below ret_res[0..k-1]
     * (Paper1/results.tex:179,241); n_ret_levels entries of ret_lev (0: no
     * schedule), one fewer of ret_res */
    int ref_indicator;
    double ref_down, ref_up;
    int n_ret_levels;
    double ret_res[8];
    int ret_lev[9];
} uqco_config;

typedef struct uqco uqco;

int uqco_create( const uqco_config* cfg, int n_nodes, const double* xy, const int* node_boundary, int n_tri, const int* tri, uqco** out );
void uqco_destroy( uqco* h );
void uqco_set_cell_bc( uqco* h, const int* codes );
/* out: n_cells, n_states, n_total, n_q, n_levels, dim_xi, n_faces, nT per level... */
void uqco_sizes( const uqco* h, int* out );
void uqco_tables( const uqco* h, double* phi, double* phiWf, double* xi, double* w );
void uqco_geometry( const uqco* h, double* area, double* max_edge, double* center, double* unit_n, double* scaled_n, int* nbr, int* boundary );
void uqco_init_state( uqco* h );
void uqco_get_state( const uqco* h, double* u, double* lambda, unsigned* level );
void uqco_set_state( uqco* h, const double* u, const double* lambda, const unsigned* level, double t );
/* Batched SolveClosure; status per cell: 0 ok, 1 not converged, 2 line search
 * exhausted, 3 Hessian not positive definite. iters: Newton iterations. */
int uqco_solve_closure( const uqco* h, int n, double* lambda, const double* u, const unsigned* n_total_cell, int* status, int* iters );
/* out = {t, dt, residual, failures} */
int uqco_step( uqco* h, int n_steps, double* out );
void uqco_mean_var( const uqco* h, double* out );
/* Ansatz evaluation at one node, for unit tests: u = U(Lambda), du = DU(Lambda). */
void uqco_ansatz( const uqco* h, const double* Lambda, double* u, double* du, int matrix_form );
void uqco_entropy_grad( const uqco* h, const double* u, double* ds );

#ifdef __cplusplus
}
#endif
#endif
