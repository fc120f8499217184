/* stmg: B200-native (sm_100a) space-time multigrid slab solve.
 *
 * C ABI of libstmg_cuda.so. Every call returns an int status (0 = OK,
 * negative = error, see STMG_ERR_*); stmg_last_error() gives the message of
 * the calling thread's last failure. Vectors are device pointers to
 * contiguous block vectors [n_t][N]: block (time dof) major, nodes of the
 * structured FE_Q(p) mesh in lexicographic order (x fastest) including the
 * Dirichlet boundary nodes, which are held at zero. Streams are
 * cudaStream_t passed as void*. Hot calls never allocate device memory;
 * handles are not re-entrant (one stream per handle at a time).
 *
 * Each entry point names the reference interface it replaces
 * (nlsmrg/dealii-stfem, file:line).
 */
#ifndef STMG_H
#define STMG_H

#if defined(__GNUC__)
#define STMG_API __attribute__((visibility("default")))
#else
#define STMG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct stmg_mesh_s     *stmg_mesh_t;
typedef struct stmg_op_s       *stmg_op_t;
typedef struct stmg_vanka_s    *stmg_vanka_t;
typedef struct stmg_transfer_s *stmg_transfer_t;
typedef struct stmg_solver_s   *stmg_solver_t;

enum
{
  STMG_OK              = 0,
  STMG_ERR_ARG         = -1, /* invalid argument */
  STMG_ERR_HANDLE      = -2, /* null or destroyed handle */
  STMG_ERR_SHAPE       = -3, /* inconsistent sizes */
  STMG_ERR_CUDA        = -4, /* CUDA runtime error */
  STMG_ERR_NONFINITE   = -5, /* NaN/Inf residual */
  STMG_ERR_NOCONV      = -6, /* iteration limit reached */
  STMG_ERR_NOMEM       = -7, /* device allocation failed */
  STMG_ERR_UNSUPPORTED = -8  /* configuration not built */
};

enum
{
  STMG_F64  = 0,
  STMG_F32  = 1,
  STMG_BF16 = 2
};

STMG_API const char *stmg_last_error(void);
STMG_API int         stmg_version(void);
/* Number of CUDA kernels the library has launched since it was loaded.
 * Diagnostic counter with no counterpart in the reference. */
STMG_API int stmg_kernel_launches(long long *count);

/* ---------------------------------------------------------- time algebra
 * Time weights of one slab of n_steps steps of size tau for time degree r
 * (time_type 1 = cGP, 2 = dG): get_fe_time_weights (fe_time.h:292-349) for
 * the heat system (problem 1: Alpha, Beta and the right-hand-side columns
 * rK, rM of tests/tp_01.cc:186-189) or the condensed wave system
 * (problem 2: get_fe_time_weights_wave, fe_time.h:98-246, with rV). Host
 * arrays: Alpha, Beta nt x nt, rK, rM, rV nt; nt = (r+1) n_steps (dG) or
 * r n_steps (cGP). rV may be NULL for heat. */
STMG_API int stmg_time_weights(int time_type, int r, double tau, int n_steps, int problem, double *Alpha,
                               double *Beta, double *rK, double *rM, double *rV);

/* Time transfer matrix of one slab (rows = fine time dofs, row-major):
 * kind 0, the k-projection from degree r-1 to r on n_steps steps
 * (get_time_projection_matrix, fe_time.h:567-623; (r n_steps) x
 * ((r-1) n_steps) for cGP, ((r+1) n_steps) x (r n_steps) for dG);
 * kind 1, the tau-prolongation from n_steps/2 to n_steps steps of degree r
 * (get_time_prolongation_matrix, fe_time.h:625-669; n_steps even). The
 * restriction is the transpose (gmg.h:77-136 with restrict_is_transpose). */
STMG_API int stmg_time_transfer(int time_type, int kind, int r, int n_steps, double *P);

/* Reorders block vectors between a caller's dof numbering and the library's
 * lexicographic node order, per time block: dst[b][i] = src[b][perm[i]]
 * (scatter = 0, caller order -> lexicographic when perm[i] is the caller's
 * index of lexicographic node i) or dst[b][perm[i]] = src[b][i] (scatter =
 * 1, back). perm: device array of n indices; src, dst: device, n_blocks x n,
 * distinct. The adapter a deal.II caller needs around every call (its
 * DoFHandler numbers the dofs of a BlockVector block, tests/tp_01.cc:260-285);
 * no counterpart in the reference. */
STMG_API int stmg_block_permute(int n_blocks, long long n, const long long *perm, int scatter, const void *src,
                                void *dst, int dtype, void *stream);

/* ---------------------------------------------------------------- mesh
 * Structured hex mesh of n_cells[0] x n_cells[1] (x n_cells[2]) cells of
 * FE_Q(degree) on Gauss-Lobatto nodes with MappingQ1 and homogeneous
 * Dirichlet conditions; replaces the DoFHandler/MatrixFree setup of
 * tests/tp_01.cc:80-100,260-285 and the coefficient tables of
 * tests/include/operators.h:435-462.
 * vertices: host array (n0+1)(n1+1)(n2+1) x dim or NULL for the box lo..hi.
 * coeff_mode 0: coefficient 1; 1: per cell (n_cells values); 2: per
 * quadrature point of QGauss(degree+1) (n_cells x (degree+1)^dim). */
STMG_API int stmg_mesh_create(int dim, const int *n_cells, int degree, const double *lo, const double *hi,
                     const double *vertices, int coeff_mode, const double *coeff, stmg_mesh_t *mesh);
STMG_API int stmg_mesh_destroy(stmg_mesh_t mesh);
STMG_API int stmg_mesh_info(stmg_mesh_t mesh, long long *n_nodes, long long *n_cells);

/* ------------------------------------------------------ space-time operator
 * dst_j = sum_i A(j,i) K src_i + B(j,i) M src_i with the Laplace matrix K
 * (coefficient at quadrature points) and mass matrix M of the mesh.
 * A, B: host, nt_out x nt_in row-major. dtype STMG_F64 or STMG_F32.
 * Replaces SystemMatrix<Number, MatrixFreeOperator> (operators.h:71-256). */
STMG_API int stmg_op_create(stmg_mesh_t mesh, int nt_out, int nt_in, const double *A, const double *B, int dtype,
                   stmg_op_t *op);
STMG_API int stmg_op_destroy(stmg_op_t op);
/* SystemMatrix::vmult (operators.h:94-122); with nt_in = 1 also
 * vmult(BlockVector&, const Vector&) (operators.h:182-187). */
STMG_API int stmg_op_vmult(stmg_op_t op, void *dst, const void *src, void *stream);
/* dst = (A (x) K + B (x) M) src on the uniform box [lo, hi] split into
 * n_cells cells, computed like stmg_op_create + stmg_op_vmult on that mesh
 * but with no handle and no device memory allocated by the call. It is for
 * callers that cannot call cudaMalloc: a host application that owns the
 * GPU's memory through its own pool or a fixed budget, or a solver loop that
 * must not stall other streams on cudaMalloc's device-wide synchronisation.
 * coeff: per-cell coefficient on the device in dtype (float for STMG_F32,
 * double for STMG_F64), or NULL for 1. dst, src: device, nt x n_nodes.
 * The tiles' face slots go to one fixed 16 MiB array in the library's device
 * code, held on every GPU that loads the library until the process exits;
 * a mesh that needs more (tiles x nt_out x face slots per tile x element
 * size) returns STMG_ERR_SHAPE: in 3-D with Q2 and four time blocks, meshes
 * up to about 40^3 cells fit in FP64 and about 52^3 in FP32. The first call
 * on each device looks up that array's device address on the current
 * device and keeps it for the life of the process, so make it before any
 * stream capture, and do not use this entry point on a device after
 * cudaDeviceReset (the library's device image is then loaded again at
 * another address). All calls share the array: calls that run at the same
 * time on one GPU race. No counterpart in the reference. */
STMG_API int stmg_op_vmult_box_noalloc(int dim, const int *n_cells, int degree, const double *lo, const double *hi,
                                       const void *coeff, int nt_out, int nt_in, const double *A, const double *B,
                                       int dtype, void *dst, const void *src, void *stream);
/* SystemMatrix::get_matrix_diagonal (inverse = 0) or
 * get_matrix_diagonal_inverse (inverse = 1), operators.h:188-215: block i
 * of dst (n_t x n_nodes, the operator's dtype) is A(i,i) diag(K) +
 * B(i,i) diag(M), or diag(K)^+ / A(i,i) + diag(M)^+ / B(i,i) with x^+ = 1/x
 * where |x| > sqrt(eps) and 1 elsewhere (MatrixFreeOperator::
 * compute_diagonal, operators.h:467-485). Dirichlet rows of diag(K) and
 * diag(M) are 1. Square operators only. */
STMG_API int stmg_op_diagonal(stmg_op_t op, int inverse, void *dst, void *stream);
/* SystemMatrix::Tvmult (operators.h:124-152): A and B transposed. */
STMG_API int stmg_op_Tvmult(stmg_op_t op, void *dst, const void *src, void *stream);
/* SystemMatrix::vmult_add (operators.h:155-180): dst += op(src). */
STMG_API int stmg_op_vmult_add(stmg_op_t op, void *dst, const void *src, void *stream);

/* ---------------------------------------------------------------- Vanka
 * Cell-patch space-time Vanka smoother of one level: per cell the inverse of
 * Alpha (x) K_c + Beta (x) M_c with K_c, M_c the assembled matrices restricted
 * to the cell's dofs, applied in factored form (generalised eigenvectors of
 * (K_c, M_c) and per-mode n_t x n_t solves), contributions weighted by
 * 1/valence. compute STMG_F32 with storage STMG_F32 or STMG_BF16, or
 * STMG_F64 with STMG_F64. Replaces PreconditionVanka's constructor
 * (gmg.h:409-474). */
STMG_API int stmg_vanka_create(stmg_mesh_t mesh, int nt, const double *Alpha, const double *Beta, int compute_dtype,
                               int storage_dtype, stmg_vanka_t *vanka);
STMG_API int stmg_vanka_destroy(stmg_vanka_t vanka);
/* PreconditionVanka::vmult (gmg.h:476-514): dst = sum_c R_c^T D_c B_c^{-1} R_c src. */
STMG_API int stmg_vanka_vmult(stmg_vanka_t vanka, void *dst, const void *src, void *stream);

/* PreconditionRelaxation<SystemMatrix, PreconditionVanka>::step, the
 * smoother sweep of MGSmootherPrecondition (gmg.h:660-664,714-730):
 * x += omega P_vanka (b - A x); tmp (same shape) receives b - A x. The
 * operator and the smoother must be of one mesh, n_t and compute type. */
STMG_API int stmg_relax_step(stmg_vanka_t vanka, stmg_op_t op, double omega, void *x, const void *b, void *tmp,
                             void *stream);

/* ------------------------------------------------------------ transfers
 * h: between a mesh and its 2x refinement (same degree), nt time blocks;
 * replaces MGTwoLevelBlockTransfer over deal.II's MGTwoLevelTransfer
 * (gmg.h:35-75, built at gmg.h:369-380).
 * t: (P (x) I) on one mesh, P nt_fine x nt_coarse, R nt_coarse x nt_fine or
 * NULL for P^T; replaces MGTwoLevelTransferST (gmg.h:77-136). */
STMG_API int stmg_transfer_h_create(stmg_mesh_t fine, stmg_mesh_t coarse, int nt, int dtype, stmg_transfer_t *tr);
STMG_API int stmg_transfer_t_create(stmg_mesh_t mesh, int nt_fine, int nt_coarse, const double *P, const double *R,
                                    int dtype, stmg_transfer_t *tr);
STMG_API int stmg_transfer_destroy(stmg_transfer_t tr);
/* STMGTransferBlockMatrixFree::prolongate (gmg.h:195-201): dst = P src. */
STMG_API int stmg_transfer_prolongate(stmg_transfer_t tr, void *dst, const void *src, void *stream);
/* ::prolongate_and_add (gmg.h:203-209): dst += P src. */
STMG_API int stmg_transfer_prolongate_add(stmg_transfer_t tr, void *dst, const void *src, void *stream);
/* ::restrict_and_add (gmg.h:211-217): dst += R src. */
STMG_API int stmg_transfer_restrict_add(stmg_transfer_t tr, void *dst, const void *src, void *stream);

/* --------------------------------------------------------------- solver
 * Slab solver of the heat (problem 1) or condensed wave (problem 2) system:
 * FP64 FGMRES preconditioned by the space-time V-cycle (FP32 or FP64) on
 * the structured mesh of subdiv cells refined `refine` times (levels as
 * tests/tp_01.cc:200-359 builds them). time_type 1 = cGP, 2 = dG. */
typedef struct
{
  int           dim, subdiv[3], refine, degree, time_degree, time_type, problem, n_steps;
  double        tau, lo[3], hi[3];
  int           smoothing_steps, fe_degree_min, n_steps_min; /* -1: reference defaults */
  int           mg_dtype, vanka_storage;                      /* STMG_F32/F64; STMG_F32/BF16/F64 */
  double        tol, abs_tol;                                 /* ReductionControl reduce, tolerance */
  int           max_iter, restart, extrapolate;
  int           rhs_mode; /* 0 manufactured (frequency), 1 nodal source f_nodal, 2 none */
  double        frequency;
  const double *fine_vertices; /* NULL or finest-mesh vertices */
  const double *fine_coeff;    /* NULL or per finest cell */
  const double *f_nodal;       /* rhs_mode 1: finest nodal values */
} stmg_solver_config;

STMG_API int stmg_solver_create(const stmg_solver_config *cfg, stmg_solver_t *solver);
STMG_API int stmg_solver_destroy(stmg_solver_t solver);
/* sizes; omegas (n_levels values, may be NULL) are the relaxation factors of
 * GMG::estimate_relaxation (gmg.h:792-844) */
STMG_API int stmg_solver_info(stmg_solver_t solver, long long *n_nodes, int *n_blocks, int *n_levels, double *omegas);
/* initial u, v on the finest nodes (host arrays of n_nodes, NULL = the
 * manufactured solution at t = 0); resets time to 0 */
STMG_API int stmg_solver_set_initial(stmg_solver_t solver, const double *u0, const double *v0);
/* replace the nodal source field (host array of n_nodes; rhs_mode 1): the
 * integrate_rhs_function of tests/tp_01.cc:390-398 for an FE source */
STMG_API int stmg_solver_set_source(stmg_solver_t solver, const double *f_nodal);
/* Point functionals of the last slab run (tests/tp_01.cc:451-619): the
 * displacement / temperature u at n_points points (host, n_points x dim,
 * inside the mesh) for every time node of each step (RemotePointEvaluation
 * with FEPointEvaluation under the Q1 map), mapped by the time evaluation
 * matrix (get_time_evaluation_matrix, fe_time.h:250-267) to samples_per_step
 * equidistant times per step (<= 0: (r+1)^2 as the reference); cGP steps
 * take the step's initial value as their first node. values (host):
 * (n_steps samples) x n_points, row-major; times (host, may be NULL):
 * n_steps samples. */
STMG_API int stmg_solver_point_values(stmg_solver_t solver, int n_points, const double *points, int samples_per_step,
                                      double *times, double *values, void *stream);
/* the FGMRES ReductionControl of the following slabs (time_integrators.h:44:
 * max_iter, abs_tol, tol as a reduction of the initial residual), as a
 * caller changes a deal.II SolverControl between solves */
STMG_API int stmg_solver_set_control(stmg_solver_t solver, double tol, double abs_tol, int max_iter);
/* the slab loop of tests/tp_01.cc:630-683 with TimeIntegratorHeat::solve /
 * TimeIntegratorWave::solve (time_integrators.h:157-180,237-280);
 * iterations: host array of n_slabs FGMRES counts (may be NULL) */
STMG_API int stmg_solver_run(stmg_solver_t solver, int n_slabs, int *iterations, void *stream);
/* copy the last slab's u (and v) blocks to host arrays of n_blocks x n_nodes */
STMG_API int stmg_solver_solution(stmg_solver_t solver, double *u, double *v);
/* the same copy without a host wait (the caller's solution vector read back
 * between slabs, time_integrators.h:174-180 and tests/tp_01.cc:630-683): the
 * blocks are copied on `stream` into device staging buffers and from there to
 * the host arrays on the library's own non-blocking stream, so the transfer
 * overlaps the next slabs (stmg_solver_run waits only for the device copy).
 * The host arrays hold the values once stmg_solver_solution_wait returns;
 * pinned host memory makes the copy asynchronous. */
STMG_API int stmg_solver_solution_async(stmg_solver_t solver, double *u, double *v, void *stream);
STMG_API int stmg_solver_solution_wait(stmg_solver_t solver);
/* SolverFGMRES::solve of the slab system (time_integrators.h:174) on device
 * vectors x (initial guess in, solution out) and rhs */
STMG_API int stmg_solver_solve(stmg_solver_t solver, double *x, const double *rhs, int *iterations, void *stream);
/* Error norms of the slabs run since the last set_initial against the
 * manufactured solution (rhs_mode 0; ErrorCalculator, exact_solution.h:
 * 217-299): L-infinity over the time and space quadrature points, L2(0,T;L2)
 * and L2(0,T;H1-seminorm), QGauss(r+1) in space and time. */
STMG_API int stmg_solver_errors(stmg_solver_t solver, double *linf, double *l2, double *h1);
/* Adjoint gradient (heat): runs n_slabs slabs from the current state and
 * returns the space-time misfit J = 1/2 sum_s |U_s - O_s|^2 over all slab
 * time dofs and nodes (u_obs: host, n_slabs x n_t x N, slab-major) and dJ/d
 * log(kappa_c) for every fine cell (grad: host, n_cells doubles; the solver's
 * fine coefficient is kappa). The adjoint slab equations A^T lambda_s =
 * U_s - O_s + E^T R^T lambda_{s+1} run backward over the slabs through a
 * multigrid built on the transposed time matrices (SystemMatrix::Tvmult,
 * operators.h:124-152); forward states are kept every checkpoint_every slabs
 * (<= 0: ceil(sqrt(n_slabs))) and recomputed per segment. its_fwd, its_adj
 * (host, n_slabs each, may be NULL) receive the FGMRES iterations. The
 * solver's state afterwards is the state after the last slab. */
STMG_API int stmg_solver_gradient(stmg_solver_t solver, int n_slabs, const double *u_obs, int checkpoint_every,
                                  double *misfit, double *grad, int *its_fwd, int *its_adj, void *stream);
/* GMG::vmult (gmg.h:846-859) on FP64 device vectors */
STMG_API int stmg_gmg_vmult(stmg_solver_t solver, double *dst, const double *src, void *stream);
/* the FP64 slab system SystemMatrix::vmult (operators.h:94-122) */
STMG_API int stmg_solver_system_vmult(stmg_solver_t solver, double *dst, const double *src, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* STMG_H */
