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
/* SystemMatrix::Tvmult (operators.h:124-152): A and B transposed. */
STMG_API int stmg_op_Tvmult(stmg_op_t op, void *dst, const void *src, void *stream);
/* SystemMatrix::vmult_add (operators.h:155-180): dst += op(src). */
STMG_API int stmg_op_vmult_add(stmg_op_t op, void *dst, const void *src, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* STMG_H */
