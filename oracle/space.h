// Oracle (test infrastructure only): CPU restatement of the reference's
// spatial pieces on a structured hex mesh:
//  - MatrixFreeOperator (tests/include/operators.h:355-562): mass / Laplace on
//    FE_Q(p) with Gauss-Lobatto support points and QGauss(p+1), MappingQ1,
//    optional coefficient at quadrature points, homogeneous Dirichlet;
//  - SystemMatrix (operators.h:71-256): sum over time blocks;
//  - PreconditionVanka (tests/include/gmg.h:402-540): cell patches of the
//    assembled matrices, Gauss-Jordan inverses, valence-weighted scatter;
//  - the h-transfer of deal.II's MGTwoLevelTransfer as used at gmg.h:35-75.
// Only tests/, the bench's CPU-baseline leg and the smoke check use it.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "time_fe.h"

namespace oracle
{
  // Structured mesh of n[0] x n[1] (x n[2]) cells; nodes of FE_Q(p) numbered
  // lexicographically with x fastest. Vertices follow the same order.
  struct Mesh
  {
    int dim = 2;
    int n[3] = {1, 1, 1};
    int p    = 1;
    // vertex coordinates, (n0+1)(n1+1)(n2+1) x dim; filled for all meshes
    std::vector<double> vert;
    // coefficient: 0 = none (constant 1), 1 = per cell, 2 = per quadrature point
    int                 coeff_mode = 0;
    std::vector<double> coeff;

    // derived
    int                 nn[3] = {1, 1, 1}; // nodes per direction
    std::size_t         n_nodes = 0, n_cells = 0;
    int                 nd = 0, nq = 0; // dofs and q-points per cell
    std::vector<double> xs;             // 1-D support points (Lobatto, p+1)
    std::vector<double> gx, gw;         // 1-D Gauss points/weights (p+1)

    void init(int dim, const int *n, int p, const double *lo, const double *hi);
    void set_vertices(const double *v); // overrides the uniform box
    void cell_nodes(std::size_t c, std::vector<std::size_t> &idx) const;
    bool is_boundary(std::size_t node) const;
    // position of a node (Q1 map of its cell at the support point)
    void node_position(std::size_t node, double *x) const;
    // Jacobian of the Q1 map of cell c at reference point xi
    void jacobian(std::size_t c, const double *xi, double J[3][3]) const;
    void map_point(std::size_t c, const double *xi, double *x) const;
    double coeff_at(std::size_t c, int q) const;
  };

  // Element matrices (mass, stiffness with coefficient) of cell c, nd x nd.
  void element_matrices(const Mesh &m, std::size_t c, std::vector<double> &Ke,
                        std::vector<double> &Me);

  // Matrix-free apply of the scalar mass (which=0) or Laplace (which=1)
  // operator: dst = A src with constrained rows/columns removed.
  template <typename Number>
  void mf_apply(const Mesh &m, int which, Number *dst, const Number *src);

  // Space-time operator dst_j = sum_i T(j,i) K src_i + S(j,i) M src_i with
  // (T,S) = (Alpha, Beta), transposed time matrices if transpose=true
  // (SystemMatrix::vmult / Tvmult, operators.h:94-152).
  template <typename Number>
  void st_apply(const Mesh &m, const DMat &Alpha, const DMat &Beta, bool transpose, Number *dst,
                const Number *src);
  // n x 1 form (operators.h:155-187): dst_j (+)= a_j K v + b_j M v.
  template <typename Number>
  void st_apply_vec(const Mesh &m, const DMat &a, const DMat &b, bool add, Number *dst,
                    const Number *src);

  // Assembled sparse matrix (CSR) with deal.II's treatment of constrained
  // rows: off-diagonals dropped, diagonal = sum over cells of |local diag|.
  struct CSR
  {
    std::size_t              n = 0;
    std::vector<std::size_t> rowptr, col;
    std::vector<double>      val;
    double                   operator()(std::size_t i, std::size_t j) const;
  };
  void assemble(const Mesh &m, CSR &K, CSR &M);

  // Cell-patch Vanka (gmg.h:409-514) with inverses kept in Number.
  template <typename Number>
  struct Vanka
  {
    const Mesh                            *mesh = nullptr;
    int                                    nt   = 0;
    std::vector<std::vector<std::size_t>>  idx;
    std::vector<Number>                    valence;
    std::vector<std::vector<Number>>       blocks; // inverses, L x L row-major
    Number                                 damp = 1;
    void setup(const Mesh &m, const CSR &K, const CSR &M, const DMat &Alpha, const DMat &Beta);
    void vmult(Number *dst, const Number *src) const; // dst overwritten
  };

  // Gauss-Jordan inversion in working precision T (FullMatrix::gauss_jordan).
  template <typename T>
  void gauss_jordan(std::vector<T> &A, int n);

  // h-transfer between nested structured meshes (same p): fine = P coarse,
  // restriction = P^T; constrained dofs are zero on both sides.
  template <typename Number>
  void h_prolongate_add(const Mesh &fine, const Mesh &coarse, int nt, Number *dst,
                        const Number *src);
  template <typename Number>
  void h_restrict_add(const Mesh &fine, const Mesh &coarse, int nt, Number *dst,
                      const Number *src);

  // (A (x) I) on block vectors (tensorproduct_add, operators.h:46-58).
  template <typename Number>
  void tensorproduct_add(std::size_t N, const DMat &A, Number *dst, const Number *src);
} // namespace oracle
