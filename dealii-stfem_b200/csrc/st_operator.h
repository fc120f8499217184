// Host object behind stmg_op_t: the space-time operator A (x) K + B (x) M on
// one mesh level (SystemMatrix, tests/include/operators.h:71-256).
#pragma once

#include "stmg_internal.h"

namespace stmg
{
  class StOperator
  {
  public:
    StOperator(Mesh *mesh, int nt_out, int nt_in, const double *A, const double *B, int dtype);

    // dst (+)= op(src) (transpose: A^T, B^T) on stream s
    void apply(bool transpose, const void *src, void *dst, bool add, cudaStream_t s) const;
    // dst = rhs + alpha op(src) + beta dst (rhs may be null): the residual
    // b - A x is alpha = -1, beta = 0
    void apply_ex(bool transpose, const void *src, void *dst, double alpha, double beta, const void *rhs,
                  cudaStream_t s) const;

    Mesh               *mesh;
    int                 nt_out, nt_in, dtype;
    std::vector<double> A, B;
    Tiling              tiling, tilingT;
    bool                big = true, bigT = true; // compile-time tile shape in use
    bool                tiny = false, tinyT = false; // 2x2x2-cell tiles (3-D degree 2, small meshes)
    int                 shp[3] = {1, 1, 1}, shpT[3] = {1, 1, 1};

    template <typename T>
    const TimeMats<T> &tm() const
    {
      if constexpr (sizeof(T) == 8)
        return tm64;
      else
        return tm32;
    }
    template <typename T>
    const TimeMats<T> &tmT() const
    {
      if constexpr (sizeof(T) == 8)
        return tmT64;
      else
        return tmT32;
    }
    template <typename T>
    const Cart1D<T> &cart() const
    {
      if constexpr (sizeof(T) == 8)
        return cart64;
      else
        return cart32;
    }
    template <typename T>
    const QTab<T> &qtab() const
    {
      if constexpr (sizeof(T) == 8)
        return qtab64;
      else
        return qtab32;
    }
    std::size_t smem_bytes(const int *shape, int nt_in, int nt_out, std::size_t elem) const;
    // SystemMatrix::get_matrix_diagonal (inverse = false) or
    // get_matrix_diagonal_inverse (operators.h:188-215) into dst (nt blocks,
    // the operator's type); the spatial diagonals are computed on first use
    void diagonal(bool inverse, void *dst, cudaStream_t s) const;

  private:
    Tiling choose_tiling(int nt_in, int nt_out, bool &big, int *shape) const;

    TimeMats<double> tm64, tmT64;
    TimeMats<float>  tm32, tmT32;
    Cart1D<double>   cart64;
    Cart1D<float>    cart32;
    QTab<double>     qtab64;
    QTab<float>      qtab32;
    DevBuf<unsigned char> shell; // tile face slots (scratch, allocated at creation)
    mutable DevBuf<double> diag_K, diag_M; // spatial diagonals (first diagonal() call)
  };

  // diagonals of K and M of a mesh (constrained rows 1), FP64, by probing
  void spatial_diagonals(Mesh *mesh, double *dK, double *dM, cudaStream_t s);

  // dst = (A (x) K + B (x) M) src on the uniform box [lo, hi] with n_cells
  // cells, allocating no device memory (face slots in a fixed device array
  // of st_operator.cu). coeff: per-cell coefficient in dtype, or null.
  void op_vmult_box_noalloc(int dim, const int *n_cells, int degree, const double *lo, const double *hi,
                            const void *coeff, int nt_out, int nt_in, const double *A, const double *B, int dtype,
                            const void *src, void *dst, cudaStream_t s);
} // namespace stmg
