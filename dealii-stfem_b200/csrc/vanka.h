// Host object behind stmg_vanka_t: the cell-patch space-time Vanka
// smoother in factored form (PreconditionVanka, tests/include/gmg.h:402-540).
#pragma once

#include "stmg_internal.h"

namespace stmg
{
  // The n_t x n_t mode systems (mu Alpha + Beta) z = y of the streamed
  // apply in the eigenbasis of C = Beta^{-1} Alpha = S Lambda S^{-1} (real
  // form: 1x1 blocks for real eigenvalues, 2x2 blocks [[a, b], [-b, a]] for
  // complex pairs a +- ib): z = S (mu Lambda + I)^{-1} G y, G = S^{-1} Beta^{-1}.
  // use = 0 keeps the pivoted elimination (decomposition failed or too
  // ill-conditioned). Kernel parameter.
  struct TimeEig
  {
    int   use, nt;
    int   kind[MAX_NT]; // 1: real eigenvalue, 2: first of a complex pair, 3: second of a pair
    float a[MAX_NT], b[MAX_NT];
    float G[16], S[16]; // n_t x n_t row-major (n_t <= 4)
  };

  // Row records (the row-record apply, FP32 compute): V as rows of
  // vk_row_stride elements per mode. FP32 rows hold the mode's nd entries,
  // then its eigenvalue mu, then zeros (a whole number of 16-byte words per
  // row); BF16 rows hold the nd entries and zeros (8-byte words), and the FP32
  // mu values follow the rows.
  template <typename TS>
  constexpr int
  vk_row_stride(int nd)
  {
    return sizeof(TS) == 4 ? (nd + 1 + 3) / 4 * 4 : (nd + 3) / 4 * 4;
  }

  // Swizzled BF16 rows of the tensor-core apply: V by rows of KT entries (KT =
  // 16 or 32, the mode/dof count padded for m16n8k16 tiles), the 16-byte
  // chunks of row m permuted so that eight consecutive rows of one chunk
  // column fall in eight different shared-memory bank groups (conflict-free
  // ldmatrix); byte offset of entry (m, d) within the V block.
  template <int KT>
  struct MmaRows
  {
    static constexpr int CPR = KT / 8; // 16-byte chunks per row
    static constexpr int RB  = 8 / CPR; // rows per swizzle step
    __host__ __device__ static constexpr int
    chunk(int m, int c)
    {
      return c ^ ((m / RB) & (CPR - 1));
    }
    __host__ __device__ static constexpr int
    offset(int m, int d)
    {
      return m * KT * 2 + chunk(m, d / 8) * 16 + (d % 8) * 2;
    }
  };

  // Set by a Vanka apply kernel whose wait for a record copy gave up (mapped
  // host memory, read by Vanka::check_fault); 0 while all is well.
  int *vanka_fault_flag_device();
  // throws Error(STMG_ERR_CUDA) if a Vanka kernel flagged a failed wait
  void vanka_check_fault();

  class Vanka
  {
  public:
    // compute: STMG_F32 (storage F32 or BF16) or STMG_F64 (storage F64).
    // A, B: host nt x nt time matrices of the level (Alpha, Beta).
    Vanka(Mesh *mesh, int nt, const double *A, const double *B, int compute, int storage);

    // dst = sum_c R_c^T diag(1/valence) B_c^{-1} R_c src (dst overwritten)
    void apply(const void *src, void *dst, cudaStream_t s) const;
    // dst = alpha P src + beta dst (the relaxation update x += omega P r is
    // alpha = omega, beta = 1)
    void apply_ex(const void *src, void *dst, double alpha, double beta, cudaStream_t s) const;

    std::size_t smem_bytes(const int *shape) const;
    template <typename T>
    const TimeMats<T> &tmats() const
    {
      if constexpr (sizeof(T) == 8)
        return tm64;
      else
        return tm32;
    }
    std::size_t inverse_bytes() const { return V.n; }

    Mesh                 *mesh;
    int                   nt, compute, storage;
    Tiling                tiling;
    // per cell one record: V as [mode][dof] in the storage type, padded to
    // 16 bytes, then the eigenvalues mu in the compute type, padded to 16 bytes
    DevBuf<unsigned char> V;
    int                   rec_bytes = 0, mu_off = 0, chunk = 8;
    // streamed: FP32 compute with 1..4 time dofs; records are then stored in
    // (tile, colour, cell) order, colour_cells records per colour at most
    bool                  streamed = false;
    // rowrec: the streamed records in row form (vk_row_stride), applied by
    // the row-record kernel (time solves in the eigenbasis, nd <= 32);
    // row_stride = elements per row, mu_stride = elements between successive
    // mu values from mu_off (in the mu type)
    bool                  rowrec     = false;
    int                   row_stride = 0, mu_stride = 1;
    // mmarec: BF16 row records in the swizzled layout of MmaRows<mma_kt>,
    // applied by the tensor-core kernel (3 or 4 time dofs, nd <= 32); teig_pf
    // is teig with complex pairs first (the kernel's lane layout)
    bool                  mmarec = false;
    // slotrec: row records on tiles of 2^dim cells applied by the small-tile
    // kernel (all cells of a tile at once, per-cell output slots): meshes
    // whose colour-phase tiles would occupy fewer CTAs than there are SMs
    bool                  slotrec = false;
    // record stages of the row-record and tensor-core applies (3..5): as
    // many colour phases in flight as two CTAs per SM leave room for
    int                   stages = 3;
    int                   mma_kt = 0;
    TimeEig               teig_pf{};
    int                   colour_cells = 1;
    bool                  big = true;                // compile-time tile shape in use
    int                   shape[3] = {1, 1, 1};
    DevBuf<unsigned char> shell; // tile face slots (scratch)
    TimeMats<double>      tm64;
    TimeMats<float>       tm32;
    TimeEig               teig{};
  };

  // apply of one (dimension, degree), defined in vanka_apply_d<D>p<P>.cu
  template <int D, int P>
  void vanka_apply_dp(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s);
#define STMG_VANKA_DP(D, P)                                                                              \
  template <>                                                                                            \
  void vanka_apply_dp<D, P>(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s);
  STMG_VANKA_DP(2, 1) STMG_VANKA_DP(2, 2) STMG_VANKA_DP(2, 3) STMG_VANKA_DP(2, 4) STMG_VANKA_DP(2, 5)
  STMG_VANKA_DP(3, 1) STMG_VANKA_DP(3, 2) STMG_VANKA_DP(3, 3)
#undef STMG_VANKA_DP

  void vanka_apply_2d(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s);
  void vanka_apply_3d(const Vanka &vk, const void *src, void *dst, double alpha, double beta, cudaStream_t s);
} // namespace stmg
