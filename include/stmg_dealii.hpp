/* stmg_dealii.hpp: C++ drop-in classes over the C ABI of libstmg_cuda.so
 * (include/stmg.h) with the method names and argument meaning of the
 * reference's operator, smoother and transfer classes, so the reference's
 * FGMRES and multigrid cycle can call them where they call
 *   SystemMatrix<Number, MatrixFreeOperator<dim, Number>>
 *       (tests/include/operators.h:71-256),
 *   PreconditionVanka<Number> inside PreconditionRelaxation
 *       (tests/include/gmg.h:402-540, 660-664),
 *   STMGTransferBlockMatrixFree<dim, Number> (tests/include/gmg.h:179-315).
 * Vectors are DeviceBlockVector<Number>: n_blocks blocks of n nodes in the
 * library's lexicographic node order on the device (the stand-in for
 * LinearAlgebra::distributed::BlockVector<Number>); DofPermutation maps a
 * caller's dof numbering (e.g. a deal.II DoFHandler's) to that order and
 * back. Errors throw std::runtime_error with stmg_last_error()'s message.
 * Header-only; link libstmg_cuda.so and the CUDA runtime. */
#ifndef STMG_DEALII_HPP
#define STMG_DEALII_HPP

#include <cuda_runtime.h>

#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "stmg.h"

namespace stmg
{
  namespace shim
  {
    inline void
    check(int rc)
    {
      if (rc != STMG_OK)
        throw std::runtime_error(std::string("stmg: ") + stmg_last_error());
    }

    inline void
    check_cuda(cudaError_t e)
    {
      if (e != cudaSuccess)
        throw std::runtime_error(std::string("stmg shim: ") + cudaGetErrorString(e));
    }

    template <typename Number>
    constexpr int
    dtype_of()
    {
      static_assert(sizeof(Number) == 8 || sizeof(Number) == 4, "Number: double or float");
      return sizeof(Number) == 8 ? STMG_F64 : STMG_F32;
    }

    /* Dense row-major time matrix (the FullMatrix<double> Alpha, Beta and
     * transfer matrices of the reference). */
    struct TimeMatrix
    {
      int                 m = 0, n = 0;
      std::vector<double> a;
      TimeMatrix() = default;
      TimeMatrix(int m_, int n_)
        : m(m_)
        , n(n_)
        , a(std::size_t(m_) * n_, 0.0)
      {}
      double &operator()(int i, int j) { return a[std::size_t(i) * n + j]; }
      double  operator()(int i, int j) const { return a[std::size_t(i) * n + j]; }
    };

    /* n_blocks blocks of n nodes on the device, owned (cudaMalloc). */
    template <typename Number>
    class DeviceBlockVector
    {
    public:
      DeviceBlockVector() = default;
      DeviceBlockVector(int n_blocks, long long n) { reinit(n_blocks, n); }
      DeviceBlockVector(const DeviceBlockVector &)            = delete;
      DeviceBlockVector &operator=(const DeviceBlockVector &) = delete;
      ~DeviceBlockVector()
      {
        if (ptr_)
          cudaFree(ptr_);
      }
      void
      reinit(int n_blocks, long long n)
      {
        if (ptr_)
          cudaFree(ptr_);
        ptr_ = nullptr;
        nb_  = n_blocks;
        n_   = n;
        check_cuda(cudaMalloc(reinterpret_cast<void **>(&ptr_), bytes()));
        check_cuda(cudaMemset(ptr_, 0, bytes()));
      }
      Number       *data() { return ptr_; }
      const Number *data() const { return ptr_; }
      Number       *block(int b) { return ptr_ + std::size_t(b) * n_; }
      int           n_blocks() const { return nb_; }
      long long     block_size() const { return n_; }
      long long     size() const { return n_ * nb_; }
      std::size_t   bytes() const { return std::size_t(size()) * sizeof(Number); }
      void
      copy_from_host(const std::vector<Number> &h)
      {
        if (static_cast<long long>(h.size()) != size())
          throw std::runtime_error("stmg shim: host vector size");
        check_cuda(cudaMemcpy(ptr_, h.data(), bytes(), cudaMemcpyHostToDevice));
      }
      std::vector<Number>
      copy_to_host() const
      {
        std::vector<Number> h(static_cast<std::size_t>(size()));
        check_cuda(cudaMemcpy(h.data(), ptr_, bytes(), cudaMemcpyDeviceToHost));
        return h;
      }

    private:
      Number   *ptr_ = nullptr;
      int       nb_  = 0;
      long long n_   = 0;
    };

    /* One mesh level (stmg_mesh_t). */
    class Mesh
    {
    public:
      Mesh(int dim, const int *n_cells, int degree, const double *lo, const double *hi,
           const double *vertices = nullptr, int coeff_mode = 0, const double *coeff = nullptr)
      {
        check(stmg_mesh_create(dim, n_cells, degree, lo, hi, vertices, coeff_mode, coeff, &h_));
        check(stmg_mesh_info(h_, &n_nodes_, &n_cells_));
      }
      Mesh(const Mesh &)            = delete;
      Mesh &operator=(const Mesh &) = delete;
      ~Mesh() { stmg_mesh_destroy(h_); }
      stmg_mesh_t handle() const { return h_; }
      long long   n_nodes() const { return n_nodes_; }
      long long   n_cells() const { return n_cells_; }

    private:
      stmg_mesh_t h_       = nullptr;
      long long   n_nodes_ = 0, n_cells_ = 0;
    };

    /* SystemMatrix<Number, MatrixFreeOperator<dim, Number>>
     * (operators.h:71-256): dst_j = sum_i Alpha(j,i) K src_i + Beta(j,i) M
     * src_i. With an n_t x 1 Alpha, Beta it is the right-hand-side matrix of
     * vmult(BlockVector&, const Vector&) and vmult_add (operators.h:155-187). */
    template <typename Number>
    class SystemMatrixGPU
    {
    public:
      SystemMatrixGPU(const Mesh &mesh, const TimeMatrix &Alpha, const TimeMatrix &Beta, cudaStream_t stream = nullptr)
        : n_nodes_(mesh.n_nodes())
        , nt_out_(Alpha.m)
        , nt_in_(Alpha.n)
        , stream_(stream)
      {
        if (Beta.m != Alpha.m || Beta.n != Alpha.n)
          throw std::runtime_error("stmg shim: Alpha and Beta differ in shape");
        check(stmg_op_create(mesh.handle(), Alpha.m, Alpha.n, Alpha.a.data(), Beta.a.data(), dtype_of<Number>(), &h_));
      }
      SystemMatrixGPU(const SystemMatrixGPU &)            = delete;
      SystemMatrixGPU &operator=(const SystemMatrixGPU &) = delete;
      ~SystemMatrixGPU() { stmg_op_destroy(h_); }

      /* operators.h:94-122; with n_t x 1 time matrices the
       * vmult(BlockVector&, const Vector&) of operators.h:182-187 */
      void
      vmult(DeviceBlockVector<Number> &dst, const DeviceBlockVector<Number> &src) const
      {
        shape(dst, nt_out_);
        shape(src, nt_in_);
        check(stmg_op_vmult(h_, dst.data(), src.data(), stream_));
      }
      /* operators.h:124-152 */
      void
      Tvmult(DeviceBlockVector<Number> &dst, const DeviceBlockVector<Number> &src) const
      {
        shape(dst, nt_in_);
        shape(src, nt_out_);
        check(stmg_op_Tvmult(h_, dst.data(), src.data(), stream_));
      }
      /* operators.h:155-180: dst += op(src) */
      void
      vmult_add(DeviceBlockVector<Number> &dst, const DeviceBlockVector<Number> &src) const
      {
        shape(dst, nt_out_);
        shape(src, nt_in_);
        check(stmg_op_vmult_add(h_, dst.data(), src.data(), stream_));
      }
      void
      initialize_dof_vector(DeviceBlockVector<Number> &v) const
      {
        v.reinit(nt_out_, n_nodes_);
      }
      /* global size of the space-time system */
      std::size_t m() const { return std::size_t(nt_out_) * std::size_t(n_nodes_); }
      /* operators.h:188-215 */
      void
      get_matrix_diagonal(DeviceBlockVector<Number> &d) const
      {
        shape(d, nt_out_);
        check(stmg_op_diagonal(h_, 0, d.data(), stream_));
      }
      void
      get_matrix_diagonal_inverse(DeviceBlockVector<Number> &d) const
      {
        shape(d, nt_out_);
        check(stmg_op_diagonal(h_, 1, d.data(), stream_));
      }
      stmg_op_t    handle() const { return h_; }
      cudaStream_t stream() const { return stream_; }

    private:
      void
      shape(const DeviceBlockVector<Number> &v, int nb) const
      {
        if (v.n_blocks() != nb || v.block_size() != n_nodes_)
          throw std::runtime_error("stmg shim: vector shape does not match the operator");
      }
      stmg_op_t    h_ = nullptr;
      long long    n_nodes_;
      int          nt_out_, nt_in_;
      cudaStream_t stream_;
    };

    /* PreconditionVanka<Number> (gmg.h:402-540): the constructor sets up the
     * cell-patch inverses (gmg.h:409-474), vmult overwrites dst
     * (gmg.h:476-514); step is PreconditionRelaxation::step with the space-
     * time operator (gmg.h:660-664). storage: STMG_F32 or STMG_BF16 for
     * float, STMG_F64 for double. */
    template <typename Number>
    class VankaGPU
    {
    public:
      VankaGPU(const Mesh &mesh, const TimeMatrix &Alpha, const TimeMatrix &Beta, int storage = dtype_of<Number>(),
               cudaStream_t stream = nullptr)
        : n_nodes_(mesh.n_nodes())
        , nt_(Alpha.m)
        , stream_(stream)
      {
        check(stmg_vanka_create(mesh.handle(), Alpha.m, Alpha.a.data(), Beta.a.data(), dtype_of<Number>(), storage, &h_));
      }
      VankaGPU(const VankaGPU &)            = delete;
      VankaGPU &operator=(const VankaGPU &) = delete;
      ~VankaGPU() { clear(); }

      void
      vmult(DeviceBlockVector<Number> &dst, const DeviceBlockVector<Number> &src) const
      {
        alive();
        check(stmg_vanka_vmult(h_, dst.data(), src.data(), stream_));
      }
      /* x += omega P (b - A x); tmp receives b - A x */
      void
      step(DeviceBlockVector<Number> &x, const DeviceBlockVector<Number> &b, const SystemMatrixGPU<Number> &A,
           double omega, DeviceBlockVector<Number> &tmp) const
      {
        alive();
        check(stmg_relax_step(h_, A.handle(), omega, x.data(), b.data(), tmp.data(), stream_));
      }
      /* releases the stored inverses (PreconditionVanka::clear) */
      void
      clear()
      {
        if (h_)
          stmg_vanka_destroy(h_);
        h_ = nullptr;
      }

    private:
      void
      alive() const
      {
        if (!h_)
          throw std::runtime_error("stmg shim: Vanka used after clear()");
      }
      stmg_vanka_t h_ = nullptr;
      long long    n_nodes_;
      int          nt_;
      cudaStream_t stream_;
    };

    /* STMGTransferBlockMatrixFree<dim, Number> (gmg.h:179-315): one two-level
     * transfer per level l >= 1 between level l and level l-1 (added coarsest
     * first), h (MGTwoLevelBlockTransfer, gmg.h:35-75) or time
     * (MGTwoLevelTransferST, gmg.h:77-136). */
    template <typename Number>
    class STTransferGPU
    {
    public:
      explicit STTransferGPU(cudaStream_t stream = nullptr)
        : stream_(stream)
      {
        levels_.push_back(nullptr); // level 0 has no transfer below it
      }
      STTransferGPU(const STTransferGPU &)            = delete;
      STTransferGPU &operator=(const STTransferGPU &) = delete;
      ~STTransferGPU()
      {
        for (auto h : levels_)
          if (h)
            stmg_transfer_destroy(h);
      }
      /* next level: the 2x refinement `fine` of `coarse`, nt time blocks */
      void
      add_h_level(const Mesh &fine, const Mesh &coarse, int nt)
      {
        stmg_transfer_t h = nullptr;
        check(stmg_transfer_h_create(fine.handle(), coarse.handle(), nt, dtype_of<Number>(), &h));
        levels_.push_back(h);
      }
      /* next level: time prolongation P (fine x coarse time dofs) on `mesh` */
      void
      add_t_level(const Mesh &mesh, const TimeMatrix &P)
      {
        stmg_transfer_t h = nullptr;
        check(stmg_transfer_t_create(mesh.handle(), P.m, P.n, P.a.data(), nullptr, dtype_of<Number>(), &h));
        levels_.push_back(h);
      }
      unsigned int n_levels() const { return unsigned(levels_.size()); }
      /* gmg.h:195-201: dst (level to_level) = P src (level to_level - 1) */
      void
      prolongate(unsigned int to_level, DeviceBlockVector<Number> &dst, const DeviceBlockVector<Number> &src) const
      {
        check(stmg_transfer_prolongate(at(to_level), dst.data(), src.data(), stream_));
      }
      /* gmg.h:203-209 */
      void
      prolongate_and_add(unsigned int to_level, DeviceBlockVector<Number> &dst,
                         const DeviceBlockVector<Number> &src) const
      {
        check(stmg_transfer_prolongate_add(at(to_level), dst.data(), src.data(), stream_));
      }
      /* gmg.h:211-217: dst (level from_level - 1) += R src (level from_level) */
      void
      restrict_and_add(unsigned int from_level, DeviceBlockVector<Number> &dst,
                       const DeviceBlockVector<Number> &src) const
      {
        check(stmg_transfer_restrict_add(at(from_level), dst.data(), src.data(), stream_));
      }

    private:
      stmg_transfer_t
      at(unsigned int l) const
      {
        if (l == 0 || l >= levels_.size())
          throw std::runtime_error("stmg shim: no transfer to this level");
        return levels_[l];
      }
      std::vector<stmg_transfer_t> levels_;
      cudaStream_t                 stream_;
    };

    /* Maps a caller's dof numbering to the library's lexicographic node
     * order. cell_dofs[c * (p+1)^dim + a] is the caller's index of the dof at
     * local lexicographic position a (x fastest) of cell c (cells
     * lexicographic, x fastest), which a deal.II caller reads from
     * DoFHandler::get_dof_indices with FE_Q's hierarchic-to-lexicographic
     * renumbering. Dofs shared by cells must agree. */
    class DofPermutation
    {
    public:
      DofPermutation(int dim, const int *n_cells, int degree, const std::vector<long long> &cell_dofs)
      {
        int       nn[3] = {1, 1, 1}, nc[3] = {1, 1, 1};
        long long cells = 1;
        n_              = 1;
        for (int d = 0; d < dim; ++d)
          {
            nc[d] = n_cells[d];
            nn[d] = n_cells[d] * degree + 1;
            n_ *= nn[d];
            cells *= nc[d];
          }
        const int p1 = degree + 1, nd = dim == 2 ? p1 * p1 : p1 * p1 * p1;
        if ((long long)cell_dofs.size() != cells * nd)
          throw std::runtime_error("stmg shim: cell_dofs size");
        std::vector<long long> perm(std::size_t(n_), -1);
        for (long long c = 0; c < cells; ++c)
          {
            const int cx = int(c % nc[0]), cy = int((c / nc[0]) % nc[1]), cz = int(c / (nc[0] * (long long)nc[1]));
            for (int a = 0; a < nd; ++a)
              {
                const int       ax = a % p1, ay = (a / p1) % p1, az = a / (p1 * p1);
                const long long lex =
                  (cx * degree + ax) + nn[0] * ((long long)(cy * degree + ay) + nn[1] * (long long)(cz * degree + az));
                const long long g = cell_dofs[std::size_t(c * nd + a)];
                if (g < 0 || g >= n_ || (perm[std::size_t(lex)] >= 0 && perm[std::size_t(lex)] != g))
                  throw std::runtime_error("stmg shim: cell dofs are not a numbering of the mesh's nodes");
                perm[std::size_t(lex)] = g;
              }
          }
        check_cuda(cudaMalloc(reinterpret_cast<void **>(&perm_), perm.size() * sizeof(long long)));
        check_cuda(cudaMemcpy(perm_, perm.data(), perm.size() * sizeof(long long), cudaMemcpyHostToDevice));
      }
      DofPermutation(const DofPermutation &)            = delete;
      DofPermutation &operator=(const DofPermutation &) = delete;
      ~DofPermutation()
      {
        if (perm_)
          cudaFree(perm_);
      }
      /* caller order -> lexicographic */
      template <typename Number>
      void
      to_lexicographic(DeviceBlockVector<Number> &dst, const DeviceBlockVector<Number> &src,
                       cudaStream_t stream = nullptr) const
      {
        check(stmg_block_permute(src.n_blocks(), n_, perm_, 0, src.data(), dst.data(), dtype_of<Number>(), stream));
      }
      /* lexicographic -> caller order */
      template <typename Number>
      void
      to_caller(DeviceBlockVector<Number> &dst, const DeviceBlockVector<Number> &src, cudaStream_t stream = nullptr) const
      {
        check(stmg_block_permute(src.n_blocks(), n_, perm_, 1, src.data(), dst.data(), dtype_of<Number>(), stream));
      }
      long long size() const { return n_; }

    private:
      long long *perm_ = nullptr;
      long long  n_    = 0;
    };
  } // namespace shim
} // namespace stmg

#endif /* STMG_DEALII_HPP */
