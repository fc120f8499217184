// Fused space-time operator dst_j = sum_i A(j,i) K src_i + B(j,i) M src_i
// (the reference's SystemMatrix over two MatrixFreeOperator objects,
// tests/include/operators.h:71-256 and 355-562), one pass over the cells for
// all time blocks at once: host side (tiling, time matrices, dispatch). The
// kernels live in op_apply_impl.cuh: per tile of cells the input brick is
// staged in shared memory, one thread per (output time dof, cell) mixes the
// time blocks and applies K and M by sum factorisation, and one thread per
// (time dof, brick node) sums the node's cells in a fixed order; nodes the
// tiles share go through per-tile face slots summed by the fix-up kernel.
// The result is deterministic (no atomics).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include <cstdlib>

#include "op_apply_impl.cuh"
#include "st_operator.h"

namespace stmg
{
  namespace
  {
    template <typename T>
    void
    launch(const StOperator &op, bool transpose, const T *src, T *dst, T *shell, const OutMode<T> &om, cudaStream_t s)
    {
      OpLaunch<T> L{op.mesh->v, transpose ? op.tilingT : op.tiling, transpose ? op.tmT<T>() : op.tm<T>(),
                    op.cart<T>(), op.qtab<T>(), src, dst, shell, om, transpose ? op.bigT : op.big, s,
                    transpose ? op.tinyT : op.tiny};
      const int dim = op.mesh->v.dim, p = op.mesh->v.p;
#define STMG_CASE(D, PP)                                                                                 \
  if (dim == D && p == PP)                                                                               \
    return op_launch_dp<D, PP, T>(L);
      STMG_CASE(2, 1) STMG_CASE(2, 2) STMG_CASE(2, 3) STMG_CASE(2, 4) STMG_CASE(2, 5)
      STMG_CASE(3, 1) STMG_CASE(3, 2) STMG_CASE(3, 3) STMG_CASE(3, 4)
#undef STMG_CASE
      throw Error(STMG_ERR_UNSUPPORTED, "operator: unsupported dim/degree");
    }

    template <typename T>
    void
    fill_mats(TimeMats<T> &tm, int nt_out, int nt_in, const std::vector<double> &A, const std::vector<double> &B,
              bool transpose)
    {
      std::memset(&tm, 0, sizeof(tm));
      tm.nt_out = transpose ? nt_in : nt_out;
      tm.nt_in  = transpose ? nt_out : nt_in;
      for (int j = 0; j < nt_out; ++j)
        for (int i = 0; i < nt_in; ++i)
          {
            const int k = transpose ? i * nt_out + j : j * nt_in + i;
            tm.A[k]     = T(A[j * nt_in + i]);
            tm.B[k]     = T(B[j * nt_in + i]);
          }
    }

    template <typename T>
    Cart1D<T>
    make_cart(const MeshView &m)
    {
      Cart1D<T>       c{};
      const FETables &t = host_tables();
      const int       n = m.p + 1;
      for (int d = 0; d < 3; ++d)
        for (int a = 0; a < n; ++a)
          for (int b = 0; b < n; ++b)
            {
              c.M[d][a * n + b] = T(t.M1[m.p][a][b] * m.h[d]);
              c.K[d][a * n + b] = T(t.K1[m.p][a][b] / m.h[d]);
            }
      return c;
    }
  } // namespace

  namespace
  {
    template <typename T>
    void
    shape_of(int dim, int p, bool big, int *T3)
    {
#define STMG_SH(D, PP)                                                                                   \
  if (dim == D && p == PP)                                                                               \
    {                                                                                                    \
      if (big)                                                                                           \
        T3[0] = op_detail::OpShape<D, PP, T, true>::TX, T3[1] = op_detail::OpShape<D, PP, T, true>::TY, T3[2] = op_detail::OpShape<D, PP, T, true>::TZ; \
      else                                                                                               \
        T3[0] = op_detail::OpShape<D, PP, T, false>::TX, T3[1] = op_detail::OpShape<D, PP, T, false>::TY, T3[2] = op_detail::OpShape<D, PP, T, false>::TZ; \
      return;                                                                                            \
    }
      STMG_SH(2, 1) STMG_SH(2, 2) STMG_SH(2, 3) STMG_SH(2, 4) STMG_SH(2, 5)
      STMG_SH(3, 1) STMG_SH(3, 2) STMG_SH(3, 3) STMG_SH(3, 4)
#undef STMG_SH
      throw Error(STMG_ERR_UNSUPPORTED, "operator: unsupported dim/degree");
    }

    // a small tile is worth taking over a partly filled GPU of big tiles
    // only while it holds four cells or more
    bool
    small_shape_worthwhile(int dim, const int *T3)
    {
      return T3[0] * T3[1] * (dim == 3 ? T3[2] : 1) >= 4;
    }
  } // namespace

  std::size_t
  StOperator::smem_bytes(const int *shape, int nt_in_, int nt_out_, std::size_t elem) const
  {
    return op_smem_bytes(mesh->v.dim, mesh->v.p, shape, nt_in_, nt_out_, elem);
  }

  // Tile shape of an operator apply on mesh m with elements of elem bytes:
  // the big shape unless it does not fit in shared memory, or it yields
  // fewer than two tiles per SM (in 3-D: than half a tile per SM) while the
  // small shape still gives each CTA several cells (a one-cell tile keeps
  // only nt_out threads of a CTA busy in phase B, far slower than a partly
  // filled GPU of big tiles). Used by StOperator and by the allocation-free
  // box apply, so both pick the same.
  Tiling
  choose_op_tiling(const MeshView &m, std::size_t elem, int nt_in_, int nt_out_, bool &big_out, int *shape)
  {
    const std::size_t budget = 200 * 1024;
    auto              shp    = [&](bool big, int *T3) {
      if (elem == 8)
        shape_of<double>(m.dim, m.p, big, T3);
      else
        shape_of<float>(m.dim, m.p, big, T3);
    };
    for (bool big : {true, false})
      {
        int T3[3];
        shp(big, T3);
        if (op_smem_bytes(m.dim, m.p, T3, nt_in_, nt_out_, elem) <= budget)
          {
            // 3-D: the big shape down to half a tile per SM (32^3 Q2: 128 big
            // tiles in one round, 37 us, against 1,024 small ones in 3.5
            // rounds, 57 us; at 16^3, 16 big tiles lose to 128 small ones)
            const long long few = m.dim == 3 ? sm_count() / 2 : 2ll * sm_count();
            if (big && make_tiling(m, T3).n_tiles < few)
              {
                int t3[3];
                shp(false, t3);
                if (small_shape_worthwhile(m.dim, t3) && op_smem_bytes(m.dim, m.p, t3, nt_in_, nt_out_, elem) <= budget)
                  continue;
              }
            big_out = big;
            for (int d = 0; d < 3; ++d)
              shape[d] = T3[d];
            return make_tiling(m, T3);
          }
      }
    throw Error(STMG_ERR_UNSUPPORTED, "operator: time blocks do not fit in shared memory");
  }

  Tiling
  StOperator::choose_tiling(int nt_in_, int nt_out_, bool &big_out, int *shape) const
  {
    return choose_op_tiling(mesh->v, dtype == STMG_F64 ? 8 : 4, nt_in_, nt_out_, big_out, shape);
  }

  StOperator::StOperator(Mesh *mesh_, int nt_out_, int nt_in_, const double *A_, const double *B_, int dtype_)
    : mesh(mesh_)
    , nt_out(nt_out_)
    , nt_in(nt_in_)
    , dtype(dtype_)
  {
    STMG_REQUIRE(nt_out >= 1 && nt_out <= MAX_NT && nt_in >= 1 && nt_in <= MAX_NT, STMG_ERR_ARG,
                 "operator: time dimensions must be 1..16");
    STMG_REQUIRE(dtype == STMG_F64 || dtype == STMG_F32, STMG_ERR_ARG, "operator: dtype must be F64 or F32");
    A.assign(A_, A_ + nt_out * nt_in);
    B.assign(B_, B_ + nt_out * nt_in);
    fill_mats(tm64, nt_out, nt_in, A, B, false);
    fill_mats(tm32, nt_out, nt_in, A, B, false);
    fill_mats(tmT64, nt_out, nt_in, A, B, true);
    fill_mats(tmT32, nt_out, nt_in, A, B, true);
    cart64 = make_cart<double>(mesh->v);
    cart32 = make_cart<float>(mesh->v);
    qtab64 = make_qtab<double>(mesh->v.p);
    qtab32 = make_qtab<float>(mesh->v.p);
    tiling  = choose_tiling(nt_in, nt_out, big, shp);
    tilingT = choose_tiling(nt_out, nt_in, bigT, shpT);
    {
      // 3-D degree 2 on meshes of at most one 2x2x2-cell tile per SM (a
      // tile of the regular shapes is a long serial chain there): tiles of
      // 2x2x2 cells, phase B by planes (STMG_OP_TINY=0 / 1 turns it off / on
      // for every 3-D degree-2 mesh)
      const char *e   = std::getenv("STMG_OP_TINY");
      const bool  can = mesh->v.dim == 3 && mesh->v.p == 2;
      const int   t2[3] = {2, 2, 2};
      const bool  few   = can && make_tiling(mesh->v, t2).n_tiles <= sm_count();
      auto        pick  = [&](Tiling &t, int *sh, bool &ti) {
        ti = can && (e ? e[0] == '1' : few);
        if (ti)
          {
            sh[0] = sh[1] = sh[2] = 2;
            t                     = make_tiling(mesh->v, sh);
          }
      };
      pick(tiling, shp, tiny);
      pick(tilingT, shpT, tinyT);
    }
    const std::size_t elem = dtype == STMG_F64 ? 8 : 4;
    const std::size_t n1   = std::size_t(tiling.n_tiles) * nt_out * tiling.tile_stride;
    const std::size_t n2   = std::size_t(tilingT.n_tiles) * nt_in * tilingT.tile_stride;
    shell.alloc(std::max(n1, n2) * elem);
  }

  void
  StOperator::apply(bool transpose, const void *src, void *dst, bool add, cudaStream_t s) const
  {
    apply_ex(transpose, src, dst, 1.0, add ? 1.0 : 0.0, nullptr, s);
  }

  void
  StOperator::apply_ex(bool transpose, const void *src, void *dst, double alpha, double beta, const void *rhs,
                       cudaStream_t s) const
  {
    STMG_REQUIRE(src && dst, STMG_ERR_ARG, "operator: null vector");
    if (dtype == STMG_F64)
      {
        const OutMode<double> om{alpha, beta, static_cast<const double *>(rhs)};
        launch<double>(*this, transpose, static_cast<const double *>(src), static_cast<double *>(dst),
                       reinterpret_cast<double *>(shell.ptr), om, s);
      }
    else
      {
        const OutMode<float> om{float(alpha), float(beta), static_cast<const float *>(rhs)};
        launch<float>(*this, transpose, static_cast<const float *>(src), static_cast<float *>(dst),
                      reinterpret_cast<float *>(shell.ptr), om, s);
      }
  }
} // namespace stmg

// ---------------------------------------------------------------------------
// Operator apply that allocates no device memory. The only scratch the
// apply needs, the tiles' face slots, lives in one fixed array of this file's
// device image, so every GPU that loads the library holds these bytes until
// the process exits. Calls share the array: two calls whose kernels overlap
// on the GPU (different streams, or different host threads on one device)
// race on it. Nothing in it has to start at zero: every face slot the fix-up
// reads is written by its tile earlier in the same call.
namespace stmg
{
  constexpr std::size_t NOALLOC_SCRATCH_BYTES = std::size_t(16) << 20; // 16 MiB

  static __device__ __align__(256) unsigned char noalloc_scratch[NOALLOC_SCRATCH_BYTES];

  namespace
  {
    constexpr int MAX_DEVICES = 64;
    std::mutex    scratch_mutex;
    void         *scratch_device_ptr[MAX_DEVICES] = {};

    // Device address of noalloc_scratch on the current device, looked up on
    // the first call per device (host code must not pass the array's name
    // to a kernel: on the host it is only a stand-in for the symbol).
    void *
    scratch_address()
    {
      int dev = 0;
      STMG_CUDA(cudaGetDevice(&dev));
      STMG_REQUIRE(dev >= 0 && dev < MAX_DEVICES, STMG_ERR_CUDA, "op_vmult_box_noalloc: device ordinal out of range");
      std::lock_guard<std::mutex> lock(scratch_mutex);
      if (!scratch_device_ptr[dev])
        {
          void             *p = nullptr;
          const cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);
          if (e != cudaSuccess || !p)
            throw Error(STMG_ERR_CUDA, std::string("op_vmult_box_noalloc: cudaGetSymbolAddress of the scratch array: ") +
                                         cudaGetErrorString(e));
          scratch_device_ptr[dev] = p;
        }
      return scratch_device_ptr[dev];
    }

    template <typename T>
    void
    box_apply(const MeshView &m, int nd, const double *A, const double *B, int nt_out, int nt_in, const T *src, T *dst,
              cudaStream_t s)
    {
      bool         big = true;
      int          shape[3];
      const Tiling tl = choose_op_tiling(m, sizeof(T), nt_in, nt_out, big, shape);
      const std::size_t need = tl.n_tiles > 1 ? std::size_t(tl.n_tiles) * nt_out * tl.tile_stride * sizeof(T) : 0;
      if (need > NOALLOC_SCRATCH_BYTES)
        throw Error(STMG_ERR_SHAPE, "op_vmult_box_noalloc: this mesh needs " + std::to_string(need) +
                                      " bytes of tile scratch, more than the fixed " +
                                      std::to_string(NOALLOC_SCRATCH_BYTES) + " bytes; use stmg_op_create instead");
      T *shell = static_cast<T *>(scratch_address());
      TimeMats<T> tm{};
      tm.nt_out = nt_out;
      tm.nt_in  = nt_in;
      for (int k = 0; k < nt_out * nt_in; ++k)
        {
          tm.A[k] = T(A[k]);
          tm.B[k] = T(B[k]);
        }
      const OpLaunch<T> L{m, tl, tm, make_cart<T>(m), make_qtab<T>(m.p), src, dst, shell, OutMode<T>{T(1), T(0), nullptr},
                          big, s};
#define STMG_BOX(D, PP)                                                                                  \
  if (m.dim == D && m.p == PP)                                                                           \
    return op_launch_dp<D, PP, T>(L);
      STMG_BOX(2, 1) STMG_BOX(2, 2) STMG_BOX(2, 3) STMG_BOX(2, 4) STMG_BOX(2, 5)
      STMG_BOX(3, 1) STMG_BOX(3, 2) STMG_BOX(3, 3) STMG_BOX(3, 4)
#undef STMG_BOX
      throw Error(STMG_ERR_UNSUPPORTED, "op_vmult_box_noalloc: unsupported dim/degree");
    }
  } // namespace

  void
  op_vmult_box_noalloc(int dim, const int *n_cells, int degree, const double *lo, const double *hi, const void *coeff,
                       int nt_out, int nt_in, const double *A, const double *B, int dtype, const void *src, void *dst,
                       cudaStream_t s)
  {
    STMG_REQUIRE(n_cells && lo && hi && A && B && src && dst, STMG_ERR_ARG, "op_vmult_box_noalloc: null argument");
    STMG_REQUIRE(dim == 2 || dim == 3, STMG_ERR_ARG, "op_vmult_box_noalloc: dim must be 2 or 3");
    STMG_REQUIRE(degree >= 1 && degree <= MAX_P && (dim == 2 || degree <= 4), STMG_ERR_UNSUPPORTED,
                 "op_vmult_box_noalloc: degree must be 1..5 (3-D: 1..4)");
    STMG_REQUIRE(nt_out >= 1 && nt_out <= MAX_NT && nt_in >= 1 && nt_in <= MAX_NT, STMG_ERR_ARG,
                 "op_vmult_box_noalloc: time dimensions must be 1..16");
    STMG_REQUIRE(dtype == STMG_F64 || dtype == STMG_F32, STMG_ERR_ARG, "op_vmult_box_noalloc: dtype must be F64 or F32");
    // the view make_mesh builds for a uniform box (no vertex array needed)
    MeshView m{};
    m.dim    = dim;
    m.p      = degree;
    m.N      = 1;
    m.ncells = 1;
    for (int d = 0; d < 3; ++d)
      {
        STMG_REQUIRE(d >= dim || (n_cells[d] >= 1 && hi[d] > lo[d]), STMG_ERR_ARG,
                     "op_vmult_box_noalloc: cell counts and box extents must be positive");
        m.n[d]  = d < dim ? n_cells[d] : 1;
        m.nn[d] = d < dim ? n_cells[d] * degree + 1 : 1;
        m.h[d]  = d < dim ? (hi[d] - lo[d]) / n_cells[d] : 1.0;
        if (d < dim)
          {
            m.N *= m.nn[d];
            m.ncells *= m.n[d];
          }
      }
    m.cartesian  = 1;
    m.box        = 1;
    m.vert       = nullptr;
    m.coeff_mode = coeff ? 1 : 0;
    m.coeff64    = dtype == STMG_F64 ? static_cast<const double *>(coeff) : nullptr;
    m.coeff32    = dtype == STMG_F32 ? static_cast<const float *>(coeff) : nullptr;
    int nd = 1;
    for (int d = 0; d < dim; ++d)
      nd *= degree + 1;
    if (dtype == STMG_F64)
      box_apply<double>(m, nd, A, B, nt_out, nt_in, static_cast<const double *>(src), static_cast<double *>(dst), s);
    else
      box_apply<float>(m, nd, A, B, nt_out, nt_in, static_cast<const float *>(src), static_cast<float *>(dst), s);
  }
} // namespace stmg
