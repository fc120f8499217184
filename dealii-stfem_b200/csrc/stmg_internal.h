// Internal declarations shared by the CUDA sources of libstmg_cuda.so.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/stmg.h"

#include <nvtx3/nvToolsExt.h>

namespace stmg
{
  constexpr int MAX_P  = 5;  // spatial degrees 1..5 (3-D up to 4 for the operator, 3 for Vanka)
  constexpr int MAX_NT = 16; // time dofs per slab

  // Error carried from the implementation to the C ABI.
  struct Error : std::runtime_error
  {
    int code;
    Error(int c, const std::string &m)
      : std::runtime_error(m)
      , code(c)
    {}
  };

  void set_last_error(const std::string &m);

  // NVTX range over a scope, named like the reference's TimerOutput sections
  // ("vmult", "Tvmult", "vanka", "gmg", "step": operators.h:97,127,158,
  // gmg.h:479,850, tp_01.cc:632), so a profiler's timeline shows the same
  // breakdown; costs nothing without a profiler attached.
  struct NvtxScope
  {
    explicit NvtxScope(const char *name) { nvtxRangePushA(name); }
    ~NvtxScope() { nvtxRangePop(); }
    NvtxScope(const NvtxScope &)            = delete;
    NvtxScope &operator=(const NvtxScope &) = delete;
  };

  // Number of kernels this library has launched (diagnostic counter).
  void      count_launch();
  void      add_launches(long long n);
  long long launch_count();

#define STMG_CUDA(call)                                                                                  \
  do                                                                                                     \
    {                                                                                                    \
      cudaError_t e_ = (call);                                                                           \
      if (e_ != cudaSuccess)                                                                             \
        throw ::stmg::Error(STMG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
    }                                                                                                    \
  while (0)

#define STMG_REQUIRE(cond, code, msg)                                                                    \
  do                                                                                                     \
    {                                                                                                    \
      if (!(cond))                                                                                       \
        throw ::stmg::Error(code, msg);                                                                  \
    }                                                                                                    \
  while (0)

  // Device buffer owned by a handle (allocation happens at setup only).
  template <typename T>
  struct DevBuf
  {
    T          *ptr = nullptr;
    std::size_t n   = 0;
    DevBuf()        = default;
    explicit DevBuf(std::size_t n_) { alloc(n_); }
    DevBuf(const DevBuf &)            = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept
      : ptr(o.ptr)
      , n(o.n)
    {
      o.ptr = nullptr;
      o.n   = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept
    {
      if (this != &o)
        {
          release();
          ptr   = o.ptr;
          n     = o.n;
          o.ptr = nullptr;
          o.n   = 0;
        }
      return *this;
    }
    ~DevBuf() { release(); }
    void alloc(std::size_t n_)
    {
      release();
      n = n_;
      if (n)
        {
          cudaError_t e = cudaMalloc(&ptr, n * sizeof(T));
          if (e != cudaSuccess)
            {
              ptr = nullptr;
              throw Error(STMG_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
            }
        }
    }
    void release()
    {
      if (ptr)
        cudaFree(ptr);
      ptr = nullptr;
      n   = 0;
    }
    void upload(const T *h, std::size_t count)
    {
      STMG_CUDA(cudaMemcpy(ptr, h, count * sizeof(T), cudaMemcpyHostToDevice));
    }
    void upload(const std::vector<T> &h)
    {
      if (h.size() != n)
        alloc(h.size());
      upload(h.data(), h.size());
    }
  };

  // 1-D finite element tables of FE_Q(p) on Gauss-Lobatto nodes with
  // QGauss(p+1), p = 1..MAX_P (held in __constant__ memory, see tables.cu).
  struct FETables
  {
    double xs[MAX_P + 1][MAX_P + 1];                   // support points
    double gx[MAX_P + 1][MAX_P + 1], gw[MAX_P + 1][MAX_P + 1]; // Gauss points, weights
    double S[MAX_P + 1][MAX_P + 1][MAX_P + 1];         // S[p][q][a] = phi_a(g_q)
    double D[MAX_P + 1][MAX_P + 1][MAX_P + 1];         // D[p][q][a] = phi_a'(g_q)
    double Dq[MAX_P + 1][MAX_P + 1][MAX_P + 1];        // collocation derivative at q-points
    double M1[MAX_P + 1][MAX_P + 1][MAX_P + 1];        // 1-D mass on [0,1]
    double K1[MAX_P + 1][MAX_P + 1][MAX_P + 1];        // 1-D stiffness on [0,1]
  };
  const FETables &host_tables();

  // Quadrature tables of one degree in working precision (kernel parameter).
  template <typename T>
  struct QTab
  {
    T S[(MAX_P + 1) * (MAX_P + 1)];  // S[q*(p+1)+a]
    T Dq[(MAX_P + 1) * (MAX_P + 1)]; // collocation derivative, Dq[q*(p+1)+r]
    T gx[MAX_P + 1], gw[MAX_P + 1];
  };
  template <typename T>
  QTab<T> make_qtab(int p);

  // Device view of one structured mesh level (passed to kernels by value).
  struct MeshView
  {
    int       dim, p;
    int       n[3];  // cells per direction (1 for unused directions)
    int       nn[3]; // nodes per direction
    long long N;     // nodes
    long long ncells;
    int       cartesian;  // axis-aligned uniform cells, coefficient constant per cell
    int       box;        // axis-aligned uniform cells (any coefficient mode)
    double    h[3];       // cell size (box / cartesian)
    const double *vert;   // vertex coordinates (general geometry), device
    int           coeff_mode; // 0 none, 1 per cell, 2 per quadrature point
    const double *coeff64;
    const float  *coeff32;
  };

  // Host-side mesh object behind stmg_mesh_t.
  struct Mesh
  {
    MeshView             v;
    std::vector<double>  vert_h;
    std::vector<double>  coeff_h;
    DevBuf<double>       vert_d, coeff64_d;
    DevBuf<float>        coeff32_d;
    int                  nq = 0, nd = 0;
  };

  std::unique_ptr<Mesh> make_mesh(int dim, const int *n, int p, const double *lo, const double *hi,
                                  const double *vertices, int coeff_mode, const double *coeff);

  // Tiling of the cell grid used by the cell-parallel kernels: tiles of
  // T[0] x T[1] x T[2] cells, each accumulating its brick of
  // (T p + 1)^dim nodes; contributions to the brick's boundary shell go to
  // per-tile face slots and are summed by the fix-up kernel.
  struct Tiling
  {
    int       T[3];
    int       ntiles[3];
    int       E[3];        // brick extent (max)
    long long face_off[6]; // offsets of the six face slots inside a tile's shell record
    long long face_len[6];
    long long tile_stride; // values per tile (per time dof)
    long long n_tiles;
  };
  Tiling make_tiling(const MeshView &m, const int *T);

  // Grid of a persistent kernel: as many CTAs as fit on the device at once
  // (occupancy with the given block size and dynamic shared memory), at most
  // `work` CTAs. Also raises the kernel's dynamic shared-memory limit.
  unsigned persistent_grid(const void *kernel, int block, std::size_t smem, long long work);
  // dst[b][i] = src[b][perm[i]] (scatter = 0) or dst[b][perm[i]] = src[b][i]
  // (scatter = 1) for n_blocks blocks of n entries; perm on the device
  void block_permute(int n_blocks, long long n, const long long *perm, int scatter, const void *src, void *dst,
                     int dtype, cudaStream_t s);
  int      sm_count();

  // Time coupling matrices of an operator (kernel parameter).
  template <typename T>
  struct TimeMats
  {
    int nt_out, nt_in;
    T   A[MAX_NT * MAX_NT]; // nt_out x nt_in row-major
    T   B[MAX_NT * MAX_NT];
  };

  // Scaled 1-D matrices of a cartesian level: Mx = M1 * h_x, Kx = K1 / h_x.
  template <typename T>
  struct Cart1D
  {
    T M[3][(MAX_P + 1) * (MAX_P + 1)];
    T K[3][(MAX_P + 1) * (MAX_P + 1)];
  };
} // namespace stmg
