// Reordering of block vectors between a caller's dof numbering and the
// library's lexicographic node order (the adapter a deal.II caller needs:
// DoFHandler numbering <-> lexicographic, per time block).
#include "stmg_internal.h"

namespace stmg
{
  namespace
  {
    // dst[b][i] = src[b][perm[i]]  (gather)  or  dst[b][perm[i]] = src[b][i]  (scatter)
    template <typename T>
    __global__ void
    permute_kernel(int n_blocks, long long n, const long long *__restrict__ perm, int scatter, const T *__restrict__ src,
                   T *__restrict__ dst)
    {
      const long long total = n * n_blocks;
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
        {
          const long long b = k / n, i = k - b * n;
          const long long j = perm[i];
          if (scatter)
            dst[b * n + j] = src[k];
          else
            dst[k] = src[b * n + j];
        }
    }
  } // namespace

  void
  block_permute(int n_blocks, long long n, const long long *perm, int scatter, const void *src, void *dst, int dtype,
                cudaStream_t s)
  {
    STMG_REQUIRE(n_blocks >= 1 && n >= 1 && perm && src && dst, STMG_ERR_ARG, "permute: bad arguments");
    STMG_REQUIRE(src != dst, STMG_ERR_ARG, "permute: source and destination must differ");
    const long long total = n * n_blocks;
    const unsigned  grid  = unsigned(std::min<long long>((total + 255) / 256, 148 * 16));
    if (dtype == STMG_F64)
      permute_kernel<double><<<grid, 256, 0, s>>>(n_blocks, n, perm, scatter, static_cast<const double *>(src),
                                                  static_cast<double *>(dst));
    else if (dtype == STMG_F32)
      permute_kernel<float><<<grid, 256, 0, s>>>(n_blocks, n, perm, scatter, static_cast<const float *>(src),
                                                 static_cast<float *>(dst));
    else
      throw Error(STMG_ERR_ARG, "permute: dtype must be F64 or F32");
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }
} // namespace stmg
