// Asynchronous global->shared copies (cp.async, sm_80+ and sm_100a) and a
// division-free row walk over tile bricks.
#pragma once

#include <cuda_runtime.h>

namespace stmg
{
  // 4/8-byte copy; src_bytes = 0 writes zeros instead of reading
  template <int BYTES>
  __device__ __forceinline__ void
  cp_async_small(void *smem, const void *gmem, bool valid)
  {
    static_assert(BYTES == 4 || BYTES == 8, "cp.async.ca copies 4 or 8 bytes");
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    const int      n = valid ? BYTES : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(BYTES), "r"(n) : "memory");
  }

  // 16-byte copy, both addresses 16-byte aligned
  __device__ __forceinline__ void
  cp_async16(void *smem, const void *gmem)
  {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
  }

  __device__ __forceinline__ void
  cp_async_commit()
  {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }

  template <int N>
  __device__ __forceinline__ void
  cp_async_wait()
  {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
  }

  // Stage the brick of a tile for nt time blocks: rows (i, z, y) over the
  // warps, x over the lanes, so the only division is per row. Dirichlet and
  // out-of-mesh nodes are zero-filled.
  template <typename T>
  __device__ __forceinline__ void
  load_brick_async(T *brick, const T *__restrict__ src, long long N, int nt, const int (&E)[3], const int (&e)[3],
                   const int (&g0)[3], const int (&nn)[3], int dim)
  {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int rows = nt * E[2] * E[1];
    for (int row = warp; row < rows; row += nw)
      {
        const int by = row % E[1], rz = row / E[1];
        const int bz = rz % E[2], i = rz / E[2];
        const int gy = g0[1] + by, gz = g0[2] + bz;
        const bool rowok = by < e[1] && bz < e[2] && gy > 0 && gy < nn[1] - 1 && (dim < 3 || (gz > 0 && gz < nn[2] - 1));
        const long long base = i * N + (long long)nn[0] * (gy + (long long)nn[1] * gz) + g0[0];
        T *dst = brick + (long long)row * E[0];
        for (int bx = lane; bx < E[0]; bx += 32)
          {
            const int  gx = g0[0] + bx;
            const bool ok = rowok && bx < e[0] && gx > 0 && gx < nn[0] - 1;
            cp_async_small<sizeof(T)>(dst + bx, ok ? src + base + bx : src, ok);
          }
      }
  }
} // namespace stmg
