// Vector kernels of the slab solve: the deal.II vector operations inside
// SolverFGMRES (time_integrators.h:113,174), PreconditionRelaxation and the
// FP64<->FP32 boundary of GMG::vmult (gmg.h:846-859). Reductions are two-pass
// with a fixed grid and fixed summation order, so results are reproducible
// bit for bit.
#include "blas.h"

namespace stmg
{
  namespace
  {
    constexpr int RED_BLOCKS  = 592; // 4 x 148 SMs
    constexpr int RED_THREADS = 256;

    // Block sums of cnt per-thread values acc[0..cnt) into partial[blockIdx.x * cnt + i]:
    // warp shuffles, then one thread per value over the warps (fixed order).
    template <int MAXV>
    __device__ __forceinline__ void
    block_sums(double (&acc)[MAXV], int cnt, double *partial)
    {
      __shared__ double sh[RED_THREADS / 32][MAXV];
      const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
      for (int i = 0; i < MAXV; ++i)
        {
          if (i >= cnt)
            break;
          double v = acc[i];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
          if (lane == 0)
            sh[warp][i] = v;
        }
      __syncthreads();
      if (threadIdx.x < cnt)
        {
          double t = 0;
          for (int w = 0; w < RED_THREADS / 32; ++w)
            t += sh[w][threadIdx.x];
          partial[blockIdx.x * cnt + threadIdx.x] = t;
        }
    }

    // partial[b * m + i] = block b's share of V_i . w; w is read once
    template <typename T, int MAXV>
    __global__ void __launch_bounds__(RED_THREADS)
    multidot_partial(long long n, int m, const __grid_constant__ VecPtrs V, const T *__restrict__ w, double *partial)
    {
      double acc[MAXV];
#pragma unroll
      for (int i = 0; i < MAXV; ++i)
        acc[i] = 0;
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        {
          const double wk = double(w[k]);
#pragma unroll
          for (int i = 0; i < MAXV; ++i)
            if (i < m)
              acc[i] += double(__ldg(static_cast<const T *>(V.p[i]) + k)) * wk;
        }
      block_sums<MAXV>(acc, m, partial);
    }

    // w -= sum_i c_i V_i; partial sums of w_new . w_new, then (if dots) of
    // V_i . w_new, with the V_i[k] kept in registers between the two uses
    template <typename T, int MAXV>
    __global__ void __launch_bounds__(RED_THREADS)
    orth_update_kernel(long long n, int m, const __grid_constant__ Coeffs c, const __grid_constant__ VecPtrs V,
                       T *__restrict__ w, int dots, double *partial)
    {
      double acc[MAXV + 1];
#pragma unroll
      for (int i = 0; i <= MAXV; ++i)
        acc[i] = 0;
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        {
          double v[MAXV];
          double s = double(w[k]);
#pragma unroll
          for (int i = 0; i < MAXV; ++i)
            {
              v[i] = i < m ? double(__ldg(static_cast<const T *>(V.p[i]) + k)) : 0.0;
              s -= c.c[i] * v[i];
            }
          const T st = T(s);
          w[k]       = st;
          const double sw = double(st);
          acc[0] += sw * sw;
#pragma unroll
          for (int i = 0; i < MAXV; ++i)
            acc[i + 1] += v[i] * sw;
        }
      block_sums<MAXV + 1>(acc, dots ? m + 1 : 1, partial);
    }

    __global__ void
    reduce_partials(int nblocks, int m, const double *partial, double *out)
    {
      const int i = threadIdx.x;
      if (i >= m)
        return;
      double s = 0;
      for (int b = 0; b < nblocks; ++b)
        s += partial[b * m + i];
      out[i] = s;
    }

    // w = alpha * w + sum_i c_i V_i   (c in kernel parameters)
    template <typename T>
    __global__ void
    multi_axpy(long long n, int m, double alpha, const __grid_constant__ Coeffs c, const __grid_constant__ VecPtrs V,
               T *__restrict__ w)
    {
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        {
          double s = alpha == 0.0 ? 0.0 : alpha * double(w[k]);
#pragma unroll 4
          for (int i = 0; i < m; ++i)
            s += c.c[i] * double(static_cast<const T *>(V.p[i])[k]);
          w[k] = T(s);
        }
    }

    template <typename Tout, typename Tin>
    __global__ void
    convert_kernel(long long n, const Tin *__restrict__ x, Tout *__restrict__ y)
    {
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        y[k] = Tout(x[k]);
    }

    // y = a x + b y
    template <typename T>
    __global__ void
    axpby_kernel(long long n, T a, const T *__restrict__ x, T b, T *__restrict__ y)
    {
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        y[k] = a * x[k] + b * y[k];
    }

    // r = b - r
    template <typename T>
    __global__ void
    sub_from_kernel(long long n, const T *__restrict__ b, T *__restrict__ r)
    {
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        r[k] = b[k] - r[k];
    }

    template <typename T>
    __global__ void
    fill_kernel(long long n, T v, T *__restrict__ y)
    {
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        y[k] = v;
    }

    unsigned
    grid_for(long long n)
    {
      const long long b = (n + 255) / 256;
      return unsigned(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
    }
  } // namespace

  Blas::Blas()
  {
    partial.alloc(std::size_t(RED_BLOCKS) * (MAX_DOTS + 1));
    result.alloc(MAX_DOTS + 1);
    STMG_CUDA(cudaMallocHost(&host_result, (MAX_DOTS + 1) * sizeof(double)));
  }

  Blas::~Blas()
  {
    if (host_result)
      cudaFreeHost(host_result);
  }

  // reduce the block partials of m values and copy them to out (host)
  void
  Blas::fetch(int m, double *out, cudaStream_t s)
  {
    reduce_partials<<<1, 64, 0, s>>>(RED_BLOCKS, m, partial.ptr, result.ptr);
    count_launch();
    STMG_CUDA(cudaGetLastError());
    STMG_CUDA(cudaMemcpyAsync(host_result, result.ptr, m * sizeof(double), cudaMemcpyDeviceToHost, s));
    STMG_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < m; ++i)
      out[i] = host_result[i];
  }

  template <typename T>
  void
  Blas::multidot(long long n, int m, const T *const *V, const T *w, double *out, cudaStream_t s)
  {
    STMG_REQUIRE(m >= 1 && m <= MAX_DOTS, STMG_ERR_ARG, "multidot: 1..32 vectors");
    VecPtrs vp{};
    for (int i = 0; i < m; ++i)
      vp.p[i] = V[i];
    if (m <= 8)
      multidot_partial<T, 8><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, m, vp, w, partial.ptr);
    else if (m <= 16)
      multidot_partial<T, 16><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, m, vp, w, partial.ptr);
    else
      multidot_partial<T, 32><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, m, vp, w, partial.ptr);
    count_launch();
    STMG_CUDA(cudaGetLastError());
    fetch(m, out, s);
  }

  template <typename T>
  double
  Blas::dot(long long n, const T *x, const T *y, cudaStream_t s)
  {
    const T *V[1] = {x};
    double   r;
    multidot<T>(n, 1, V, y, &r, s);
    return r;
  }

  template <typename T>
  void
  Blas::combine(long long n, double alpha, int m, const double *c, const T *const *V, T *w, cudaStream_t s)
  {
    STMG_REQUIRE(m >= 0 && m <= MAX_DOTS, STMG_ERR_ARG, "combine: 0..32 vectors");
    Coeffs  cc{};
    VecPtrs vp{};
    for (int i = 0; i < m; ++i)
      {
        cc.c[i] = c[i];
        vp.p[i] = V[i];
      }
    multi_axpy<T><<<grid_for(n), 256, 0, s>>>(n, m, alpha, cc, vp, w);
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }

  template <typename T>
  double
  Blas::orth_update(long long n, int m, const double *c, const T *const *V, T *w, double *dots, cudaStream_t s)
  {
    STMG_REQUIRE(m >= 1 && m <= MAX_DOTS, STMG_ERR_ARG, "orth_update: 1..32 vectors");
    Coeffs  cc{};
    VecPtrs vp{};
    for (int i = 0; i < m; ++i)
      {
        cc.c[i] = c[i];
        vp.p[i] = V[i];
      }
    const int d = dots ? 1 : 0;
    if (m <= 8)
      orth_update_kernel<T, 8><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, m, cc, vp, w, d, partial.ptr);
    else if (m <= 16)
      orth_update_kernel<T, 16><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, m, cc, vp, w, d, partial.ptr);
    else
      orth_update_kernel<T, 32><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, m, cc, vp, w, d, partial.ptr);
    count_launch();
    STMG_CUDA(cudaGetLastError());
    double out[MAX_DOTS + 1];
    fetch(dots ? m + 1 : 1, out, s);
    if (dots)
      for (int i = 0; i < m; ++i)
        dots[i] = out[i + 1];
    return out[0];
  }

  template <typename Tout, typename Tin>
  void
  convert(long long n, const Tin *x, Tout *y, cudaStream_t s)
  {
    convert_kernel<Tout, Tin><<<grid_for(n), 256, 0, s>>>(n, x, y);
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }

  template <typename T>
  void
  axpby(long long n, T a, const T *x, T b, T *y, cudaStream_t s)
  {
    axpby_kernel<T><<<grid_for(n), 256, 0, s>>>(n, a, x, b, y);
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }

  template <typename T>
  void
  sub_from(long long n, const T *b, T *r, cudaStream_t s)
  {
    sub_from_kernel<T><<<grid_for(n), 256, 0, s>>>(n, b, r);
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }

  template <typename T>
  void
  fill(long long n, T v, T *y, cudaStream_t s)
  {
    fill_kernel<T><<<grid_for(n), 256, 0, s>>>(n, v, y);
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }

#define STMG_BLAS_INST(T)                                                                                \
  template void   Blas::multidot<T>(long long, int, const T *const *, const T *, double *, cudaStream_t);  \
  template double Blas::dot<T>(long long, const T *, const T *, cudaStream_t);                              \
  template void   Blas::combine<T>(long long, double, int, const double *, const T *const *, T *, cudaStream_t); \
  template double Blas::orth_update<T>(long long, int, const double *, const T *const *, T *, double *, cudaStream_t); \
  template void   axpby<T>(long long, T, const T *, T, T *, cudaStream_t);                                  \
  template void   sub_from<T>(long long, const T *, T *, cudaStream_t);                                     \
  template void   fill<T>(long long, T, T *, cudaStream_t);
  STMG_BLAS_INST(double)
  STMG_BLAS_INST(float)
#undef STMG_BLAS_INST
  template void convert<float, double>(long long, const double *, float *, cudaStream_t);
  template void convert<double, float>(long long, const float *, double *, cudaStream_t);
  template void convert<double, double>(long long, const double *, double *, cudaStream_t);
  template void convert<float, float>(long long, const float *, float *, cudaStream_t);
} // namespace stmg
