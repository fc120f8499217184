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

    template <typename T>
    __device__ __forceinline__ double
    block_sum(double v, double *sh)
    {
      for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      if (lane == 0)
        sh[warp] = v;
      __syncthreads();
      double s = 0;
      if (threadIdx.x == 0)
        for (int w = 0; w < int(blockDim.x >> 5); ++w)
          s += sh[w];
      return s;
    }

    // partial[b * m + i] = sum over block b's slice of V_i . w
    template <typename T>
    __global__ void
    multidot_partial(long long n, int m, const T *const *__restrict__ V, const T *__restrict__ w, double *partial)
    {
      __shared__ double sh[32];
      for (int i = 0; i < m; ++i)
        {
          const T *v = V[i];
          double   s = 0;
          for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
            s += double(v[k]) * double(w[k]);
          const double t = block_sum<T>(s, sh);
          if (threadIdx.x == 0)
            partial[blockIdx.x * m + i] = t;
          __syncthreads();
        }
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
    multi_axpy(long long n, int m, double alpha, const __grid_constant__ Coeffs c, const T *const *__restrict__ V,
               T *__restrict__ w)
    {
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        {
          double s = alpha == 0.0 ? 0.0 : alpha * double(w[k]);
          for (int i = 0; i < m; ++i)
            s += c.c[i] * double(V[i][k]);
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
    partial.alloc(std::size_t(RED_BLOCKS) * MAX_DOTS);
    result.alloc(MAX_DOTS);
    ptrs.alloc(MAX_DOTS * 2);
    STMG_CUDA(cudaMallocHost(&host_result, MAX_DOTS * sizeof(double)));
    STMG_CUDA(cudaMallocHost(&host_ptrs, MAX_DOTS * 2 * sizeof(void *)));
  }

  Blas::~Blas()
  {
    if (host_result)
      cudaFreeHost(host_result);
    if (host_ptrs)
      cudaFreeHost(host_ptrs);
  }

  template <typename T>
  void
  Blas::multidot(long long n, int m, const T *const *V, const T *w, double *out, cudaStream_t s)
  {
    STMG_REQUIRE(m >= 1 && m <= MAX_DOTS, STMG_ERR_ARG, "multidot: 1..32 vectors");
    // vector pointers staged through pinned memory (ordered on the stream)
    STMG_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < m; ++i)
      host_ptrs[i] = const_cast<T *>(V[i]);
    STMG_CUDA(cudaMemcpyAsync(ptrs.ptr, host_ptrs, m * sizeof(void *), cudaMemcpyHostToDevice, s));
    multidot_partial<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, m, reinterpret_cast<const T *const *>(ptrs.ptr), w,
                                                          partial.ptr);
    count_launch();
    STMG_CUDA(cudaGetLastError());
    reduce_partials<<<1, 32, 0, s>>>(RED_BLOCKS, m, partial.ptr, result.ptr);
    count_launch();
    STMG_CUDA(cudaGetLastError());
    STMG_CUDA(cudaMemcpyAsync(host_result, result.ptr, m * sizeof(double), cudaMemcpyDeviceToHost, s));
    STMG_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < m; ++i)
      out[i] = host_result[i];
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
    Coeffs cc{};
    for (int i = 0; i < m; ++i)
      cc.c[i] = c[i];
    STMG_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < m; ++i)
      host_ptrs[MAX_DOTS + i] = const_cast<T *>(V[i]);
    void **dptr = reinterpret_cast<void **>(ptrs.ptr) + MAX_DOTS;
    if (m > 0)
      STMG_CUDA(cudaMemcpyAsync(dptr, host_ptrs + MAX_DOTS, m * sizeof(void *), cudaMemcpyHostToDevice, s));
    multi_axpy<T><<<grid_for(n), 256, 0, s>>>(n, m, alpha, cc, reinterpret_cast<const T *const *>(dptr), w);
    count_launch();
    STMG_CUDA(cudaGetLastError());
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
