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
    constexpr int RED_BLOCKS  = 592; // 4 x 148 SMs: the grid of a large reduction
    constexpr int RED_THREADS = 256;

    // Reduction grid for n entries: about four entries per thread, at most
    // RED_BLOCKS blocks (small vectors take a few blocks, so their partial
    // sums are few).
    unsigned
    red_grid(long long n)
    {
      const long long b = (n + 4 * RED_THREADS - 1) / (4 * RED_THREADS);
      return unsigned(b < 1 ? 1 : (b > RED_BLOCKS ? RED_BLOCKS : b));
    }

    // What the last block does with the cnt reduced values r_i: with
    // nscale > 0, h_i = r_i sc_i and c_i = h_i sc_i for i < nscale (the
    // Gram-Schmidt coefficients of basis vectors stored divided by sc_i; c
    // stays on the device for the update pass); every value goes to out (a
    // mapped pinned host buffer).
    struct Finish
    {
      double       *out;
      double       *c;
      int           nscale;
      Coeffs        sc;
      unsigned     *counter;
    };

    // Block sums of cnt per-thread values acc[0..cnt) into partial[blockIdx.x * cnt + i]
    // (warp shuffles, then one thread per value over the warps, fixed order);
    // the block that finishes last reduces all blocks' partials (each value
    // by one warp: lanes take blocks lane, lane + 32, ..., then a shuffle
    // tree) and applies `fin`. The order depends on the grid only, so the
    // result is reproducible bit for bit.
    template <int MAXV>
    __device__ __forceinline__ void
    block_sums(double (&acc)[MAXV], int cnt, double *partial, const Finish &fin)
    {
      __shared__ double sh[RED_THREADS / 32][MAXV];
      __shared__ bool   last;
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
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0)
        last = atomicAdd(fin.counter, 1u) == gridDim.x - 1;
      __syncthreads();
      if (!last)
        return;
      const int nb = gridDim.x;
      for (int i = warp; i < cnt; i += RED_THREADS / 32)
        {
          double t = 0;
          for (int b = lane; b < nb; b += 32)
            t += __ldcg(partial + b * cnt + i);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1)
            t += __shfl_xor_sync(0xffffffffu, t, o);
          if (lane == 0)
            {
              if (i < fin.nscale)
                {
                  t *= fin.sc.c[i];
                  fin.c[i] = t * fin.sc.c[i];
                }
              fin.out[i] = t;
            }
        }
      if (threadIdx.x == 0)
        *fin.counter = 0u; // ready for the next reduction on this stream
    }

    // partial[b * m + i] = block b's share of V_i . w; w is read once
    template <typename T, int MAXV>
    __global__ void __launch_bounds__(RED_THREADS)
    multidot_partial(long long n, int m, const __grid_constant__ VecPtrs V, const T *__restrict__ w, double *partial,
                     const __grid_constant__ Finish fin)
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
      block_sums<MAXV>(acc, m, partial, fin);
    }

    // w -= sum_i c_i V_i with c on the device (written by the multidot's last
    // block); partial sums of w_new . w_new
    template <typename T, int MAXV>
    __global__ void __launch_bounds__(RED_THREADS)
    orth_update_kernel(long long n, int m, const double *__restrict__ cdev, const __grid_constant__ VecPtrs V,
                       T *__restrict__ w, double *partial, const __grid_constant__ Finish fin)
    {
      double c[MAXV];
#pragma unroll
      for (int i = 0; i < MAXV; ++i)
        c[i] = i < m ? cdev[i] : 0.0;
      double acc[1] = {0.0};
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        {
          double s = double(w[k]);
#pragma unroll
          for (int i = 0; i < MAXV; ++i)
            if (i < m)
              s -= c[i] * double(__ldg(static_cast<const T *>(V.p[i]) + k));
          const T st = T(s);
          w[k]       = st;
          const double sw = double(st);
          acc[0] += sw * sw;
        }
      block_sums<1>(acc, 1, partial, fin);
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

    // y = Tout(scale x); scale is a power of two (or 1), so the product is
    // exact and the conversion rounds as without it
    template <typename Tout, typename Tin>
    __global__ void
    convert_kernel(long long n, const Tin *__restrict__ x, Tout *__restrict__ y, double scale)
    {
      for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        y[k] = Tout(double(x[k]) * scale);
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
    coef.alloc(MAX_DOTS + 1);
    counter.alloc(1);
    STMG_CUDA(cudaMemset(counter.ptr, 0, sizeof(unsigned)));
    STMG_CUDA(cudaHostAlloc(&host_result, (MAX_DOTS + 2) * sizeof(double), cudaHostAllocMapped));
    STMG_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&dev_result), host_result, 0));
  }

  Blas::~Blas()
  {
    if (host_result)
      cudaFreeHost(host_result);
  }

  template <typename T>
  void
  Blas::launch_multidot(long long n, int m, const T *const *V, const T *w, int nscale, const double *sc,
                        double *out_dev, cudaStream_t s)
  {
    STMG_REQUIRE(m >= 1 && m <= MAX_DOTS, STMG_ERR_ARG, "multidot: 1..32 vectors");
    VecPtrs vp{};
    for (int i = 0; i < m; ++i)
      vp.p[i] = V[i];
    Finish fin{};
    fin.out     = out_dev;
    fin.c       = coef.ptr;
    fin.nscale  = nscale;
    fin.counter = reinterpret_cast<unsigned *>(counter.ptr);
    for (int i = 0; i < nscale; ++i)
      fin.sc.c[i] = sc[i];
    const unsigned g = red_grid(n);
    if (m <= 8)
      multidot_partial<T, 8><<<g, RED_THREADS, 0, s>>>(n, m, vp, w, partial.ptr, fin);
    else if (m <= 16)
      multidot_partial<T, 16><<<g, RED_THREADS, 0, s>>>(n, m, vp, w, partial.ptr, fin);
    else
      multidot_partial<T, MAX_DOTS><<<g, RED_THREADS, 0, s>>>(n, m, vp, w, partial.ptr, fin);
    count_launch();
    STMG_CUDA(cudaGetLastError());
  }

  template <typename T>
  void
  Blas::multidot(long long n, int m, const T *const *V, const T *w, double *out, cudaStream_t s)
  {
    STMG_REQUIRE(m >= 1 && m <= MAX_DOTS, STMG_ERR_ARG, "multidot: 1..32 vectors");
    launch_multidot<T>(n, m, V, w, 0, nullptr, dev_result, s);
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
  Blas::gs_pass(long long n, int m, const T *const *V, const double *sc, T *w, bool with_self, double *h,
                cudaStream_t s)
  {
    STMG_REQUIRE(m >= 1 && m <= MAX_DOTS, STMG_ERR_ARG, "gs_pass: 1..32 basis vectors");
    const T *vw[MAX_DOTS + 1];
    for (int i = 0; i < m; ++i)
      vw[i] = V[i];
    vw[m]        = w;
    const int md = with_self ? m + 1 : m;
    STMG_REQUIRE(md <= MAX_DOTS, STMG_ERR_ARG, "gs_pass: basis plus self dot beyond 32 vectors");
    // h_i = sc_i (V_i . w), c_i = h_i sc_i (and w . w), reduced by the last block
    launch_multidot<T>(n, md, vw, w, m, sc, dev_result, s);
    // w -= sum_i c_i V_i with the c_i left on the device; w . w after the update
    VecPtrs vp{};
    for (int i = 0; i < m; ++i)
      vp.p[i] = V[i];
    Finish fin{};
    fin.out        = dev_result + MAX_DOTS + 1;
    fin.counter    = reinterpret_cast<unsigned *>(counter.ptr);
    const unsigned g = red_grid(n);
    if (m <= 8)
      orth_update_kernel<T, 8><<<g, RED_THREADS, 0, s>>>(n, m, coef.ptr, vp, w, partial.ptr, fin);
    else if (m <= 16)
      orth_update_kernel<T, 16><<<g, RED_THREADS, 0, s>>>(n, m, coef.ptr, vp, w, partial.ptr, fin);
    else
      orth_update_kernel<T, MAX_DOTS><<<g, RED_THREADS, 0, s>>>(n, m, coef.ptr, vp, w, partial.ptr, fin);
    count_launch();
    STMG_CUDA(cudaGetLastError());
    STMG_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < md; ++i)
      h[i] = host_result[i];
    return host_result[MAX_DOTS + 1];
  }

  template <typename Tout, typename Tin>
  void
  convert(long long n, const Tin *x, Tout *y, cudaStream_t s, double scale)
  {
    convert_kernel<Tout, Tin><<<grid_for(n), 256, 0, s>>>(n, x, y, scale);
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
  template double Blas::gs_pass<T>(long long, int, const T *const *, const double *, T *, bool, double *, cudaStream_t); \
  template void   axpby<T>(long long, T, const T *, T, T *, cudaStream_t);                                  \
  template void   sub_from<T>(long long, const T *, T *, cudaStream_t);                                     \
  template void   fill<T>(long long, T, T *, cudaStream_t);
  STMG_BLAS_INST(double)
  STMG_BLAS_INST(float)
#undef STMG_BLAS_INST
  template void convert<float, double>(long long, const double *, float *, cudaStream_t, double);
  template void convert<double, float>(long long, const float *, double *, cudaStream_t, double);
  template void convert<double, double>(long long, const double *, double *, cudaStream_t, double);
  template void convert<float, float>(long long, const float *, float *, cudaStream_t, double);
} // namespace stmg
