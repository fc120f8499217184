// Vector kernels used by the V-cycle and FGMRES (device vectors).
#pragma once

#include "stmg_internal.h"

namespace stmg
{
  constexpr int MAX_DOTS = 32;

  struct Coeffs
  {
    double c[MAX_DOTS];
  };

  // vector pointers of one call, passed by value to the kernels
  struct VecPtrs
  {
    const void *p[MAX_DOTS];
  };

  // Reductions with FP64 accumulation in a fixed order; owns its scratch
  // (block partial sums, a completion counter, the Gram-Schmidt coefficients
  // and a mapped pinned result buffer), allocated once. One stream at a time.
  class Blas
  {
  public:
    Blas();
    ~Blas();
    Blas(const Blas &)            = delete;
    Blas &operator=(const Blas &) = delete;

    // out[i] = V_i . w, i < m (synchronises the stream)
    template <typename T>
    void multidot(long long n, int m, const T *const *V, const T *w, double *out, cudaStream_t s);
    template <typename T>
    double dot(long long n, const T *x, const T *y, cudaStream_t s);
    // w = alpha w + sum_i c_i V_i
    template <typename T>
    void combine(long long n, double alpha, int m, const double *c, const T *const *V, T *w, cudaStream_t s);
    // One classical Gram-Schmidt pass against basis vectors stored divided
    // by sc_i: h_i = sc_i (V_i . w) for i < m (and h_m = w . w before the
    // pass if with_self), then w -= sum_i (h_i sc_i) V_i with the
    // coefficients kept on the device; returns w . w after the update.
    // Two kernels and one host wait (synchronises the stream).
    template <typename T>
    double gs_pass(long long n, int m, const T *const *V, const double *sc, T *w, bool with_self, double *h,
                   cudaStream_t s);

  private:
    template <typename T>
    void launch_multidot(long long n, int m, const T *const *V, const T *w, int nscale, const double *sc,
                         double *out_dev, cudaStream_t s);
    DevBuf<double> partial, coef, counter;
    double        *host_result = nullptr, *dev_result = nullptr;
  };

  // y = scale x in the output type; scale must be a power of two (exact)
  template <typename Tout, typename Tin>
  void convert(long long n, const Tin *x, Tout *y, cudaStream_t s, double scale = 1.0);
  template <typename T>
  void axpby(long long n, T a, const T *x, T b, T *y, cudaStream_t s); // y = a x + b y
  template <typename T>
  void sub_from(long long n, const T *b, T *r, cudaStream_t s);        // r = b - r
  template <typename T>
  void fill(long long n, T v, T *y, cudaStream_t s);
} // namespace stmg
