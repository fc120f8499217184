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
  // (block partial sums and a pinned result), allocated once.
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
    // one Gram-Schmidt update in a single pass: w -= sum_i c_i V_i, then
    // dots[i] = V_i . w (if dots) and returns w . w (synchronises)
    template <typename T>
    double orth_update(long long n, int m, const double *c, const T *const *V, T *w, double *dots, cudaStream_t s);

  private:
    void fetch(int m, double *out, cudaStream_t s);
    DevBuf<double> partial, result;
    double        *host_result = nullptr;
  };

  template <typename Tout, typename Tin>
  void convert(long long n, const Tin *x, Tout *y, cudaStream_t s);
  template <typename T>
  void axpby(long long n, T a, const T *x, T b, T *y, cudaStream_t s); // y = a x + b y
  template <typename T>
  void sub_from(long long n, const T *b, T *r, cudaStream_t s);        // r = b - r
  template <typename T>
  void fill(long long n, T v, T *y, cudaStream_t s);
} // namespace stmg
