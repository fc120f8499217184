// Oracle (test infrastructure only): CPU FP64 restatement of the reference's
// time finite-element algebra, tests/include/fe_time.h of nlsmrg/dealii-stfem.
// Only tests/, the bench's CPU-baseline leg and the smoke check use this code,
// and only to check results against; the product never links it.
#pragma once

#include <array>
#include <cstddef>
#include <string>
#include <vector>

namespace oracle
{
  // Dense row-major matrix (stands in for dealii::FullMatrix<double>).
  struct DMat
  {
    std::size_t         m = 0, n = 0;
    std::vector<double> a;
    DMat() = default;
    DMat(std::size_t m_, std::size_t n_)
      : m(m_)
      , n(n_)
      , a(m_ * n_, 0.0)
    {}
    double &operator()(std::size_t i, std::size_t j) { return a[i * n + j]; }
    double  operator()(std::size_t i, std::size_t j) const { return a[i * n + j]; }
    bool    all_zero() const;
    void    scale(double s);
  };

  DMat mmult(const DMat &A, const DMat &B);
  DMat transpose(const DMat &A);
  DMat invert(const DMat &A); // Gauss-Jordan with partial pivoting
  // deal.II FullMatrix::fill(src, dst_i, dst_j, src_i, src_j): copy as much
  // of src[src_i:, src_j:] as fits into this[dst_i:, dst_j:] (overwrites).
  void fill(DMat &dst, const DMat &src, std::size_t di, std::size_t dj, std::size_t si, std::size_t sj);

  enum class TimeType : int
  {
    CGP = 1,
    DG  = 2
  };
  enum class TimeMG : int
  {
    tau  = 1,
    k    = 2,
    none = 3
  };

  // Quadratures on [0,1] (deal.II QGauss, QGaussLobatto, QGaussRadau(right)).
  void gauss(unsigned n, std::vector<double> &x, std::vector<double> &w);
  void gauss_lobatto(unsigned n, std::vector<double> &x, std::vector<double> &w);
  void gauss_radau_right(unsigned n, std::vector<double> &x);

  // Lagrange basis through `pts`, value / derivative of basis i at x.
  double lagrange(const std::vector<double> &pts, unsigned i, double x);
  double lagrange_d(const std::vector<double> &pts, unsigned i, double x);

  // Support points of the time basis (fe_time.h:414-425).
  std::vector<double> time_basis_points(TimeType type, unsigned r);

  std::array<DMat, 3> get_dg_weights(unsigned r);                 // fe_time.h:514-555
  std::array<DMat, 2> get_cg_weights(unsigned r);                 // fe_time.h:473-512
  std::array<DMat, 4> split_lhs_rhs(const std::array<DMat, 2> &); // fe_time.h:431-460
  std::array<DMat, 4> split_lhs_rhs(const std::array<DMat, 3> &); // fe_time.h:462-471
  std::array<DMat, 4> get_fe_time_weights(TimeType type, unsigned r, double tau,
                                          unsigned n_steps); // fe_time.h:292-349
  std::array<DMat, 5> get_fe_time_weights_wave(TimeType type, const DMat &Alpha, const DMat &Beta,
                                               const DMat &Gamma, const DMat &Zeta,
                                               unsigned n_steps); // fe_time.h:98-246
  std::vector<std::array<DMat, 4>> get_fe_time_weights_levels(TimeType type, unsigned r, double tau,
                                                              unsigned n_steps,
                                                              const std::vector<TimeMG> &seq); // fe_time.h:351-381
  std::vector<std::array<DMat, 5>> get_fe_time_weights_wave_levels(TimeType type, unsigned r, double tau,
                                                                   unsigned n_steps,
                                                                   const std::vector<TimeMG> &seq); // fe_time.h:383-412

  std::vector<TimeMG> get_time_mg_sequence(unsigned n_sp_lvl, unsigned k_max, unsigned k_min,
                                           unsigned n_steps, unsigned n_steps_min,
                                           TimeMG lower = TimeMG::k,
                                           bool   time_before_space = false); // fe_time.h:43-69
  // Level -> spatial-mesh index map (fe_time.h:71-96). spatial index 0 is
  // the coarsest mesh; the result has seq.size()+1 entries.
  std::vector<unsigned> get_space_time_levels(const std::vector<TimeMG> &seq, unsigned n_sp_lvl);

  DMat get_time_projection_matrix(TimeType type, unsigned r_src, unsigned r_dst,
                                  unsigned n_steps); // fe_time.h:567-623
  DMat get_time_prolongation_matrix(TimeType type, unsigned r,
                                    unsigned n_steps = 2); // fe_time.h:625-669
  DMat get_time_restriction_matrix(TimeType type, unsigned r,
                                   unsigned n_steps = 2); // fe_time.h:671-716
  DMat get_time_evaluation_matrix(const std::vector<double> &pts, unsigned samples); // fe_time.h:248-267

  // The 2-decimal printer the reference tests use (tests/tp_02.cc:9-30).
  std::string print_formatted(const DMat &M);
} // namespace oracle
