// Oracle (test infrastructure only): CPU restatement of the reference's slab
// solve: level hierarchy and V-cycle (tests/include/gmg.h:317-400,652-906 with
// deal.II's Multigrid / MGSmootherPrecondition / PreconditionRelaxation),
// FGMRES (time_integrators.h:44,113,174), heat and wave slab loops
// (time_integrators.h:60-180,237-280; tests/tp_01.cc:630-683) and the
// space-time error norms (tests/include/exact_solution.h:217-299).
#pragma once

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "space.h"

namespace oracle
{
  enum class Problem : int
  {
    heat = 1,
    wave = 2
  };

  struct Config
  {
    int      dim        = 2;
    int      subdiv[3]  = {1, 1, 1};
    int      refine     = 2;
    int      p          = 2; // spatial degree
    int      r          = 1; // time degree
    TimeType type       = TimeType::DG;
    Problem  problem    = Problem::heat;
    int      n_steps    = 1; // time steps per slab
    double   tau        = 0.125;
    int      n_slabs    = 8;
    double   lo[3]      = {0, 0, 0};
    double   hi[3]      = {1, 1, 1};
    // multigrid (gmg.h:542-559)
    int    smoothing_steps       = 1;
    bool   variable              = true;
    bool   estimate_relaxation   = true;
    bool   restrict_is_transpose = true;
    int    fe_degree_min         = -1;
    int    n_steps_min           = -1;
    bool   space_time_mg         = true;
    bool   time_before_space     = false;
    // outer solver
    double tol      = 1e-12; // ReductionControl reduce and abs tolerance
    double abs_tol  = 1e-12;
    int    max_iter = 200;
    int    restart  = 30;
    bool   extrapolate = true;
    // data
    int                 rhs_mode  = 0; // 0 manufactured (frequency), 1 nodal field f, 2 zero
    double              frequency = 1.0;
    std::vector<double> f_nodal;   // rhs_mode 1: nodal values on the finest mesh
    std::vector<double> u0_nodal;  // initial u (finest nodes); empty = exact solution at t=0
    std::vector<double> v0_nodal;  // initial v (wave)
    std::vector<double> fine_vertices; // empty = uniform box
    std::vector<double> fine_coeff;    // empty = 1; else per finest cell
    bool                compute_errors = true;
    bool                mg_float       = true; // FP32 V-cycle (tests/tp_01.cc:767,776)
    bool                keep_all       = false; // Result::u_all: every slab's blocks
  };

  struct Result
  {
    std::vector<int>    iterations; // per slab
    int                 total_iterations = 0;
    double              l8 = -1, l2 = 0, h1 = 0; // L-inf-L-inf, L2-L2, L2-H1semi
    std::vector<double> omega;                   // per level
    std::vector<double> u_last;                  // all blocks of the last slab
    std::vector<double> u_all;                   // all blocks of every slab (Config::keep_all)
    std::vector<double> v_last;
    std::size_t         n_dofs = 0, n_cells = 0;
    int                 n_blocks = 0, n_levels = 0;
  };

  // One level of the space-time hierarchy.
  struct LevelInfo
  {
    int      sp;       // spatial mesh index (0 = coarsest)
    int      r;        // time degree
    int      n_steps;  // steps per slab
    int      nt;       // time dofs
    TimeMG   to_finer; // type of the transfer to the next finer level
    DMat     Alpha, Beta;
  };

  struct Hierarchy
  {
    std::vector<Mesh>      meshes; // spatial meshes, coarsest first
    std::vector<LevelInfo> levels; // coarsest first
    std::vector<TimeMG>    seq;
  };

  // Builds meshes, level schedule and level time matrices (tp_01.cc:200-328).
  Hierarchy build_hierarchy(const Config &cfg, double tau);

  // FP64 or FP32 V-cycle preconditioner.
  class GMGBase
  {
  public:
    virtual ~GMGBase() = default;
    virtual void vmult(double *dst, const double *src) = 0;
    virtual std::vector<double> omegas() const        = 0;
  };
  std::unique_ptr<GMGBase> make_gmg(const Config &cfg, const Hierarchy &h);

  // Right-preconditioned FGMRES with deal.II's SolverFGMRES / ReductionControl
  // semantics; returns the iteration count (throws on no convergence).
  int fgmres(std::size_t n, const std::function<void(double *, const double *)> &A,
             const std::function<void(double *, const double *)> &P, double *x, const double *b,
             double abs_tol, double reduce, int max_iter, int basis_size);

  Result run(const Config &cfg);

  // Output in the layout of tests/tp_01.output for one config file line.
  std::string convergence_report(const Config &base, int k0, int n_deg, int r0, int n_ref);
} // namespace oracle
