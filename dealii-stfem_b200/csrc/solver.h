// Host C++ of the slab solve on the GPU: level hierarchy, V-cycle
// preconditioner (GMG, tests/include/gmg.h:652-906), FP64 FGMRES
// (SolverFGMRES with ReductionControl, time_integrators.h:44,113,174) and the
// heat / wave slab loops (time_integrators.h:60-180,237-280).
#pragma once

#include <memory>
#include <vector>

#include "blas.h"
#include "st_operator.h"
#include "stmg_internal.h"
#include "time_fe.h"
#include "transfer.h"
#include "vanka.h"

namespace stmg
{
  struct SolverConfig
  {
    int    dim = 2, subdiv[3] = {1, 1, 1}, refine = 2, degree = 2, time_degree = 1, time_type = 2, problem = 1,
        n_steps = 1;
    double tau = 0.125, lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    int    smoothing_steps = 1, fe_degree_min = -1, n_steps_min = -1;
    int    mg_dtype = STMG_F32, vanka_storage = STMG_F32;
    double tol = 1e-12, abs_tol = 1e-12;
    int    max_iter = 200, restart = 30, extrapolate = 1;
    int    rhs_mode = 0; // 0 manufactured (frequency), 1 nodal source field, 2 none
    double frequency = 1.0;
    std::vector<double> fine_vertices, fine_coeff, f_nodal;
  };

  // One level of the space-time hierarchy (operator, smoother, transfer to
  // the next coarser level) and its V-cycle vectors.
  struct Level
  {
    Mesh                       *mesh = nullptr;
    int                         nt   = 0, r = 0, n_steps = 0;
    tfe::Mat                    A, B;
    std::unique_ptr<StOperator> op;
    std::unique_ptr<Vanka>      vanka;
    std::unique_ptr<Transfer>   to_coarser; // between this level and level-1
    double                      omega = 1.0;
    DevBuf<unsigned char>       sol, def, t, r_, z;
    long long                   size() const { return mesh->v.N * nt; }
  };

  class GMG
  {
  public:
    // transpose_time: every level uses Alpha^T, Beta^T (the preconditioner
    // of the adjoint system A^T)
    GMG(const SolverConfig &cfg, std::vector<std::unique_ptr<Mesh>> &meshes, Blas &blas,
        bool transpose_time = false);
    ~GMG();
    GMG(const GMG &)            = delete;
    GMG &operator=(const GMG &) = delete;
    // FP64 in, FP64 out; FP32 or FP64 inside (GMG::vmult, gmg.h:846-859)
    // dst = V-cycle(src); scale (a power of two) is applied to src before
    // the cycle and undone after it, exactly
    void vmult(double *dst, const double *src, cudaStream_t s, double scale = 1.0);
    std::vector<double> omegas() const;
    std::vector<Level>  levels; // coarsest first
    int                 dtype;
    std::vector<tfe::MG> seq;
    // Levels 0..tail (tail >= 0) run as one dense matrix C: with fixed
    // relaxation weights and sweep counts the V-cycle from level `tail` down
    // is the linear map sol = C def, composed once in FP64 from dense copies
    // of the levels' operators, smoothers and transfers, and applied in FP64
    // (the coarse-grid solve stays FP64 in the FP32 V-cycle). -1: none.
    int tail = -1;
    static constexpr long long DENSE_TAIL_MAX = 4096; // entries per level vector

  private:
    template <typename T>
    void cycle(cudaStream_t s);
    template <typename T>
    void vstep(int l, cudaStream_t s);
    template <typename T>
    void relax_step(int l, T *x, const T *b, cudaStream_t s);
    template <typename T>
    void smooth(int l, T *x, const T *b, bool zero_start, cudaStream_t s);
    template <typename T>
    double estimate_relaxation(int l, cudaStream_t s);
    unsigned steps(int l) const;
    void     build_tail();
    std::unique_ptr<Transfer> make_transfer(int l, int dt) const;

    SolverConfig    cfg;
    Blas           &blas;
    bool            use_graph = true;
    cudaGraphExec_t graph     = nullptr;
    cudaStream_t    cap       = nullptr;
    long long       graph_nodes = 0;
    DevBuf<unsigned char> tail_mat; // n x n row-major, FP64 (applied in FP64 in either V-cycle type)
  };

  // FGMRES(restart) with CGS2 orthogonalisation on device vectors.
  class FGMRES
  {
  public:
    FGMRES(long long n, int basis, Blas &blas);
    template <typename Aop, typename Pop>
    int solve(Aop &&A, Pop &&P, double *x, const double *b, double abs_tol, double reduce, int max_iter,
              cudaStream_t s);
    double last_residual = 0, initial_residual = 0;

  private:
    long long                            n;
    int                                  basis;
    Blas                                &blas;
    std::vector<DevBuf<double>>          V, Z;
    DevBuf<double>                       aux;
  };

  class SlabSolver
  {
  public:
    explicit SlabSolver(const SolverConfig &cfg);
    // initial values on the finest nodes (host); null = the manufactured
    // solution at t = 0 (exact_solution.h:18-51,136-161)
    void set_initial(const double *u0, const double *v0);
    // nodal source field on the finest nodes (host): rhs = M f
    void set_source(const double *f_nodal);
    // run n slabs, iteration counts to `its` (host)
    void run(int n_slabs, int *its, cudaStream_t s);
    // one FGMRES solve of the slab system for device vectors x, rhs
    int  solve(double *x, const double *rhs, cudaStream_t s);
    void system_vmult(double *dst, const double *src, cudaStream_t s);
    void download(double *u, double *v) const;
    // download without a host wait: the last slab's u (and v) blocks are
    // copied on `s` into device staging buffers, then to the host arrays on
    // a non-blocking copy stream, so the host transfer overlaps later slabs
    // (run() waits only for the device copy). download_wait() returns once
    // the host arrays hold the values; pinned host arrays make the copy
    // asynchronous.
    void download_async(double *u, double *v, cudaStream_t s);
    void download_wait();
    // Heat only: runs n_slabs slabs from the current state and returns the
    // misfit J = 1/2 sum_s |U_s - O_s|^2 (obs: host, n_slabs x n_t x N) and
    // dJ/d(log kappa_c) per fine cell (grad: host), by the discrete adjoint
    // run backward over the slabs (A^T lambda_s = U_s - O_s + E^T R^T
    // lambda_{s+1}); forward states are kept every `checkpoint_every` slabs
    // and recomputed segment by segment. Leaves the state after the last slab.
    double gradient(int n_slabs, const double *obs, int checkpoint_every, double *grad, int *its_fwd,
                    int *its_adj, cudaStream_t s);

    // Point functionals of the last slab (tests/tp_01.cc:451-619): u at the
    // n_pts points (host, n_pts x dim) for each time node, mapped to
    // `samples` equidistant times per step by the Lagrange time basis;
    // values: host, (n_steps samples) x n_pts; times (may be null): the
    // sample times
    void point_values(int n_pts, const double *pts, int samples, double *times, double *values, cudaStream_t s);

    SolverConfig                        cfg;
    std::vector<std::unique_ptr<Mesh>>  meshes; // coarsest first
    Blas                                blas;
    std::unique_ptr<GMG>                gmg;
    std::unique_ptr<StOperator>         A64, rhs64, rhsv64, mass64;
    std::unique_ptr<FGMRES>             gmres;
    int                                 nb = 0, ni = 0;
    long long                           N  = 0;
    double                              time = 0;
    tfe::Mat                            w1[4];
    tfe::Mat                            AixB, AixG, AixZ;
    DevBuf<double>                      x, v, prev_x, prev_v, rhs, F, Mf, fsrc;
    std::vector<double>                 node_x; // node coordinates (host), N x dim
    tfe::Mat                            lhsK_, rK_; // time matrices of K in the system and the rhs
    // error norms against the manufactured solution over the slabs run since
    // set_initial (rhs_mode 0): sums of squares and the maximum
    double                              err_l2sq = 0, err_h1sq = 0, err_l8 = 0;
    std::unique_ptr<GMG>                gmgT;       // preconditioner of A^T (built on first use)
    std::vector<int>                    last_iterations;

  private:
    // copy stream and events of download_async (created on first use)
    struct AsyncCopy
    {
      cudaStream_t stream = nullptr;
      cudaEvent_t  ready = nullptr, snapped = nullptr, copied = nullptr;
      bool         pending = false;
      AsyncCopy()                             = default;
      AsyncCopy(const AsyncCopy &)            = delete;
      AsyncCopy &operator=(const AsyncCopy &) = delete;
      ~AsyncCopy();
    };
    DevBuf<double> stage_u, stage_v; // declared first: the copy stream is drained before they go
    AsyncCopy      acopy;
    // the work queued on s, or the host, waits for a pending download's
    // device copy before x and v change
    void wait_snapshot(cudaStream_t s);
    void wait_snapshot_host();
    void force(double t, double *out, cudaStream_t s);
    void accumulate_errors(const std::vector<double> &tq, cudaStream_t s);
    DevBuf<double> err_buf, err_num;
  };

  std::vector<std::unique_ptr<Mesh>> build_meshes(const SolverConfig &cfg);
} // namespace stmg
