// Drives the C++ drop-in classes of include/stmg_dealii.hpp through the C ABI
// on a GPU and checks them against identities of the operators they replace:
//  * SystemMatrixGPU: <y, A x> = <A^T y, x>; vmult_add adds; the diagonal
//    equals (A e_i)_i for unit vectors e_i (get_matrix_diagonal), and the
//    inverse follows the reference's composition;
//  * VankaGPU::step = x + omega P (b - A x) from separate vmult calls;
//  * STTransferGPU: restrict_and_add is the transpose of prolongate_and_add
//    (h and time levels), prolongate overwrites;
//  * DofPermutation: a random cell-consistent numbering goes to the
//    lexicographic order and back.
// Prints "ALL OK" and exits 0 when every check passes.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "stmg_dealii.hpp"

using namespace stmg::shim;

namespace
{
  int failures = 0;

  void
  expect(bool ok, const char *what, double a = 0, double b = 0)
  {
    if (!ok)
      {
        std::printf("FAIL %s (%.17g vs %.17g)\n", what, a, b);
        ++failures;
      }
  }

  template <typename T>
  double
  dot(const std::vector<T> &a, const std::vector<T> &b)
  {
    double s = 0;
    for (std::size_t i = 0; i < a.size(); ++i)
      s += double(a[i]) * double(b[i]);
    return s;
  }

  // random values, zero on the Dirichlet nodes of an n0 x n1 x n2 node grid
  template <typename T>
  std::vector<T>
  random_block(int nb, const int *nn, std::mt19937_64 &rng)
  {
    std::normal_distribution<double> N01;
    const long long                  n = (long long)nn[0] * nn[1] * nn[2];
    std::vector<T>                   v(std::size_t(n * nb));
    for (int b = 0; b < nb; ++b)
      for (long long i = 0; i < n; ++i)
        {
          const long long x = i % nn[0], y = (i / nn[0]) % nn[1], z = i / ((long long)nn[0] * nn[1]);
          const bool      bd = x == 0 || y == 0 || z == 0 || x == nn[0] - 1 || y == nn[1] - 1 || z == nn[2] - 1;
          v[std::size_t(b * n + i)] = bd ? T(0) : T(N01(rng));
        }
    return v;
  }

  TimeMatrix
  random_matrix(int m, int n, std::mt19937_64 &rng, double diag)
  {
    std::uniform_real_distribution<double> U(-0.5, 0.5);
    TimeMatrix                             M(m, n);
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < n; ++j)
        M(i, j) = U(rng) + (i == j ? diag : 0.0);
    return M;
  }
} // namespace

int
main()
{
  std::mt19937_64 rng(20261203);
  const int       dim = 3, p = 2, nt = 3;
  const int       nc[3] = {6, 5, 4}, ncc[3] = {3, 5, 2};
  const double    lo[3] = {0, 0, 0}, hi[3] = {1.5, 1.0, 0.8};
  std::vector<double> kappa(nc[0] * nc[1] * nc[2]);
  std::uniform_real_distribution<double> Uk(-1, 1);
  for (auto &k : kappa)
    k = std::pow(10.0, Uk(rng));
  Mesh      mesh(dim, nc, p, lo, hi, nullptr, 1, kappa.data());
  const int nn[3] = {nc[0] * p + 1, nc[1] * p + 1, nc[2] * p + 1};
  const long long N = mesh.n_nodes();

  // ---------------------------------------------------- SystemMatrixGPU
  const TimeMatrix Alpha = random_matrix(nt, nt, rng, 2.0), Beta = random_matrix(nt, nt, rng, 3.0);
  SystemMatrixGPU<double> A(mesh, Alpha, Beta);
  expect(A.m() == std::size_t(nt * N), "m()");
  DeviceBlockVector<double> x, y, Ax, ATy;
  A.initialize_dof_vector(x);
  A.initialize_dof_vector(y);
  A.initialize_dof_vector(Ax);
  A.initialize_dof_vector(ATy);
  const auto hx = random_block<double>(nt, nn, rng), hy = random_block<double>(nt, nn, rng);
  x.copy_from_host(hx);
  y.copy_from_host(hy);
  A.vmult(Ax, x);
  A.Tvmult(ATy, y);
  const double yAx = dot(hy, Ax.copy_to_host()), ATyx = dot(ATy.copy_to_host(), hx);
  expect(std::abs(yAx - ATyx) <= 1e-12 * std::abs(yAx), "<y, A x> = <A^T y, x>", yAx, ATyx);
  // vmult_add: Ax + A x = 2 A x
  DeviceBlockVector<double> twice;
  A.initialize_dof_vector(twice);
  twice.copy_from_host(Ax.copy_to_host());
  A.vmult_add(twice, x);
  {
    const auto t = twice.copy_to_host(), a = Ax.copy_to_host();
    double     err = 0, mx = 0;
    for (std::size_t i = 0; i < t.size(); ++i)
      {
        err = std::max(err, std::abs(t[i] - 2 * a[i]));
        mx  = std::max(mx, std::abs(a[i]));
      }
    expect(err <= 1e-13 * mx, "vmult_add", err, mx);
  }
  // diagonal against A e_i at a few interior nodes of every block
  DeviceBlockVector<double> diag, dinv, e, Ae;
  A.initialize_dof_vector(diag);
  A.initialize_dof_vector(dinv);
  A.initialize_dof_vector(e);
  A.initialize_dof_vector(Ae);
  A.get_matrix_diagonal(diag);
  A.get_matrix_diagonal_inverse(dinv);
  const auto hd = diag.copy_to_host(), hdi = dinv.copy_to_host();
  const long long probes[3] = {1 + nn[0] * (1 + nn[1] * 1), 2 + nn[0] * (3 + nn[1] * 2), 5 + nn[0] * (4 + nn[1] * 3)};
  for (int b = 0; b < nt; ++b)
    for (long long i : probes)
      {
        std::vector<double> he(std::size_t(nt * N), 0.0);
        he[std::size_t(b * N + i)] = 1.0;
        e.copy_from_host(he);
        A.vmult(Ae, e);
        const double aii = Ae.copy_to_host()[std::size_t(b * N + i)];
        expect(std::abs(aii - hd[std::size_t(b * N + i)]) <= 1e-12 * std::abs(aii), "get_matrix_diagonal", aii,
               hd[std::size_t(b * N + i)]);
      }
  {
    // inverse: block b = diag(K)^+ / Alpha(b,b) + diag(M)^+ / Beta(b,b)
    TimeMatrix                I(1, 1), Z(1, 1);
    I(0, 0) = 1.0;
    SystemMatrixGPU<double>   K(mesh, I, Z), M(mesh, Z, I);
    DeviceBlockVector<double> dK(1, N), dM(1, N);
    K.get_matrix_diagonal(dK);
    M.get_matrix_diagonal(dM);
    const auto hk = dK.copy_to_host(), hm = dM.copy_to_host();
    double     err = 0, mx = 0;
    for (int b = 0; b < nt; ++b)
      for (long long i = 0; i < N; ++i)
        {
          const double ki = std::abs(hk[std::size_t(i)]) > 1.4901161193847656e-08 ? 1.0 / hk[std::size_t(i)] : 1.0;
          const double mi = std::abs(hm[std::size_t(i)]) > 1.4901161193847656e-08 ? 1.0 / hm[std::size_t(i)] : 1.0;
          const double r  = ki / Alpha(b, b) + mi / Beta(b, b);
          err             = std::max(err, std::abs(r - hdi[std::size_t(b * N + i)]));
          mx              = std::max(mx, std::abs(r));
        }
    expect(err <= 1e-13 * mx, "get_matrix_diagonal_inverse", err, mx);
  }

  // ----------------------------------------------------------- VankaGPU
  {
    SystemMatrixGPU<float>   Af(mesh, Alpha, Beta);
    VankaGPU<float>          P(mesh, Alpha, Beta);
    DeviceBlockVector<float> xf, bf, tmp, r, Pr, xs;
    for (auto *v : {&xf, &bf, &tmp, &r, &Pr, &xs})
      Af.initialize_dof_vector(*v);
    const auto hxf = random_block<float>(nt, nn, rng), hbf = random_block<float>(nt, nn, rng);
    xf.copy_from_host(hxf);
    bf.copy_from_host(hbf);
    xs.copy_from_host(hxf);
    const double omega = 0.7;
    P.step(xs, bf, Af, omega, tmp);
    Af.vmult(r, xf);
    auto hr = r.copy_to_host();
    for (std::size_t i = 0; i < hr.size(); ++i)
      hr[i] = hbf[i] - hr[i];
    r.copy_from_host(hr);
    P.vmult(Pr, r);
    const auto hp = Pr.copy_to_host(), hs = xs.copy_to_host();
    double     err = 0, mx = 0;
    for (std::size_t i = 0; i < hs.size(); ++i)
      {
        const double ref = double(hxf[i]) + omega * double(hp[i]);
        err              = std::max(err, std::abs(double(hs[i]) - ref));
        mx               = std::max(mx, std::abs(ref));
      }
    expect(err <= 1e-5 * mx, "VankaGPU::step", err, mx);
    P.clear();
    bool threw = false;
    try
      {
        P.vmult(Pr, r);
      }
    catch (const std::exception &)
      {
        threw = true;
      }
    expect(threw, "VankaGPU used after clear() throws");
  }

  // ------------------------------------------------------ STTransferGPU
  {
    Mesh                   coarse(dim, ncc, p, lo, hi);
    const int              ncf[3] = {6, 10, 4};
    Mesh                   fine(dim, ncf, p, lo, hi);
    STTransferGPU<double>  T;
    T.add_h_level(fine, coarse, nt);                             // level 1
    TimeMatrix             Pt = random_matrix(2 * nt, nt, rng, 0.0); // level 2: time prolongation on `fine`
    T.add_t_level(fine, Pt);
    expect(T.n_levels() == 3, "n_levels");
    const int nnc[3] = {ncc[0] * p + 1, ncc[1] * p + 1, ncc[2] * p + 1};
    const int nnf[3] = {ncf[0] * p + 1, ncf[1] * p + 1, ncf[2] * p + 1};
    const long long Nc = coarse.n_nodes(), Nf = fine.n_nodes();
    DeviceBlockVector<double> xc(nt, Nc), yf(nt, Nf), Pxc(nt, Nf), Ryf(nt, Nc);
    const auto hxc = random_block<double>(nt, nnc, rng), hyf = random_block<double>(nt, nnf, rng);
    xc.copy_from_host(hxc);
    yf.copy_from_host(hyf);
    T.prolongate(1, Pxc, xc);
    T.restrict_and_add(1, Ryf, yf);
    const double a = dot(hyf, Pxc.copy_to_host()), b = dot(Ryf.copy_to_host(), hxc);
    expect(std::abs(a - b) <= 1e-12 * std::abs(a), "h: <y, P x> = <R y, x>", a, b);
    // prolongate overwrites, prolongate_and_add adds
    T.prolongate_and_add(1, Pxc, xc);
    T.prolongate(1, yf, xc);
    {
      const auto p2 = Pxc.copy_to_host(), p1 = yf.copy_to_host();
      double     err = 0, mx = 0;
      for (std::size_t i = 0; i < p1.size(); ++i)
        {
          err = std::max(err, std::abs(p2[i] - 2 * p1[i]));
          mx  = std::max(mx, std::abs(p1[i]));
        }
      expect(err <= 1e-13 * mx, "prolongate / prolongate_and_add", err, mx);
    }
    DeviceBlockVector<double> xt(nt, Nf), yt(2 * nt, Nf), Pxt(2 * nt, Nf), Ryt(nt, Nf);
    const auto hxt = random_block<double>(nt, nnf, rng), hyt = random_block<double>(2 * nt, nnf, rng);
    xt.copy_from_host(hxt);
    yt.copy_from_host(hyt);
    T.prolongate(2, Pxt, xt);
    T.restrict_and_add(2, Ryt, yt);
    const double c = dot(hyt, Pxt.copy_to_host()), d = dot(Ryt.copy_to_host(), hxt);
    expect(std::abs(c - d) <= 1e-12 * std::abs(c), "tau: <y, P x> = <R y, x>", c, d);
    bool threw = false;
    try
      {
        T.prolongate(0, Pxc, xc);
      }
    catch (const std::exception &)
      {
        threw = true;
      }
    expect(threw, "no transfer to level 0");
  }

  // ------------------------------------------------------ DofPermutation
  {
    std::vector<long long> pi(static_cast<std::size_t>(N));
    for (long long i = 0; i < N; ++i)
      pi[std::size_t(i)] = i;
    std::shuffle(pi.begin(), pi.end(), rng);
    const int              p1 = p + 1, nd = p1 * p1 * p1;
    std::vector<long long> cell_dofs;
    for (int cz = 0; cz < nc[2]; ++cz)
      for (int cy = 0; cy < nc[1]; ++cy)
        for (int cx = 0; cx < nc[0]; ++cx)
          for (int a = 0; a < nd; ++a)
            {
              const int       ax = a % p1, ay = (a / p1) % p1, az = a / (p1 * p1);
              const long long lex = (cx * p + ax) + nn[0] * ((long long)(cy * p + ay) + nn[1] * (long long)(cz * p + az));
              cell_dofs.push_back(pi[std::size_t(lex)]);
            }
    DofPermutation            perm(dim, nc, p, cell_dofs);
    DeviceBlockVector<double> caller(nt, N), lex(nt, N), back(nt, N);
    std::vector<double>       hc(std::size_t(nt * N));
    std::normal_distribution<double> N01;
    for (auto &v : hc)
      v = N01(rng);
    caller.copy_from_host(hc);
    perm.to_lexicographic(lex, caller);
    perm.to_caller(back, lex);
    const auto hl = lex.copy_to_host(), hb = back.copy_to_host();
    bool       ok = true;
    for (int b = 0; b < nt && ok; ++b)
      for (long long i = 0; i < N; ++i)
        if (hl[std::size_t(b * N + i)] != hc[std::size_t(b * N + pi[std::size_t(i)])])
          {
            ok = false;
            break;
          }
    expect(ok, "DofPermutation::to_lexicographic");
    expect(hb == hc, "DofPermutation round trip");
  }

  if (failures == 0)
    std::printf("ALL OK\n");
  return failures == 0 ? 0 : 1;
}
