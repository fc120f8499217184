// Structured mesh levels (device copies of vertices and coefficients) and
// the cell tiling used by the cell-parallel kernels.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>

#include "stmg_internal.h"

namespace stmg
{
  template <typename T>
  QTab<T>
  make_qtab(int p)
  {
    const FETables &t = host_tables();
    QTab<T>         q{};
    const int       n = p + 1;
    for (int i = 0; i < n; ++i)
      {
        q.gx[i] = T(t.gx[p][i]);
        q.gw[i] = T(t.gw[p][i]);
        for (int j = 0; j < n; ++j)
          {
            q.S[i * n + j]  = T(t.S[p][i][j]);
            q.Dq[i * n + j] = T(t.Dq[p][i][j]);
          }
      }
    return q;
  }
  template QTab<float>  make_qtab<float>(int);
  template QTab<double> make_qtab<double>(int);

  std::unique_ptr<Mesh>
  make_mesh(int dim, const int *n, int p, const double *lo, const double *hi, const double *vertices, int coeff_mode,
            const double *coeff)
  {
    STMG_REQUIRE(dim == 2 || dim == 3, STMG_ERR_ARG, "dim must be 2 or 3");
    STMG_REQUIRE(p >= 1 && p <= MAX_P && (dim == 2 || p <= 4), STMG_ERR_UNSUPPORTED, "degree must be 1..5 (3-D: 1..4)");
    STMG_REQUIRE(coeff_mode >= 0 && coeff_mode <= 2, STMG_ERR_ARG, "coeff_mode must be 0, 1 or 2");
    STMG_REQUIRE(coeff_mode == 0 || coeff, STMG_ERR_ARG, "coefficient array missing");
    auto       m = std::make_unique<Mesh>();
    MeshView  &v = m->v;
    v.dim        = dim;
    v.p          = p;
    v.N          = 1;
    v.ncells     = 1;
    long long nv = 1;
    for (int d = 0; d < 3; ++d)
      {
        v.n[d]  = d < dim ? n[d] : 1;
        v.nn[d] = d < dim ? n[d] * p + 1 : 1;
        STMG_REQUIRE(v.n[d] >= 1, STMG_ERR_ARG, "cell counts must be positive");
        if (d < dim)
          {
            v.N *= v.nn[d];
            v.ncells *= v.n[d];
            nv *= v.n[d] + 1;
          }
        v.h[d] = d < dim ? (hi[d] - lo[d]) / n[d] : 1.0;
      }
    m->nd = m->nq = 1;
    for (int d = 0; d < dim; ++d)
      m->nd *= p + 1, m->nq *= p + 1;
    // vertices: uniform box unless given
    m->vert_h.resize(nv * dim);
    const int nvd[3] = {v.n[0] + 1, dim > 1 ? v.n[1] + 1 : 1, dim > 2 ? v.n[2] + 1 : 1};
    for (long long i = 0; i < nv; ++i)
      {
        const long long ijk[3] = {i % nvd[0], (i / nvd[0]) % nvd[1], i / (nvd[0] * nvd[1])};
        for (int d = 0; d < dim; ++d)
          m->vert_h[i * dim + d] = vertices ? vertices[i * dim + d] : lo[d] + (hi[d] - lo[d]) * double(ijk[d]) / n[d];
      }
    // cartesian if every vertex sits on the uniform box lattice
    v.cartesian = 1;
    if (vertices)
      for (long long i = 0; i < nv && v.cartesian; ++i)
        {
          const long long ijk[3] = {i % nvd[0], (i / nvd[0]) % nvd[1], i / (nvd[0] * nvd[1])};
          for (int d = 0; d < dim; ++d)
            {
              const double ref = lo[d] + (hi[d] - lo[d]) * double(ijk[d]) / n[d];
              if (std::abs(vertices[i * dim + d] - ref) > 1e-14 * (1.0 + std::abs(ref)))
                v.cartesian = 0;
            }
        }
    v.box = v.cartesian;
    if (coeff_mode == 2)
      v.cartesian = 0; // a coefficient varying inside cells needs quadrature
    m->vert_d.upload(m->vert_h);
    v.vert       = m->vert_d.ptr;
    v.coeff_mode = coeff_mode;
    v.coeff64    = nullptr;
    v.coeff32    = nullptr;
    if (coeff_mode)
      {
        const long long nc = coeff_mode == 1 ? v.ncells : v.ncells * m->nq;
        m->coeff_h.assign(coeff, coeff + nc);
        std::vector<float> c32(m->coeff_h.begin(), m->coeff_h.end());
        m->coeff64_d.upload(m->coeff_h);
        m->coeff32_d.upload(c32);
        v.coeff64 = m->coeff64_d.ptr;
        v.coeff32 = m->coeff32_d.ptr;
      }
    return m;
  }

  Tiling
  make_tiling(const MeshView &m, const int *T)
  {
    Tiling t{};
    t.n_tiles = 1;
    for (int d = 0; d < 3; ++d)
      {
        t.T[d]      = d < m.dim ? std::min(T[d], m.n[d]) : 1;
        t.ntiles[d] = d < m.dim ? (m.n[d] + t.T[d] - 1) / t.T[d] : 1;
        t.E[d]      = d < m.dim ? t.T[d] * m.p + 1 : 1;
        t.n_tiles *= t.ntiles[d];
      }
    // faces x0,x1 (E1 x E2), y0,y1 (E0 x E2), z0,z1 (E0 x E1)
    const long long len[3] = {(long long)t.E[1] * t.E[2], (long long)t.E[0] * t.E[2], (long long)t.E[0] * t.E[1]};
    long long       off    = 0;
    for (int f = 0; f < 6; ++f)
      {
        const int d   = f / 2;
        t.face_len[f] = d < m.dim ? len[d] : 0;
        t.face_off[f] = off;
        off += t.face_len[f];
      }
    t.tile_stride = off;
    return t;
  }

  int
  sm_count()
  {
    static int n = [] {
      int dev = 0, c = 0;
      STMG_CUDA(cudaGetDevice(&dev));
      STMG_CUDA(cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev));
      return c;
    }();
    return n;
  }

  unsigned
  persistent_grid(const void *kernel, int block, std::size_t smem, long long work)
  {
    // the dynamic shared-memory limit is a per-kernel attribute: keep it at
    // the largest size any caller needs
    static std::mutex                                              mu;
    static std::map<const void *, std::size_t>                     limit;
    static std::map<std::pair<const void *, std::size_t>, int>     cache;
    int                                                            per_sm = 0;
    std::lock_guard<std::mutex>                                    lk(mu);
    std::size_t                                                   &lim = limit[kernel];
    if (smem > lim)
      {
        STMG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        lim = smem;
      }
    auto it = cache.find({kernel, smem});
    if (it == cache.end())
      {
        STMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem));
        STMG_REQUIRE(per_sm > 0, STMG_ERR_UNSUPPORTED, "kernel does not fit on a multiprocessor");
        cache[{kernel, smem}] = per_sm;
      }
    else
      per_sm = it->second;
    const long long g = std::min<long long>(work, (long long)per_sm * sm_count());
    return unsigned(std::max<long long>(g, 1));
  }
} // namespace stmg
