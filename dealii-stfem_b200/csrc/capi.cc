// extern "C" entry points of libstmg_cuda.so (declared in include/stmg.h).
#include <cstring>
#include <exception>
#include <string>

#include "st_operator.h"
#include "stmg_internal.h"

struct stmg_mesh_s
{
  std::unique_ptr<stmg::Mesh> m;
};
struct stmg_op_s
{
  std::unique_ptr<stmg::StOperator> op;
};

namespace stmg
{
  namespace
  {
    thread_local std::string last_error;
  }
  void
  set_last_error(const std::string &m)
  {
    last_error = m;
  }

  template <typename F>
  int
  guard(F &&f)
  {
    try
      {
        f();
        return STMG_OK;
      }
    catch (const Error &e)
      {
        last_error = e.what();
        return e.code;
      }
    catch (const std::bad_alloc &)
      {
        last_error = "host allocation failed";
        return STMG_ERR_NOMEM;
      }
    catch (const std::exception &e)
      {
        last_error = e.what();
        return STMG_ERR_ARG;
      }
  }

  const char *
  last_error_cstr()
  {
    return last_error.c_str();
  }
} // namespace stmg

using namespace stmg;

extern "C"
{
  const char *
  stmg_last_error(void)
  {
    return last_error_cstr();
  }

  int
  stmg_version(void)
  {
    return 1;
  }

  int
  stmg_mesh_create(int dim, const int *n_cells, int degree, const double *lo, const double *hi, const double *vertices,
                   int coeff_mode, const double *coeff, stmg_mesh_t *mesh)
  {
    return guard([&] {
      STMG_REQUIRE(n_cells && lo && hi && mesh, STMG_ERR_ARG, "mesh_create: null argument");
      auto h = new stmg_mesh_s;
      try
        {
          h->m = make_mesh(dim, n_cells, degree, lo, hi, vertices, coeff_mode, coeff);
        }
      catch (...)
        {
          delete h;
          throw;
        }
      *mesh = h;
    });
  }

  int
  stmg_mesh_destroy(stmg_mesh_t mesh)
  {
    return guard([&] {
      STMG_REQUIRE(mesh, STMG_ERR_HANDLE, "mesh_destroy: null handle");
      delete mesh;
    });
  }

  int
  stmg_mesh_info(stmg_mesh_t mesh, long long *n_nodes, long long *n_cells)
  {
    return guard([&] {
      STMG_REQUIRE(mesh && mesh->m, STMG_ERR_HANDLE, "mesh_info: null handle");
      if (n_nodes)
        *n_nodes = mesh->m->v.N;
      if (n_cells)
        *n_cells = mesh->m->v.ncells;
    });
  }

  int
  stmg_op_create(stmg_mesh_t mesh, int nt_out, int nt_in, const double *A, const double *B, int dtype, stmg_op_t *op)
  {
    return guard([&] {
      STMG_REQUIRE(mesh && mesh->m, STMG_ERR_HANDLE, "op_create: null mesh");
      STMG_REQUIRE(A && B && op, STMG_ERR_ARG, "op_create: null argument");
      auto h = new stmg_op_s;
      try
        {
          h->op = std::make_unique<StOperator>(mesh->m.get(), nt_out, nt_in, A, B, dtype);
        }
      catch (...)
        {
          delete h;
          throw;
        }
      *op = h;
    });
  }

  int
  stmg_op_destroy(stmg_op_t op)
  {
    return guard([&] {
      STMG_REQUIRE(op, STMG_ERR_HANDLE, "op_destroy: null handle");
      delete op;
    });
  }

  int
  stmg_op_vmult(stmg_op_t op, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(op && op->op, STMG_ERR_HANDLE, "op_vmult: null handle");
      op->op->apply(false, src, dst, false, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_op_Tvmult(stmg_op_t op, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(op && op->op, STMG_ERR_HANDLE, "op_Tvmult: null handle");
      op->op->apply(true, src, dst, false, static_cast<cudaStream_t>(stream));
    });
  }

  int
  stmg_op_vmult_add(stmg_op_t op, void *dst, const void *src, void *stream)
  {
    return guard([&] {
      STMG_REQUIRE(op && op->op, STMG_ERR_HANDLE, "op_vmult_add: null handle");
      op->op->apply(false, src, dst, true, static_cast<cudaStream_t>(stream));
    });
  }
}
