// Oracle (test infrastructure only): command-line driver running the
// restated slab solve for the reference's 2-D convergence tests
// (tests/tp_01.cc with tests/json/tf01..tf08.json).
//   stmg_oracle <heat|wave> <DG|CGP> <steps_per_slab> <k0> <n_deg> <r0> <n_ref> [fp64]
// The minimum time degree is the one the reference derives from the JSON's
// feDegree (gmg.h:637-648): 0 for dG and 1 for cGP.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>

#include "solver.h"

using namespace oracle;

int
main(int argc, char **argv)
{
  if (argc < 8)
    {
      std::fprintf(stderr, "usage: %s heat|wave DG|CGP steps k0 n_deg r0 n_ref [fp64]\n", argv[0]);
      return 2;
    }
  Config c;
  c.problem       = std::strcmp(argv[1], "wave") == 0 ? Problem::wave : Problem::heat;
  c.type          = std::strcmp(argv[2], "CGP") == 0 ? TimeType::CGP : TimeType::DG;
  c.n_steps       = std::atoi(argv[3]);
  c.fe_degree_min = c.type == TimeType::DG ? 0 : 1;
  c.n_steps_min   = std::max(1, c.n_steps / 2);
  c.mg_float      = !(argc > 8 && std::strcmp(argv[8], "fp64") == 0);
  try
    {
      std::cout << convergence_report(c, std::atoi(argv[4]), std::atoi(argv[5]), std::atoi(argv[6]),
                                       std::atoi(argv[7]));
    }
  catch (const std::exception &e)
    {
      std::fprintf(stderr, "error: %s\n", e.what());
      return 1;
    }
  return 0;
}
