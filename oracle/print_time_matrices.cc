// Oracle (test infrastructure only): prints the time-weight and time-transfer
// matrices in the layout of the reference's known-answer programs
// tests/tp_02.cc (mode "tp_02") and tests/transfer_02.cc (mode "transfer_02"),
// so that the restatement can be diffed against tests/tp_02.output and
// tests/transfer_02.output line by line.
#include <cstring>
#include <iostream>

#include "time_fe.h"

using namespace oracle;

static void
tp02_test(TimeType type, unsigned r) // tests/tp_02.cc:32-78
{
  if (type == TimeType::CGP)
    {
      std::cout << "CG(" << r << ")" << std::endl;
      auto m = get_cg_weights(r);
      std::cout << print_formatted(m[0]) << print_formatted(m[1]);
      auto s = split_lhs_rhs(m);
      auto w = get_fe_time_weights_wave(TimeType::CGP, s[0], s[1], s[2], s[3], 1);
      std::cout << "Waves" << std::endl;
      for (auto &x : w)
        std::cout << print_formatted(x);
    }
  else
    {
      std::cout << "DG(" << r << ")" << std::endl;
      auto m = get_dg_weights(r);
      std::cout << print_formatted(m[2]) << print_formatted(m[0]) << print_formatted(m[1]);
      auto w = get_fe_time_weights_wave(TimeType::DG, m[0], m[1], m[2], DMat(), 1);
      std::cout << "Waves" << std::endl;
      for (auto &x : w)
        std::cout << print_formatted(x);
    }
}

static void
tp02_test2(TimeType type, unsigned r, unsigned n) // tests/tp_02.cc:81-105
{
  const char *t = type == TimeType::CGP ? "CG(" : "DG(";
  std::cout << t << r << ") - " << n << " timesteps in one system" << std::endl;
  auto w = get_fe_time_weights(type, r, 1.0, n);
  for (auto &x : w)
    std::cout << print_formatted(x);
  auto w1 = get_fe_time_weights(type, r, 1.0, 1);
  auto ww = get_fe_time_weights_wave(type, w1[0], w1[1], w1[2], w1[3], n);
  std::cout << "Waves " << t << r << ") - " << n << " timesteps in one system" << std::endl;
  for (auto &x : ww)
    std::cout << print_formatted(x);
}

static void
tr02_test_r(TimeType type, unsigned rs, unsigned rd, unsigned n) // tests/transfer_02.cc:40-55
{
  std::cout << "- Projection\n"
            << (type == TimeType::CGP ? "CG " : "DG ") << "From " << rs << " to " << rd
            << "\nTimesteps at once: " << n << std::endl;
  std::cout << print_formatted(get_time_projection_matrix(type, rs, rd, n));
  std::cout << std::endl;
}

static void
tr02_test_t(TimeType type, unsigned r, unsigned n = 2) // tests/transfer_02.cc:57-76
{
  const char *t = type == TimeType::CGP ? "CG(" : "DG(";
  std::cout << "- Prolongation\n" << t << r << ")" << std::endl;
  std::cout << print_formatted(get_time_prolongation_matrix(type, r, n));
  std::cout << "- Restriction\n" << t << r << ")" << std::endl;
  std::cout << print_formatted(get_time_restriction_matrix(type, r, n));
  std::cout << std::endl;
}

static void
tr02_test_tw(TimeType type, unsigned r, unsigned n = 4) // tests/transfer_02.cc:78-119
{
  std::cout << "Test MG in time operators\n";
  auto seq = get_time_mg_sequence(1, r, type == TimeType::DG ? 0 : 1, n, 1, TimeMG::k);
  auto tw  = get_fe_time_weights_levels(type, r, 0.25, n, seq);
  auto ww  = get_fe_time_weights_wave_levels(type, r, 0.25, n, seq);
  for (auto &el : tw)
    {
      std::cout << "- Alpha heat\n" << print_formatted(el[0]);
      std::cout << "- Beta heat\n" << print_formatted(el[1]);
      std::cout << "- Gamma heat\n" << print_formatted(el[2]);
      std::cout << "- Zeta heat\n" << print_formatted(el[3]);
    }
  for (auto &el : ww)
    {
      std::cout << "- Alpha wave u\n" << print_formatted(el[0]);
      std::cout << "- Beta wave u\n" << print_formatted(el[1]);
      std::cout << "- Gamma wave u\n" << print_formatted(el[2]);
      std::cout << "- Zeta wave u\n" << print_formatted(el[3]);
      std::cout << "- Gamma wave v\n" << print_formatted(el[4]);
    }
}

int
main(int argc, char **argv)
{
  const char *mode = argc > 1 ? argv[1] : "tp_02";
  if (std::strcmp(mode, "tp_02") == 0)
    {
      for (unsigned r = 1; r <= 5; ++r)
        tp02_test(TimeType::CGP, r);
      for (unsigned r = 1; r <= 5; ++r)
        tp02_test(TimeType::DG, r);
      for (unsigned n : {2u, 3u, 4u})
        {
          tp02_test2(TimeType::CGP, 1, n);
          tp02_test2(TimeType::CGP, 2, n);
          tp02_test2(TimeType::DG, 1, n);
          tp02_test2(TimeType::DG, 2, n);
        }
      return 0;
    }
  // transfer_02 (tests/transfer_02.cc:121-163); the FE_Q permutation check
  // prints nothing when it passes, and the lexicographic bases used here
  // have no permutation to get wrong.
  for (unsigned i = 1; i < 6; ++i)
    tr02_test_t(TimeType::CGP, i);
  for (unsigned i = 0; i < 6; ++i)
    tr02_test_t(TimeType::DG, i);
  for (unsigned i = 2; i < 6; ++i)
    {
      tr02_test_r(TimeType::CGP, i - 1, i, 1);
      tr02_test_r(TimeType::CGP, i, i - 1, 1);
    }
  for (unsigned i = 1; i < 6; ++i)
    {
      tr02_test_r(TimeType::DG, i - 1, i, 1);
      tr02_test_r(TimeType::DG, i, i - 1, 1);
    }
  tr02_test_r(TimeType::CGP, 1, 2, 2);
  tr02_test_r(TimeType::CGP, 2, 1, 2);
  tr02_test_r(TimeType::CGP, 2, 3, 2);
  tr02_test_r(TimeType::CGP, 3, 2, 2);
  tr02_test_r(TimeType::DG, 0, 1, 2);
  tr02_test_r(TimeType::DG, 1, 0, 2);
  tr02_test_r(TimeType::DG, 1, 2, 2);
  tr02_test_r(TimeType::DG, 2, 1, 2);
  tr02_test_t(TimeType::CGP, 1, 4);
  tr02_test_t(TimeType::CGP, 2, 4);
  tr02_test_t(TimeType::CGP, 3, 4);
  tr02_test_t(TimeType::DG, 0, 4);
  tr02_test_t(TimeType::DG, 1, 4);
  tr02_test_t(TimeType::DG, 2, 4);
  tr02_test_tw(TimeType::DG, 4, 4);
  tr02_test_tw(TimeType::CGP, 4, 4);
  return 0;
}
