// Test program: the classical step loop of run.cpp:204-394 written against the reference's classes
// as nnpe.hpp provides them (one thread, NVE, no g(r) steps), for a water box:
//   adapter_loop <init-file> <table-file> <total_steps> <log_interval> <positions-out> [sqd-out]
// Prints the log lines of run.cpp:383-390 and writes the final positions (float32, atom-id order);
// with sqd-out, the direct S(q) of the final state to 6 A^-1 on 60 points (run.cpp:420-432).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "nnpe.hpp"

using namespace nnpe;

int main(int argc, char** argv) {
  if (argc != 6 && argc != 7) return 2;
  const int total_steps = std::atoi(argv[3]), log_interval = std::atoi(argv[4]);
  const numtype pair_cutoff = 10, skin = 2, gr_cutoff = 10;
  ENVIRON::initialize(argv[1]);
  const numtype comm_cutoff = skin + (gr_cutoff > pair_cutoff ? gr_cutoff : pair_cutoff);
  LOCAL::set_ghost_lim(comm_cutoff);
  ENVIRON::init_grid(0.5f * (skin + pair_cutoff), comm_cutoff);
  int** bin_list_pair = NEIGHLIST::build_bin_list(pair_cutoff + skin, 126);
  LJTableCoulDSF pair(pair_cutoff, 1000);
  BOND bond(1, 0);
  bond.setParam(0, 1.0f, 0, 0, 450.0f);
  bond.autoGenerate();
  ANGLE angle(1, 0);
  angle.setParam(0, 109.47f, 0, 0, 62.0f);
  angle.autoGenerate();
  DIHEDRAL dihedral(0, 0);
  dihedral.autoGenerate();
  ENVIRON::initV(0);
  LOCAL local(0);
  NEIGHLIST list_pair(0, pair_cutoff, skin, 2048, bin_list_pair);
  pair.loadPotential(0, argv[2]);
  pair.loadPotential(1);
  VERLET::setDt(-1);
  VERLET verlet(0);
  local.clear_vector(nullptr, 3);
  verlet.updateX();
  VERLET::setDt(1);
  double erg = 0, virial = 0, ekin = 0;
  for (int md_step = 0; md_step <= total_steps; ++md_step) {
    const bool f_log = !(md_step % log_interval);
    verlet.updateX();
    if (!list_pair.isvalid()) {
      local.refold_and_tag();
      ENVIRON::sort();
      local.generate_ghost();
      ENVIRON::tidyup_ghost();
      local.update_ghost_pos<true>();
      ENVIRON::sort_ghost();
      local.update_ghost_and_info();
      list_pair.build<false>();
    } else {
      local.update_ghost_pos<false>();
    }
    local.clear_vector_cs(nullptr, 3);
    numtype e = 0, w = 0;
    if (f_log) {
      bond.compute<true>(0, &e, &w);
      angle.compute<true>(0, &e, &w);
      dihedral.compute<true>(0, &e, &w);
      pair.compute<true, false>(&list_pair, &e, &w);
      erg = e;
      virial = w;
    } else {
      bond.compute<false>(0, nullptr, nullptr);
      angle.compute<false>(0, nullptr, nullptr);
      dihedral.compute<false>(0, nullptr, nullptr);
      pair.compute<false, false>(&list_pair, nullptr, nullptr);
    }
    verlet.updateV();
    ekin = verlet.computeKE();
    if (f_log) {
      const double temperature = ekin / ENVIRON::natom * ENVIRON::ek_T;
      const double press = (virial + ekin * 2) / 3 * ENVIRON::ev_GPa / ((double)ENVIRON::bl * ENVIRON::bl * ENVIRON::bl);
      std::printf("%7d%18.6e%18.6e%18.6e%18.6e%10d\n", md_step, temperature, press, erg, 0.0, list_pair.nbuild);
    }
  }
  std::vector<float> x((size_t)ENVIRON::natom * 3);
  nnpe_get_positions(ENVIRON::ctx, x.data());
  FILE* fp = std::fopen(argv[5], "wb");
  std::fwrite(x.data(), sizeof(float), x.size(), fp);
  std::fclose(fp);
  if (argc == 7) {
    SQD sqd(60, 6.0f);
    sqd.compute(0);
    sqd.dump(argv[6]);
  }
  nnpe_destroy(ENVIRON::ctx);
  return 0;
}
