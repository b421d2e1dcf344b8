// nnpe_run: the reference's step drivers on the B200 force step.
//
//   nnpe_run classical <input-file> [--seed S] [--device D] [--fp32-state] [--no-graph]
//   nnpe_run nnp_run   <input-file> [--seed S] [--device D] [--fp32-state] [--no-graph] [--fp32-network]
//
// Reads the input files of NNPEngine's `classical` (run.cpp:53-457) and `nnp_run`
// (run.cpp:968-1403) modes line by line with the same rules (blank lines skipped, trailing
// annotations ignored, ${VAR} expanded from the environment), sets up one context through the C ABI
// (include/nnpe.h) and runs md_step = 0..total_steps as the reference's loop does: updateX, list
// check/rebuild, g(r)/S(q)/RMDF on gr_interval, forces, updateV, Andersen thermostat (fraction 0.1)
// on scale_interval with the temperature ramp, and the log line of run.cpp:376-392 on stdout. The
// output section writes the xyz, g(r), S(q), RMDF S(q) and force-table files in the reference's
// formats (environ.cpp:178-188, grsq.cpp:221-256, 324-360, 1380-1416, pair.cpp:421-437).
//
// Differences: the velocity generator is seeded (--seed; the reference seeds from random_device,
// main.cpp:16); positions and velocities advance in FP64 unless --fp32-state. A non-zero status
// from the library ends the program
// with its message, as END_PROGRAM does (util.cpp:117-124).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nnpe.h"

namespace {

constexpr int kBuf = 4096;
nnpe_ctx* g_ctx = nullptr;

[[noreturn]] void die(const char* where, const std::string& msg) {
  fprintf(stderr, "%s -> %s\n", where, msg.c_str());
  exit(EXIT_FAILURE);
}
void ok(int rc, const char* where) {
  if (rc) die(where, g_ctx ? nnpe_last_error(g_ctx) : "error");
}

bool non_empty(const char* s) {
  for (; *s; ++s)
    if (*s != ' ' && *s != '\n' && *s != '\r' && *s != '\t') return true;
  return false;
}

// fgets_non_empty + string_get_env (util.cpp:126-210): the next non-blank line with ${VAR} / $VAR
// replaced by the environment's value.
std::string next_line(FILE* fp) {
  char buf[kBuf];
  while (fgets(buf, kBuf, fp)) {
    if (!non_empty(buf)) continue;
    std::string in(buf), out;
    for (size_t i = 0; i < in.size(); ++i) {
      if (in[i] != '$') { out += in[i]; continue; }
      std::string name;
      size_t j = i + 1;
      for (; j < in.size() && in[j] != '}'; ++j)
        if (in[j] != '{') name += in[j];
      const char* v = std::getenv(name.c_str());
      if (!v) die("string_get_env", "getenv failed: " + name);
      out += v;
      i = j;
    }
    return out;
  }
  die("input", "read error (end of file)");
}

struct Opts {
  uint64_t seed = 12345;
  int device = 0;
  bool fp64 = true, graph = true, bf16 = true;
};

void dump_xyz(const char* fname, bool append, int natom, double bl, const std::vector<int>& typ,
              const std::vector<int>& mol) {
  std::vector<float> x((size_t)natom * 3);
  ok(nnpe_get_positions(g_ctx, x.data()), "dump");
  // whole molecules: every atom at the periodic image nearest its molecule's first atom
  std::vector<int> first(natom, -1);
  for (int i = 0; i < natom; ++i) {
    int& f = first[mol[i]];
    if (f < 0) f = i;
    for (int d = 0; d < 3; ++d) {
      const double dx = x[3 * i + d] - x[3 * f + d];
      x[3 * i + d] -= (float)(std::nearbyint(dx / bl) * bl);
    }
  }
  FILE* fp = fopen(fname, append ? "a" : "w");
  if (!fp) die("dump", std::string("cannot write ") + fname);
  fprintf(fp, "%d\nx y z w %.15e %.15e\n", natom, -bl / 2, bl / 2);
  for (int i = 0; i < natom; ++i) fprintf(fp, "T%d %.15e %.15e %.15e\n", typ[i], x[3 * i], x[3 * i + 1], x[3 * i + 2]);
  fclose(fp);
}

// "# num" + rows "x y_0 .. y_{n-1}", averaged with an existing file over up to 100 dumps when
// appending (GR::dump / SQ::dump, grsq.cpp:221-256, 324-360).
void dump_avg(const char* fname, bool append, const std::vector<double>& xs, std::vector<double> y, int ncol) {
  const int n = (int)xs.size();
  int num = 1;
  double factor = 1, cofactor = 0;
  FILE* fp;
  if (append && (fp = fopen(fname, "r"))) {
    if (fscanf(fp, "# %d ", &num) == 1) {
      num = std::min(num + 1, 100);
      factor = 1.0 / num;
      cofactor = 1 - factor;
      for (int i = 0; i < n; ++i) {
        double v;
        if (fscanf(fp, "%lf ", &v) != 1) break;
        for (int p = 0; p < ncol; ++p) {
          if (fscanf(fp, "%lf ", &v) != 1) break;
          y[(size_t)p * n + i] = y[(size_t)p * n + i] * factor + cofactor * v;
        }
      }
    }
    fclose(fp);
  }
  fp = fopen(fname, "w");
  if (!fp) die("dump", std::string("cannot write ") + fname);
  fprintf(fp, "# %d\n", num);
  for (int i = 0; i < n; ++i) {
    fprintf(fp, "%.15e", xs[i]);
    for (int p = 0; p < ncol; ++p) fprintf(fp, " %.15e", y[(size_t)p * n + i]);
    fprintf(fp, "\n");
  }
  fclose(fp);
}

struct Setup {
  int total_steps = 0, log_interval = 1, scale_interval = 1, gr_interval = -1, gr_interval_long = -1;
  double temp_start = 0, temp_end = 0, pair_cutoff = 10, skin = 1, gr_cutoff = 19;
  int nbin_gr = 0, nq = 0;
  double qmax = 0;
  int nbin_table = 0;
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: nnpe_run classical|nnp_run <input-file> [--seed S] [--device D] [--fp32-state] "
                    "[--no-graph] [--fp32-network]\n");
    return 2;
  }
  const std::string mode = argv[1];
  if (mode != "classical" && mode != "nnp_run") die("main", "invalid arg");   // main.cpp:18-21
  Opts o;
  for (int k = 3; k < argc; ++k) {
    std::string a = argv[k];
    if (a == "--seed" && k + 1 < argc) o.seed = std::strtoull(argv[++k], nullptr, 10);
    else if (a == "--device" && k + 1 < argc) o.device = std::atoi(argv[++k]);
    else if (a == "--fp32-state") o.fp64 = false;
    else if (a == "--no-graph") o.graph = false;
    else if (a == "--fp32-network") o.bf16 = false;
    else die("main", "unknown option " + a);
  }
  FILE* fp = fopen(argv[2], "r");
  if (!fp) die("main", std::string("cannot open ") + argv[2]);
  const bool nnp = mode == "nnp_run";
  ok(nnpe_create(o.device, &g_ctx), "nnpe_create");

  // initial configuration (ENVIRON::initialize)
  std::string l = next_line(fp);
  char name[kBuf];
  if (sscanf(l.c_str(), "%s", name) != 1) die("input", "read error (init)");
  ok(nnpe_load_system_file(g_ctx, name), "ENVIRON::initialize");
  const int natom = nnpe_natom(g_ctx), npair = nnpe_npair(g_ctx);

  Setup S;
  l = next_line(fp);
  if (sscanf(l.c_str(), "%lf %lf %lf", &S.pair_cutoff, &S.skin, &S.gr_cutoff) != 3) die("input", "read error (cutoffs)");
  fprintf(stderr, "cutoff %g %g skin %g\n", S.pair_cutoff, S.gr_cutoff, S.skin);
  ok(nnpe_setup(g_ctx, S.pair_cutoff, S.skin, S.gr_cutoff, 2048), "setup");   // NEIGH_SZ (run.h:2)

  std::vector<float> bc, ac, dc;
  int nbt = 0, nat = 0, ndt = 0;
  char potfile[kBuf], paramfile[kBuf], wtfile[kBuf];
  if (!nnp) {
    l = next_line(fp);
    if (sscanf(l.c_str(), "%d %s", &S.nbin_table, potfile) != 2) die("input", "read error (table)");
    ok(nnpe_pair_load_table(g_ctx, S.nbin_table, potfile), "LJTableCoulDSF::loadPotential");
    // bond: b0 k -> setParam(i, b0, 0, 0, k) (run.cpp:117-123)
    l = next_line(fp);
    if (sscanf(l.c_str(), "%d", &nbt) != 1) die("input", "read error (bond)");
    for (int i = 0; i < nbt; ++i) {
      double b0, k;
      l = next_line(fp);
      if (sscanf(l.c_str(), "%lf %lf", &b0, &k) != 2) die("input", "read error (bond coef)");
      float c[4];
      nnpe_bond_coef(b0, 0, 0, k, c);
      bc.insert(bc.end(), c, c + 4);
    }
    l = next_line(fp);
    if (sscanf(l.c_str(), "%d", &nat) != 1) die("input", "read error (angle)");
    for (int i = 0; i < nat; ++i) {
      double t0, a, b, c3;
      l = next_line(fp);
      if (sscanf(l.c_str(), "%lf %lf %lf %lf", &t0, &a, &b, &c3) != 4) die("input", "read error (angle coef)");
      float c[4];
      nnpe_angle_coef(t0, a, b, c3, c);
      ac.insert(ac.end(), c, c + 4);
    }
    l = next_line(fp);
    if (sscanf(l.c_str(), "%d", &ndt) != 1) die("input", "read error (dihedral)");
    for (int i = 0; i < ndt; ++i) {
      double c0, c1, c2, c3;
      l = next_line(fp);
      if (sscanf(l.c_str(), "%lf %lf %lf %lf", &c0, &c1, &c2, &c3) != 4) die("input", "read error (dihedral coef)");
      float c[4];
      nnpe_dihedral_coef(c0, c1, c2, c3, c);
      dc.insert(dc.end(), c, c + 4);
    }
    ok(nnpe_bonded_autogen(g_ctx, nbt, bc.empty() ? nullptr : bc.data(), nat, ac.empty() ? nullptr : ac.data(), ndt,
                           dc.empty() ? nullptr : dc.data()),
       "autoGenerate");
  } else {
    // nnp_run: bond/angle/dihedral type counts; coefficients come from the weight file (pair_nnp.cpp:507-512)
    l = next_line(fp);
    if (sscanf(l.c_str(), "%d", &nbt) != 1) die("input", "read error (bond)");
    l = next_line(fp);
    if (sscanf(l.c_str(), "%d", &nat) != 1) die("input", "read error (angle)");
    l = next_line(fp);
    if (sscanf(l.c_str(), "%d", &ndt) != 1) die("input", "read error (dihedral)");
    std::vector<float> zb(4 * std::max(nbt, 1), 0.f), za(4 * std::max(nat, 1), 0.f), zd(4 * std::max(ndt, 1), 0.f);
    ok(nnpe_bonded_autogen(g_ctx, nbt, zb.data(), nat, za.data(), ndt, zd.data()), "autoGenerate");
    l = next_line(fp);
    if (sscanf(l.c_str(), "%s", paramfile) != 1) die("input", "read error (paramfile)");
    l = next_line(fp);
    if (sscanf(l.c_str(), "%s", wtfile) != 1) die("input", "read error (weight file)");
    l = next_line(fp);
    if (sscanf(l.c_str(), "%d", &S.nbin_table) != 1) die("input", "read error (table bins)");
    ok(nnpe_pair_enable(g_ctx, 0), "pair");
    ok(nnpe_nnp_load(g_ctx, S.pair_cutoff, S.nbin_table, paramfile, wtfile), "NNPOTENTIAL_TBL");
    int din = 0, kind = 0;
    nnpe_nnp_info(g_ctx, &din, &kind);
    if (kind == 1) ok(nnpe_nnp_precision(g_ctx, o.bf16 ? 1 : 0), "network precision");
    fprintf(stderr, "NNP: %s\nWGT: %s\n", paramfile, wtfile);
  }

  // g(r) / S(q) / RMDF lines
  l = next_line(fp);
  if (sscanf(l.c_str(), "%d %d %lf", &S.nbin_gr, &S.nq, &S.qmax) != 3) die("input", "read error (gr/sq)");
  double strength = 0, gamma = 1;
  l = next_line(fp);
  if (sscanf(l.c_str(), "%lf %lf", &strength, &gamma) != 2) die("input", "read error (rmdf)");
  l = next_line(fp);
  int nsq = 0, used = 0;
  if (sscanf(l.c_str(), "%d %n", &nsq, &used) != 1) die("input", "read error (rmdf files)");
  if (nsq > 2) die("input", "max n_sq is 2");
  std::vector<std::string> sqfiles;
  {
    const char* p = l.c_str() + used;
    for (int i = 0; i < nsq; ++i) {
      char f[kBuf];
      int n = 0;
      if (sscanf(p, "%s %n", f, &n) != 1) die("input", "read error (rmdf file)");
      sqfiles.push_back(f);
      p += n;
    }
  }
  l = next_line(fp);
  char deltafile[kBuf];
  if (sscanf(l.c_str(), "%s", deltafile) != 1) die("input", "read error (rmdf weights)");
  l = next_line(fp);
  if (sscanf(l.c_str(), "%lf %lf", &S.temp_start, &S.temp_end) != 2) die("input", "read error (temperature)");
  l = next_line(fp);
  if (sscanf(l.c_str(), "%d %d %d %d %d", &S.total_steps, &S.log_interval, &S.scale_interval, &S.gr_interval,
             &S.gr_interval_long) < 3)
    die("input", "read error (steps)");
  if (S.gr_interval < 0) S.gr_interval = S.total_steps;
  if (S.gr_interval_long < 0) S.gr_interval_long = S.total_steps;
  if ((S.total_steps % S.log_interval) || (S.total_steps % S.scale_interval)) die("input", "bad steps");
  fprintf(stderr, "MD steps: total %d; log %d; scale %d; gr %d; long %d\n", S.total_steps, S.log_interval,
          S.scale_interval, S.gr_interval, S.gr_interval_long);

  ok(nnpe_gr_setup(g_ctx, S.nbin_gr, S.nq, S.qmax, S.gr_interval, S.gr_interval_long), "GR/SQ");
  if (nsq > 0) {
    std::vector<const char*> names;
    for (auto& f : sqfiles) names.push_back(f.c_str());
    ok(nnpe_rmdf_load(g_ctx, nsq, names.data(), strength, gamma), "RMDF");
    ok(nnpe_rmdf_load_delta(g_ctx, deltafile), "RMDF::loadDeltaSQ");
  }

  ok(nnpe_init_velocities(g_ctx, S.temp_start, 1.0, o.seed), "ENVIRON::initV");
  ok(nnpe_verlet_setup(g_ctx, 1.0, o.fp64 ? 1 : 0), "VERLET::setDt");   // dt = 1 fs (run.cpp:224)
  ok(nnpe_thermostat(g_ctx, 1, S.temp_start, S.temp_end, S.scale_interval, 0.1, o.seed + 1), "thermostat");
  ok(nnpe_set_total_steps(g_ctx, S.total_steps), "steps");

  fprintf(stderr, "%7s%18s%18s%18s%18s%10s\n", "md_step", "temp [K]", "press [GPa]", "erg [kcal/mol]", "dif [kcal/mol]",
          "nbuild");
  // md_step = 0..total_steps in blocks, printing each block's log lines as they come back
  const int block = std::max(S.log_interval, std::min(S.total_steps + 1, 1000 / S.log_interval * S.log_interval));
  std::vector<nnpe_thermo> log(block / S.log_interval + 2);
  for (int done = 0; done <= S.total_steps;) {
    const int n = std::min(block, S.total_steps + 1 - done);
    int nlog = 0;
    ok((o.graph ? nnpe_run_graph : nnpe_run)(g_ctx, n, S.log_interval, log.data(), (int)log.size(), &nlog), "MD");
    for (int k = 0; k < nlog; ++k)
      printf("%7d%18.6g%18.6g%18.6g%18.6g%10d\n", log[k].step, log[k].temperature, log[k].pressure, log[k].erg,
             log[k].erg_exp, log[k].nbuild);
    fflush(stdout);
    done += n;
  }

  // output section (run.cpp:397-454, 1357-1401)
  std::vector<int> typ(natom), mol(natom);
  double bl = 0;
  ok(nnpe_atom_info(g_ctx, typ.data(), mol.data(), &bl), "atom info");
  char f1[kBuf];
  int app = 0;
  l = next_line(fp);
  if (sscanf(l.c_str(), "%s %d", f1, &app) != 2) die("input", "read error (xyz)");
  if (f1[0] != '*') dump_xyz(f1, app, natom, bl, typ, mol);
  l = next_line(fp);
  if (sscanf(l.c_str(), "%s %d", f1, &app) != 2) die("input", "read error (gr)");
  if (f1[0] != '*') {
    const int nb = nnpe_gr_nbin(g_ctx, 0);
    std::vector<uint64_t> cnt((size_t)npair * nb);
    std::vector<double> gr((size_t)npair * nb), rr(nb);
    ok(nnpe_gr_get(g_ctx, 0, cnt.data(), gr.data()), "GR::dump");
    const double dr = S.pair_cutoff / S.nbin_gr;
    for (int i = 0; i < nb; ++i) rr[i] = (float)((i + 0.5F) * (float)dr);
    dump_avg(f1, app, rr, gr, npair);
  }
  l = next_line(fp);
  if (sscanf(l.c_str(), "%s %d", f1, &app) != 2) die("input", "read error (sq)");
  if (f1[0] != '*') {
    std::vector<double> sq((size_t)npair * S.nq), q(S.nq);
    ok(nnpe_sq_compute(g_ctx, 0, sq.data(), q.data()), "SQ::dump");
    dump_avg(f1, app, q, sq, npair);
  }
  l = next_line(fp);
  {  // file append q_max nq (run.cpp:420-432)
    float sqd_qmax = 0;
    int sqd_nq = 0;
    if (sscanf(l.c_str(), "%s %d %f %d", f1, &app, &sqd_qmax, &sqd_nq) != 4) die("input", "read error (sqd)");
    if (f1[0] != '*') {
      fprintf(stderr, "sqd = %s; append = %d\n", f1, (int)(app != 0));
      int ngv = 0;
      ok(nnpe_sqd_setup(g_ctx, sqd_nq, sqd_qmax, &ngv), "SQD::SQD");
      fprintf(stderr, "SQDIRECT::SQDIRECT %d G vecs\n", ngv);
      ok(nnpe_sqd_compute(g_ctx), "SQD::compute");
      ok(nnpe_sqd_dump(g_ctx, f1, app), "SQD::dump");
    }
  }
  l = next_line(fp);
  if (sscanf(l.c_str(), "%s %d", f1, &app) != 2) die("input", "read error (sqx)");
  if (f1[0] != '*' && nsq > 0) ok(nnpe_rmdf_dump_sq(g_ctx, f1, app), "RMDF::dumpSQ");
  if (!nnp) {
    l = next_line(fp);
    if (sscanf(l.c_str(), "%s %d", f1, &app) != 2) die("input", "read error (force)");
    if (f1[0] != '*') {
      const int nb1 = S.nbin_table + 1;
      std::vector<float> F((size_t)npair * nb1), U((size_t)npair * nb1);
      ok(nnpe_pair_get_table(g_ctx, F.data(), U.data()), "dumpForce");
      FILE* out = fopen(f1, app ? "a+" : "w");
      if (!out) die("dumpForce", std::string("cannot write ") + f1);
      const float dr = (float)S.pair_cutoff / S.nbin_table;
      for (int i = 0; i < S.nbin_table; ++i) {
        fprintf(out, "%.15e", (double)((i + .5F) * dr));
        for (int p = 0; p < npair; ++p) fprintf(out, " %.15e %.15e", (double)F[(size_t)p * nb1 + i], (double)U[(size_t)p * nb1 + i]);
        fprintf(out, "\n");
      }
      fclose(out);
    }
  }
  fclose(fp);
  nnpe_destroy(g_ctx);
  return 0;
}
