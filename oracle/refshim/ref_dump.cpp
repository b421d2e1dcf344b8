// Test infrastructure only: a harness around the reference's own C++ classes.
//
// Linked against the reference's translation units compiled in place (oracle/Makefile), it
// composes ENVIRON/LOCAL (environ.cpp), NEIGHLIST (neighlist.cpp), LJTableCoulDSF (pair.cpp),
// NNPOTENTIAL_TBL (pair_nnp.cpp, network via tf_shim.cpp), BOND/ANGLE/DIHEDRAL, VERLET and
// GR/SQ (grsq.cpp) in the order of the reference's step loops (run.cpp:204-394 for the
// classical step, run.cpp:1214-1307 for the NNP force block), and writes their results as raw
// little-endian arrays in atom-id order. It is the checker for the CUDA path and the timed CPU
// baseline ("kind": "reference"); nothing in the product links it.
//
// Differences from run.cpp, all outside the reference's arithmetic:
//  * the random seed is an argument (main.cpp:16 draws it from random_device);
//  * initial velocities can be read from a file instead of ENVIRON::initV;
//  * per-thread energy/virial/KE partial sums are added in thread order after a barrier rather
//    than in a `critical` section, so that repeated runs are bit-identical;
//  * the thermostat can be switched off (scale_interval 0) for NVE parity runs;
//  * g(r) steps (gr.tally, reduce_local, SQ::compute, RMDF::compute_Qspace/Rspace/Potential,
//    run.cpp:286-299) run only when `gr_interval` is given, and RMDF only with an `rmdf` line
//    (run.cpp always constructs RMDF and needs at least one target file for it).
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "angle.h"
#include "bond.h"
#include "dihedral.h"
#include "environ.h"
#include "grsq.h"
#include "mathlib.h"
#include "memory.h"
#include "neighlist.h"
#include "pair.h"
#include "pair_nnp.h"
#include "util.h"
#include "verlet.h"

namespace {

struct Cfg {
  std::string init, vel, table, out = ".", mode = "snapshot", nnp_param, nnp_wt;
  float cutoff = 10, skin = 2, gr_cutoff = 10, nnp_cutoff = 6, qmax = 20, dt = 1, temp = 300;
  int nbin = 1000, nnp_nbin = 0, nq = 512, steps = 0, scale_interval = 0, log_interval = 1, neigh_sz = 2048;
  unsigned seed = 12345;
  bool lj = true;
  std::vector<std::vector<float>> bond, angle, dih;
  std::vector<std::string> rmdf_files;
  float rmdf_strength = 0, rmdf_gamma = 1;
  int gr_interval = 0, gr_interval_long = 0;
  int sqd_nq = 0;          // direct S(q) (SQD, grsq.cpp:362-585) of the final state when > 0
  float sqd_qmax = 0;
};

void die(const char* m) { fprintf(stderr, "ref_dump: %s\n", m); exit(2); }

Cfg parse(const char* path) {
  Cfg c;
  FILE* fp = fopen(path, "r");
  if (!fp) die("cannot open config");
  char line[1024];
  while (fgets(line, sizeof line, fp)) {
    char key[64], s1[512], s2[512];
    if (sscanf(line, "%63s", key) != 1 || key[0] == '#') continue;
    std::string k(key);
    auto fl = [&](float& v) { sscanf(line, "%*s %f", &v); };
    auto in = [&](int& v) { sscanf(line, "%*s %d", &v); };
    if (k == "init") { sscanf(line, "%*s %511s", s1); c.init = s1; }
    else if (k == "velocity") { sscanf(line, "%*s %511s", s1); c.vel = s1; }
    else if (k == "out") { sscanf(line, "%*s %511s", s1); c.out = s1; }
    else if (k == "mode") { sscanf(line, "%*s %511s", s1); c.mode = s1; }
    else if (k == "table") { sscanf(line, "%*s %d %511s", &c.nbin, s1); c.table = s1; }
    else if (k == "nnp") { sscanf(line, "%*s %f %d %511s %511s", &c.nnp_cutoff, &c.nnp_nbin, s1, s2); c.nnp_param = s1; c.nnp_wt = s2; }
    else if (k == "no_lj") c.lj = false;
    else if (k == "rmdf") {
      char f1[512] = "", f2[512] = "";
      int n = sscanf(line, "%*s %f %f %511s %511s", &c.rmdf_strength, &c.rmdf_gamma, f1, f2);
      if (n < 3) die("bad rmdf line");
      c.rmdf_files.push_back(f1);
      if (n == 4) c.rmdf_files.push_back(f2);
    } else if (k == "gr_interval") {
      if (sscanf(line, "%*s %d %d", &c.gr_interval, &c.gr_interval_long) != 2) die("bad gr_interval line");
    }
    else if (k == "sqd") { if (sscanf(line, "%*s %d %f", &c.sqd_nq, &c.sqd_qmax) != 2) die("bad sqd line"); }
    else if (k == "cutoff") fl(c.cutoff);
    else if (k == "skin") fl(c.skin);
    else if (k == "gr_cutoff") fl(c.gr_cutoff);
    else if (k == "qmax") fl(c.qmax);
    else if (k == "nq") in(c.nq);
    else if (k == "dt") fl(c.dt);
    else if (k == "temp") fl(c.temp);
    else if (k == "steps") in(c.steps);
    else if (k == "scale_interval") in(c.scale_interval);
    else if (k == "log_interval") in(c.log_interval);
    else if (k == "neigh_sz") in(c.neigh_sz);
    else if (k == "seed") { unsigned s; sscanf(line, "%*s %u", &s); c.seed = s; }
    else if (k == "bond" || k == "angle" || k == "dihedral") {
      std::vector<float> v(4, 0.f);
      int n = sscanf(line, "%*s %f %f %f %f", &v[0], &v[1], &v[2], &v[3]);
      if (n < 2) die("bad bonded line");
      (k == "bond" ? c.bond : k == "angle" ? c.angle : c.dih).push_back(v);
    } else die(("unknown key " + k).c_str());
  }
  fclose(fp);
  return c;
}

template <typename T>
void dump(const Cfg& c, const char* name, const T* p, size_t n) {
  std::string path = c.out + "/" + name;
  FILE* fp = fopen(path.c_str(), "wb");
  if (!fp) die("cannot write output");
  fwrite(p, sizeof(T), n, fp);
  fclose(fp);
}

// Per-atom arrays of the sorted state, written in atom-id order.
void dump_by_id(const Cfg& c, const char* name, numtype** a, int width) {
  std::vector<float> out((size_t)ENVIRON::natom * width);
  for (int i = 0; i < ENVIRON::natom; ++i)
    for (int d = 0; d < width; ++d) out[(size_t)ENVIRON::atom_id[i] * width + d] = (float)a[i][d];
  dump(c, name, out.data(), out.size());
}

int shift_code(int j) {
  // image of entry j: 13 for a real atom, else (sx+1)*9+(sy+1)*3+(sz+1) of the ghost shift
  if (j < ENVIRON::natom) return 13;
  numtype* g = ENVIRON::g_ghost[j - ENVIRON::natom];
  int s[3];
  for (int d = 0; d < 3; ++d) s[d] = g[d] > 0 ? 1 : (g[d] < 0 ? -1 : 0);
  return (s[0] + 1) * 9 + (s[1] + 1) * 3 + (s[2] + 1);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 2) die("usage: ref_dump <config>");
  Cfg c = parse(argv[1]);
  random_set_seed(c.seed);
  ENVIRON::initialize(c.init.c_str());
  random_set_gamma_ndof(ENVIRON::natom * 3);

  const numtype list_cut = c.lj ? c.cutoff : c.nnp_cutoff;
  const numtype comm_cutoff = c.skin + std::max((numtype)c.gr_cutoff, list_cut);
  LOCAL::set_ghost_lim(comm_cutoff);
  ENVIRON::init_grid(0.5 * (c.skin + list_cut), comm_cutoff);
  int** bin_list_pair = NEIGHLIST::build_bin_list(list_cut + c.skin, 126);
  int** bin_list_gr = NEIGHLIST::build_bin_list(c.gr_cutoff + c.skin, 8192);

  LJTableCoulDSF* pair = nullptr;
  if (c.lj) {
    pair = new LJTableCoulDSF(c.cutoff, c.nbin);
    pair->loadPotential(0, c.table.c_str());
    pair->loadPotential(1);
  }
  int nb = 0, na = 0, nd = 0;
  for (int im = 0; im < ENVIRON::nmol; ++im) {
    MOLECULE* m = ENVIRON::moltype + ENVIRON::mol_type[im];
    nb += m->n_bond; na += m->n_angle; nd += m->n_dihedral;
  }
  BOND bond((int)std::max<size_t>(c.bond.size(), 1), nb);
  for (size_t i = 0; i < c.bond.size(); ++i) bond.setParam((int)i, c.bond[i][0], 0, 0, c.bond[i][1]);
  bond.autoGenerate();
  ANGLE angle((int)std::max<size_t>(c.angle.size(), 1), na);
  for (size_t i = 0; i < c.angle.size(); ++i) angle.setParam((int)i, c.angle[i][0], c.angle[i][1], c.angle[i][2], c.angle[i][3]);
  angle.autoGenerate();
  DIHEDRAL dihedral((int)std::max<size_t>(c.dih.size(), 1), nd);
  for (size_t i = 0; i < c.dih.size(); ++i) dihedral.setParam((int)i, c.dih[i][0], c.dih[i][1], c.dih[i][2], c.dih[i][3]);
  dihedral.autoGenerate();

  NNPOTENTIAL_TBL* nnp = nullptr;
  if (!c.nnp_param.empty()) {
    nnp = new NNPOTENTIAL_TBL(c.nnp_cutoff, c.nnp_nbin, c.nnp_param.c_str(), c.nnp_wt.c_str(), &bond, &angle, &dihedral);
    nnp->allocateTable();
  }
  GR gr(c.lj ? c.nbin : c.nnp_nbin, c.gr_cutoff, list_cut);
  SQ sq(c.nq, c.qmax, &gr);
  RMDF* rmdf = nullptr;
  if (!c.rmdf_files.empty()) {
    std::vector<char*> names;
    for (auto& f : c.rmdf_files) names.push_back(const_cast<char*>(f.c_str()));
    rmdf = new RMDF((int)names.size(), names.data(), &sq, c.rmdf_strength, c.rmdf_gamma, pair, pair ? nullptr : nnp);
  }

  if (!c.vel.empty()) {
    FILE* fp = fopen(c.vel.c_str(), "rb");
    if (!fp) die("cannot open velocity file");
    std::vector<float> v((size_t)ENVIRON::natom * 3);
    if (fread(v.data(), sizeof(float), v.size(), fp) != v.size()) die("short velocity file");
    fclose(fp);
    for (int i = 0; i < ENVIRON::natom; ++i)
      for (int d = 0; d < 3; ++d) ENVIRON::v[i][d] = v[(size_t)i * 3 + d];
  } else {
    ENVIRON::initV(c.temp / 300);
  }

  const int NT = ENVIRON::NUM_THREAD;
  std::vector<double> erg_t(NT), vir_t(NT), ke_t(NT), enn_t(NT), exp_t(NT, 0.0);
  std::vector<double> log_exp;
  std::vector<int> valid_t(NT);
  std::vector<double> log_e, log_w, log_k, log_enn;
  std::vector<int> log_build;
  bool is_list_valid = true;
  double erg = 0, vir = 0, ekin = 0, enn = 0;
  long long total_pairs_full = 0;
  const bool snapshot = c.mode == "snapshot";
  const int total_steps = snapshot ? 0 : c.steps;
  double t_loop = 0;
  std::chrono::steady_clock::time_point t0;

  VERLET::setDt(-c.dt);   // run.cpp:193 undoes the first updateX with dt=-1 (its dt is fixed at 1)
#pragma omp parallel num_threads(NT)
  {
    if (omp_get_num_threads() != NT) END_PROGRAM("omp failed to start");
    const int me = omp_get_thread_num();
    LOCAL local(me);
    NEIGHLIST list_pair(me, list_cut, c.skin, c.neigh_sz, bin_list_pair);
    VERLET verlet(me);
    local.clear_vector(ENVIRON::f, 3);
#pragma omp barrier
    verlet.updateX();
#pragma omp barrier
#pragma omp single
    { VERLET::setDt(c.dt); }
#pragma omp single
    { t0 = std::chrono::steady_clock::now(); }
    for (int md_step = 0; md_step <= total_steps; ++md_step) {
      const bool f_log = !(md_step % c.log_interval) || snapshot;
      verlet.updateX();
      valid_t[me] = list_pair.isvalid();
#pragma omp barrier
#pragma omp single
      {
        is_list_valid = true;
        for (int t = 0; t < NT; ++t) is_list_valid = is_list_valid && valid_t[t];
      }
      if (!is_list_valid) {
        local.refold_and_tag();
#pragma omp barrier
#pragma omp single
        { ENVIRON::sort(); }
        local.generate_ghost();
#pragma omp barrier
#pragma omp single
        { ENVIRON::tidyup_ghost(); }
        local.update_ghost_pos<true>();
#pragma omp barrier
#pragma omp single
        { ENVIRON::sort_ghost(); }
        local.update_ghost_and_info();
#pragma omp barrier
        list_pair.build<false>();
      } else {
        local.update_ghost_pos<false>();
      }
#pragma omp barrier
      if (snapshot) {
        // full list (build<true>) of this thread's atoms, written after the step's forces
        NEIGHLIST full(me, list_cut, c.skin, c.neigh_sz, bin_list_pair);
        full.build<true>();
        std::vector<int> rec;
        for (int i = 0; i < full.n_local; ++i) {
          int ii = full.local_list[i];
          for (int k = 0; k < full.num_neigh[i]; ++k) {
            int j = full.nei_list[i][k];
            rec.push_back(ENVIRON::atom_id[ii]);
            rec.push_back(ENVIRON::atom_id[j]);
            rec.push_back(shift_code(j));
            rec.push_back(full.special[i][k]);
          }
        }
#pragma omp critical
        {
          std::string p = c.out + "/fulllist_t" + std::to_string(me) + ".i32";
          FILE* fp = fopen(p.c_str(), "wb");
          fwrite(rec.data(), sizeof(int), rec.size(), fp);
          fclose(fp);
          total_pairs_full += (long long)rec.size() / 4;
        }
        // g(r): cell-based tally to gr_cutoff (grsq.cpp:151-205) and list-based (grsq.cpp:94-149)
        gr.tally(bin_list_gr, &local);
#pragma omp barrier
#pragma omp single
        {
          std::vector<long long> cnt((size_t)ENVIRON::npair * gr.nbin_r, 0);
          for (int t = 0; t < NT; ++t)
            for (size_t k = 0; k < cnt.size(); ++k) cnt[k] += gr.gr_local[t][0][k];
          dump(c, "gr_counts.i64", cnt.data(), cnt.size());
        }
        gr.reduce_local(me);
#pragma omp barrier
        sq.compute(me);
#pragma omp barrier
#pragma omp single
        {
          dump(c, "gr.f32", gr.gr[0], (size_t)ENVIRON::npair * gr.nbin_r);
          dump(c, "sq.f32", sq.sq[0], (size_t)ENVIRON::npair * sq.nbin_q);
          dump(c, "qq.f32", sq.qq, (size_t)sq.nbin_q);
          dump(c, "rr.f32", gr.rr, (size_t)gr.nbin_r);
        }
        if (rmdf) {
          // one refinement update on this S(q): compute_Qspace, compute_Rspace, compute_Potential
          exp_t[me] = rmdf->compute_Qspace(me);
#pragma omp barrier
          if (pair) { rmdf->compute_Rspace(me); rmdf->compute_Potential(me); }
          else { rmdf->compute_Rspace_NNP(me); rmdf->compute_Potential_NNP(me); }
#pragma omp barrier
#pragma omp single
          {
            double e = 0;
            for (int t = 0; t < NT; ++t) e += exp_t[t];
            dump(c, "rmdf_erg.f64", &e, 1);
            dump(c, "rmdf_sq.f32", rmdf->sq[0], (size_t)c.rmdf_files.size() * sq.nbin_q);
            if (pair) {
              dump(c, "tbl_force.f32", pair->force[0], (size_t)ENVIRON::npair * (pair->nbin_r + 1));
              dump(c, "tbl_pot.f32", pair->potential[0], (size_t)ENVIRON::npair * (pair->nbin_r + 1));
            } else {
              dump(c, "tbl_force.f32", nnp->tbl_f_pair[0][0], (size_t)ENVIRON::npair * 4 * (nnp->nbin_r + 1));
              dump(c, "tbl_pot.f32", nnp->tbl_pair[0][0], (size_t)ENVIRON::npair * 4 * (nnp->nbin_r + 1));
            }
          }
        }
        gr.tally<true>(&list_pair);
#pragma omp barrier
#pragma omp single
        {
          std::vector<long long> cnt((size_t)ENVIRON::npair * gr.nbin_r_inner, 0);
          for (int t = 0; t < NT; ++t)
            for (int p = 0; p < ENVIRON::npair; ++p)
              for (int k = 0; k < gr.nbin_r_inner; ++k) cnt[(size_t)p * gr.nbin_r_inner + k] += gr.gr_local[t][p][k];
          dump(c, "gr_inner_counts.i64", cnt.data(), cnt.size());
        }
      }

      // g(r) step: tally, reduce, S(q), RMDF (run.cpp:286-299)
      if (!snapshot && c.gr_interval > 0 && !(md_step % c.gr_interval)) {
#pragma omp barrier
        if (md_step % c.gr_interval_long) gr.tally<true>(&list_pair);
        else gr.tally(bin_list_gr, &local);
#pragma omp barrier
        gr.reduce_local(me);
#pragma omp barrier
        sq.compute(me);
        if (rmdf) exp_t[me] = rmdf->compute_Qspace(me);
#pragma omp barrier
        if (rmdf) {
          if (pair) rmdf->compute_Rspace(me);
          else rmdf->compute_Rspace_NNP(me);
          if (f_log && c.rmdf_gamma != 1) {
            if (pair) rmdf->compute_Potential(me);
            else rmdf->compute_Potential_NNP(me);
          }
        }
      }

      // forces: the classical block (run.cpp:302-342) and/or the NNP block (run.cpp:1234-1263)
      local.clear_vector_cs(*ENVIRON::f, 3);
      numtype e_l = 0, w_l = 0, e_n = 0;
#pragma omp barrier
      if (nnp) {
        local.clear_vector_cs(*nnp->descriptor, nnp->n_descriptor);
#pragma omp barrier
        nnp->computeDescriptor(&list_pair);
      }
      if (f_log) {
        bond.compute<true>(me, &e_l, &w_l);
#pragma omp barrier
        angle.compute<true>(me, &e_l, &w_l);
#pragma omp barrier
        dihedral.compute<true>(me, &e_l, &w_l);
#pragma omp barrier
        if (pair) pair->compute<true, false>(&list_pair, &e_l, &w_l);
      } else {
        bond.compute<false>(me, nullptr, nullptr);
#pragma omp barrier
        angle.compute<false>(me, nullptr, nullptr);
#pragma omp barrier
        dihedral.compute<false>(me, nullptr, nullptr);
#pragma omp barrier
        if (pair) pair->compute<false, false>(&list_pair, nullptr, nullptr);
      }
#pragma omp barrier
      if (nnp) {
#pragma omp single
        { nnp->nnEval(); }
        nnp->evalFinalize(&local);
#pragma omp barrier
        if (snapshot) {
#pragma omp single
          {
            // bonded + LJ forces before the NNP term, for a separate check of each block
            dump_by_id(c, "f_classical.f32", ENVIRON::f, 3);
            dump(c, "desc.f32", nnp->descriptor[0], (size_t)ENVIRON::natom * nnp->n_descriptor);
            dump(c, "dedg.f32", nnp->dedg[0], (size_t)ENVIRON::natom * nnp->n_descriptor);
          }
        }
        numtype e2 = 0, w2 = 0;
        if (f_log) nnp->compute<true>(&list_pair, &e2, &w2);
        else nnp->compute<false>(&list_pair, nullptr, nullptr);
        e_n = e2; w_l += w2;
#pragma omp barrier
#pragma omp single
        {
          enn = **(nnp->tfcall->outputs);
          nnp->tfcall->clearOutput();
        }
      }
      erg_t[me] = e_l; vir_t[me] = w_l; enn_t[me] = e_n;
#pragma omp barrier
      if (snapshot) {
#pragma omp single
        { dump_by_id(c, "force.f32", ENVIRON::f, 3); }
      }
      verlet.updateV();
      if (c.scale_interval > 0 && !(md_step % c.scale_interval)) {
        ke_t[me] = verlet.computeKE();
#pragma omp barrier
#pragma omp single
        { ENVIRON::initV(c.temp / 300, 0.1); }
      } else {
        ke_t[me] = verlet.computeKE();
      }
#pragma omp barrier
#pragma omp single
      {
        if (f_log) {
          float e = 0, w = 0;
          double k = 0;
          for (int t = 0; t < NT; ++t) { e += (float)erg_t[t] + (float)enn_t[t]; w += (float)vir_t[t]; k += ke_t[t]; }
          erg = e + (nnp ? enn : 0); vir = w; ekin = k;
          log_e.push_back(erg); log_w.push_back(vir); log_k.push_back(ekin);
          log_enn.push_back(nnp ? enn : 0);
          float ex = 0;
          for (int t = 0; t < NT; ++t) ex += (float)exp_t[t];
          log_exp.push_back(ex);
          log_build.push_back((int)list_pair.nbuild);
        }
      }
    }
#pragma omp single
    { t_loop = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
  }

  dump_by_id(c, "f.f32", ENVIRON::f, 3);   // holds accelerations after updateV
  dump_by_id(c, "x.f32", ENVIRON::x, 3);
  dump_by_id(c, "v.f32", ENVIRON::v, 3);
  dump(c, "log_e.f64", log_e.data(), log_e.size());
  dump(c, "log_w.f64", log_w.data(), log_w.size());
  dump(c, "log_k.f64", log_k.data(), log_k.size());
  dump(c, "log_enn.f64", log_enn.data(), log_enn.size());
  dump(c, "log_exp.f64", log_exp.data(), log_exp.size());
  if (rmdf && !snapshot) {
    if (pair) {
      dump(c, "tbl_force.f32", pair->force[0], (size_t)ENVIRON::npair * (pair->nbin_r + 1));
      dump(c, "tbl_pot.f32", pair->potential[0], (size_t)ENVIRON::npair * (pair->nbin_r + 1));
    }
    dump(c, "rmdf_sq.f32", rmdf->sq[0], (size_t)c.rmdf_files.size() * sq.nbin_q);
  }
  int sqd_ngv = 0;
  double t_sqd = 0;
  if (c.sqd_nq > 0) {   // as run.cpp:420-432: SQD of the final positions, computed by every thread
    SQD sqd(c.sqd_nq, c.sqd_qmax);
    const auto ts = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(NT)
    { sqd.compute(omp_get_thread_num()); }
    t_sqd = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
    std::vector<int> cnt(sqd.nbin_q);
    for (int i = 0; i < sqd.nbin_q; ++i) cnt[i] = sqd.vend[i] - sqd.vbegin[i];
    dump(c, "sqd_q.f32", sqd.qq, (size_t)sqd.nbin_q);
    dump(c, "sqd_sq.f32", sqd.sq[0], (size_t)sqd.nbin_q * ENVIRON::npair);
    dump(c, "sqd_count.i32", cnt.data(), cnt.size());
    sqd.dump((c.out + "/sqd.txt").c_str(), false);
    sqd_ngv = sqd.ngv;
  }
  FILE* fp = fopen((c.out + "/info.txt").c_str(), "w");
  fprintf(fp, "natom %d\nnghost %d\nntot %d\nnum_gx %d\nnpair %d\nnbin_r %d\nnbin_r_inner %d\nnbin_q %d\n"
          "full_pairs %lld\nnbuild_last %d\nt_loop %.9f\nsteps %d\nthreads %d\nsqd_ngv %d\nt_sqd %.9f\n",
          ENVIRON::natom, ENVIRON::nghost, ENVIRON::ntot, ENVIRON::num_gx, ENVIRON::npair, gr.nbin_r,
          gr.nbin_r_inner, sq.nbin_q, total_pairs_full, log_build.empty() ? 0 : log_build.back(), t_loop,
          total_steps, NT, sqd_ngv, t_sqd);
  fclose(fp);
  return 0;
}
