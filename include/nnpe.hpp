/* nnpe.hpp — the reference's C++ classes over the C ABI of the B200 force step (nnpe.h).
 *
 * A run loop written against NNPEngine's ENVIRON / LOCAL / NEIGHLIST / LJTableCoulDSF /
 * NNPOTENTIAL_TBL / BOND / ANGLE / DIHEDRAL / VERLET / GR / SQ / RMDF (run.cpp:53-457,
 * 968-1403) compiles against these classes with the same names, constructors and methods, and
 * runs its force step on the GPU. Namespace nnpe; `using namespace nnpe;` in place of the
 * reference's headers.
 *
 * Semantics where the device differs from the reference's per-thread objects:
 *  - One context (ENVIRON::ctx) holds the whole system in HBM. Every per-thread object acts only
 *    for thread 0 (the thread id given to its constructor, or the list's); the calls of the other
 *    OpenMP threads return at once, so the reference's barriers/single/critical stay harmless.
 *  - The rebuild pipeline (refold_and_tag, sort, generate_ghost, tidyup_ghost,
 *    update_ghost_pos<true>, sort_ghost, update_ghost_and_info, build) runs as one device pass in
 *    NEIGHLIST::build; the other calls of that sequence return at once.
 *  - The force block (bond, angle, dihedral, pair and network compute, run.cpp:302-342,
 *    1217-1263) is one device evaluation: the first compute call after clear_vector_cs runs it and
 *    adds the whole energy and virial to its erg/virial (FP64 sums), the later calls add nothing,
 *    so the sum the reference forms under `critical` is the same.
 *  - g(r) tallies are exact uint64 counts; S(q) and RMDF are FP64 (float in the reference).
 *  - Errors end the process with the library's message, as END_PROGRAM does (util.cpp:117-124).
 */
#ifndef NNPE_HPP
#define NNPE_HPP
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "nnpe.h"

namespace nnpe {

using numtype = float;

inline void check(int rc, const char* what, nnpe_ctx* c) {
  if (rc) {
    std::fprintf(stderr, "%s -> %s\n", what, c ? nnpe_last_error(c) : "nnpe error");
    std::exit(EXIT_FAILURE);
  }
}

class NEIGHLIST;
class LOCAL;

/* environ.h:20-123 */
class ENVIRON {
 public:
  inline static nnpe_ctx* ctx = nullptr;
  inline static int natom = 0, npair = 0, device = 0;
  inline static numtype bl = 0, comm_cutoff = 0;
  inline static uint64_t seed = 12345;   /* the reference draws its seed from random_device */
  inline static constexpr numtype ek_T = 335.47968899917714, ev_GPa = 6.9476954570553735;
  inline static bool force_pending = true;   /* set by clear_vector_cs, cleared by the force block */

  static void initialize(const char* init_file) {
    if (!ctx) check(nnpe_create(device, &ctx), "nnpe_create", ctx);
    check(nnpe_load_system_file(ctx, init_file), "ENVIRON::initialize", ctx);
    natom = nnpe_natom(ctx);
    npair = nnpe_npair(ctx);
    double b = 0;
    nnpe_atom_info(ctx, nullptr, nullptr, &b);
    bl = (numtype)b;
  }
  /* init_grid(dx, comm_cutoff) (environ.cpp:143-155): the grid follows from the cutoffs, set up
   * when the pair list is constructed */
  static void init_grid(numtype, numtype comm) { comm_cutoff = comm; }
  static void initV(numtype tempera_rel_300, numtype fraction = 1) {
    check(nnpe_init_velocities(ctx, 300.0 * tempera_rel_300, fraction, seed++), "ENVIRON::initV", ctx);
  }
  static void sort() {}
  static void tidyup_ghost() {}
  static void sort_ghost() {}
  /* verify_grid (environ.cpp:638-683): the cell sort's invariants on the device's sort; a
   * violation ends the program as the reference's END_PROGRAM("verify_grid fail") does */
  static void verify_grid() { check(nnpe_verify_grid(ctx), "verify_grid fail", ctx); }
  static void dump(const char* xyzfile, bool append = false) {
    std::vector<float> x((size_t)natom * 3);
    std::vector<int> typ(natom);
    check(nnpe_get_positions(ctx, x.data()), "ENVIRON::dump", ctx);
    nnpe_atom_info(ctx, typ.data(), nullptr, nullptr);
    FILE* fp = std::fopen(xyzfile, append ? "a" : "w");
    if (!fp) return;
    std::fprintf(fp, "%d\nx y z w %.15e %.15e\n", natom, -0.5 * bl, 0.5 * bl);
    for (int i = 0; i < natom; ++i) std::fprintf(fp, "T%d %.15e %.15e %.15e\n", typ[i], x[3 * i], x[3 * i + 1], x[3 * i + 2]);
    std::fclose(fp);
  }
};

/* LOCAL (environ.h:125-153): the per-thread view of the rebuild; the device runs it in
 * NEIGHLIST::build */
class LOCAL {
 public:
  int thread_id;
  explicit LOCAL(int thr) : thread_id(thr) {}
  static void set_ghost_lim(numtype) {}
  void refold_and_tag() {}
  void generate_ghost() {}
  void update_ghost_and_info() {}
  template <bool tag>
  void update_ghost_pos() {
    if (!tag && thread_id == 0) check(nnpe_ghost_update(ENVIRON::ctx), "update_ghost_pos", ENVIRON::ctx);
  }
  template <typename T>
  void clear_vector(T, int = 3) {}
  template <typename T>
  void clear_vector_cs(T, int = 3) {
    if (thread_id == 0) ENVIRON::force_pending = true;
  }
};

/* neighlist.h:6-47 */
/* run.h:9-21, run.cpp:688-729: a new box length per configuration (variable-box training). setBL
 * re-derives the grid, stencils and ghost limit on the device (nnpe_set_box); the stencil it
 * returns in the reference lives on the device here, so the returned pointer is null, as
 * NEIGHLIST::build_bin_list's. */
class BL_MANAGER {
 public:
  BL_MANAGER(numtype /*grid_length*/, numtype /*ghost_cutoff*/, numtype /*list_cutoff*/) {}
  int** setBL(numtype bl) {
    check(nnpe_set_box(ENVIRON::ctx, bl), "BL_MANAGER::setBL", ENVIRON::ctx);
    ENVIRON::bl = bl;
    return nullptr;
  }
};

class NEIGHLIST {
 public:
  int thread_id, nbuild = 0;
  numtype cutoff, skin;
  int capacity;
  NEIGHLIST(int thr, numtype cf, numtype sk, int cap, int** /*bin_l*/) : thread_id(thr), cutoff(cf), skin(sk), capacity(cap) {
    if (thr != 0) return;
    const numtype gr_cut = ENVIRON::comm_cutoff > 0 ? ENVIRON::comm_cutoff - sk : cf;
    check(nnpe_setup(ENVIRON::ctx, cf, sk, gr_cut > cf ? gr_cut : cf, cap), "NEIGHLIST", ENVIRON::ctx);
  }
  /* the stencils live on the device (built by nnpe_setup) */
  static int** build_bin_list(numtype, int, numtype = 0, numtype = 0) { return nullptr; }
  template <bool full>
  int build() {
    if (thread_id != 0) return 0;
    check(nnpe_list_build(ENVIRON::ctx), "NEIGHLIST::build", ENVIRON::ctx);
    int ng = 0, nb = 0, gx = 0;
    int64_t ne = 0;
    nnpe_list_info(ENVIRON::ctx, &ng, &ne, &nb, &gx);
    nbuild = nb;
    return (int)ne;
  }
  bool isvalid() {
    if (thread_id != 0) return true;
    int v = 0;
    check(nnpe_list_isvalid(ENVIRON::ctx, &v), "NEIGHLIST::isvalid", ENVIRON::ctx);
    return v != 0;
  }
};

/* the force block: one device evaluation per step (see the header comment) */
inline void force_block(bool ev, numtype* erg, numtype* virial) {
  if (!ENVIRON::force_pending) return;
  ENVIRON::force_pending = false;
  double e = 0, w = 0;
  check(nnpe_compute_forces(ENVIRON::ctx, ev ? 1 : 0, ev ? &e : nullptr, ev ? &w : nullptr), "force block", ENVIRON::ctx);
  if (ev && erg) *erg += (numtype)e;
  if (ev && virial) *virial += (numtype)w;
}

/* BOND / ANGLE / DIHEDRAL (bond.h:6-21, angle.h:6-21, dihedral.h:4-17): coefficients are stored in
 * setParam form; the terms are generated on the device when the force field is complete */
struct Bonded {
  inline static std::vector<float> b, a, d;
  inline static int nb = 0, na = 0, nd = 0;
  inline static bool dirty = true;
  static void commit() {
    if (!dirty || !ENVIRON::ctx) return;
    dirty = false;
    check(nnpe_bonded_autogen(ENVIRON::ctx, nb, b.empty() ? nullptr : b.data(), na, a.empty() ? nullptr : a.data(), nd,
                              d.empty() ? nullptr : d.data()),
          "autoGenerate", ENVIRON::ctx);
  }
};
class BOND {
 public:
  BOND(int ntyp, int) { Bonded::nb = ntyp; Bonded::b.assign(4 * (ntyp > 0 ? ntyp : 1), 0.f); Bonded::dirty = true; }
  void setParam(int i, numtype b0, numtype ka, numtype kb, numtype kc) { nnpe_bond_coef(b0, ka, kb, kc, &Bonded::b[4 * i]); }
  void autoGenerate() { Bonded::dirty = true; }
  template <bool ev>
  void compute(int thread_id, numtype* erg, numtype* virial) {
    if (thread_id == 0) { Bonded::commit(); force_block(ev, erg, virial); }
  }
};
class ANGLE {
 public:
  ANGLE(int ntyp, int) { Bonded::na = ntyp; Bonded::a.assign(4 * (ntyp > 0 ? ntyp : 1), 0.f); Bonded::dirty = true; }
  void setParam(int i, numtype t0, numtype ka, numtype kb, numtype kc) { nnpe_angle_coef(t0, ka, kb, kc, &Bonded::a[4 * i]); }
  void autoGenerate() { Bonded::dirty = true; }
  template <bool ev>
  void compute(int thread_id, numtype* erg, numtype* virial) {
    if (thread_id == 0) { Bonded::commit(); force_block(ev, erg, virial); }
  }
};
class DIHEDRAL {
 public:
  DIHEDRAL(int ntyp, int) { Bonded::nd = ntyp; Bonded::d.assign(4 * (ntyp > 0 ? ntyp : 1), 0.f); Bonded::dirty = true; }
  void setParam(int i, numtype c0, numtype c1, numtype c2, numtype c3) { nnpe_dihedral_coef(c0, c1, c2, c3, &Bonded::d[4 * i]); }
  void autoGenerate() { Bonded::dirty = true; Bonded::commit(); }
  template <bool ev>
  void compute(int thread_id, numtype* erg, numtype* virial) {
    if (thread_id == 0) { Bonded::commit(); force_block(ev, erg, virial); }
  }
};

/* pair.h:30-54 */
class LJTableCoulDSF {
 public:
  numtype cutoff, dr, r_dr;
  int nbin_r;
  LJTableCoulDSF(numtype cf, int nbin) : cutoff(cf), dr(cf / nbin), r_dr(nbin / cf), nbin_r(nbin) {}
  /* kind 0 reads the base table; 1 (the refined copy) and 2 (no-special copy) are device-side */
  void loadPotential(int kind, const char* potfile = nullptr) {
    if (kind == 0 && potfile) check(nnpe_pair_load_table(ENVIRON::ctx, nbin_r, potfile), "loadPotential", ENVIRON::ctx);
  }
  template <bool ev, bool nsp>
  void compute(NEIGHLIST* list, numtype* erg, numtype* viral) {
    if (list->thread_id == 0) { Bonded::commit(); force_block(ev, erg, viral); }
  }
  void dumpForce(const char* fname, bool /*nsp*/, bool append = false) {
    const int P = ENVIRON::npair, nb1 = nbin_r + 1;
    std::vector<float> F((size_t)P * nb1), U((size_t)P * nb1);
    check(nnpe_pair_get_table(ENVIRON::ctx, F.data(), U.data()), "dumpForce", ENVIRON::ctx);
    FILE* fp = std::fopen(fname, append ? "a+" : "w");
    if (!fp) return;
    for (int i = 0; i < nbin_r; ++i) {
      std::fprintf(fp, "%.15e", (double)((i + .5F) * dr));
      for (int p = 0; p < P; ++p) std::fprintf(fp, " %.15e %.15e", (double)F[(size_t)p * nb1 + i], (double)U[(size_t)p * nb1 + i]);
      std::fprintf(fp, "\n");
    }
    std::fclose(fp);
  }
};

/* pair_nnp.h:54-75 (the tabulated deploy path): the descriptor, network and back-projection run on
 * the device inside the force block; computeDescriptor / nnEval / evalFinalize return at once */
class NNPOTENTIAL_TBL {
 public:
  static constexpr int n_descriptor = 20;
  numtype cutoff;
  int nbin_r;
  NNPOTENTIAL_TBL(numtype cf, int nbr, const char* paramfile, const char* wtfile, class BOND*, class ANGLE*,
                  class DIHEDRAL*)
      : cutoff(cf), nbin_r(nbr) {
    Bonded::commit();
    check(nnpe_pair_enable(ENVIRON::ctx, 0), "NNPOTENTIAL_TBL", ENVIRON::ctx);
    check(nnpe_nnp_load(ENVIRON::ctx, cf, nbr, paramfile, wtfile), "NNPOTENTIAL_TBL", ENVIRON::ctx);
  }
  void allocateTable() {}
  void computeDescriptor(NEIGHLIST*) {}
  void nnEval() {}
  void evalFinalize(LOCAL*) {}
  template <bool ev>
  void compute(NEIGHLIST* list, numtype* erg, numtype* viral) {
    if (list->thread_id == 0) force_block(ev, erg, viral);
  }
};

/* verlet.h:4-22 */
class VERLET {
 public:
  inline static numtype dt = 1;
  inline static double ekin = 0;
  int thread_id;
  explicit VERLET(int thr) : thread_id(thr) {}
  /* VERLET::setDt (verlet.cpp:18-22); the state advances in FP64 on the device */
  static void setDt(numtype d) {
    dt = d;
    if (ENVIRON::ctx) check(nnpe_verlet_setup(ENVIRON::ctx, d, 1), "VERLET::setDt", ENVIRON::ctx);
  }
  void updateX() {
    if (thread_id == 0) check(nnpe_verlet_update_x(ENVIRON::ctx, dt), "VERLET::updateX", ENVIRON::ctx);
  }
  void updateV() {
    if (thread_id == 0) check(nnpe_verlet_update_v(ENVIRON::ctx, &ekin), "VERLET::updateV", ENVIRON::ctx);
  }
  /* the kinetic energy of the last updateV (whole system on thread 0) */
  numtype computeKE() { return thread_id == 0 ? (numtype)ekin : 0; }
};

/* grsq.h:8-38 */
class GR {
 public:
  int nbin_r_inner, nbin_r;
  numtype dr;
  GR(int nbi, numtype r_max, numtype r_max_inner) : nbin_r_inner(nbi), dr(r_max_inner / nbi) {
    nbin_r = (int)(r_max * (nbi / r_max_inner));
  }
  void setup(int nq, numtype qmax) {
    check(nnpe_gr_setup(ENVIRON::ctx, nbin_r_inner, nq, qmax, 0, 0), "GR", ENVIRON::ctx);
  }
  template <bool inner>
  void tally(NEIGHLIST* list) {
    if (list->thread_id == 0) check(nnpe_gr_tally(ENVIRON::ctx, inner ? 1 : 0), "GR::tally", ENVIRON::ctx);
  }
  void tally(int**, LOCAL* local) {
    if (local->thread_id == 0) check(nnpe_gr_tally(ENVIRON::ctx, 0), "GR::tally", ENVIRON::ctx);
  }
  void reduce_local(int) {}
};
class SQ {
 public:
  int nbin_q;
  numtype q_max;
  GR* gr;
  SQ(int nq, numtype qmax, GR* g) : nbin_q(nq), q_max(qmax), gr(g) { g->setup(nq, qmax); }
  void compute(int thread_id) {
    if (thread_id == 0) check(nnpe_sq_compute(ENVIRON::ctx, 0, nullptr, nullptr), "SQ::compute", ENVIRON::ctx);
  }
};
// SQD (grsq.h:40-61): S(q) summed over reciprocal lattice vectors, of the positions at compute().
class SQD {
 public:
  int nbin_q, ngv = 0;
  numtype q_max;
  SQD(int nq, numtype qmax) : nbin_q(nq), q_max(qmax) {
    check(nnpe_sqd_setup(ENVIRON::ctx, nq, qmax, &ngv), "SQD::SQD", ENVIRON::ctx);
  }
  void compute(int thread_id) {
    if (thread_id == 0) check(nnpe_sqd_compute(ENVIRON::ctx), "SQD::compute", ENVIRON::ctx);
  }
  void dump(const char* fname, bool append = false) {
    check(nnpe_sqd_dump(ENVIRON::ctx, fname, append), "SQD::dump", ENVIRON::ctx);
  }
};
class RMDF {
 public:
  bool on;
  RMDF(int nexp, char** fexp, SQ*, numtype strength, numtype gamma, LJTableCoulDSF*, NNPOTENTIAL_TBL*) : on(nexp > 0) {
    if (on) check(nnpe_rmdf_load(ENVIRON::ctx, nexp, fexp, strength, gamma), "RMDF", ENVIRON::ctx);
  }
  numtype compute_Qspace(int thread_id) {
    double e = 0;
    if (on && thread_id == 0) check(nnpe_rmdf_step(ENVIRON::ctx, 1, &e), "RMDF::compute_Qspace", ENVIRON::ctx);
    return (numtype)e;
  }
  void compute_Rspace(int thread_id) { part(thread_id, 2); }
  void compute_Potential(int thread_id) { part(thread_id, 4); }
  void compute_Rspace_NNP(int thread_id) { part(thread_id, 2); }
  void compute_Potential_NNP(int thread_id) { part(thread_id, 4); }
  void dumpSQ(const char* fname, bool append = false) {
    if (on) check(nnpe_rmdf_dump_sq(ENVIRON::ctx, fname, append), "RMDF::dumpSQ", ENVIRON::ctx);
  }
  void loadDeltaSQ(const char* fname) {
    if (on) check(nnpe_rmdf_load_delta(ENVIRON::ctx, fname), "RMDF::loadDeltaSQ", ENVIRON::ctx);
  }

 private:
  void part(int thread_id, int bit) {
    if (on && thread_id == 0) check(nnpe_rmdf_step(ENVIRON::ctx, bit, nullptr), "RMDF", ENVIRON::ctx);
  }
};

}  // namespace nnpe
#endif /* NNPE_HPP */
