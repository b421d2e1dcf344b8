/* ORACLE (test infrastructure only): a CPU restatement of NNPEngine's short-range force step.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load this library, and
 * only as the checker. It is compiled twice from this file: ORC_REAL=float follows the
 * reference's single-precision arithmetic step by step (no FMA contraction), ORC_REAL=double
 * is the FP64 oracle against which the FP32 and BF16 device results state their errors.
 *
 * Each routine cites the reference function it restates (paths within NNPEngine's src/).
 * The restatement builds the full neighbour list (neighlist.cpp:190-331 with full=true) and
 * accumulates each ordered pair on its first atom, which gives the same pair set, forces and
 * energies as the reference's half list plus ownership rule (pair.cpp:360-411) up to
 * summation order. Parity of this file is pinned against the reference's own compiled code
 * (oracle/_ref) by the tests.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <tgmath.h>

#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL real;

#define ELECTRIC_K ((real)332.06371)
static const real SPECIAL_LJ[4] = {1, 0, 0, 0.5};
static const real SPECIAL_COUL[4] = {1, 0, 0, (real)(5 / 6.)};
#define MASK_BIN 0xFFFFFF
#define MASK_NO_CHECK (1 << 24)

typedef struct {
  int natom, ntype, npair, nmoltype, nmax;
  real bl, r_bl, h_bl;
  int *typ, *mol_id, *intra, *amoltype, *spec, *pairtype;
  real* q;
  /* grid (environ.cpp:143-155) */
  real g_dx, g_rdx, g_offset, ghost_lim;
  int num_gx, num_gxsq, num_grid;
  /* sorted real atoms then ghosts */
  int nghost, ntot;
  int* order;      /* sorted index -> atom id (ghosts: atom id of owner) */
  int* shift;      /* per sorted entry: image code 13 = none */
  int *cell, *gstart, *gend, *ggstart, *ggend;
  real* xs;        /* ntot*3 */
  int* stencil;    /* num_grid x (sw) entries, -1 terminated (bin_list) */
  int sw;
  /* full list in sorted index space */
  long* lstart;
  int* lcount;
  int* lj;
  long lsize, lcap;
  int* mol_shift;  /* per atom id: image code of x_mol (environ.cpp:461-469) */
} orc_t;

static int code_of(int sx, int sy, int sz) { return (sx + 1) * 9 + (sy + 1) * 3 + (sz + 1); }
static void shift_vec(const orc_t* o, int code, real* s) {
  int c[3] = {code / 9 - 1, (code / 3) % 3 - 1, code % 3 - 1};
  for (int d = 0; d < 3; ++d) s[d] = c[d] == 0 ? (real)0 : (c[d] > 0 ? o->bl : -o->bl);
}
static int special_of(const orc_t* o, int ia, int ja) {
  if (o->mol_id[ia] != o->mol_id[ja]) return 0;
  return o->spec[(o->amoltype[ia] * o->nmax + o->intra[ia]) * o->nmax + o->intra[ja]];
}
static real sqr(real a) { return a * a; }

orc_t* orc_create(int natom, int ntype, double bl, const int* typ, const float* q, const int* mol_id,
                  const int* intra, const int* amoltype, int nmoltype, int nmax, const int* spec) {
  orc_t* o = (orc_t*)calloc(1, sizeof(orc_t));
  o->natom = natom; o->ntype = ntype; o->nmoltype = nmoltype; o->nmax = nmax;
  o->bl = (real)bl; o->r_bl = 1 / o->bl; o->h_bl = o->bl * 0.5f;     /* ENVIRON::set_bl */
  o->typ = (int*)malloc(sizeof(int) * natom); memcpy(o->typ, typ, sizeof(int) * natom);
  o->mol_id = (int*)malloc(sizeof(int) * natom); memcpy(o->mol_id, mol_id, sizeof(int) * natom);
  o->intra = (int*)malloc(sizeof(int) * natom); memcpy(o->intra, intra, sizeof(int) * natom);
  o->amoltype = (int*)malloc(sizeof(int) * natom); memcpy(o->amoltype, amoltype, sizeof(int) * natom);
  o->spec = (int*)malloc(sizeof(int) * nmoltype * nmax * nmax);
  memcpy(o->spec, spec, sizeof(int) * nmoltype * nmax * nmax);
  o->q = (real*)malloc(sizeof(real) * natom);
  for (int i = 0; i < natom; ++i) o->q[i] = (real)q[i];
  o->pairtype = (int*)malloc(sizeof(int) * ntype * ntype);
  int n = 0;                                                          /* environ.cpp:130-138 */
  for (int i = 0; i < ntype; ++i)
    for (int j = i; j < ntype; ++j) o->pairtype[i * ntype + j] = o->pairtype[j * ntype + i] = n++;
  o->npair = n;
  o->mol_shift = (int*)calloc(natom, sizeof(int));
  return o;
}

static void free_state(orc_t* o) {
  free(o->order); free(o->shift); free(o->cell); free(o->gstart); free(o->gend); free(o->ggstart);
  free(o->ggend); free(o->xs); free(o->stencil); free(o->lstart); free(o->lcount); free(o->lj);
  o->order = o->shift = o->cell = o->gstart = o->gend = o->ggstart = o->ggend = o->stencil = o->lcount = o->lj = NULL;
  o->xs = NULL; o->lstart = NULL;
}

void orc_destroy(orc_t* o) {
  if (!o) return;
  free_state(o);
  free(o->typ); free(o->mol_id); free(o->intra); free(o->amoltype); free(o->spec); free(o->q);
  free(o->pairtype); free(o->mol_shift); free(o);
}

/* NEIGHLIST::build_bin_list (neighlist.cpp:35-168) for one cutoff, no secondary cutoffs. */
static int build_stencil(orc_t* o, real cutoff, int max_nbin) {
  int ng = o->num_gx, ngsq = o->num_gxsq;
  real t = cutoff * o->g_rdx;
  int max_d = (int)ceil(t * t);
  o->sw = max_nbin + 1;
  o->stencil = (int*)malloc(sizeof(int) * (size_t)o->num_grid * o->sw);
  for (int i = 0; i < ng; ++i)
    for (int j = 0; j < ng; ++j)
      for (int k = 0; k < ng; ++k) {
        int* il = o->stencil + (size_t)(i * ngsq + j * ng + k) * o->sw;
        int num = 0;
        for (int l = 0; l < ng; ++l) {
          int mx, mxx;
          if (l == i) { mx = 0; mxx = 1; }
          else { int tp = l > i ? l - i : i - l; if ((mx = (tp - 1) * (tp - 1)) >= max_d) continue; mxx = (tp + 1) * (tp + 1); }
          for (int m = 0; m < ng; ++m) {
            int my, mxy;
            if (m == j) { my = mx; mxy = mxx + 1; }
            else { int tp = m > j ? m - j : j - m; if ((my = mx + (tp - 1) * (tp - 1)) >= max_d) continue; mxy = mxx + (tp + 1) * (tp + 1); }
            for (int nn = 0; nn < ng; ++nn) {
              int mz, mxz;
              if (nn == k) { mz = my; mxz = mxy + 1; }
              else { int tp = nn > k ? nn - k : k - nn; if ((mz = my + (tp - 1) * (tp - 1)) >= max_d) continue; mxz = mxy + (tp + 1) * (tp + 1); }
              int index = l * ngsq + m * ng + nn;
              if (mxz < max_d) index |= MASK_NO_CHECK;
              if (num >= max_nbin) return -1;                         /* "bin_list overflow" */
              il[num++] = index;
            }
          }
        }
        il[num] = -1;
      }
  return 0;
}

static int cell_of(const orc_t* o, const real* x) {
  int ix = (int)((o->g_offset + x[0]) * o->g_rdx);                   /* environ.cpp:252-260 */
  int iy = (int)((o->g_offset + x[1]) * o->g_rdx);
  int iz = (int)((o->g_offset + x[2]) * o->g_rdx);
  if (ix < 0 || iy < 0 || iz < 0 || ix >= o->num_gx || iy >= o->num_gx || iz >= o->num_gx) return -1;
  return ix * o->num_gxsq + iy * o->num_gx + iz;
}

/* Rebuild: refold_and_tag (environ.cpp:234-262), sort (:303-362), generate_ghost (:401-442),
 * tidyup_ghost/update_ghost_pos<true>/sort_ghost (:157-176, :488-522, :364-399),
 * update_ghost_and_info (:444-485) and NEIGHLIST::build<true> (neighlist.cpp:190-331).
 * Returns 0, or -1 bad cell, -2 list overflow, -3 stencil overflow. */
int orc_rebuild(orc_t* o, const float* x_by_id, double cutoff_d, double skin_d, double comm_d, int cap, int max_nbin) {
  free_state(o);
  const int N = o->natom;
  const real cutoff = (real)cutoff_d, skin = (real)skin_d, comm = (real)comm_d;
  o->g_dx = (real)(0.5 * (skin + cutoff));
  o->g_rdx = 1 / o->g_dx;
  o->g_offset = comm + o->h_bl;
  o->num_gx = (int)ceil((o->g_offset * 2) * o->g_rdx);
  o->num_gxsq = o->num_gx * o->num_gx;
  o->num_grid = o->num_gxsq * o->num_gx;
  o->ghost_lim = o->h_bl - comm;
  if (build_stencil(o, cutoff + skin, max_nbin)) return -3;

  real* xr = (real*)malloc(sizeof(real) * 3 * N);
  int* c0 = (int*)malloc(sizeof(int) * N);
  for (int a = 0; a < N; ++a) {
    for (int d = 0; d < 3; ++d) {
      real v = (real)x_by_id[3 * a + d];
      v -= nearbyint(v * o->r_bl) * o->bl;
      xr[3 * a + d] = v;
    }
    c0[a] = cell_of(o, xr + 3 * a);
    if (c0[a] < 0) { free(xr); free(c0); return -1; }
  }
  /* stable counting sort by cell of the atom-id order */
  int G = o->num_grid;
  o->gstart = (int*)calloc(G, sizeof(int)); o->gend = (int*)calloc(G, sizeof(int));
  for (int a = 0; a < N; ++a) o->gend[c0[a]]++;
  for (int c = 0, s = 0; c < G; ++c) { o->gstart[c] = s; s += o->gend[c]; o->gend[c] = s; }
  int* pos = (int*)malloc(sizeof(int) * G);
  memcpy(pos, o->gstart, sizeof(int) * G);
  int* ord = (int*)malloc(sizeof(int) * N);
  for (int a = 0; a < N; ++a) ord[pos[c0[a]]++] = a;
  /* ghosts in (owner sorted index, shift loop) order, then stable sort by cell */
  int gcap = 27 * N + 16, ng = 0;
  int* gown = (int*)malloc(sizeof(int) * gcap);
  int* gcode = (int*)malloc(sizeof(int) * gcap);
  for (int i = 0; i < N; ++i) {
    const real* xl = xr + 3 * ord[i];
    int xs = xl[0] > o->ghost_lim ? -1 : 0, xe = xl[0] < -o->ghost_lim ? 1 : 0;
    int ys = xl[1] > o->ghost_lim ? -1 : 0, ye = xl[1] < -o->ghost_lim ? 1 : 0;
    int zs = xl[2] > o->ghost_lim ? -1 : 0, ze = xl[2] < -o->ghost_lim ? 1 : 0;
    if (xs == xe && ys == ye && zs == ze) continue;
    for (int ix = xs; ix <= xe; ++ix)
      for (int iy = ys; iy <= ye; ++iy)
        for (int iz = zs; iz <= ze; ++iz) {
          if (!ix && !iy && !iz) continue;
          gown[ng] = i; gcode[ng] = code_of(ix, iy, iz); ++ng;
        }
  }
  o->nghost = ng; o->ntot = N + ng;
  o->xs = (real*)malloc(sizeof(real) * 3 * o->ntot);
  o->order = (int*)malloc(sizeof(int) * o->ntot);
  o->shift = (int*)malloc(sizeof(int) * o->ntot);
  o->cell = (int*)malloc(sizeof(int) * o->ntot);
  for (int i = 0; i < N; ++i) {
    o->order[i] = ord[i]; o->shift[i] = 13; o->cell[i] = c0[ord[i]];
    for (int d = 0; d < 3; ++d) o->xs[3 * i + d] = xr[3 * ord[i] + d];
  }
  real* gx = (real*)malloc(sizeof(real) * 3 * (ng + 1));
  int* gc = (int*)malloc(sizeof(int) * (ng + 1));
  for (int k = 0; k < ng; ++k) {
    real s[3];
    shift_vec(o, gcode[k], s);
    for (int d = 0; d < 3; ++d) gx[3 * k + d] = o->xs[3 * gown[k] + d] + s[d];
    gc[k] = cell_of(o, gx + 3 * k);
    if (gc[k] < 0) { free(xr); free(c0); free(pos); free(ord); free(gown); free(gcode); free(gx); free(gc); return -1; }
  }
  o->ggstart = (int*)calloc(G, sizeof(int)); o->ggend = (int*)calloc(G, sizeof(int));
  for (int k = 0; k < ng; ++k) o->ggend[gc[k]]++;
  for (int c = 0, s = N; c < G; ++c) { o->ggstart[c] = s; s += o->ggend[c]; o->ggend[c] = s; }
  memcpy(pos, o->ggstart, sizeof(int) * G);
  for (int k = 0; k < ng; ++k) {
    int dst = pos[gc[k]]++;
    o->order[dst] = ord[gown[k]]; o->shift[dst] = gcode[k]; o->cell[dst] = gc[k];
    for (int d = 0; d < 3; ++d) o->xs[3 * dst + d] = gx[3 * k + d];
  }
  /* x_mol image per atom (environ.cpp:461-469): a ghost within h_bl of the representative */
  memset(o->mol_shift, 0, sizeof(int) * N);
  for (int a = 0; a < N; ++a) o->mol_shift[a] = 13;
  {
    int* rep_of_mol = (int*)malloc(sizeof(int) * N);
    for (int a = 0; a < N; ++a) if (o->intra[a] == 0) rep_of_mol[o->mol_id[a]] = a;
    for (int g = N; g < o->ntot; ++g) {
      int a = o->order[g];
      if (!o->intra[a]) continue;
      const real* xg = o->xs + 3 * g;
      const real* xp = xr + 3 * rep_of_mol[o->mol_id[a]];
      if (fabs(xg[0] - xp[0]) < o->h_bl && fabs(xg[1] - xp[1]) < o->h_bl && fabs(xg[2] - xp[2]) < o->h_bl)
        o->mol_shift[a] = o->shift[g];
    }
    free(rep_of_mol);
  }
  free(xr); free(c0); free(pos); free(ord); free(gown); free(gcode); free(gx); free(gc);

  /* full list (neighlist.cpp:190-331, full=true): real cells then ghost cells */
  const real c_s = cutoff + skin, cutsq = c_s * c_s;
  o->lstart = (long*)malloc(sizeof(long) * (N + 1));
  o->lcount = (int*)malloc(sizeof(int) * N);
  o->lcap = (long)N * cap;
  o->lj = (int*)malloc(sizeof(int) * o->lcap);
  long tot = 0;
  int overflow = 0;
  for (int i = 0; i < N; ++i) {
    o->lstart[i] = tot;
    const real *xi = o->xs + 3 * i;
    int cnt = 0;
    const int* il = o->stencil + (size_t)o->cell[i] * o->sw;
    for (int pass = 0; pass < 2; ++pass) {
      for (int b = 0; il[b] >= 0; ++b) {
        int cb = il[b] & MASK_BIN, nocheck = il[b] & MASK_NO_CHECK;
        int j0 = pass ? o->ggstart[cb] : o->gstart[cb], j1 = pass ? o->ggend[cb] : o->gend[cb];
        for (int j = j0; j < j1; ++j) {
          if (!pass && j == i) continue;
          if (!nocheck) {
            const real* xj = o->xs + 3 * j;
            real rsq = sqr(xi[0] - xj[0]) + sqr(xi[1] - xj[1]) + sqr(xi[2] - xj[2]);
            if (!(rsq < cutsq)) continue;
          }
          if (cnt < cap) o->lj[tot + cnt] = j;
          ++cnt;
        }
      }
    }
    if (cnt >= cap) overflow = 1;                                        /* "nei_list overflow" */
    o->lcount[i] = cnt < cap ? cnt : cap;
    tot += o->lcount[i];
  }
  o->lstart[N] = tot;
  o->lsize = tot;
  return overflow ? -2 : 0;
}

long orc_list_size(const orc_t* o) { return o->lsize; }
int orc_nghost(const orc_t* o) { return o->nghost; }
int orc_num_gx(const orc_t* o) { return o->num_gx; }

/* Full list as records (id_i, id_j, image, special), grouped by sorted i. */
void orc_get_list(const orc_t* o, int* rec) {
  long k = 0;
  for (int i = 0; i < o->natom; ++i)
    for (long e = o->lstart[i]; e < o->lstart[i + 1]; ++e) {
      int j = o->lj[e];
      rec[4 * k] = o->order[i];
      rec[4 * k + 1] = o->order[j];
      rec[4 * k + 2] = o->shift[j];
      rec[4 * k + 3] = special_of(o, o->order[i], o->order[j]);
      ++k;
    }
}

void orc_get_sorted(const orc_t* o, int* order, int* shift, double* xs) {
  for (int i = 0; i < o->ntot; ++i) {
    order[i] = o->order[i]; shift[i] = o->shift[i];
    for (int d = 0; d < 3; ++d) xs[3 * i + d] = (double)o->xs[3 * i + d];
  }
}

/* LJTableCoulDSF::compute<ev,false> (pair.cpp:289-419), linear interpolation, analytic DSF
 * Coulomb with erfc off (pair.cpp:190-194, 353-357, 381-385). Tables are [npair][nbin+1]. */
int orc_pair_forces(const orc_t* o, const float* Ftab, const float* Utab, int nbin, double cutoff_d,
                    double* f_by_id, double* erg, double* vir) {
  const real cutoff = (real)cutoff_d, cutsq = cutoff * cutoff;
  const real r_dr = (real)nbin / cutoff;
  const real vc = -1 / cutoff, fc = vc / cutoff;
  double e = 0, w = 0;
  for (int i = 0; i < o->natom; ++i) {
    const int ia = o->order[i];
    const real* xi = o->xs + 3 * i;
    real fx = 0, fy = 0, fz = 0;
    for (long k = o->lstart[i]; k < o->lstart[i + 1]; ++k) {
      const int j = o->lj[k], ja = o->order[j];
      const real* xj = o->xs + 3 * j;
      real dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
      real rsq = sqr(dx) + sqr(dy) + sqr(dz);
      if (!(rsq < cutsq)) continue;
      real r = sqrt(rsq);
      int p = o->pairtype[o->typ[ia] * o->ntype + o->typ[ja]];
      int s = special_of(o, ia, ja);
      real ipw1 = r * r_dr - 0.5f;
      int t1 = (int)ipw1, t2 = t1 + 1;
      real ipw2 = ipw1 - t1;
      ipw1 = 1 - ipw2;
      const float* ft = Ftab + (size_t)p * (nbin + 1);
      real fpair = ((real)ft[t1] * ipw1 + (real)ft[t2] * ipw2) * SPECIAL_LJ[s];
      real qq = o->q[ia] * o->q[ja] * ELECTRIC_K;
      fpair += qq * (1 / (r * rsq) + fc / r) * SPECIAL_COUL[s];
      fx += dx * fpair; fy += dy * fpair; fz += dz * fpair;
      const float* ut = Utab + (size_t)p * (nbin + 1);
      real u = ((real)ut[t1] * ipw1 + (real)ut[t2] * ipw2) * SPECIAL_LJ[s];
      u += qq * (1 / r + vc + fc * (cutoff - r)) * SPECIAL_COUL[s];
      e += 0.5 * (double)u;
      w += 0.5 * (double)(fpair * rsq);
    }
    f_by_id[3 * ia] += (double)fx; f_by_id[3 * ia + 1] += (double)fy; f_by_id[3 * ia + 2] += (double)fz;
  }
  *erg += e; *vir += w;
  return 0;
}

static void xmol(const orc_t* o, const int* inv, int a, real* out) {
  real s[3];
  shift_vec(o, o->mol_shift[a], s);
  const real* x = o->xs + 3 * inv[a];
  for (int d = 0; d < 3; ++d) out[d] = x[d] + s[d];
}

/* BOND/ANGLE/DIHEDRAL::compute<true> (bond.cpp:108-137, angle.cpp:245-294,
 * dihedral.cpp:403-460) on the x_mol images, coefficients already in the stored form
 * (b0,2a,b,2c) / (cos t0,2a,b,2c) / (c0-c2, c1-3c3, 4c2, 12c3). Atom indices are atom ids. */
int orc_bonded(const orc_t* o, int nb, const int* bonds, const float* bcoef, int na, const int* angles,
               const float* acoef, int nd, const int* dihs, const float* dcoef, double* f_by_id, double* erg, double* vir) {
  int* inv = (int*)malloc(sizeof(int) * o->natom);
  for (int i = 0; i < o->natom; ++i) inv[o->order[i]] = i;
  double e = 0, w = 0;
  for (int b = 0; b < nb; ++b) {
    const float* c = bcoef + 4 * bonds[3 * b];
    int a1 = bonds[3 * b + 1], a2 = bonds[3 * b + 2];
    real xi[3], xj[3];
    xmol(o, inv, a1, xi); xmol(o, inv, a2, xj);
    real dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
    real rr = sqrt(sqr(dx) + sqr(dy) + sqr(dz));
    real dr = rr - (real)c[0], bdr = (real)c[2] - dr;
    real ff = dr * ((real)c[3] + (real)c[1] * bdr * (bdr - dr)) / rr;
    dx *= ff; dy *= ff; dz *= ff;
    f_by_id[3 * a1] -= dx; f_by_id[3 * a1 + 1] -= dy; f_by_id[3 * a1 + 2] -= dz;
    f_by_id[3 * a2] += dx; f_by_id[3 * a2 + 1] += dy; f_by_id[3 * a2 + 2] += dz;
    e += 0.5f * sqr(dr) * ((real)c[1] * sqr(bdr) + (real)c[3]);
    w -= ff * rr * rr;
  }
  for (int t = 0; t < na; ++t) {
    const float* c = acoef + 4 * angles[4 * t];
    int a1 = angles[4 * t + 1], a2 = angles[4 * t + 2], a3 = angles[4 * t + 3];
    real xi[3], xj[3], xk[3];
    xmol(o, inv, a1, xi); xmol(o, inv, a2, xj); xmol(o, inv, a3, xk);
    real dx1 = xi[0] - xj[0], dy1 = xi[1] - xj[1], dz1 = xi[2] - xj[2];
    real dx2 = xk[0] - xj[0], dy2 = xk[1] - xj[1], dz2 = xk[2] - xj[2];
    real r1 = 1 / sqrt(sqr(dx1) + sqr(dy1) + sqr(dz1));
    real r2 = 1 / sqrt(sqr(dx2) + sqr(dy2) + sqr(dz2));
    dx1 *= r1; dy1 *= r1; dz1 *= r1; dx2 *= r2; dy2 *= r2; dz2 *= r2;
    real cq = dx1 * dx2 + dy1 * dy2 + dz1 * dz2;
    real dcq = cq - (real)c[0], b_dcq = (real)c[2] - dcq;
    real fe = dcq * ((real)c[3] + (real)c[1] * b_dcq * (b_dcq - dcq));
    real ff = fe * r1;
    real fx = ff * (cq * dx1 - dx2), fy = ff * (cq * dy1 - dy2), fz = ff * (cq * dz1 - dz2);
    f_by_id[3 * a1] += fx; f_by_id[3 * a1 + 1] += fy; f_by_id[3 * a1 + 2] += fz;
    f_by_id[3 * a2] -= fx; f_by_id[3 * a2 + 1] -= fy; f_by_id[3 * a2 + 2] -= fz;
    ff = fe * r2;
    fx = ff * (dx1 - cq * dx2); fy = ff * (dy1 - cq * dy2); fz = ff * (dz1 - cq * dz2);
    f_by_id[3 * a3] -= fx; f_by_id[3 * a3 + 1] -= fy; f_by_id[3 * a3 + 2] -= fz;
    f_by_id[3 * a2] += fx; f_by_id[3 * a2 + 1] += fy; f_by_id[3 * a2 + 2] += fz;
    e += 0.5f * sqr(dcq) * ((real)c[1] * sqr(b_dcq) + (real)c[3]);
  }
  for (int t = 0; t < nd; ++t) {
    const float* c = dcoef + 4 * dihs[5 * t];
    int a1 = dihs[5 * t + 1], a2 = dihs[5 * t + 2], a3 = dihs[5 * t + 3], a4 = dihs[5 * t + 4];
    real xi[3], xj[3], xk[3], xl[3];
    xmol(o, inv, a1, xi); xmol(o, inv, a2, xj); xmol(o, inv, a3, xk); xmol(o, inv, a4, xl);
    real dx1 = xi[0] - xj[0], dy1 = xi[1] - xj[1], dz1 = xi[2] - xj[2];
    real dx2 = xk[0] - xj[0], dy2 = xk[1] - xj[1], dz2 = xk[2] - xj[2];
    real dx3 = xl[0] - xk[0], dy3 = xl[1] - xk[1], dz3 = xl[2] - xk[2];
    real r_rsq2 = 1 / (sqr(dx2) + sqr(dy2) + sqr(dz2));
    real dot12 = (dx1 * dx2 + dy1 * dy2 + dz1 * dz2) * r_rsq2;
    real dot32 = (dx3 * dx2 + dy3 * dy2 + dz3 * dz2) * r_rsq2;
    dx1 -= dx2 * dot12; dy1 -= dy2 * dot12; dz1 -= dz2 * dot12;
    dx3 -= dx2 * dot32; dy3 -= dy2 * dot32; dz3 -= dz2 * dot32;
    real r1 = 1 / sqrt(sqr(dx1) + sqr(dy1) + sqr(dz1)), r3 = 1 / sqrt(sqr(dx3) + sqr(dy3) + sqr(dz3));
    dx1 *= r1; dy1 *= r1; dz1 *= r1; dx3 *= r3; dy3 *= r3; dz3 *= r3;
    real cq = dx1 * dx3 + dy1 * dy3 + dz1 * dz3;
    real ff = ((real)c[3] * cq + (real)c[2]) * cq + (real)c[1];
    r1 *= ff; r3 *= ff;
    real f1x = r1 * (cq * dx1 - dx3), f1y = r1 * (cq * dy1 - dy3), f1z = r1 * (cq * dz1 - dz3);
    real f3x = r3 * (cq * dx3 - dx1), f3y = r3 * (cq * dy3 - dy1), f3z = r3 * (cq * dz3 - dz1);
    real f2x = f1x * dot12 + f3x * dot32, f2y = f1y * dot12 + f3y * dot32, f2z = f1z * dot12 + f3z * dot32;
    f_by_id[3 * a1] += f1x; f_by_id[3 * a1 + 1] += f1y; f_by_id[3 * a1 + 2] += f1z;
    f_by_id[3 * a4] += f3x; f_by_id[3 * a4 + 1] += f3y; f_by_id[3 * a4 + 2] += f3z;
    f_by_id[3 * a2] += f2x - f1x; f_by_id[3 * a2 + 1] += f2y - f1y; f_by_id[3 * a2 + 2] += f2z - f1z;
    f_by_id[3 * a3] -= f2x + f3x; f_by_id[3 * a3 + 1] -= f2y + f3y; f_by_id[3 * a3 + 2] -= f2z + f3z;
    e += (((real)c[3] / 3 * cq + (real)c[2] / 2) * cq + (real)c[1]) * cq + (real)c[0];
  }
  free(inv);
  *erg += e; *vir += w;
  return 0;
}

/* GR (grsq.cpp:28-80) bin geometry and the cell-based tally (grsq.cpp:151-205), written as
 * +1 per ordered (real i, any j) pair; the reference's +2 for real j>i and +1 per ghost pair
 * give the same integers. Uses the current grid and a stencil for gr_cutoff+skin. */
int orc_gr_counts(orc_t* o, double gr_cutoff_d, double skin_d, int nbin_inner, double r_inner_d, int64_t* counts,
                  int* nbin_out) {
  const real r_max = (real)gr_cutoff_d, r_inner = (real)r_inner_d;
  const real dr = r_inner / nbin_inner, r_dr = nbin_inner / r_inner;
  const int nbin = (int)(r_max * r_dr);
  const real r_maxsq = sqr(nbin * dr);
  *nbin_out = nbin;
  int* saved = o->stencil; int saved_w = o->sw;
  o->stencil = NULL;
  if (build_stencil(o, r_max + (real)skin_d, 8192)) { o->stencil = saved; o->sw = saved_w; return -3; }
  memset(counts, 0, sizeof(int64_t) * (size_t)o->npair * nbin);
  for (int i = 0; i < o->natom; ++i) {
    const real* xi = o->xs + 3 * i;
    const int ti = o->typ[o->order[i]];
    const int* il = o->stencil + (size_t)o->cell[i] * o->sw;
    for (int pass = 0; pass < 2; ++pass)
      for (int b = 0; il[b] >= 0; ++b) {
        int cb = il[b] & MASK_BIN;
        int j0 = pass ? o->ggstart[cb] : o->gstart[cb], j1 = pass ? o->ggend[cb] : o->gend[cb];
        for (int j = j0; j < j1; ++j) {
          if (!pass && j == i) continue;
          const real* xj = o->xs + 3 * j;
          real rsq = sqr(xi[0] - xj[0]) + sqr(xi[1] - xj[1]) + sqr(xi[2] - xj[2]);
          if (!(rsq < r_maxsq)) continue;
          int bin = (int)(sqrt(rsq) * r_dr);
          if (bin >= nbin) continue;
          counts[(size_t)o->pairtype[ti * o->ntype + o->typ[o->order[j]]] * nbin + bin] += 1;
        }
      }
  }
  free(o->stencil);
  o->stencil = saved; o->sw = saved_w;
  return 0;
}

/* ---------------------------------------------------------------------------------------- */
/* NNP (NNPOTENTIAL_TBL, pair_nnp.cpp:433-793) and the per-atom fitting network              */
/* ---------------------------------------------------------------------------------------- */

/* Fitting network per atom of species t: din -> h1 -> h2 -> 1 with tanh; returns E_t and
 * writes dE/dG. Weight block per species: A1[din][h1] c1[h1] A2[h1][h2] c2[h2] A3[h2] c3. */
static double fit_eval(const float* w, int din, int h1, int h2, const real* G, real* dG) {
  const float *A1 = w, *c1 = A1 + (size_t)din * h1, *A2 = c1 + h1, *c2 = A2 + (size_t)h1 * h2, *A3 = c2 + h2, *c3 = A3 + h2;
  real* z1 = (real*)malloc(sizeof(real) * (h1 + h2 + h1 + h2));
  real *z2 = z1 + h1, *g1 = z2 + h2, *g2 = g1 + h1;
  for (int k = 0; k < h1; ++k) {
    real s = (real)c1[k];
    for (int d = 0; d < din; ++d) s += G[d] * (real)A1[(size_t)d * h1 + k];
    z1[k] = tanh(s);
  }
  real e = (real)c3[0];
  for (int m = 0; m < h2; ++m) {
    real s = (real)c2[m];
    for (int k = 0; k < h1; ++k) s += z1[k] * (real)A2[(size_t)k * h2 + m];
    z2[m] = tanh(s);
    e += z2[m] * (real)A3[m];
  }
  for (int m = 0; m < h2; ++m) g2[m] = (real)A3[m] * (1 - z2[m] * z2[m]);
  for (int k = 0; k < h1; ++k) {
    real s = 0;
    for (int m = 0; m < h2; ++m) s += (real)A2[(size_t)k * h2 + m] * g2[m];
    g1[k] = s * (1 - z1[k] * z1[k]);
  }
  for (int d = 0; d < din; ++d) {
    real s = 0;
    for (int k = 0; k < h1; ++k) s += (real)A1[(size_t)d * h1 + k] * g1[k];
    dG[d] = s;
  }
  free(z1);
  return (double)e;
}
static size_t fit_block(int din, int h1, int h2) { return (size_t)din * h1 + h1 + (size_t)h1 * h2 + h2 + h2 + 1; }

/* Table generation of NNPOTENTIAL_TBL (pair_nnp.cpp:521-590): pair part from coef_p and the
 * 4x20 Gaussian descriptor functions with the cutoff factor cff = 1-1/(1+(r-rc)^2). Tables:
 * pair/f_pair [npair][4][nbin+1], desc/f_desc [npair][80][nbin+1]. coef_p is modified in the
 * reference (the powers are pre-multiplied); here a local copy is used. */
void orc_nnp_tables(int npair, double cutoff_d, int nbin, const float* coef_p_in, const float* coef_w,
                    const float* coef_d, const float* coef_r, real* tp, real* tfp, real* td, real* tfd) {
  const int szd = 80, nb1 = nbin + 1;
  const real cutoff = (real)cutoff_d;
  const real dr = cutoff / nbin;
  float* cp = (float*)malloc(sizeof(float) * npair * 24);
  memcpy(cp, coef_p_in, sizeof(float) * npair * 24);
  for (int p = 0; p < npair; ++p) {
    for (int k = 0; k < 4; ++k) {
      float* c = cp + p * 24 + k * 6;
      real src2 = sqr((real)c[1] / cutoff), src6 = src2 * src2 * src2;
      real elim = -2 * (real)c[5] / cutoff - (real)c[0] * src6 * (-7 + src2 * (9 * (real)c[2] + src2 * (11 * (real)c[3] + src2 * 13 * (real)c[4])));
      real c2 = (real)c[2] * 8, c3 = (real)c[3] * 10, c4 = (real)c[4] * 12;
      real flim = ((real)c[5] / cutoff + (real)c[0] * src6 * (-6 + src2 * (c2 + src2 * (c3 + src2 * c4)))) / cutoff;
      real s2 = (real)c[1] * (real)c[1];
      real* pir = tp + ((size_t)p * 4 + k) * nb1;
      real* fir = tfp + ((size_t)p * 4 + k) * nb1;
      for (int i = 0; i < nbin; ++i) {
        real rr = (real)(dr * (i + 0.5));
        real rsq = sqr(rr);
        real sr2 = s2 / rsq, sr6 = sr2 * sr2 * sr2;
        fir[i] = ((real)c[5] / rr + (real)c[0] * sr6 * (-6 + sr2 * (c2 + sr2 * (c3 + sr2 * c4)))) / rsq - flim / rr;
        pir[i] = (real)c[5] / rr + (real)c[0] * sr6 * (-1 + sr2 * (c2 * 0.125f + sr2 * (c3 * 0.1f + sr2 * c4 * 0.08333333333333333333f))) + flim * rr + elim;
      }
      pir[nbin] = fir[nbin] = 0;
    }
    const float *w = coef_w + (size_t)p * szd, *d = coef_d + (size_t)p * szd, *r0 = coef_r + (size_t)p * szd;
    for (int i = 0; i < nbin; ++i) {
      real rr = (real)(dr * (i + 0.5));
      real cf2 = rr - cutoff;
      real rrcsq_1 = 1 + sqr(cf2);
      real cff = 1 - 1 / rrcsq_1;
      real cfr = (-2 * cff) / rr;
      cf2 /= (-.5f * rr * sqr(rrcsq_1));
      for (int k = 0; k < szd; ++k) {
        real rr0 = rr - (real)r0[k];
        real drr0 = (real)d[k] * rr0;
        real wexp = exp(drr0 * rr0) * (real)w[k];
        tfd[((size_t)p * szd + k) * nb1 + i] = wexp * (cf2 + drr0 * cfr);
        td[((size_t)p * szd + k) * nb1 + i] = wexp * cff;
      }
    }
    for (int k = 0; k < szd; ++k) td[((size_t)p * szd + k) * nb1 + nbin] = tfd[((size_t)p * szd + k) * nb1 + nbin] = 0;
  }
  free(cp);
}

static void interp_w(real r, real r_dr, int* t1, real* w1, real* w2) {
  real u = r * r_dr - 0.5f;
  *t1 = (int)u;
  *w2 = u - *t1;
  *w1 = 1 - *w2;
}

/* NNPOTENTIAL_TBL computeDescriptor (pair_nnp.cpp:625-688), network, compute<true>
 * (pair_nnp.cpp:710-793). Fitting weights: per species, din=20. Outputs by atom id. */
int orc_nnp_tbl(const orc_t* o, double cutoff_d, int nbin, const float* coef_p, const float* coef_w,
                const float* coef_d, const float* coef_r, int h1, int h2, const float* fitw,
                double* G_out, double* dEdG_out, double* f_by_id, double* e_pair, double* e_net, double* vir) {
  const int N = o->natom, nd = 20, nb1 = nbin + 1, P = o->npair;
  const real cutoff = (real)cutoff_d, cutsq = cutoff * cutoff, r_dr = nbin / cutoff;
  real* tp = (real*)malloc(sizeof(real) * P * 4 * nb1);
  real* tfp = (real*)malloc(sizeof(real) * P * 4 * nb1);
  real* td = (real*)malloc(sizeof(real) * P * 80 * nb1);
  real* tfd = (real*)malloc(sizeof(real) * P * 80 * nb1);
  orc_nnp_tables(P, cutoff_d, nbin, coef_p, coef_w, coef_d, coef_r, tp, tfp, td, tfd);
  real* G = (real*)calloc((size_t)N * nd, sizeof(real));
  real* dG = (real*)calloc((size_t)N * nd, sizeof(real));
  for (int i = 0; i < N; ++i) {
    const int ia = o->order[i];
    const real* xi = o->xs + 3 * i;
    for (long k = o->lstart[i]; k < o->lstart[i + 1]; ++k) {
      const int j = o->lj[k], ja = o->order[j];
      const real* xj = o->xs + 3 * j;
      real rsq = sqr(xi[0] - xj[0]) + sqr(xi[1] - xj[1]) + sqr(xi[2] - xj[2]);
      if (!(rsq < cutsq)) continue;
      int t1; real w1, w2;
      interp_w(sqrt(rsq), r_dr, &t1, &w1, &w2);
      int p = o->pairtype[o->typ[ia] * o->ntype + o->typ[ja]], s = special_of(o, ia, ja);
      for (int c = 0; c < nd; ++c) {
        const real* t = td + ((size_t)p * 80 + nd * s + c) * nb1;
        G[(size_t)ia * nd + c] += t[t1] * w1 + t[t1 + 1] * w2;
      }
    }
  }
  double en = 0;
  const size_t fb = fit_block(nd, h1, h2);
  for (int a = 0; a < N; ++a) en += fit_eval(fitw + fb * o->typ[a], nd, h1, h2, G + (size_t)a * nd, dG + (size_t)a * nd);
  double ep = 0, w = 0;
  for (int i = 0; i < N; ++i) {
    const int ia = o->order[i];
    const real* xi = o->xs + 3 * i;
    real fx = 0, fy = 0, fz = 0;
    for (long k = o->lstart[i]; k < o->lstart[i + 1]; ++k) {
      const int j = o->lj[k], ja = o->order[j];
      const real* xj = o->xs + 3 * j;
      real dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
      real rsq = sqr(dx) + sqr(dy) + sqr(dz);
      if (!(rsq < cutsq)) continue;
      int t1; real w1, w2;
      interp_w(sqrt(rsq), r_dr, &t1, &w1, &w2);
      int p = o->pairtype[o->typ[ia] * o->ntype + o->typ[ja]], s = special_of(o, ia, ja);
      const real* tf = tfp + ((size_t)p * 4 + s) * nb1;
      real fpair = tf[t1] * w1 + tf[t1 + 1] * w2;
      for (int c = 0; c < nd; ++c) {
        const real* t = tfd + ((size_t)p * 80 + nd * s + c) * nb1;
        fpair += (dG[(size_t)ia * nd + c] + dG[(size_t)ja * nd + c]) * (t[t1] * w1 + t[t1 + 1] * w2);
      }
      fx += dx * fpair; fy += dy * fpair; fz += dz * fpair;
      const real* tq = tp + ((size_t)p * 4 + s) * nb1;
      ep += 0.5 * (double)(tq[t1] * w1 + tq[t1 + 1] * w2);
      w += 0.5 * (double)(fpair * rsq);
    }
    f_by_id[3 * ia] += fx; f_by_id[3 * ia + 1] += fy; f_by_id[3 * ia + 2] += fz;
  }
  if (G_out) for (size_t k = 0; k < (size_t)N * nd; ++k) { G_out[k] = G[k]; dEdG_out[k] = dG[k]; }
  *e_pair += ep; *e_net += en; *vir += w;
  free(tp); free(tfp); free(td); free(tfd); free(G); free(dG);
  return 0;
}

/* d/dr of sum_c a_c * scale * y_c(r) * cff(r) for the embedding net at W1 (W1, b1, W2, b2 in a row),
 * with h and t scratch of e1 + e2 and e1 entries. */
static real emb_dedr(const float* W1, int e1, int e2, real u, real r_rc, real cff, real dcff, real scale,
                     const real* a, real* h, real* t) {
  const float *b1 = W1 + e1, *W2 = b1 + e1, *b2 = W2 + (size_t)e1 * e2;
  for (int q = 0; q < e1; ++q) { h[q] = tanh((real)W1[q] * u + (real)b1[q]); t[q] = 0; }
  real dEdr = 0;
  for (int c = 0; c < e2; ++c) {
    real z = (real)b2[c];
    for (int q = 0; q < e1; ++q) z += h[q] * (real)W2[(size_t)q * e2 + c];
    real yc = tanh(z), ac = scale * a[c];
    dEdr += ac * yc * dcff;
    real gc = ac * cff * (1 - yc * yc);
    for (int q = 0; q < e1; ++q) t[q] += gc * (real)W2[(size_t)q * e2 + c];
  }
  for (int q = 0; q < e1; ++q) dEdr += t[q] * (1 - h[q] * h[q]) * (real)W1[q] * r_rc;
  return dEdr;
}

/* Radial-embedding NNP (the network of the 96k-atom workload; no counterpart in the reference's
 * C++, whose network sits behind TF). Per neighbour species t_j an embedding net
 * u=r/rc -> e1 (tanh) -> e2 (tanh); the pair's contribution scale*y_c(r)*cff(r), with the
 * reference's cutoff factor cff = 1-1/(1+(r-rc)^2) (pair_nnp.cpp:573-584), is accumulated into
 * descriptor slot s*e2+c of atom i by special class s (the reference selects its descriptor
 * functions by special class the same way, pair_nnp.cpp:663); a per-species fitting network on
 * the 4*e2 inputs gives E_i. Forces follow the reference's back-projection (pair_nnp.cpp:753-764),
 * fpair = -dE/dr / r with dE/dr = sum_c dE/dG_i[s*e2+c] d(phi^{t_j}_c)/dr + dE/dG_j[s*e2+c]
 * d(phi^{t_i}_c)/dr: the pair sits in G_i through the net of t_j and in G_j through that of t_i.
 * Embedding block per species: W1[e1] b1[e1] W2[e1][e2] b2[e2]. */
int orc_nnp_emb(const orc_t* o, double cutoff_d, double scale_d, int e1, int e2, const float* embw, int h1, int h2,
                const float* fitw, double* G_out, double* dEdG_out, double* e_atom, double* f_by_id,
                double* e_net, double* vir) {
  const int N = o->natom, din = 4 * e2;
  const real rc = (real)cutoff_d, cutsq = rc * rc, r_rc = 1 / rc, scale = (real)scale_d;
  const size_t eb = (size_t)e1 + e1 + (size_t)e1 * e2 + e2;
  real* G = (real*)calloc((size_t)N * din, sizeof(real));
  real* dG = (real*)calloc((size_t)N * din, sizeof(real));
  double* ea_all = (double*)calloc((size_t)N, sizeof(double));
  double* w_all = (double*)calloc((size_t)N, sizeof(double));
  /* Each loop writes only the rows of its own atom i and sums them in list order, and the
   * energy and virial are summed over atoms serially afterwards: the result does not depend on
   * the thread count. */
#pragma omp parallel
  {
    real* h = (real*)malloc(sizeof(real) * (e1 + e2 + e1));
    real* t = h + e1 + e2;
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < N; ++i) {
      const int ia = o->order[i];
      const real* xi = o->xs + 3 * i;
      for (long k = o->lstart[i]; k < o->lstart[i + 1]; ++k) {
        const int j = o->lj[k], ja = o->order[j];
        const real* xj = o->xs + 3 * j;
        real rsq = sqr(xi[0] - xj[0]) + sqr(xi[1] - xj[1]) + sqr(xi[2] - xj[2]);
        if (!(rsq < cutsq)) continue;
        real r = sqrt(rsq), u = r * r_rc;
        int s = special_of(o, ia, ja);
        const float *W1 = embw + eb * o->typ[ja], *b1 = W1 + e1, *W2 = b1 + e1, *b2 = W2 + (size_t)e1 * e2;
        real cf = r - rc, cff = 1 - 1 / (1 + cf * cf);
        for (int a = 0; a < e1; ++a) h[a] = tanh((real)W1[a] * u + (real)b1[a]);
        for (int c = 0; c < e2; ++c) {
          real z = (real)b2[c];
          for (int a = 0; a < e1; ++a) z += h[a] * (real)W2[(size_t)a * e2 + c];
          G[(size_t)ia * din + s * e2 + c] += scale * tanh(z) * cff;
        }
      }
    }
    const size_t fb = fit_block(din, h1, h2);
#pragma omp for schedule(static)
    for (int a = 0; a < N; ++a)
      ea_all[a] = fit_eval(fitw + fb * o->typ[a], din, h1, h2, G + (size_t)a * din, dG + (size_t)a * din);
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < N; ++i) {
      const int ia = o->order[i];
      const real* xi = o->xs + 3 * i;
      real fx = 0, fy = 0, fz = 0;
      double wi = 0;
      for (long k = o->lstart[i]; k < o->lstart[i + 1]; ++k) {
        const int j = o->lj[k], ja = o->order[j];
        const real* xj = o->xs + 3 * j;
        real dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
        real rsq = sqr(dx) + sqr(dy) + sqr(dz);
        if (!(rsq < cutsq)) continue;
        real r = sqrt(rsq), u = r * r_rc;
        int s = special_of(o, ia, ja);
        real cf = r - rc, den = 1 + cf * cf, cff = 1 - 1 / den, dcff = 2 * cf / (den * den);
        /* dE/dr_ij: G_i holds y_{t_j}(r) and G_j holds y_{t_i}(r), both in slot s */
        real dEdr = emb_dedr(embw + eb * o->typ[ja], e1, e2, u, r_rc, cff, dcff, scale, dG + (size_t)ia * din + s * e2, h, t) +
                    emb_dedr(embw + eb * o->typ[ia], e1, e2, u, r_rc, cff, dcff, scale, dG + (size_t)ja * din + s * e2, h, t);
        real fpair = -dEdr / r;
        fx += dx * fpair; fy += dy * fpair; fz += dz * fpair;
        wi += 0.5 * (double)(fpair * rsq);
      }
      f_by_id[3 * ia] += fx; f_by_id[3 * ia + 1] += fy; f_by_id[3 * ia + 2] += fz;
      w_all[i] = wi;
    }
    free(h);
  }
  double en = 0, w = 0;
  for (int a = 0; a < N; ++a) {
    if (e_atom) e_atom[a] = ea_all[a];
    en += ea_all[a];
  }
  for (int i = 0; i < N; ++i) w += w_all[i];
  if (G_out) for (size_t k = 0; k < (size_t)N * din; ++k) { G_out[k] = G[k]; dEdG_out[k] = dG[k]; }
  *e_net += en; *vir += w;
  free(G); free(dG); free(ea_all); free(w_all);
  return 0;
}

/* S(q) of grsq.cpp:258-322: ftmx[q][r] = sin(q r) 4 pi rho dr r / q, S_p(q) = sum_r ftmx g_p(r).
 * gr here is g(r)-1 as reduce_local leaves it (grsq.cpp:218). */
void orc_sq(int natom, double bl_d, int nbin_r, double dr_d, int nq, double qmax_d, int npair, const double* gr,
            double* sq, double* qq) {
  const real bl = (real)bl_d, dr = (real)dr_d, qmax = (real)qmax_d;
  const real dq = qmax / nq;
  const real four_pi = (real)(4 * 3.141592653589793238462643383279502884);
  const real fprd = four_pi * natom / (bl * bl * bl) * dr;
  for (int i = 0; i < nq; ++i) {
    real qi = (i + .5f) * dq;
    qq[i] = (double)qi;
    for (int p = 0; p < npair; ++p) {
      real acc = 0;
      for (int j = 0; j < nbin_r; ++j) {
        real rj = (j + 0.5f) * dr;
        acc += sin(qi * rj) * fprd * rj / qi * (real)gr[(size_t)p * nbin_r + j];
      }
      sq[(size_t)p * nq + i] = (double)acc;
    }
  }
}
