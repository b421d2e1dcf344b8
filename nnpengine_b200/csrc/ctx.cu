// Context lifetime, system/table/topology upload, grid and stencil set-up, state export.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <random>
#include <mutex>
#include <unordered_map>
#include <string>
#include <vector>

#include "internal.cuh"

int nnpe_fail(nnpe_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int nnpe_sm_count(int device) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  return n > 0 ? n : 148;
}

static std::mutex g_alloc_mu;
static std::unordered_map<void*, std::pair<nnpe_ctx*, size_t>> g_allocs;

cudaError_t dev_malloc(nnpe_ctx* c, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    g_allocs[*p] = {c, bytes};
    c->dev_bytes += (int64_t)bytes;
  }
  return e;
}

void dev_free(void* p) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    auto it = g_allocs.find(p);
    if (it != g_allocs.end()) {
      it->second.first->dev_bytes -= (int64_t)it->second.second;
      g_allocs.erase(it);
    }
  }
  cudaFree(p);
}

template <typename T>
static int dalloc(nnpe_ctx* c, T** p, size_t n) {
  if (*p) { dev_free(*p); *p = nullptr; }
  if (n == 0) n = 1;
  NNPE_CUDA(c, dev_malloc(c, (void**)p, n * sizeof(T)));
  return 0;
}
template <typename T>
static void dfree(T** p) {
  if (*p) dev_free(*p);
  *p = nullptr;
}
#define TRY(x) do { int rc_ = (x); if (rc_) return rc_; } while (0)

// API functions below take C linkage from their declarations in nnpe.h.

int nnpe_create(int device, nnpe_ctx** out) {
  if (!out) return NNPE_EARG;
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return NNPE_ECUDA;
  auto* c = new nnpe_ctx();
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return NNPE_ECUDA; }
  if (dev_malloc(c, (void**)&c->d_ctrl, sizeof(int) * CTRL_WORDS) != cudaSuccess ||
      cudaMallocHost(&c->h_ctrl, sizeof(int) * CTRL_WORDS) != cudaSuccess ||
      dev_malloc(c, (void**)&c->d_red, sizeof(double) * 16) != cudaSuccess ||
      dev_malloc(c, (void**)&c->d_red_part, sizeof(double) * 4 * 256) != cudaSuccess ||
      cudaMallocHost(&c->h_red, sizeof(double) * 16) != cudaSuccess) {
    delete c;
    return NNPE_ECUDA;
  }
  cudaMemsetAsync(c->d_ctrl, 0, sizeof(int) * CTRL_WORDS, c->stream);
  cudaMemsetAsync(c->d_red, 0, sizeof(double) * 16, c->stream);
  *out = c;
  return NNPE_OK;
}

static void free_graphs(nnpe_ctx* c) {
  for (auto& g : c->graph_exec)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto& g : c->fs_graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  c->graph_valid = false;
  c->fs_valid = false;
}

static void free_state(nnpe_ctx* c) {
  free_graphs(c);
  dfree(&c->d_xd); dfree(&c->d_vd); dfree(&c->d_acc); dfree(&c->d_frc); dfree(&c->d_pos); dfree(&c->d_xbuild);
  dfree(&c->d_info); dfree(&c->d_cell); dfree(&c->d_atom_id); dfree(&c->d_sorted_of_id); dfree(&c->d_qm);
  dfree(&c->d_gowner); dfree(&c->d_gshift); dfree(&c->d_ccount); dfree(&c->d_cstart); dfree(&c->d_cend);
  dfree(&c->d_gccount); dfree(&c->d_gcstart); dfree(&c->d_gcend); dfree(&c->d_slot); dfree(&c->d_ctmp);
  dfree(&c->d_perm); dfree(&c->d_gcnt); dfree(&c->d_goff); dfree(&c->d_gtmp_owner); dfree(&c->d_gtmp_shift);
  dfree(&c->d_gtmp_cell); dfree(&c->d_gtmp_slot); dfree(&c->d_sxd); dfree(&c->d_svd); dfree(&c->d_sacc);
  dfree(&c->d_sinfo); dfree(&c->d_satom); dfree(&c->d_sqm); dfree(&c->d_list); dfree(&c->d_ncount);
  dfree(&c->d_plist); dfree(&c->d_pcount); dfree(&c->d_xprune);
  dfree(&c->d_eatom); dfree(&c->d_watom); dfree(&c->d_kin); dfree(&c->d_log);
  dfree(&c->d_xstage); dfree(&c->d_fstage);
  c->force_step_init = false;
  dfree(&c->st_pair.rows); dfree(&c->st_pair.nrows); dfree(&c->st_gr.rows); dfree(&c->st_gr.nrows);
}

void nnpe_destroy(nnpe_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_state(c);
  nnp_free(c);
  rmdf_free(c);
  sqd_free(c);
  dfree(&c->d_table); dfree(&c->d_bond); dfree(&c->d_angle); dfree(&c->d_dih); dfree(&c->d_bcoef);
  dfree(&c->d_acoef); dfree(&c->d_dcoef); dfree(&c->d_mol_terms); dfree(&c->d_mol_atoms); dfree(&c->d_molshift);
  dfree(&c->d_mol_rep); dfree(&c->d_special); dfree(&c->d_pairtype); dfree(&c->d_emol); dfree(&c->d_wmol);
  dfree(&c->d_gr_counts); dfree(&c->d_gr_counts_inner); dfree(&c->d_gr); dfree(&c->d_sq); dfree(&c->d_gr_norm);
  dfree(&c->d_qq); dfree(&c->d_ctrl); dfree(&c->d_red); dfree(&c->d_red_part); dfree(&c->d_xstage); dfree(&c->d_fstage);
  if (c->h_ctrl) cudaFreeHost(c->h_ctrl);
  if (c->h_red) cudaFreeHost(c->h_red);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* nnpe_last_error(const nnpe_ctx* c) { return c ? c->err.c_str() : "null context"; }

int nnpe_device_bytes(const nnpe_ctx* c, int64_t* bytes) {
  if (!c || !bytes) return NNPE_EARG;
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  *bytes = c->dev_bytes;
  return NNPE_OK;
}
void* nnpe_stream(nnpe_ctx* c) { return c ? (void*)c->stream : nullptr; }
int nnpe_natom(const nnpe_ctx* c) { return c ? c->natom : 0; }
int nnpe_npair(const nnpe_ctx* c) { return c ? c->npair : 0; }

int nnpe_device_errors(nnpe_ctx* c, int* bits) {
  if (!c || !bits) return NNPE_EARG;
  NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  *bits = c->h_ctrl[CTRL_ERR];
  NNPE_CUDA(c, cudaMemsetAsync(c->d_ctrl + CTRL_ERR, 0, sizeof(int), c->stream));
  return NNPE_OK;
}

int nnpe_set_system(nnpe_ctx* c, int natom, int ntype, double bl, const int* typ, const float* mass, const float* q,
                    const float* x, const int* mol_id, const int* intra_id, const int* atom_moltype, int nmoltype,
                    int nmax, const int* special) {
  if (!c || natom <= 0 || ntype <= 0 || !(bl > 0) || !typ || !mass || !q || !x || !mol_id || !intra_id ||
      !atom_moltype || nmoltype <= 0 || nmax <= 0 || !special)
    return nnpe_fail(c, NNPE_EARG, "nnpe_set_system: bad argument");
  if (ntype > NNPE_MAX_TYPES) return nnpe_fail(c, NNPE_EARG, "nnpe_set_system: at most 8 atom types");
  if (nmax > 255 || nmoltype > 32767) return nnpe_fail(c, NNPE_EARG, "nnpe_set_system: molecule too large");
  cudaSetDevice(c->device);
  free_state(c);
  c->have_setup = false;
  c->first_step_done = false;
  c->natom = natom; c->ntype = ntype; c->npair = ntype * (ntype + 1) / 2; c->bl = bl;
  c->nmoltype = nmoltype; c->nmax = nmax;
  c->h_typ.assign(typ, typ + natom); c->h_mass.assign(mass, mass + natom); c->h_q.assign(q, q + natom);
  c->h_mol_id.assign(mol_id, mol_id + natom); c->h_intra.assign(intra_id, intra_id + natom);
  c->h_amoltype.assign(atom_moltype, atom_moltype + natom);
  c->h_special.assign(special, special + (size_t)nmoltype * nmax * nmax);
  int nmol = 0;
  for (int i = 0; i < natom; ++i) {
    if (typ[i] < 0 || typ[i] >= ntype) return nnpe_fail(c, NNPE_EARG, "nnpe_set_system: type out of range");
    if (intra_id[i] < 0 || intra_id[i] >= nmax) return nnpe_fail(c, NNPE_EARG, "nnpe_set_system: intra id out of range");
    nmol = std::max(nmol, mol_id[i] + 1);
  }
  c->nmol = nmol;
  c->h_mol_rep.assign(nmol, -1);
  for (int i = 0; i < natom; ++i)
    if (intra_id[i] == 0) c->h_mol_rep[mol_id[i]] = i;
  for (int m = 0; m < nmol; ++m)
    if (c->h_mol_rep[m] < 0) return nnpe_fail(c, NNPE_EARG, "nnpe_set_system: molecule without intra id 0");
  // set_bl (environ.h:105), in float as the reference's numtype
  float blf = (float)bl;
  c->grid.bl = blf; c->grid.r_bl = 1.0f / blf; c->grid.h_bl = blf * .5F; c->grid.m_bl = -blf;
  // pair type table (environ.cpp:130-138)
  std::vector<int> pt(ntype * ntype);
  for (int i = 0, n = 0; i < ntype; ++i)
    for (int j = i; j < ntype; ++j) pt[i * ntype + j] = pt[j * ntype + i] = n++;
  TRY(dalloc(c, &c->d_pairtype, pt.size()));
  NNPE_CUDA(c, cudaMemcpy(c->d_pairtype, pt.data(), sizeof(int) * pt.size(), cudaMemcpyHostToDevice));
  TRY(dalloc(c, &c->d_special, c->h_special.size()));
  NNPE_CUDA(c, cudaMemcpy(c->d_special, c->h_special.data(), sizeof(int) * c->h_special.size(), cudaMemcpyHostToDevice));
  TRY(dalloc(c, &c->d_mol_rep, nmol));
  NNPE_CUDA(c, cudaMemcpy(c->d_mol_rep, c->h_mol_rep.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice));
  TRY(dalloc(c, &c->d_molshift, natom));
  TRY(dalloc(c, &c->d_emol, nmol));
  TRY(dalloc(c, &c->d_wmol, nmol));
  // state arrays in atom-id order until the first sort
  TRY(dalloc(c, &c->d_xd, natom)); TRY(dalloc(c, &c->d_vd, natom)); TRY(dalloc(c, &c->d_acc, natom));
  TRY(dalloc(c, &c->d_frc, natom)); TRY(dalloc(c, &c->d_atom_id, natom)); TRY(dalloc(c, &c->d_qm, natom));
  TRY(dalloc(c, &c->d_sorted_of_id, natom));
  std::vector<double4> xd(natom), vd(natom, make_double4(0, 0, 0, 0));
  std::vector<int> aid(natom);
  std::vector<float2> qm(natom);
  for (int i = 0; i < natom; ++i) {
    xd[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0);
    aid[i] = i;
    qm[i] = make_float2(q[i], 1.0f / mass[i]);   // r_m[idd]=1/r_m[idd] (environ.cpp:117)
  }
  NNPE_CUDA(c, cudaMemcpy(c->d_xd, xd.data(), sizeof(double4) * natom, cudaMemcpyHostToDevice));
  NNPE_CUDA(c, cudaMemcpy(c->d_vd, vd.data(), sizeof(double4) * natom, cudaMemcpyHostToDevice));
  NNPE_CUDA(c, cudaMemset(c->d_acc, 0, sizeof(float4) * natom));
  NNPE_CUDA(c, cudaMemset(c->d_frc, 0, sizeof(float4) * natom));
  NNPE_CUDA(c, cudaMemcpy(c->d_atom_id, aid.data(), sizeof(int) * natom, cudaMemcpyHostToDevice));
  NNPE_CUDA(c, cudaMemcpy(c->d_sorted_of_id, aid.data(), sizeof(int) * natom, cudaMemcpyHostToDevice));
  NNPE_CUDA(c, cudaMemcpy(c->d_qm, qm.data(), sizeof(float2) * natom, cudaMemcpyHostToDevice));
  c->have_system = true;
  return NNPE_OK;
}

// Current sorted -> atom id map (host copy).
static int get_atom_ids(nnpe_ctx* c, std::vector<int>& aid) {
  aid.resize(c->natom);
  NNPE_CUDA(c, cudaMemcpyAsync(aid.data(), c->d_atom_id, sizeof(int) * c->natom, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  return 0;
}

int nnpe_set_positions(nnpe_ctx* c, const float* x) {
  if (!c || !c->have_system || !x) return nnpe_fail(c, NNPE_EARG, "nnpe_set_positions: no system");
  std::vector<int> aid;
  TRY(get_atom_ids(c, aid));
  std::vector<double4> xd(c->natom);
  for (int i = 0; i < c->natom; ++i) {
    const float* p = x + 3 * (size_t)aid[i];
    xd[i] = make_double4(p[0], p[1], p[2], 0);
  }
  NNPE_CUDA(c, cudaMemcpy(c->d_xd, xd.data(), sizeof(double4) * c->natom, cudaMemcpyHostToDevice));
  int one = 1;
  NNPE_CUDA(c, cudaMemcpy(c->d_ctrl + CTRL_REBUILD, &one, sizeof(int), cudaMemcpyHostToDevice));
  return NNPE_OK;
}

int nnpe_atom_info(const nnpe_ctx* c, int* typ, int* mol_id, double* bl) {
  if (!c || !c->have_system) return NNPE_EARG;
  if (typ) std::copy(c->h_typ.begin(), c->h_typ.end(), typ);
  if (mol_id) std::copy(c->h_mol_id.begin(), c->h_mol_id.end(), mol_id);
  if (bl) *bl = c->bl;
  return NNPE_OK;
}

// ENVIRON::initV (environ.cpp:190-205): each atom, with probability `frac`, gets velocity
// components drawn from N(0, sqrt(T/300 * 300 / m) * kT_m_sqrt); a seeded 64-bit Mersenne twister
// stands in for the reference's random_device-seeded generator (mathlib.cpp:6-19).
int nnpe_init_velocities(nnpe_ctx* c, double temperature, double frac, uint64_t seed) {
  if (!c || !c->have_system || temperature < 0) return nnpe_fail(c, NNPE_EARG, "nnpe_init_velocities");
  std::vector<float> v((size_t)c->natom * 3, 0.f);
  if (frac < 1) TRY(nnpe_get_velocities(c, v.data()));
  std::mt19937_64 gen(seed);
  std::uniform_real_distribution<double> uni(0.0, 1.0);
  std::normal_distribution<double> nrm(0.0, 1.0);
  const double kTmSqrt = 0.0009118367518929329;   // environ.h:80
  for (int i = 0; i < c->natom; ++i) {
    if (uni(gen) >= frac) continue;
    const double fc = std::sqrt(temperature / c->h_mass[i]) * kTmSqrt;
    for (int d = 0; d < 3; ++d) v[(size_t)i * 3 + d] = (float)(fc * nrm(gen));
  }
  return nnpe_set_velocities(c, v.data());
}

int nnpe_set_velocities(nnpe_ctx* c, const float* v) {
  if (!c || !c->have_system || !v) return nnpe_fail(c, NNPE_EARG, "nnpe_set_velocities: no system");
  std::vector<int> aid;
  TRY(get_atom_ids(c, aid));
  std::vector<double4> vd(c->natom);
  for (int i = 0; i < c->natom; ++i) {
    const float* p = v + 3 * (size_t)aid[i];
    vd[i] = make_double4(p[0], p[1], p[2], 0);
  }
  NNPE_CUDA(c, cudaMemcpy(c->d_vd, vd.data(), sizeof(double4) * c->natom, cudaMemcpyHostToDevice));
  return NNPE_OK;
}

// ---------------------------------------------------------------------------------------------
// stencil: NEIGHLIST::build_bin_list (neighlist.cpp:35-168) computed once on the host, stored
// per cell as rows of z-contiguous cells with a per-cell "no distance check" bit mask.
// ---------------------------------------------------------------------------------------------
int build_stencil_host(nnpe_ctx* c, float cutoff, int max_nbin, Stencil* out) {
  const GridParams& g = c->grid;
  const int ng = g.num_gx, ngsq = g.num_gxsq;
  float t = cutoff * g.g_rdx;
  const int max_d = (int)std::ceil(t * t);
  std::vector<std::vector<int4>> rows(g.num_grid);
  size_t maxrows = 0;
  for (int i = 0; i < ng; ++i)
    for (int j = 0; j < ng; ++j)
      for (int k = 0; k < ng; ++k) {
        std::vector<int4>& R = rows[i * ngsq + j * ng + k];
        int num = 0;
        for (int l = 0; l < ng; ++l) {
          int mx, mxx;
          if (l == i) { mx = 0; mxx = 1; }
          else { int tp = std::abs(l - i); if ((mx = (tp - 1) * (tp - 1)) >= max_d) continue; mxx = (tp + 1) * (tp + 1); }
          for (int m = 0; m < ng; ++m) {
            int my, mxy;
            if (m == j) { my = mx; mxy = mxx + 1; }
            else { int tp = std::abs(m - j); if ((my = mx + (tp - 1) * (tp - 1)) >= max_d) continue; mxy = mxx + (tp + 1) * (tp + 1); }
            int4 row = make_int4(-1, -1, 0, 0);
            for (int n = 0; n < ng; ++n) {
              int mz, mxz;
              if (n == k) { mz = my; mxz = mxy + 1; }
              else { int tp = std::abs(n - k); if ((mz = my + (tp - 1) * (tp - 1)) >= max_d) continue; mxz = mxy + (tp + 1) * (tp + 1); }
              (void)mz;
              int cell = l * ngsq + m * ng + n;
              if (row.x < 0) row.x = cell;
              else if (cell != row.y + 1) return nnpe_fail(c, NNPE_EOVERFLOW, "stencil row not contiguous");
              row.y = cell;
              if (cell - row.x >= NNPE_MAX_ROW) return nnpe_fail(c, NNPE_EOVERFLOW, "stencil row longer than 32 cells");
              if (mxz < max_d) row.z |= 1 << (cell - row.x);
              ++num;
            }
            if (row.x >= 0) R.push_back(row);
          }
        }
        if (num >= max_nbin) return nnpe_fail(c, NNPE_EOVERFLOW, "bin_list overflow");   // neighlist.cpp:138
        maxrows = std::max(maxrows, R.size());
      }
  out->maxrows = (int)maxrows;
  out->cut = cutoff;
  std::vector<int4> flat((size_t)g.num_grid * maxrows, make_int4(0, -1, 0, 0));
  std::vector<int> nr(g.num_grid);
  for (int cidx = 0; cidx < g.num_grid; ++cidx) {
    nr[cidx] = (int)rows[cidx].size();
    std::copy(rows[cidx].begin(), rows[cidx].end(), flat.begin() + (size_t)cidx * maxrows);
  }
  TRY(dalloc(c, &out->rows, flat.size()));
  TRY(dalloc(c, &out->nrows, nr.size()));
  NNPE_CUDA(c, cudaMemcpy(out->rows, flat.data(), sizeof(int4) * flat.size(), cudaMemcpyHostToDevice));
  NNPE_CUDA(c, cudaMemcpy(out->nrows, nr.data(), sizeof(int) * nr.size(), cudaMemcpyHostToDevice));
  return 0;
}

int alloc_state(nnpe_ctx* c) {
  const int N = c->natom;
  const GridParams& g = c->grid;
  // expected images per atom for a uniform density (see generate_ghost, environ.cpp:401-442)
  double f = std::min(1.0, (double)c->comm_cutoff / c->bl);
  double per = std::pow(1 + 2 * f, 3) - 1;
  long gcap = (long)(1.3 * N * per) + 4096;
  gcap = std::min(gcap, 26L * N + 4096);
  if (c->Gcap > gcap) gcap = c->Gcap;   // a grown capacity is kept
  c->Gcap = (int)gcap;
  const long T = (long)N + gcap;
  TRY(dalloc(c, &c->d_pos, T)); TRY(dalloc(c, &c->d_info, T)); TRY(dalloc(c, &c->d_cell, T));
  TRY(dalloc(c, &c->d_xbuild, N));
  TRY(dalloc(c, &c->d_gowner, gcap)); TRY(dalloc(c, &c->d_gshift, gcap));
  TRY(dalloc(c, &c->d_ccount, g.num_grid)); TRY(dalloc(c, &c->d_cstart, g.num_grid + 1)); TRY(dalloc(c, &c->d_cend, g.num_grid));
  TRY(dalloc(c, &c->d_gccount, g.num_grid)); TRY(dalloc(c, &c->d_gcstart, g.num_grid + 1)); TRY(dalloc(c, &c->d_gcend, g.num_grid));
  TRY(dalloc(c, &c->d_slot, N)); TRY(dalloc(c, &c->d_ctmp, N)); TRY(dalloc(c, &c->d_perm, std::max<long>(N, gcap)));
  TRY(dalloc(c, &c->d_gcnt, N)); TRY(dalloc(c, &c->d_goff, N + 1));
  TRY(dalloc(c, &c->d_gtmp_owner, gcap)); TRY(dalloc(c, &c->d_gtmp_shift, gcap));
  TRY(dalloc(c, &c->d_gtmp_cell, gcap)); TRY(dalloc(c, &c->d_gtmp_slot, gcap));
  TRY(dalloc(c, &c->d_sxd, N)); TRY(dalloc(c, &c->d_svd, N)); TRY(dalloc(c, &c->d_sacc, N));
  TRY(dalloc(c, &c->d_sinfo, N)); TRY(dalloc(c, &c->d_satom, N)); TRY(dalloc(c, &c->d_sqm, N));
  TRY(dalloc(c, &c->d_list, (size_t)N * c->cap)); TRY(dalloc(c, &c->d_ncount, N));
  TRY(dalloc(c, &c->d_plist, (size_t)N * c->cap)); TRY(dalloc(c, &c->d_pcount, N)); TRY(dalloc(c, &c->d_xprune, N));
  TRY(dalloc(c, &c->d_eatom, N)); TRY(dalloc(c, &c->d_watom, N)); TRY(dalloc(c, &c->d_kin, N));
  NNPE_CUDA(c, cudaMemset(c->d_eatom, 0, sizeof(double) * N));
  NNPE_CUDA(c, cudaMemset(c->d_watom, 0, sizeof(double) * N));
  NNPE_CUDA(c, cudaMemset(c->d_ncount, 0, sizeof(int) * N));
  NNPE_CUDA(c, cudaMemset(c->d_pcount, 0, sizeof(int) * N));
  // info of real atoms in the current (atom-id or sorted) order
  std::vector<int> aid;
  TRY(get_atom_ids(c, aid));
  std::vector<int2> info(N);
  for (int i = 0; i < N; ++i) {
    int a = aid[i];
    info[i] = make_int2(c->h_mol_id[a], c->h_typ[a] | (c->h_intra[a] << 8) | (c->h_amoltype[a] << 16));
  }
  NNPE_CUDA(c, cudaMemcpy(c->d_info, info.data(), sizeof(int2) * N, cudaMemcpyHostToDevice));
  return 0;
}

int nnpe_setup(nnpe_ctx* c, double pair_cutoff, double skin, double gr_cutoff, int neigh_cap) {
  if (!c || !c->have_system) return nnpe_fail(c, NNPE_EARG, "nnpe_setup: no system");
  if (!(pair_cutoff > 0) || !(skin >= 0) || neigh_cap <= 0) return nnpe_fail(c, NNPE_EARG, "nnpe_setup: bad cutoff");
  cudaSetDevice(c->device);
  free_graphs(c);
  c->pair_cutoff = (float)pair_cutoff;
  c->skin = (float)skin;
  c->gr_cutoff = (float)(gr_cutoff > 0 ? gr_cutoff : pair_cutoff);
  c->cap = neigh_cap;
  // run.cpp:76-79 in numtype (float) arithmetic
  c->comm_cutoff = c->skin + std::max(c->gr_cutoff, c->pair_cutoff);
  GridParams& g = c->grid;
  g.ghost_lim = g.h_bl - c->comm_cutoff;
  g.g_dx = (float)(0.5 * (c->skin + c->pair_cutoff));
  g.g_rdx = 1 / g.g_dx;
  g.g_offset = c->comm_cutoff + g.h_bl;
  g.num_gx = (int)std::ceil((g.g_offset * 2) * g.g_rdx);
  g.num_gxsq = g.num_gx * g.num_gx;
  g.num_grid = g.num_gx * g.num_gxsq;
  if ((double)c->natom + 27.0 * c->natom >= (double)NNPE_J_MASK)
    return nnpe_fail(c, NNPE_EARG, "nnpe_setup: system too large for 27-bit list indices");
  TRY(build_stencil_host(c, c->pair_cutoff + c->skin, 126, &c->st_pair));
  TRY(build_stencil_host(c, c->gr_cutoff + c->skin, 8192, &c->st_gr));
  TRY(alloc_state(c));
  int ctrl[CTRL_WORDS] = {0};
  ctrl[CTRL_REBUILD] = 1;   // x_prev=INFINITY makes the first isvalid() false (neighlist.cpp:29)
  NNPE_CUDA(c, cudaMemcpy(c->d_ctrl, ctrl, sizeof(ctrl), cudaMemcpyHostToDevice));
  TRY(noalloc_stage_prepare(c));
  c->have_setup = true;
  c->first_step_done = false;
  c->poisoned = false;
  return NNPE_OK;
}

// A new box length for a set-up context: ENVIRON::set_bl plus BL_MANAGER::setBL (run.cpp:688-712),
// i.e. the box constants in float, the grid re-derived with the same cell length, the ghost limit
// and the stencils for the new grid; the device arrays that depend on the grid or on the number of
// images are reallocated for it. The positions stay as they are (set new ones with
// nnpe_set_positions or pass them to nnpe_force_step); the next force evaluation rebuilds the list.
int nnpe_set_box(nnpe_ctx* c, double bl) {
  if (!c || !c->have_setup || !(bl > 0)) return nnpe_fail(c, NNPE_EARG, "nnpe_set_box: not set up, or box length <= 0");
  if (int rc = refuse_if_poisoned(c)) return rc;
  const float blf = (float)bl;
  c->bl = bl;
  c->grid.bl = blf; c->grid.r_bl = 1.0f / blf; c->grid.h_bl = blf * .5F; c->grid.m_bl = -blf;
  c->force_step_init = false;
  return nnpe_setup(c, c->pair_cutoff, c->skin, c->gr_cutoff, c->cap);
}

// ---------------------------------------------------------------------------------------------
// pair table
// ---------------------------------------------------------------------------------------------
int nnpe_pair_set_table(nnpe_ctx* c, int nbin, const float* force, const float* potential) {
  if (!c || !c->have_system || nbin <= 0 || !force || !potential) return nnpe_fail(c, NNPE_EARG, "nnpe_pair_set_table");
  cudaSetDevice(c->device);
  std::vector<float2> t((size_t)c->npair * (nbin + 1));
  for (int p = 0; p < c->npair; ++p)
    for (int i = 0; i <= nbin; ++i)
      t[(size_t)p * (nbin + 1) + i] = make_float2(force[(size_t)p * (nbin + 1) + i], potential[(size_t)p * (nbin + 1) + i]);
  TRY(dalloc(c, &c->d_table, t.size()));
  NNPE_CUDA(c, cudaMemcpy(c->d_table, t.data(), sizeof(float2) * t.size(), cudaMemcpyHostToDevice));
  c->nbin = nbin;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

int nnpe_pair_get_table(nnpe_ctx* c, float* force, float* potential) {
  if (!c || !c->d_table) return nnpe_fail(c, NNPE_EARG, "nnpe_pair_get_table: no table");
  std::vector<float2> t((size_t)c->npair * (c->nbin + 1));
  NNPE_CUDA(c, cudaMemcpyAsync(t.data(), c->d_table, sizeof(float2) * t.size(), cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  for (size_t k = 0; k < t.size(); ++k) { force[k] = t[k].x; potential[k] = t[k].y; }
  return NNPE_OK;
}

int nnpe_pair_exact(nnpe_ctx* c, int on) {
  if (!c) return NNPE_EARG;
  c->exact_forces = on != 0;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

int nnpe_pair_enable(nnpe_ctx* c, int on) {
  if (!c) return NNPE_EARG;
  c->pair_on = on != 0;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

// LJTableCoulDSF::loadPotential(0, potfile) (pair.cpp:219-243): nbin rows of
// r F_00/r U_00 F_01/r U_01 ... ; the extra column nbin is zero.
int nnpe_pair_load_table(nnpe_ctx* c, int nbin, const char* potfile) {
  if (!c || !c->have_system || nbin <= 0 || !potfile) return nnpe_fail(c, NNPE_EARG, "nnpe_pair_load_table");
  FILE* fp = fopen(potfile, "r");
  if (!fp) return nnpe_fail(c, NNPE_EFILE, std::string("cannot open ") + potfile);
  const int P = c->npair;
  std::vector<float> F((size_t)P * (nbin + 1), 0.f), U((size_t)P * (nbin + 1), 0.f);
  for (int i = 0; i < nbin; ++i) {
    float r;
    if (fscanf(fp, "%f ", &r) != 1) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, "pair table: short file"); }
    for (int p = 0; p < P; ++p)
      if (fscanf(fp, "%f ", &F[(size_t)p * (nbin + 1) + i]) != 1 || fscanf(fp, "%f ", &U[(size_t)p * (nbin + 1) + i]) != 1) {
        fclose(fp);
        return nnpe_fail(c, NNPE_EFILE, "pair table: short row");
      }
  }
  fclose(fp);
  return nnpe_pair_set_table(c, nbin, F.data(), U.data());
}

// ---------------------------------------------------------------------------------------------
// bonded topology, grouped per molecule so that one thread owns every term of a molecule
// ---------------------------------------------------------------------------------------------
int nnpe_bonded_set(nnpe_ctx* c, int nbond, const int* bonds, int nbtyp, const float* bcoef, int nangle,
                    const int* angles, int natyp, const float* acoef, int ndih, const int* dihs, int ndtyp,
                    const float* dcoef) {
  if (!c || !c->have_system) return nnpe_fail(c, NNPE_EARG, "nnpe_bonded_set: no system");
  cudaSetDevice(c->device);
  const int nmol = c->nmol;
  auto mol_of = [&](int a) { return c->h_mol_id[a]; };
  std::vector<std::vector<int4>> B(nmol), A(nmol);
  std::vector<std::vector<std::array<int, 5>>> D(nmol);
  for (int k = 0; k < nbond; ++k) {
    const int* b = bonds + 3 * k;
    if (b[0] < 0 || b[0] >= nbtyp || b[1] < 0 || b[2] < 0 || b[1] >= c->natom || b[2] >= c->natom || mol_of(b[1]) != mol_of(b[2]))
      return nnpe_fail(c, NNPE_EARG, "auto generate error (bond)");   // bond.cpp:80-86
    B[mol_of(b[1])].push_back(make_int4(b[0], b[1], b[2], 0));
  }
  for (int k = 0; k < nangle; ++k) {
    const int* a = angles + 4 * k;
    if (a[0] < 0 || a[0] >= natyp || mol_of(a[1]) != mol_of(a[2]) || mol_of(a[1]) != mol_of(a[3]))
      return nnpe_fail(c, NNPE_EARG, "auto generate error (angle)");
    A[mol_of(a[1])].push_back(make_int4(a[0], a[1], a[2], a[3]));
  }
  for (int k = 0; k < ndih; ++k) {
    const int* d = dihs + 5 * k;
    if (d[0] < 0 || d[0] >= ndtyp || mol_of(d[1]) != mol_of(d[2]) || mol_of(d[1]) != mol_of(d[3]) || mol_of(d[1]) != mol_of(d[4]))
      return nnpe_fail(c, NNPE_EARG, "auto generate error (dihedral)");
    D[mol_of(d[1])].push_back({d[0], d[1], d[2], d[3], d[4]});
  }
  std::vector<int4> fb, fa;
  std::vector<int> fd;
  std::vector<int> terms(3 * (nmol + 1));
  for (int m = 0; m < nmol; ++m) {
    terms[3 * m] = (int)fb.size(); terms[3 * m + 1] = (int)fa.size(); terms[3 * m + 2] = (int)(fd.size() / 5);
    fb.insert(fb.end(), B[m].begin(), B[m].end());
    fa.insert(fa.end(), A[m].begin(), A[m].end());
    for (auto& d : D[m]) fd.insert(fd.end(), d.begin(), d.end());
  }
  terms[3 * nmol] = (int)fb.size(); terms[3 * nmol + 1] = (int)fa.size(); terms[3 * nmol + 2] = (int)(fd.size() / 5);
  c->nbond = nbond; c->nangle = nangle; c->ndih = ndih;
  TRY(dalloc(c, &c->d_bond, fb.size())); TRY(dalloc(c, &c->d_angle, fa.size())); TRY(dalloc(c, &c->d_dih, fd.size()));
  TRY(dalloc(c, &c->d_mol_terms, terms.size()));
  if (!fb.empty()) NNPE_CUDA(c, cudaMemcpy(c->d_bond, fb.data(), sizeof(int4) * fb.size(), cudaMemcpyHostToDevice));
  if (!fa.empty()) NNPE_CUDA(c, cudaMemcpy(c->d_angle, fa.data(), sizeof(int4) * fa.size(), cudaMemcpyHostToDevice));
  if (!fd.empty()) NNPE_CUDA(c, cudaMemcpy(c->d_dih, fd.data(), sizeof(int) * fd.size(), cudaMemcpyHostToDevice));
  NNPE_CUDA(c, cudaMemcpy(c->d_mol_terms, terms.data(), sizeof(int) * terms.size(), cudaMemcpyHostToDevice));
  auto up = [&](float4** d, const float* h, int n) -> int {
    std::vector<float4> v(std::max(n, 1), make_float4(0, 0, 0, 0));
    for (int i = 0; i < n; ++i) v[i] = make_float4(h[4 * i], h[4 * i + 1], h[4 * i + 2], h[4 * i + 3]);
    TRY(dalloc(c, d, v.size()));
    NNPE_CUDA(c, cudaMemcpy(*d, v.data(), sizeof(float4) * v.size(), cudaMemcpyHostToDevice));
    return 0;
  };
  TRY(up(&c->d_bcoef, bcoef, bcoef ? nbtyp : 0));
  TRY(up(&c->d_acoef, acoef, acoef ? natyp : 0));
  TRY(up(&c->d_dcoef, dcoef, dcoef ? ndtyp : 0));
  c->nbtyp = nbtyp; c->natyp = natyp; c->ndtyp = ndtyp;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

// Replace the bonded coefficients (stored form) keeping the topology.
int nnpe_bonded_coefs(nnpe_ctx* c, const float* bcoef, const float* acoef, const float* dcoef) {
  auto up = [&](float4* d, const float* h, int n) -> int {
    if (n <= 0 || !d) return 0;
    std::vector<float4> v(n);
    for (int i = 0; i < n; ++i) v[i] = make_float4(h[4 * i], h[4 * i + 1], h[4 * i + 2], h[4 * i + 3]);
    NNPE_CUDA(c, cudaMemcpy(d, v.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    return 0;
  };
  TRY(up(c->d_bcoef, bcoef, c->nbtyp));
  TRY(up(c->d_acoef, acoef, c->natyp));
  TRY(up(c->d_dcoef, dcoef, c->ndtyp));
  return NNPE_OK;
}

int nnpe_verlet_setup(nnpe_ctx* c, double dt, int fp64_state) {
  if (!c) return NNPE_EARG;
  c->dt = dt;
  c->fp64_state = fp64_state != 0;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

int nnpe_thermostat(nnpe_ctx* c, int kind, double t_start, double t_end, int interval, double frac, uint64_t seed) {
  if (!c || kind < 0 || kind > 2 || (kind && interval <= 0)) return nnpe_fail(c, NNPE_EARG, "nnpe_thermostat");
  c->thermo_kind = kind; c->t_start = t_start; c->t_end = t_end; c->thermo_interval = interval;
  c->thermo_frac = frac; c->seed = seed;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

// ---------------------------------------------------------------------------------------------
// state export
// ---------------------------------------------------------------------------------------------
template <typename T, typename F>
static int export_by_id(nnpe_ctx* c, const T* dsrc, F&& put) {
  std::vector<int> aid;
  TRY(get_atom_ids(c, aid));
  std::vector<T> h(c->natom);
  NNPE_CUDA(c, cudaMemcpyAsync(h.data(), dsrc, sizeof(T) * c->natom, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int i = 0; i < c->natom; ++i) put(aid[i], h[i]);
  return 0;
}

int nnpe_get_forces(nnpe_ctx* c, int kind, float* f) {
  if (!c || !c->have_system || !f) return nnpe_fail(c, NNPE_EARG, "nnpe_get_forces");
  return export_by_id(c, kind ? c->d_acc : c->d_frc, [&](int a, float4 v) { f[3 * a] = v.x; f[3 * a + 1] = v.y; f[3 * a + 2] = v.z; });
}
int nnpe_get_positions(nnpe_ctx* c, float* x) {
  if (!c || !c->have_system || !x) return nnpe_fail(c, NNPE_EARG, "nnpe_get_positions");
  return export_by_id(c, c->d_xd, [&](int a, double4 v) { x[3 * a] = (float)v.x; x[3 * a + 1] = (float)v.y; x[3 * a + 2] = (float)v.z; });
}
int nnpe_get_positions_f64(nnpe_ctx* c, double* x) {
  if (!c || !c->have_system || !x) return nnpe_fail(c, NNPE_EARG, "nnpe_get_positions_f64");
  return export_by_id(c, c->d_xd, [&](int a, double4 v) { x[3 * a] = v.x; x[3 * a + 1] = v.y; x[3 * a + 2] = v.z; });
}
int nnpe_get_velocities(nnpe_ctx* c, float* v) {
  if (!c || !c->have_system || !v) return nnpe_fail(c, NNPE_EARG, "nnpe_get_velocities");
  return export_by_id(c, c->d_vd, [&](int a, double4 u) { v[3 * a] = (float)u.x; v[3 * a + 1] = (float)u.y; v[3 * a + 2] = (float)u.z; });
}
int nnpe_get_velocities_f64(nnpe_ctx* c, double* v) {
  if (!c || !c->have_system || !v) return nnpe_fail(c, NNPE_EARG, "nnpe_get_velocities_f64");
  return export_by_id(c, c->d_vd, [&](int a, double4 u) { v[3 * a] = u.x; v[3 * a + 1] = u.y; v[3 * a + 2] = u.z; });
}
int nnpe_get_atom_energy(nnpe_ctx* c, double* e) {
  if (!c || !c->have_setup || !e) return nnpe_fail(c, NNPE_EARG, "nnpe_get_atom_energy");
  return export_by_id(c, c->d_eatom, [&](int a, double v) { e[a] = v; });
}

int nnpe_list_info(nnpe_ctx* c, int* nghost, int64_t* nentries, int* nbuild, int* num_gx) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_list_info: not set up");
  NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
  std::vector<int> cnt(c->natom);
  NNPE_CUDA(c, cudaMemcpyAsync(cnt.data(), c->d_ncount, sizeof(int) * c->natom, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  if (nghost) *nghost = c->h_ctrl[CTRL_NGHOST];
  if (nbuild) *nbuild = c->h_ctrl[CTRL_NBUILD];
  if (num_gx) *num_gx = c->grid.num_gx;
  if (nentries) {
    int64_t s = 0;
    for (int v : cnt) s += v;
    *nentries = s;
  }
  return NNPE_OK;
}

int nnpe_set_prune(nnpe_ctx* c, double delta) {
  if (!c || !(delta == delta) || delta > 1e3) return nnpe_fail(c, NNPE_EARG, "nnpe_set_prune: bad delta");
  c->prune_delta = delta > 0 ? (float)delta : 0.f;
  free_graphs(c);   // captured steps hold the list pointers of the old setting
  if (c->d_ctrl) {  // the next evaluation makes a fresh copy
    int one = 1;
    NNPE_CUDA(c, cudaMemcpyAsync(c->d_ctrl + CTRL_PRUNE, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  return NNPE_OK;
}

int nnpe_prune_info(nnpe_ctx* c, double* delta, int* active, int* nprune, int64_t* nentries) {
  if (!c) return NNPE_EARG;
  if (delta) *delta = c->prune_delta;
  if (active) *active = prune_active(c) ? 1 : 0;
  if (nentries) {
    *nentries = 0;
    if (c->d_pcount && prune_active(c)) {
      std::vector<int> cnt(c->natom);
      NNPE_CUDA(c, cudaMemcpyAsync(cnt.data(), c->d_pcount, sizeof(int) * c->natom, cudaMemcpyDeviceToHost, c->stream));
      NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
      for (int v : cnt) *nentries += v;
    }
  }
  if (nprune) {
    *nprune = 0;
    if (c->d_ctrl) {
      NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
      NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
      *nprune = c->h_ctrl[CTRL_NPRUNE];
    }
  }
  return NNPE_OK;
}

int nnpe_list_get(nnpe_ctx* c, int64_t cap, int* rec, int64_t* n) {
  if (!c || !c->have_setup || !rec || !n) return nnpe_fail(c, NNPE_EARG, "nnpe_list_get");
  const int N = c->natom;
  NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  const int G = c->h_ctrl[CTRL_NGHOST];
  std::vector<int> cnt(N), aid(N), gown(std::max(G, 1)), gsh(std::max(G, 1));
  std::vector<uint32_t> L((size_t)N * c->cap);
  NNPE_CUDA(c, cudaMemcpyAsync(cnt.data(), c->d_ncount, sizeof(int) * N, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(aid.data(), c->d_atom_id, sizeof(int) * N, cudaMemcpyDeviceToHost, c->stream));
  if (G) {
    NNPE_CUDA(c, cudaMemcpyAsync(gown.data(), c->d_gowner, sizeof(int) * G, cudaMemcpyDeviceToHost, c->stream));
    NNPE_CUDA(c, cudaMemcpyAsync(gsh.data(), c->d_gshift, sizeof(int) * G, cudaMemcpyDeviceToHost, c->stream));
  }
  NNPE_CUDA(c, cudaMemcpyAsync(L.data(), c->d_list, sizeof(uint32_t) * L.size(), cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  int64_t k = 0;
  for (int i = 0; i < N; ++i)
    for (int e = 0; e < cnt[i]; ++e) {
      uint32_t v = L[(size_t)i * c->cap + e];
      int j = (int)(v & NNPE_J_MASK), s = (int)(v >> 30);
      int ja, code;
      if (j < N) { ja = aid[j]; code = 13; }
      else { ja = aid[gown[j - N]]; code = gsh[j - N]; }
      if (k < cap) { rec[4 * k] = aid[i]; rec[4 * k + 1] = ja; rec[4 * k + 2] = code; rec[4 * k + 3] = s; }
      ++k;
    }
  *n = k;
  return k <= cap ? NNPE_OK : nnpe_fail(c, NNPE_EOVERFLOW, "nnpe_list_get: record capacity too small");
}


// setParam of the bonded classes in the reference's float arithmetic (bond.cpp:48-55,
// angle.cpp:184-191, dihedral.cpp:340-348): the stored coefficient forms the kernels read.
int nnpe_bond_coef(double b0, double ka, double kb, double kc, float* out) {
  if (!out) return NNPE_EARG;
  const float a = (float)ka, c = (float)kc;
  out[0] = (float)b0; out[1] = a * 2; out[2] = (float)kb; out[3] = c * 2;
  return NNPE_OK;
}
int nnpe_angle_coef(double theta0, double ka, double kb, double kc, float* out) {
  if (!out) return NNPE_EARG;
  const float t = (float)theta0, pi = 3.141592653589793238462643383279502884f;
  const float a = (float)ka, c = (float)kc;
  out[0] = std::cos(t * pi / 180); out[1] = a * 2; out[2] = (float)kb; out[3] = c * 2;
  return NNPE_OK;
}
int nnpe_dihedral_coef(double c0, double c1, double c2, double c3, float* out) {
  if (!out) return NNPE_EARG;
  const float f0 = (float)c0, f1 = (float)c1, f2 = (float)c2, f3 = (float)c3;
  out[0] = f0 - f2; out[1] = f1 - 3 * f3; out[2] = f2 * 2 * 2; out[3] = f3 * 4 * 3;
  return NNPE_OK;
}

// ---------------------------------------------------------------------------------------------
// reference input formats
// ---------------------------------------------------------------------------------------------
namespace {
// fgets_non_empty (util.cpp:138-145): next line with a non-blank character
bool next_line(FILE* fp, char* buf, int n) {
  while (fgets(buf, n, fp)) {
    for (char* p = buf; *p; ++p)
      if (*p != ' ' && *p != '\n' && *p != '\r' && *p != '\t') return true;
  }
  return false;
}
struct MolFile {
  int n_atom = 0;
  std::vector<std::array<int, 5>> bonds, angles, dihs;   // 0-based (type, atoms...)
  std::vector<int> special;                               // n_atom*n_atom
};
// MOLECULE::from_file (molecule.cpp:145-254)
int read_molecule(nnpe_ctx* c, const char* path, MolFile& m) {
  FILE* fp = fopen(path, "r");
  if (!fp) return nnpe_fail(c, NNPE_EFILE, std::string("cannot open molecule file ") + path);
  enum { HEADER, BOND, ANGLE, DIH, OTHER } st = HEADER;
  char buf[256], w[256];
  while (fgets(buf, sizeof buf, fp)) {
    char* s = buf;
    while (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r') ++s;
    if (!*s) continue;
    if (!strncmp(s, "Coords", 6) || !strncmp(s, "Types", 5) || !strncmp(s, "Charges", 7)) { st = OTHER; continue; }
    if (!strncmp(s, "Bonds", 5)) { st = BOND; continue; }
    if (!strncmp(s, "Angles", 6)) { st = ANGLE; continue; }
    if (!strncmp(s, "Dihedrals", 9)) { st = DIH; continue; }
    std::array<int, 5> r{0, 0, 0, 0, 0};
    switch (st) {
      case HEADER: {
        int v;
        if (sscanf(s, "%d %255s", &v, w) != 2) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, "molecule header read error"); }
        if (!strncmp(w, "atoms", 5)) m.n_atom = v;
        else if (strncmp(w, "bonds", 5) && strncmp(w, "angles", 6) && strncmp(w, "dihedrals", 9)) {
          fclose(fp);
          return nnpe_fail(c, NNPE_EFILE, "molecule header read error");
        }
        break;
      }
      case BOND:
        if (sscanf(s, "%*d %d %d %d", &r[0], &r[1], &r[2]) != 3) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, "bond read error"); }
        m.bonds.push_back({r[0] - 1, r[1] - 1, r[2] - 1, 0, 0});
        break;
      case ANGLE:
        if (sscanf(s, "%*d %d %d %d %d", &r[0], &r[1], &r[2], &r[3]) != 4) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, "angle read error"); }
        m.angles.push_back({r[0] - 1, r[1] - 1, r[2] - 1, r[3] - 1, 0});
        break;
      case DIH:
        if (sscanf(s, "%*d %d %d %d %d %d", &r[0], &r[1], &r[2], &r[3], &r[4]) != 5) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, "dihedral read error"); }
        m.dihs.push_back({r[0] - 1, r[1] - 1, r[2] - 1, r[3] - 1, r[4] - 1});
        break;
      default:
        break;
    }
  }
  fclose(fp);
  if (m.n_atom <= 0) return nnpe_fail(c, NNPE_EFILE, "molecule without atoms");
  m.special.assign((size_t)m.n_atom * m.n_atom, 0);
  auto in = [&](int a) { return a >= 0 && a < m.n_atom; };
  for (auto& b : m.bonds) {
    if (!in(b[1]) || !in(b[2])) return nnpe_fail(c, NNPE_EFILE, "bond atom out of range");
    m.special[b[1] * m.n_atom + b[2]] = m.special[b[2] * m.n_atom + b[1]] = 1;
  }
  for (auto& a : m.angles) {
    if (!in(a[1]) || !in(a[3])) return nnpe_fail(c, NNPE_EFILE, "angle atom out of range");
    m.special[a[1] * m.n_atom + a[3]] = m.special[a[3] * m.n_atom + a[1]] = 2;
  }
  for (auto& d : m.dihs) {
    if (!in(d[1]) || !in(d[4])) return nnpe_fail(c, NNPE_EFILE, "dihedral atom out of range");
    m.special[d[1] * m.n_atom + d[4]] = m.special[d[4] * m.n_atom + d[1]] = 3;
  }
  return 0;
}
}  // namespace

// ENVIRON::initialize (environ.cpp:22-141). The molecules' bonded terms, expanded per molecule
// as autoGenerate does (bond.cpp:66-86), are kept for nnpe_bonded_autogen.
int nnpe_load_system_file(nnpe_ctx* c, const char* path) {
  if (!c || !path) return nnpe_fail(c, NNPE_EARG, "nnpe_load_system_file");
  FILE* fp = fopen(path, "r");
  if (!fp) return nnpe_fail(c, NNPE_EFILE, std::string("cannot open ") + path);
  char buf[512], w[512];
  int nmoltype = 0, nmol = 0, ntype = 0, natom = 0;
  float bl = 0;
  auto bad = [&](const char* m) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, std::string("read error: ") + m); };
  if (!next_line(fp, buf, sizeof buf) || sscanf(buf, "%d %d", &nmoltype, &nmol) != 2 || nmoltype <= 0) return bad("header");
  std::vector<MolFile> mols(nmoltype);
  for (int i = 0; i < nmoltype; ++i) {
    if (!next_line(fp, buf, sizeof buf) || sscanf(buf, "%511s", w) != 1) return bad("molecule file line");
    if (int rc = read_molecule(c, w, mols[i])) { fclose(fp); return rc; }
  }
  if (!next_line(fp, buf, sizeof buf) || sscanf(buf, "%d %d %f", &ntype, &natom, &bl) != 3 || natom <= 0) return bad("ntype natom BL");
  std::vector<int> typ(natom), mol_id(natom), intra(natom), amt(natom);
  std::vector<float> mass(natom), q(natom), x(3 * (size_t)natom);
  int in_mol = 0, imol = 0, mt_prev = 0;
  for (int i = 0; i < natom; ++i) {
    int mt;
    if (!next_line(fp, buf, sizeof buf) ||
        sscanf(buf, "%d %d %f %f %f %f %f", &mt, &typ[i], &mass[i], &q[i], &x[3 * i], &x[3 * i + 1], &x[3 * i + 2]) != 7)
      return bad("atom line");
    if (typ[i] >= ntype || typ[i] < 0 || mt < 0 || mt >= nmoltype) return bad("atom type");
    if (in_mol && mt != mt_prev) return bad("molecule type changes inside a molecule");
    intra[i] = in_mol; mol_id[i] = imol; amt[i] = mt;
    if (mols[mt].n_atom == ++in_mol) { ++imol; in_mol = 0; }
    mt_prev = mt;
  }
  fclose(fp);
  if (imol != nmol) return nnpe_fail(c, NNPE_EFILE, "read error: molecule count");
  int nmax = 0;
  for (auto& m : mols) nmax = std::max(nmax, m.n_atom);
  std::vector<int> special((size_t)nmoltype * nmax * nmax, 0);
  for (int t = 0; t < nmoltype; ++t)
    for (int a = 0; a < mols[t].n_atom; ++a)
      for (int b = 0; b < mols[t].n_atom; ++b)
        special[((size_t)t * nmax + a) * nmax + b] = mols[t].special[a * mols[t].n_atom + b];
  if (int rc = nnpe_set_system(c, natom, ntype, bl, typ.data(), mass.data(), q.data(), x.data(), mol_id.data(),
                               intra.data(), amt.data(), nmoltype, nmax, special.data()))
    return rc;
  c->top_bonds.clear(); c->top_angles.clear(); c->top_dihs.clear();
  for (int i = 0; i < natom; ++i) {
    if (intra[i]) continue;
    const MolFile& m = mols[amt[i]];
    for (auto& b : m.bonds) c->top_bonds.insert(c->top_bonds.end(), {b[0], b[1] + i, b[2] + i});
    for (auto& a : m.angles) c->top_angles.insert(c->top_angles.end(), {a[0], a[1] + i, a[2] + i, a[3] + i});
    for (auto& d : m.dihs) c->top_dihs.insert(c->top_dihs.end(), {d[0], d[1] + i, d[2] + i, d[3] + i, d[4] + i});
  }
  return NNPE_OK;
}

// BOND/ANGLE/DIHEDRAL::autoGenerate (bond.cpp:66-103) over the topology read with the system.
int nnpe_bonded_autogen(nnpe_ctx* c, int nbtyp, const float* bcoef, int natyp, const float* acoef, int ndtyp,
                        const float* dcoef) {
  if (!c || !c->have_system) return nnpe_fail(c, NNPE_EARG, "nnpe_bonded_autogen: no system");
  return nnpe_bonded_set(c, (int)c->top_bonds.size() / 3, c->top_bonds.data(), nbtyp, bcoef,
                         (int)c->top_angles.size() / 4, c->top_angles.data(), natyp, acoef,
                         (int)c->top_dihs.size() / 5, c->top_dihs.data(), ndtyp, dcoef);
}
