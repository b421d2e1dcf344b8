// RMDF: reverse-MD / FMIRL refinement of the pair table against target structure factors
// (grsq.h:82-112, grsq.cpp:899-1443), on the device so that the tables the force kernels read
// are rewritten in HBM on the same stream, before the same step's forces (run.cpp:286-302).
//
// Per g(r) step, after the g(r) tally and the S(q) transform:
//   k_rmdf_q   compute_Qspace (grsq.cpp:1061-1118): per target n the weighted total
//              S_n(q) = sum_p S_p(q) sqwt[n][p][q], the penalty sum_q wt (S_n - S_exp)^2,
//              deltaS <- deltaS + gamma (S_n - S_exp - deltaS) and force_q[p][q] = sum_n deltaS fwt[n][p][q];
//              the penalty times natom/4 is the logged erg_exp.
//   k_rmdf_r   compute_Rspace / compute_Potential (grsq.cpp:1120-1210): table row r of pair p is
//              base + sum_q force_q[p][q] ftmx[r][q] (force, F/r) or potmx[r][q] (potential), with
//              ftmx = (j0(qr) - cos(qr)) / r^2, potmx = j0(qr) = sin(qr)/(qr); the network variant
//              (compute_Rspace_NNP, grsq.cpp:1213-1294) writes special class 0 and class 3 scaled by
//              special_lj[3].
// All sums are FP64 in a fixed order (one warp per table row, fixed shuffle tree), so the rewritten
// tables are the same bits run to run; the grid points r and q are the reference's float grids.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "internal.cuh"
#include "nnp.cuh"

struct RmdfState {
  int n_sq = 0, nq = 0, nbin = 0, P = 0;
  double gamma = 1, strength = 0;
  bool nnp = false;          // tables of the network term (NNPOTENTIAL_TBL) instead of LJTableCoulDSF
  double *d_sqwt = nullptr, *d_fwt = nullptr;       // [n_sq][P][nq]
  double *d_sqex = nullptr, *d_wt = nullptr;        // [n_sq][nq]
  double *d_dsq = nullptr, *d_sqn = nullptr;        // deltaS, weighted S_n [n_sq][nq]
  double* d_fq = nullptr;                           // force_q [P][nq]
  double *d_ftmx = nullptr, *d_potmx = nullptr;     // [nbin][nq]
  float2* d_base = nullptr;                         // table as loaded (the *_base arrays)
  std::vector<float> h_qq;                          // SQ's q grid (grsq.cpp:270-274)
  std::vector<double> h_dsq_acc;                    // deltasq_accu [n_sq][nq] (dumpSQ running average)
};

namespace {

constexpr double kSpecialLj14 = 0.5;   // MOLECULE::special_lj[3] (molecule.h:11)

__global__ void k_rmdf_q(const double* __restrict__ sq, const double* __restrict__ sqwt, const double* __restrict__ fwt,
                         const double* __restrict__ sqex, const double* __restrict__ wt, double* dsq, double* sqn,
                         double* __restrict__ fq, int n_sq, int P, int nq, double gamma, double natom, double* red) {
  __shared__ double sh[512];
  const int t = threadIdx.x;
  double e = 0;
  for (int q = t; q < nq; q += blockDim.x) {
    double f[NNPE_MAX_TYPES * (NNPE_MAX_TYPES + 1) / 2];
    for (int p = 0; p < P; ++p) f[p] = 0;
    for (int n = 0; n < n_sq; ++n) {
      const double* sw = sqwt + (size_t)n * P * nq;
      double s = 0;
      for (int p = 0; p < P; ++p) s += sq[(size_t)p * nq + q] * sw[(size_t)p * nq + q];
      const double d = s - sqex[(size_t)n * nq + q];
      e += d * d * wt[(size_t)n * nq + q];
      double ds = dsq[(size_t)n * nq + q];
      ds += gamma * (d - ds);
      dsq[(size_t)n * nq + q] = ds;
      sqn[(size_t)n * nq + q] = s;
      const double* fw = fwt + (size_t)n * P * nq;
      for (int p = 0; p < P; ++p) f[p] += ds * fw[(size_t)p * nq + q];
    }
    for (int p = 0; p < P; ++p) fq[(size_t)p * nq + q] = f[p];
  }
  sh[t] = e;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s) sh[t] += sh[t + s];
    __syncthreads();
  }
  if (t == 0) red[4] = sh[0] * natom * 0.25;
}

// One warp per (pair p, row r): acc = sum_q fq[p][q] mx[r][q]; the table entry becomes base + acc.
// NNP: rows of class 0 and 3 of the [P][4][nbin+1] table, class 3 as base + acc * special_lj[3].
// comp: 0 writes the force slot, 1 the potential slot of the float2 entry (classical tables hold
// (F/r, U), the network's (U, F/r)).
template <bool NNP>
__global__ void k_rmdf_r(const double* __restrict__ fq, const double* __restrict__ mx, const float2* __restrict__ base,
                         float2* table, int P, int nbin, int nq, int comp) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= P * nbin) return;
  const int p = warp / nbin, r = warp % nbin;
  double acc = 0;
  for (int q = lane; q < nq; q += 32) acc += fq[(size_t)p * nq + q] * mx[(size_t)r * nq + q];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane != 0) return;
  const int nb1 = nbin + 1;
  if (!NNP) {
    const size_t k = (size_t)p * nb1 + r;
    float2 v = table[k];
    const float2 b = base[k];
    if (comp == 0) v.x = (float)((double)b.x + acc);
    else v.y = (float)((double)b.y + acc);
    table[k] = v;
  } else {
    const size_t k0 = (size_t)(p * 4 + 0) * nb1 + r, k3 = (size_t)(p * 4 + 3) * nb1 + r;
    float2 v0 = table[k0], v3 = table[k3];
    const float2 b0 = base[k0], b3 = base[k3];
    if (comp == 0) {   // (U, F/r): force in .y
      v0.y = (float)((double)b0.y + acc);
      v3.y = (float)((double)b3.y + acc * kSpecialLj14);
    } else {
      v0.x = (float)((double)b0.x + acc);
      v3.x = (float)((double)b3.x + acc * kSpecialLj14);
    }
    table[k0] = v0;
    table[k3] = v3;
  }
}

template <typename T>
int dput(nnpe_ctx* c, T** d, const std::vector<T>& h) {
  if (*d) dev_free(*d);
  *d = nullptr;
  NNPE_CUDA(c, dev_malloc(c, (void**)d, sizeof(T) * std::max<size_t>(h.size(), 1)));
  if (!h.empty()) NNPE_CUDA(c, cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return 0;
}

float2* rmdf_table(nnpe_ctx* c) { return c->rmdf->nnp ? c->nnp->d_tpair : c->d_table; }

}  // namespace

void rmdf_free(nnpe_ctx* c) {
  RmdfState* r = c->rmdf;
  if (!r) return;
  for (void* p : {(void*)r->d_sqwt, (void*)r->d_fwt, (void*)r->d_sqex, (void*)r->d_wt, (void*)r->d_dsq, (void*)r->d_sqn,
                  (void*)r->d_fq, (void*)r->d_ftmx, (void*)r->d_potmx, (void*)r->d_base})
    if (p) dev_free(p);
  delete r;
  c->rmdf = nullptr;
}

// Parts of an update on the S(q) of the last g(r) step (bit 1 compute_Qspace, 2 compute_Rspace,
// 4 compute_Potential); erg_exp lands in d_red[4].
static int rmdf_parts_enqueue(nnpe_ctx* c, int parts) {
  RmdfState* r = c->rmdf;
  if (!r) return 0;
  if (parts & 1)
    k_rmdf_q<<<1, 512, 0, c->stream>>>(c->d_sq, r->d_sqwt, r->d_fwt, r->d_sqex, r->d_wt, r->d_dsq, r->d_sqn, r->d_fq,
                                       r->n_sq, r->P, r->nq, r->gamma, (double)c->natom, c->d_red);
  float2* tbl = rmdf_table(c);
  const int warps = r->P * r->nbin, blocks = nblocks((long)warps * 32, 256);
  for (int comp = 0; comp < 2; ++comp) {
    if (!(parts & (comp == 0 ? 2 : 4))) continue;
    const double* mx = comp == 0 ? r->d_ftmx : r->d_potmx;
    if (r->nnp) k_rmdf_r<true><<<blocks, 256, 0, c->stream>>>(r->d_fq, mx, r->d_base, tbl, r->P, r->nbin, r->nq, comp);
    else k_rmdf_r<false><<<blocks, 256, 0, c->stream>>>(r->d_fq, mx, r->d_base, tbl, r->P, r->nbin, r->nq, comp);
  }
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

// compute_Qspace + compute_Rspace (+ compute_Potential) of a g(r) step of the loop.
int rmdf_step_enqueue(nnpe_ctx* c, bool potential) { return rmdf_parts_enqueue(c, potential ? 7 : 3); }

bool rmdf_potential_on_log(const nnpe_ctx* c) { return c->rmdf && c->rmdf->gamma != 1.0; }

// RMDF constructor (grsq.cpp:899-1059) from arrays: per target n and q point, sqex, wt (before
// `strength`) and the ntype scattering factors ff[n][q][t].
extern "C" int nnpe_rmdf_set(nnpe_ctx* c, int n_sq, const double* sqex, const double* wt, const double* ff,
                             double strength, double gamma) {
  if (!c || !c->d_gr_counts || n_sq <= 0 || !sqex || !wt || !ff)
    return nnpe_fail(c, NNPE_EARG, "nnpe_rmdf_set: needs nnpe_gr_setup and at least one target");
  if (!(gamma >= 0 && gamma <= 1)) return nnpe_fail(c, NNPE_EARG, "invalid gamma");   // grsq.cpp:904
  cudaSetDevice(c->device);
  const bool nnp = !c->pair_on || !c->d_table;
  int nbin;
  float tdr;
  if (!nnp) {
    nbin = c->nbin;
    tdr = c->pair_cutoff / c->nbin;
  } else {
    if (!c->nnp || !c->nnp->d_tpair) return nnpe_fail(c, NNPE_EARG, "nnpe_rmdf_set: no pair table to refine");
    nbin = c->nnp->nbin;
    tdr = c->nnp->rc / c->nnp->nbin;
  }
  // grsq.cpp:926-947: the table grid must be the g(r) grid (EPSILON = 1e-5, environ.h)
  if (nbin != c->gr_nbin_inner || std::fabs(tdr - c->gr_dr) > 1e-5f) return nnpe_fail(c, NNPE_EARG, "RMDF mismatch");
  rmdf_free(c);
  auto* r = new RmdfState();
  c->rmdf = r;
  const int P = c->npair, nq = c->gr_nq, T = c->ntype;
  r->n_sq = n_sq; r->nq = nq; r->nbin = nbin; r->P = P; r->gamma = gamma; r->strength = strength; r->nnp = nnp;
  std::vector<long long> cnt(T, 0);
  for (int t : c->h_typ) ++cnt[t];
  const double natom = c->natom, natsq = natom * natom;
  std::vector<double> vsqwt((size_t)n_sq * P * nq), vfwt((size_t)n_sq * P * nq), vsqex(sqex, sqex + (size_t)n_sq * nq),
      vwt((size_t)n_sq * nq);
  for (int n = 0; n < n_sq; ++n)
    for (int i = 0; i < nq; ++i) {
      const double w = wt[(size_t)n * nq + i] * strength;
      vwt[(size_t)n * nq + i] = w;
      const double* f = ff + ((size_t)n * nq + i) * T;
      double cifi2 = 0;
      for (int j = 0; j < T; ++j) cifi2 += f[j] * cnt[j];
      cifi2 = (cifi2 / natom) * (cifi2 / natom);
      for (int j = 0, ip = 0; j < T; ++j) {
        const double ni = cnt[j] / natsq;
        for (int k = j; k < T; ++k, ++ip) {
          const double fw = f[j] * f[k] / cifi2;
          vsqwt[((size_t)n * P + ip) * nq + i] = fw * cnt[k] * ni * (k == j ? 1 : 2);
          vfwt[((size_t)n * P + ip) * nq + i] = fw * w;
        }
      }
    }
  // grids: rr = (i+.5F)dr of GR (grsq.cpp:53), qq = (i+.5F)dq of SQ (grsq.cpp:272), as floats
  r->h_qq.resize(nq);
  const float dq = (float)c->gr_qmax / nq;
  for (int i = 0; i < nq; ++i) r->h_qq[i] = (i + .5F) * dq;
  std::vector<double> ftmx((size_t)nbin * nq), potmx((size_t)nbin * nq);
  for (int i = 0; i < nbin; ++i) {
    const double rr = (double)((i + 0.5F) * c->gr_dr), fi = 1 / (rr * rr);
    for (int j = 0; j < nq; ++j) {
      const double qr = (double)r->h_qq[j] * rr, j0 = std::sin(qr) / qr;
      potmx[(size_t)i * nq + j] = j0;
      ftmx[(size_t)i * nq + j] = fi * (j0 - std::cos(qr));
    }
  }
  std::vector<double> zero((size_t)n_sq * nq, 0.0);
  r->h_dsq_acc = zero;
  if (int rc = dput(c, &r->d_sqwt, vsqwt)) return rc;
  if (int rc = dput(c, &r->d_fwt, vfwt)) return rc;
  if (int rc = dput(c, &r->d_sqex, vsqex)) return rc;
  if (int rc = dput(c, &r->d_wt, vwt)) return rc;
  if (int rc = dput(c, &r->d_dsq, zero)) return rc;
  if (int rc = dput(c, &r->d_sqn, zero)) return rc;
  if (int rc = dput(c, &r->d_fq, std::vector<double>((size_t)P * nq, 0.0))) return rc;
  if (int rc = dput(c, &r->d_ftmx, ftmx)) return rc;
  if (int rc = dput(c, &r->d_potmx, potmx)) return rc;
  // the *_base tables: the table as it stands now (loadPotential(1) copies base to force, pair.cpp:245-250)
  const size_t tsz = nnp ? (size_t)P * 4 * (nbin + 1) : (size_t)P * (nbin + 1);
  NNPE_CUDA(c, dev_malloc(c, (void**)&r->d_base, sizeof(float2) * tsz));
  NNPE_CUDA(c, cudaMemcpy(r->d_base, rmdf_table(c), sizeof(float2) * tsz, cudaMemcpyDeviceToDevice));
  double zero5 = 0;
  NNPE_CUDA(c, cudaMemcpy(c->d_red + 4, &zero5, sizeof(double), cudaMemcpyHostToDevice));
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

// Target files in the reference's format (grsq.cpp:897, 974-1018): nq lines of
// q S_exp(q) wt(q) f_0(q) ... f_{ntype-1}(q); at most 2 targets (run.cpp:163).
extern "C" int nnpe_rmdf_load(nnpe_ctx* c, int n_sq, const char* const* files, double strength, double gamma) {
  if (!c || !c->d_gr_counts || n_sq <= 0 || n_sq > 2 || !files) return nnpe_fail(c, NNPE_EARG, "nnpe_rmdf_load: 1 or 2 targets");
  const int nq = c->gr_nq, T = c->ntype;
  std::vector<double> sqex((size_t)n_sq * nq), wt((size_t)n_sq * nq), ff((size_t)n_sq * nq * T);
  for (int n = 0; n < n_sq; ++n) {
    FILE* fp = fopen(files[n], "r");
    if (!fp) return nnpe_fail(c, NNPE_EFILE, std::string("read error: ") + files[n]);
    for (int i = 0; i < nq; ++i) {
      float q, s, w;
      if (fscanf(fp, "%f %f %f", &q, &s, &w) != 3) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, std::string("short S(q) file ") + files[n]); }
      sqex[(size_t)n * nq + i] = s;
      wt[(size_t)n * nq + i] = w;
      for (int t = 0; t < T; ++t) {
        float f;
        if (fscanf(fp, "%f", &f) != 1) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, std::string("short S(q) file ") + files[n]); }
        ff[((size_t)n * nq + i) * T + t] = f;
      }
    }
    fclose(fp);
  }
  return nnpe_rmdf_set(c, n_sq, sqex.data(), wt.data(), ff.data(), strength, gamma);
}

// Parts of one refinement update on the current g(r) (tally + S(q) of the last call to
// nnpe_sq_compute or of the step loop).
extern "C" int nnpe_rmdf_step(nnpe_ctx* c, int parts, double* erg_exp) {
  if (!c || !c->rmdf) return nnpe_fail(c, NNPE_EARG, "nnpe_rmdf_step: no RMDF set up");
  cudaSetDevice(c->device);
  if (int rc = rmdf_parts_enqueue(c, parts)) return rc;
  if (erg_exp) NNPE_CUDA(c, cudaMemcpyAsync(erg_exp, c->d_red + 4, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  return NNPE_OK;
}

// Weighted S_n(q), deltaS_n(q) [n_sq][nq] and force_q [npair][nq] of the last update (any may be NULL).
extern "C" int nnpe_rmdf_get(nnpe_ctx* c, double* sq, double* deltasq, double* force_q) {
  if (!c || !c->rmdf) return nnpe_fail(c, NNPE_EARG, "nnpe_rmdf_get: no RMDF set up");
  RmdfState* r = c->rmdf;
  const size_t ns = (size_t)r->n_sq * r->nq;
  if (sq) NNPE_CUDA(c, cudaMemcpyAsync(sq, r->d_sqn, sizeof(double) * ns, cudaMemcpyDeviceToHost, c->stream));
  if (deltasq) NNPE_CUDA(c, cudaMemcpyAsync(deltasq, r->d_dsq, sizeof(double) * ns, cudaMemcpyDeviceToHost, c->stream));
  if (force_q) NNPE_CUDA(c, cudaMemcpyAsync(force_q, r->d_fq, sizeof(double) * r->P * r->nq, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  return NNPE_OK;
}

// RMDF::loadDeltaSQ (grsq.cpp:1419-1443): deltaS from a dumpSQ file (column 2 of each target, or
// column 3, the running average, when gamma == 0). A missing file is not an error, as there.
extern "C" int nnpe_rmdf_load_delta(nnpe_ctx* c, const char* fname) {
  if (!c || !c->rmdf || !fname) return nnpe_fail(c, NNPE_EARG, "nnpe_rmdf_load_delta");
  RmdfState* r = c->rmdf;
  FILE* fp = fopen(fname, "r");
  if (!fp) return NNPE_OK;
  std::vector<double> d((size_t)r->n_sq * r->nq);
  int num;
  if (fscanf(fp, "# %d ", &num) != 1) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, "bad deltaS file"); }
  for (int i = 0; i < r->nq; ++i) {
    float q;
    if (fscanf(fp, "%f ", &q) != 1) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, "short deltaS file"); }
    for (int n = 0; n < r->n_sq; ++n) {
      float a, b, e;
      if (fscanf(fp, "%f %f %f ", &a, &b, &e) != 3) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, "short deltaS file"); }
      d[(size_t)n * r->nq + i] = r->gamma == 0 ? e : b;
    }
  }
  fclose(fp);
  NNPE_CUDA(c, cudaMemcpy(r->d_dsq, d.data(), sizeof(double) * d.size(), cudaMemcpyHostToDevice));
  return NNPE_OK;
}

// RMDF::dumpSQ (grsq.cpp:1380-1416): "# num" then per q: q and, per target, S_n, deltaS_n and the
// running average of deltaS over up to 100 appended dumps (S_n averaged the same way).
extern "C" int nnpe_rmdf_dump_sq(nnpe_ctx* c, const char* fname, int append) {
  if (!c || !c->rmdf || !fname) return nnpe_fail(c, NNPE_EARG, "nnpe_rmdf_dump_sq");
  RmdfState* r = c->rmdf;
  const size_t ns = (size_t)r->n_sq * r->nq;
  std::vector<double> sq(ns), dsq(ns);
  if (int rc = nnpe_rmdf_get(c, sq.data(), dsq.data(), nullptr)) return rc;
  int num = 1;
  double factor = 1, cofactor = 0;
  FILE* fp;
  if (append && (fp = fopen(fname, "r"))) {
    if (fscanf(fp, "# %d ", &num) == 1) {
      num = std::min(num + 1, 100);   // MAXACC (grsq.cpp:25)
      factor = 1.0 / num;
      cofactor = 1 - factor;
      for (int i = 0; i < r->nq; ++i) {
        double q;
        if (fscanf(fp, "%lf ", &q) != 1) break;
        for (int n = 0; n < r->n_sq; ++n) {
          double a, b, e;
          if (fscanf(fp, "%lf %lf %lf ", &a, &b, &e) != 3) break;
          sq[(size_t)n * r->nq + i] = sq[(size_t)n * r->nq + i] * factor + cofactor * a;
          r->h_dsq_acc[(size_t)n * r->nq + i] = e;
        }
      }
    }
    fclose(fp);
  }
  fp = fopen(fname, "w");
  if (!fp) return nnpe_fail(c, NNPE_EFILE, std::string("cannot write ") + fname);
  fprintf(fp, "# %d\n", num);
  for (int i = 0; i < r->nq; ++i) {
    fprintf(fp, "%.15e", (double)r->h_qq[i]);
    for (int n = 0; n < r->n_sq; ++n) {
      const size_t k = (size_t)n * r->nq + i;
      fprintf(fp, " %.15e %.15e %.15e", sq[k], dsq[k], dsq[k] * factor + cofactor * r->h_dsq_acc[k]);
    }
    fprintf(fp, "\n");
  }
  fclose(fp);
  return NNPE_OK;
}
