// Network term: NNPOTENTIAL_TBL (pair_nnp.cpp:433-793) and the radial-embedding network.
//
// Two descriptor kinds share one pipeline (computeDescriptor -> nnEval -> compute, the call
// sequence of run.cpp:1234-1249):
//  * gauss: the reference's tabulated NNP. Tables tbl_pair/tbl_f_pair [npair][4][nbin+1] and
//    tbl_desc/tbl_f_desc [npair][80][nbin+1] are generated on the host with the reference's float
//    arithmetic (pair_nnp.cpp:521-590); 20 descriptor slots per atom, the special class selecting
//    which 20 functions a pair adds (pair_nnp.cpp:663-683).
//  * embed: per neighbour species an embedding net u=r/rc -> e1 -> e2 (tanh), times the
//    reference's cutoff factor cff(r) and a descriptor scale, accumulated into slot s*e2+c.
// Both feed a per-species fitting network din -> h1 -> h2 -> 1 (tanh) whose hand-written backward
// gives dE/dG; forces are the reference's back-projection
// fpair = f_pair(r) + sum_c (dE/dG_i + dE/dG_j)[c] f_desc_c(r),  F_i += fpair (x_i - x_j).
//
// Work split: a compact per-step list of the pairs inside the network cutoff (exact float test as
// the reference's rsq<cutsq, pair_nnp.cpp:656) is filtered from the Verlet list; descriptor and
// force kernels run one warp per atom over it (no atomics); the fitting network runs as tiled
// GEMMs per species. precision 0 = FP32 on CUDA cores; precision 1 = BF16 tcgen05 (nnp_tc.cu).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.cuh"
#include "nnp.cuh"

// ---------------------------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------------------------
template <typename T>
static int nalloc(nnpe_ctx* c, T** p, size_t n) {
  if (*p) dev_free(*p);
  *p = nullptr;
  NNPE_CUDA(c, dev_malloc(c, (void**)p, std::max<size_t>(n, 1) * sizeof(T)));
  return 0;
}
template <typename T>
static void nfree(T** p) {
  if (*p) dev_free(*p);
  *p = nullptr;
}

void nnp_free(nnpe_ctx* c) {
  NnpModel* m = c->nnp;
  if (!m) return;
  nfree(&m->d_embw); nfree(&m->d_fitw); nfree(&m->d_fitg); nfree(&m->d_tdesc); nfree(&m->d_tpair); nfree(&m->d_G); nfree(&m->d_dG);
  nfree(&m->d_enet); nfree(&m->d_list6); nfree(&m->d_n6); nfree(&m->d_sidx); nfree(&m->d_scount);
  nfree(&m->d_H1); nfree(&m->d_G2); nfree(&m->d_G1); nfree(&m->d_soff_dev);
  nnp_tc_free(m);
  delete m;
  c->nnp = nullptr;
}

const double* nnp_atom_energy_ptr(nnpe_ctx* c) { return c->nnp && c->nnp->enabled ? c->nnp->d_enet : nullptr; }
bool nnp_enabled(nnpe_ctx* c) { return c->nnp && c->nnp->enabled; }
float nnp_cutoff(nnpe_ctx* c) { return c->nnp ? c->nnp->rc : 0.f; }
bool nnp_list6(nnpe_ctx* c, uint32_t** list6, int** n6, int* cap6, float* cut6) {
  if (!c->nnp) return false;
  *list6 = c->nnp->d_list6; *n6 = c->nnp->d_n6; *cap6 = c->nnp->cap6; *cut6 = c->nnp->rc;
  return true;
}

int nnpe_nnp_enable(nnpe_ctx* c, int on) {
  if (!c || !c->nnp) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_enable: no network");
  c->nnp->enabled = on != 0;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

// pair_nnp.cpp:521-590 in the reference's float arithmetic (exp is the C library's float exp).
static void gen_tables(int npair, float cutoff, int nbin, const float* coef_p_in, const float* coef_w,
                       const float* coef_d, const float* coef_r, std::vector<float2>& tpair, std::vector<float2>& tdesc) {
  const int szd = 80, nb1 = nbin + 1;
  tpair.assign((size_t)npair * 4 * nb1, make_float2(0, 0));
  tdesc.assign((size_t)npair * szd * nb1, make_float2(0, 0));
  std::vector<float> cp(coef_p_in, coef_p_in + (size_t)npair * 24);
  const float dr = cutoff / nbin;
  auto sqr = [](float a) { return a * a; };
  for (int p = 0; p < npair; ++p) {
    for (int k = 0; k < 4; ++k) {
      float* q = cp.data() + p * 24 + k * 6;
      float src2 = sqr(q[1] / cutoff), src6 = src2 * src2 * src2;
      const float elim = -2 * q[5] / cutoff - q[0] * src6 * (-7 + src2 * (9 * q[2] + src2 * (11 * q[3] + src2 * 13 * q[4])));
      const float flim = (q[5] / cutoff + q[0] * src6 * (-6 + src2 * ((q[2] *= 8) + src2 * ((q[3] *= 10) + src2 * (q[4] *= 12))))) / cutoff;
      q[1] *= q[1];
      float2* t = tpair.data() + ((size_t)p * 4 + k) * nb1;
      for (int i = 0; i < nbin; ++i) {
        float rr, rsq;
        rsq = sqr(rr = dr * (i + 0.5));
        src2 = q[1] / rsq;
        src6 = src2 * src2 * src2;
        const float f = (q[5] / rr + (*q) * src6 * (-6 + src2 * (q[2] + src2 * (q[3] + src2 * q[4])))) / rsq - (flim) / rr;
        const float u = q[5] / rr + (*q) * src6 * (-1 + src2 * (q[2] * .125F + src2 * (q[3] * .1F + src2 * q[4] * .08333333333333333333F))) +
                        (flim) * rr + elim;
        t[i] = make_float2(u, f);   // (U, F/r)
      }
      t[nbin] = make_float2(0, 0);
    }
    const float *w = coef_w + (size_t)p * szd, *d = coef_d + (size_t)p * szd, *r0 = coef_r + (size_t)p * szd;
    for (int i = 0; i < nbin; ++i) {
      float rr = dr * (i + 0.5), cf2, rrcsq_1, cff, cfr;
      rrcsq_1 = 1 + sqr(cf2 = rr - cutoff);
      cfr = (-2 * (cff = 1 - 1 / rrcsq_1)) / rr;
      cf2 /= (-.5f * rr * sqr(rrcsq_1));
      for (int k = 0; k < szd; ++k) {
        const float rr0 = rr - r0[k];
        const float drr0 = d[k] * rr0;
        const float wexp = std::exp(drr0 * rr0) * w[k];
        tdesc[((size_t)p * szd + k) * nb1 + i] = make_float2(wexp * cff, wexp * (cf2 + drr0 * cfr));   // (desc, f_desc)
      }
    }
  }
}

static size_t fit_block(int din, int h1, int h2) { return (size_t)din * h1 + h1 + (size_t)h1 * h2 + h2 + h2 + 1; }
static constexpr int kEmbWarpsHost = 4;
static constexpr int kDescScratchHost = 32 * 32 + 3 * 32;                     // floats per warp, k_emb_desc_f32
static constexpr int kForceScratchHost = 16 * (32 + 32 + 33) + 10 * 32;   // floats per warp, k_emb_force_f32
static int nnp_set_smem_attrs(nnpe_ctx* c, int smem_desc, int smem_force);

int nnpe_nnp_set(nnpe_ctx* c, int kind, double cutoff, int nbin, double scale, int e1, int e2, int h1, int h2,
                 const float* coef_p, const float* coef_w, const float* coef_d, const float* coef_r, const float* embw,
                 const float* fitw) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_set: call nnpe_setup first");
  if ((kind != 0 && kind != 1) || !(cutoff > 0) || h1 <= 0 || h2 <= 0 || h1 > 256 || h2 > 256 || !fitw)
    return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_set: bad network shape");
  if ((float)cutoff > c->pair_cutoff + c->skin) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_set: network cutoff beyond the list");
  if (kind == 1 && (e1 != 32 || e2 != 64 || !embw)) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_set: embedding must be 1->32->64");
  if (kind == 0 && (nbin <= 0 || !coef_p || !coef_w || !coef_d || !coef_r)) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_set: tables need coefficients");
  cudaSetDevice(c->device);
  nnp_free(c);
  auto* m = new NnpModel();
  c->nnp = m;
  m->kind = kind; m->rc = (float)cutoff; m->nbin = nbin; m->scale = (float)scale; m->e1 = e1; m->e2 = e2;
  m->din = kind == 0 ? 20 : 4 * e2; m->h1 = h1; m->h2 = h2; m->ntype = c->ntype; m->npair = c->npair;
  m->cap6 = 256;
  const int N = c->natom;
  int rc = 0;
  if (kind == 0) {
    std::vector<float2> tp, td;
    gen_tables(c->npair, m->rc, nbin, coef_p, coef_w, coef_d, coef_r, tp, td);
    if ((rc = nalloc(c, &m->d_tpair, tp.size())) || (rc = nalloc(c, &m->d_tdesc, td.size()))) return rc;
    NNPE_CUDA(c, cudaMemcpy(m->d_tpair, tp.data(), sizeof(float2) * tp.size(), cudaMemcpyHostToDevice));
    NNPE_CUDA(c, cudaMemcpy(m->d_tdesc, td.data(), sizeof(float2) * td.size(), cudaMemcpyHostToDevice));
    m->h_tpair = tp;
  } else {
    const size_t eb = (size_t)e1 + e1 + (size_t)e1 * e2 + e2;
    if ((rc = nalloc(c, &m->d_embw, eb * c->ntype))) return rc;
    NNPE_CUDA(c, cudaMemcpy(m->d_embw, embw, sizeof(float) * eb * c->ntype, cudaMemcpyHostToDevice));
    m->h_embw.assign(embw, embw + eb * c->ntype);
  }
  const size_t fb = fit_block(m->din, h1, h2);
  if ((rc = nalloc(c, &m->d_fitw, fb * c->ntype))) return rc;
  NNPE_CUDA(c, cudaMemcpy(m->d_fitw, fitw, sizeof(float) * fb * c->ntype, cudaMemcpyHostToDevice));
  m->h_fitw.assign(fitw, fitw + fb * c->ntype);
  {   // aligned copies for the FP32 GEMMs, with the backward's transposed weights
    const int D = m->din;
    auto up4 = [](size_t n) { return (n + 3) & ~(size_t)3; };
    const size_t o2 = up4((size_t)D * h1), o2t = o2 + up4((size_t)h1 * h2), o1t = o2t + up4((size_t)h2 * h1),
                 oc1 = o1t + up4((size_t)h1 * D), oc2 = oc1 + up4(h1), oa3 = oc2 + up4(h2);
    m->fitg_block = oa3 + up4(h2);
    std::vector<float> g(m->fitg_block * c->ntype, 0.f);
    for (int t = 0; t < c->ntype; ++t) {
      const float* w = fitw + fb * t;
      const float *A1 = w, *c1 = A1 + (size_t)D * h1, *A2 = c1 + h1, *c2 = A2 + (size_t)h1 * h2, *A3 = c2 + h2;
      float* o = g.data() + m->fitg_block * t;
      std::copy(A1, A1 + (size_t)D * h1, o);
      std::copy(A2, A2 + (size_t)h1 * h2, o + o2);
      for (int k = 0; k < h2; ++k)
        for (int n2 = 0; n2 < h1; ++n2) o[o2t + (size_t)k * h1 + n2] = A2[(size_t)n2 * h2 + k];
      for (int k = 0; k < h1; ++k)
        for (int n2 = 0; n2 < D; ++n2) o[o1t + (size_t)k * D + n2] = A1[(size_t)n2 * h1 + k];
      std::copy(c1, c1 + h1, o + oc1);
      std::copy(c2, c2 + h2, o + oc2);
      std::copy(A3, A3 + h2, o + oa3);
    }
    if ((rc = nalloc(c, &m->d_fitg, g.size()))) return rc;
    NNPE_CUDA(c, cudaMemcpy(m->d_fitg, g.data(), sizeof(float) * g.size(), cudaMemcpyHostToDevice));
  }
  if ((rc = nalloc(c, &m->d_G, (size_t)N * m->din)) || (rc = nalloc(c, &m->d_dG, (size_t)N * m->din)) ||
      (rc = nalloc(c, &m->d_enet, N)) || (rc = nalloc(c, &m->d_list6, (size_t)N * m->cap6)) ||
      (rc = nalloc(c, &m->d_n6, N)) || (rc = nalloc(c, &m->d_sidx, N)) || (rc = nalloc(c, &m->d_scount, NNPE_MAX_TYPES)) ||
      (rc = nalloc(c, &m->d_H1, (size_t)N * h1)) || (rc = nalloc(c, &m->d_G2, (size_t)N * h2)) ||
      (rc = nalloc(c, &m->d_G1, (size_t)N * h1)))
    return rc;
  NNPE_CUDA(c, cudaMemset(m->d_enet, 0, sizeof(double) * N));
  NNPE_CUDA(c, cudaMemset(m->d_n6, 0, sizeof(int) * N));
  // species offsets are fixed (type counts); membership follows the sort
  m->soff.assign(c->ntype + 1, 0);
  std::vector<int> cnt(c->ntype, 0);
  for (int t : c->h_typ) ++cnt[t];
  for (int t = 0; t < c->ntype; ++t) m->soff[t + 1] = m->soff[t] + cnt[t];
  if ((rc = nalloc(c, &m->d_soff_dev, NNPE_MAX_TYPES + 1))) return rc;
  NNPE_CUDA(c, cudaMemcpy(m->d_soff_dev, m->soff.data(), sizeof(int) * m->soff.size(), cudaMemcpyHostToDevice));
  // species lists: counters start at zero, and the next evaluation builds the lists (k_species)
  NNPE_CUDA(c, cudaMemset(m->d_scount, 0, sizeof(int) * NNPE_MAX_TYPES));
  {
    const int one = 1;
    NNPE_CUDA(c, cudaMemcpy(c->d_ctrl + CTRL_RESORT, &one, sizeof(int), cudaMemcpyHostToDevice));
  }
  if (kind == 1) {
    const size_t eb = (size_t)32 + 32 + 32 * (size_t)e2 + e2;
    const int smem_desc = (int)(sizeof(float) * (eb * c->ntype + kEmbWarpsHost * kDescScratchHost));
    const int smem_force = (int)(sizeof(float) * (eb * c->ntype + kEmbWarpsHost * kForceScratchHost));
    if (int r2 = nnp_set_smem_attrs(c, smem_desc, smem_force)) return r2;
  }
  c->graph_valid = false;
  c->fs_valid = false;
  return nnp_tc_setup(c);
}

int nnpe_nnp_precision(nnpe_ctx* c, int bf16) {
  if (!c || !c->nnp) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_precision: no network");
  if (bf16 && c->nnp->kind != 1) return nnpe_fail(c, NNPE_EARG, "BF16 tensor-core path is for the embedding network");
  c->nnp->bf16 = bf16 != 0;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

// ---------------------------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------------------------
namespace {

// Pairs inside the network cutoff, in list order, with the reference's float test rsq<cutsq.
__global__ void __launch_bounds__(128) k_filter6(const float4* __restrict__ pos, const uint32_t* __restrict__ list,
                                                 const int* __restrict__ ncount, int cap, uint32_t* __restrict__ list6,
                                                 int* __restrict__ n6, int cap6, float cutsq, int N, int* ctrl) {
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= N) return;
  const float4 xi = pos[i];
  const uint32_t* row = list + (size_t)i * cap;
  uint32_t* out = list6 + (size_t)i * cap6;
  const int n = ncount[i];
  int cnt = 0;
  for (int base = 0; base < n; base += 32) {
    const int k = base + lane;
    bool ok = false;
    uint32_t e = 0;
    if (k < n) {
      e = row[k];
      const float4 xj = pos[e & NNPE_J_MASK];
      ok = rsq3(fsub(xi.x, xj.x), fsub(xi.y, xj.y), fsub(xi.z, xj.z)) < cutsq;
    }
    const unsigned b = __ballot_sync(0xffffffffu, ok);
    if (ok) {
      const int idx = cnt + __popc(b & ((1u << lane) - 1));
      if (idx < cap6) out[idx] = e;
    }
    cnt += __popc(b);
  }
  if (lane == 0) {
    n6[i] = min(cnt, cap6);
    if (cnt > cap6) atomicOr(ctrl + CTRL_ERR, NNPE_DEV_LIST_OVERFLOW);
  }
}

// Species membership lists (sorted atom indices grouped by type) for the per-species fitting net.
// (The order within a species is arbitrary: every fitting row depends on its own atom only.)
// One counter update per warp and species. The lists change only with the sorted order, so the
// kernel works only when CTRL_RESORT is set (a rebuild or a new network) and returns at once
// otherwise; the last block to finish clears the flag and the counters (zero for the next time).
__global__ void k_species(const int2* __restrict__ info, int* __restrict__ sidx, int* __restrict__ scount,
                          const int* __restrict__ soff, int N, int ntype, int* ctrl) {
  if (*reinterpret_cast<volatile int*>(ctrl + CTRL_RESORT) == 0) return;   // grid-uniform
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int t = i < N ? (info[i].y & 0xFF) : -1;
  for (int sp = 0; sp < ntype; ++sp) {
    const unsigned m = __ballot_sync(0xffffffffu, t == sp);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&scount[sp], __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (t == sp) sidx[soff[sp] + base + __popc(m & ((1u << lane) - 1))] = i;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(reinterpret_cast<unsigned*>(ctrl + CTRL_RESORT_DONE), 1u) == gridDim.x - 1) {
      for (int sp = 0; sp < ntype; ++sp) scount[sp] = 0;
      ctrl[CTRL_RESORT] = 0;
      ctrl[CTRL_RESORT_DONE] = 0;
    }
  }
}

__device__ __forceinline__ int owner_of(int j, int N, const int* __restrict__ gowner) { return j < N ? j : gowner[j - N]; }

// ---- gauss (tabulated) descriptor: computeDescriptor (pair_nnp.cpp:625-688) ----
__global__ void __launch_bounds__(128) k_gauss_desc(NnpArgs a) {
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= a.N) return;
  const float4 xi = a.pos[i];
  const int* ptrow = a.pairtype + (a.info[i].y & 0xFF) * a.ntype;
  const uint32_t* row = a.list6 + (size_t)i * a.cap6;
  const int n = a.n6[i];
  float acc[20];
#pragma unroll
  for (int k = 0; k < 20; ++k) acc[k] = 0.f;
  const int nb1 = a.nbin + 1;
  for (int k = lane; k < n; k += 32) {
    const uint32_t e = row[k];
    const float4 xj = a.pos[e & NNPE_J_MASK];
    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz);
    float ipw1 = r * a.r_dr - 0.5F;
    const int t1 = (int)ipw1;
    const float ipw2 = ipw1 - (float)t1;
    ipw1 = 1 - ipw2;
    const int s = e >> 30, p = ptrow[(e >> 27) & 7];
    const float2* t = a.tdesc + ((size_t)p * 80 + 20 * s) * nb1 + t1;
#pragma unroll
    for (int c = 0; c < 20; ++c) {
      const float2 u = __ldg(t + (size_t)c * nb1), v = __ldg(t + (size_t)c * nb1 + 1);
      acc[c] += u.x * ipw1 + v.x * ipw2;
    }
  }
#pragma unroll
  for (int c = 0; c < 20; ++c) {
    float v = acc[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[c] = v;
  }
  if (lane < 20) {
    float v = 0.f;
#pragma unroll
    for (int c = 0; c < 20; ++c) v = lane == c ? acc[c] : v;
    a.G[(size_t)i * 20 + lane] = v;
  }
}

// ---- gauss force: NNPOTENTIAL_TBL::compute<ev> (pair_nnp.cpp:710-793) ----
template <bool EV>
__global__ void __launch_bounds__(128) k_gauss_force(NnpArgs a) {
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= a.N) return;
  const float4 xi = a.pos[i];
  const int* ptrow = a.pairtype + (a.info[i].y & 0xFF) * a.ntype;
  const uint32_t* row = a.list6 + (size_t)i * a.cap6;
  const int n = a.n6[i];
  const float* dGi = a.dG + (size_t)i * 20;
  const int nb1 = a.nbin + 1;
  float fx = 0, fy = 0, fz = 0;
  double e = 0, w = 0;
  for (int k = lane; k < n; k += 32) {
    const uint32_t ent = row[k];
    const int j = ent & NNPE_J_MASK;
    const float4 xj = a.pos[j];
    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    const float rsq = dx * dx + dy * dy + dz * dz;
    const float r = sqrtf(rsq);
    float ipw1 = r * a.r_dr - 0.5F;
    const int t1 = (int)ipw1;
    const float ipw2 = ipw1 - (float)t1;
    ipw1 = 1 - ipw2;
    const int s = ent >> 30, p = ptrow[(ent >> 27) & 7];
    const float2* tp = a.tpair + ((size_t)p * 4 + s) * nb1 + t1;
    const float2 pa = __ldg(tp), pb = __ldg(tp + 1);
    float fpair = pa.y * ipw1 + pb.y * ipw2;
    const float* dGj = a.dG + (size_t)owner_of(j, a.N, a.gowner) * 20;
    const float2* t = a.tdesc + ((size_t)p * 80 + 20 * s) * nb1 + t1;
#pragma unroll 4
    for (int c = 0; c < 20; ++c) {
      const float2 u = __ldg(t + (size_t)c * nb1), v = __ldg(t + (size_t)c * nb1 + 1);
      fpair += (dGi[c] + dGj[c]) * (u.y * ipw1 + v.y * ipw2);
    }
    fx += dx * fpair; fy += dy * fpair; fz += dz * fpair;
    if (EV) {
      e += 0.5 * (double)(pa.x * ipw1 + pb.x * ipw2);
      w += 0.5 * (double)(fpair * rsq);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
    if (EV) {
      e += __shfl_xor_sync(0xffffffffu, e, o);
      w += __shfl_xor_sync(0xffffffffu, w, o);
    }
  }
  if (lane == 0) {
    const float4 f = a.frc[i];
    a.frc[i] = make_float4(f.x + fx, f.y + fy, f.z + fz, f.w);
    if (EV) { a.eatom[i] += e; a.watom[i] += w; }
  }
}

// ---- FP32 embedding network on CUDA cores (the plain form). One warp per atom. Lane l owns output
// channels 2l and 2l+1, and the warp takes the atom's pairs one neighbour species at a time, so that
// it holds that species' second-layer weights W2[q][2l], W2[q][2l+1] (64 values) in registers. Per
// group of up to 32 pairs of the species (ballot-compacted from the list), lane q computes
// first-layer unit q of every pair into shared memory; then pair by pair every lane reads the pair's
// 32 first-layer values as 16-byte broadcasts and runs its two channels' sums: one weight register
// per FMA and no weight traffic, 64 FMAs per lane per pair and layer.
// The embedding net wt of one species is W1[32] b1[32] W2[32][64] b2[64] (e1 = 32, e2 = 64).
constexpr int kEmbWarps = 4;
constexpr int kEmbBlock = 32 + 32 + 32 * 64 + 64;

// tanh(x) = 1 - 2 / (exp(2x) + 1), with the exponential as 2^(2 x log2 e) on the hardware base-2
// unit and the quotient on the hardware reciprocal: absolute error a few 1e-7, saturating exactly
// (the exponential overflows to +inf -> 1, underflows to 0 -> -1).
__device__ __forceinline__ float tanh_fast(float x) {
  float e, r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(x * 2.8853900817779268f));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e + 1.f));
  return fmaf(-2.f, r, 1.f);
}

// One species' embedding weights as lane l holds them.
struct EmbLane {
  float wa[32], wb[32];   // W2[q][2l], W2[q][2l + 1]
  float w1, b1, w1r;      // first-layer unit q = l: W1[l], b1[l], W1[l] / rc
  float b2a, b2b;         // b2[2l], b2[2l + 1]
};
__device__ __forceinline__ void emb_lane_load(const float* wt, int lane, float r_rc, EmbLane& L) {
  L.w1 = wt[lane];
  L.b1 = wt[32 + lane];
  L.w1r = L.w1 * r_rc;
#pragma unroll
  for (int q = 0; q < 32; ++q) {
    const float2 w = *reinterpret_cast<const float2*>(wt + 64 + q * 64 + 2 * lane);
    L.wa[q] = w.x;
    L.wb[q] = w.y;
  }
  const float2 b = *reinterpret_cast<const float2*>(wt + 64 + 32 * 64 + 2 * lane);
  L.b2a = b.x;
  L.b2b = b.y;
}

// za += sum_q W2[q][2l] h_q, zb += sum_q W2[q][2l + 1] h_q over one pair's row h (32 first-layer
// values, 16-byte aligned in shared memory, read as broadcasts), q in order.
__device__ __forceinline__ void emb_row(const EmbLane& L, const float* h, float& za, float& zb) {
  const float4* h4 = reinterpret_cast<const float4*>(h);
#pragma unroll
  for (int q4 = 0; q4 < 8; ++q4) {
    const float4 v = h4[q4];
    za = fmaf(L.wa[4 * q4], v.x, za); zb = fmaf(L.wb[4 * q4], v.x, zb);
    za = fmaf(L.wa[4 * q4 + 1], v.y, za); zb = fmaf(L.wb[4 * q4 + 1], v.y, zb);
    za = fmaf(L.wa[4 * q4 + 2], v.z, za); zb = fmaf(L.wb[4 * q4 + 2], v.z, zb);
    za = fmaf(L.wa[4 * q4 + 3], v.w, za); zb = fmaf(L.wb[4 * q4 + 3], v.w, zb);
  }
}

// acc[s] += (ya, yb) for a warp-uniform special class s.
__device__ __forceinline__ void add_class(float (&acc)[4][2], int s, float ya, float yb) {
#pragma unroll
  for (int c = 0; c < 4; ++c)
    if (s == c) { acc[c][0] += ya; acc[c][1] += yb; }
}

// ---- embedding descriptor (FP32): G_i[s][c] = sum over the pairs of class s of scale cff(r) y_c(r),
// y = tanh(b2 + W2^T tanh(W1 u + b1)) of the neighbour's species, u = r / rc. Sums per lane in a fixed
// order (species by species, list order within), so deterministic.
// Shared memory per warp (kDescScratch floats): first-layer rows [32][32], then per pair u, scale cff, s.
constexpr int kDescScratch = 32 * 32 + 3 * 32;
__global__ void __launch_bounds__(kEmbWarps * 32, 4) k_emb_desc_f32(NnpArgs a) {
  extern __shared__ __align__(16) float sm[];
  float* W = sm;   // [ntype][kEmbBlock]
  for (int k = threadIdx.x; k < kEmbBlock * a.ntype; k += blockDim.x) W[k] = a.embw[k];
  __syncthreads();
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int i = blockIdx.x * kEmbWarps + wi;
  if (i >= a.N) return;
  float* hb = sm + kEmbBlock * a.ntype + wi * kDescScratch;
  float* su = hb + 32 * 32;
  float* scs = su + 32;
  int* ss = reinterpret_cast<int*>(scs + 32);
  const float4 xi = a.pos[i];
  const uint32_t* row = a.list6 + (size_t)i * a.cap6;
  const int n = a.n6[i];
  const float r_rc = 1.f / a.rc;
  float acc[4][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
  for (int t = 0; t < a.ntype; ++t) {
    EmbLane L;
    bool loaded = false;
    for (int base = 0; base < n; base += 32) {
      const int k = base + lane;
      const uint32_t ent = k < n ? row[k] : 0u;
      const bool sel = k < n && (int)((ent >> 27) & 7) == t;
      const unsigned mask = __ballot_sync(0xffffffffu, sel);
      if (!mask) continue;   // warp-uniform
      if (!loaded) { emb_lane_load(W + kEmbBlock * t, lane, r_rc, L); loaded = true; }
      const int m = __popc(mask);
      if (sel) {
        const int rk = __popc(mask & ((1u << lane) - 1u));
        const float4 xj = a.pos[ent & NNPE_J_MASK];
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float r = sqrtf(dx * dx + dy * dy + dz * dz);
        const float cf = r - a.rc;
        su[rk] = r * r_rc;
        scs[rk] = a.scale * (1.f - 1.f / (1.f + cf * cf));
        ss[rk] = (int)(ent >> 30);
      }
      __syncwarp();
      for (int p = 0; p < m; ++p) hb[p * 32 + lane] = tanh_fast(fmaf(L.w1, su[p], L.b1));
      __syncwarp();
      for (int p = 0; p < m; p += 2) {   // two pairs at a time (four independent sums); a lone last pair is doubled
        const int p1 = min(p + 1, m - 1);
        float z0 = L.b2a, z1 = L.b2b, z2 = L.b2a, z3 = L.b2b;
        emb_row(L, hb + p * 32, z0, z1);
        emb_row(L, hb + p1 * 32, z2, z3);
        const float c0 = scs[p];
        add_class(acc, ss[p], tanh_fast(z0) * c0, tanh_fast(z1) * c0);
        if (p + 1 < m) {
          const float c1 = scs[p1];
          add_class(acc, ss[p1], tanh_fast(z2) * c1, tanh_fast(z3) * c1);
        }
      }
      __syncwarp();
    }
  }
  float* Gi = a.G + (size_t)i * 256;
#pragma unroll
  for (int s = 0; s < 4; ++s) *reinterpret_cast<float2*>(Gi + s * 64 + 2 * lane) = make_float2(acc[s][0], acc[s][1]);
}

// ---- embedding force (FP32): per pair (i, j) of i's full list, fpair = -dE/dr / r from the pair's
// two descriptor terms, applied to i only (a warp-level gather, no atomics):
//   the term in G_i, through the net of j's species with dE/dG_i, and
//   the term in G_j, through the net of i's species with dE/dG_j,
// dE/dr = scale sum_c D_c [dcff y_c + cff (1 - y_c^2) k_c], k_c = sum_q W2[q][c] (1 - h_q^2) W1[q] / rc.
// Pass t = species of i evaluates that net once per pair with D = dE/dG_j (+ dE/dG_i when j has the
// same species); a pass t != species of i evaluates it on the pairs whose j is of species t with
// D = dE/dG_i. Each lane leaves its two channels' share of dE/dr in shared memory; the lane that
// owns the pair adds the 32 shares in a fixed order.
// Shared memory per warp (kForceScratch floats): h rows [16][32], dh/dr rows [16][32], shares
// [16][33] of a group of up to 16 pairs, then per pair of the 32-entry chunk u, scale cff, scale dcff,
// dx, dy, dz, rsq, r, dE/dG_j row offset, flags.
constexpr int kForceGroup = 16;
constexpr int kForceScratch = kForceGroup * (32 + 32 + 33) + 10 * 32;
template <bool EV>
__global__ void __launch_bounds__(kEmbWarps * 32, 4) k_emb_force_f32(NnpArgs a) {
  extern __shared__ __align__(16) float sm[];
  float* W = sm;
  for (int k = threadIdx.x; k < kEmbBlock * a.ntype; k += blockDim.x) W[k] = a.embw[k];
  __syncthreads();
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int i = blockIdx.x * kEmbWarps + wi;
  if (i >= a.N) return;
  float* hb = sm + kEmbBlock * a.ntype + wi * kForceScratch;
  float* gb = hb + kForceGroup * 32;
  float* vb = gb + kForceGroup * 32;
  float* su = vb + kForceGroup * 33;
  float* scf = su + 32;
  float* sdcf = scf + 32;
  float* sdx = sdcf + 32;
  float* sdy = sdx + 32;
  float* sdz = sdy + 32;
  float* srsq = sdz + 32;
  float* sr = srsq + 32;
  int* sjo = reinterpret_cast<int*>(sr + 32);
  int* sfl = sjo + 32;
  const float4 xi = a.pos[i];
  const uint32_t* row = a.list6 + (size_t)i * a.cap6;
  const int n = a.n6[i];
  const int ti = a.info[i].y & 0xFF;
  const float r_rc = 1.f / a.rc;
  const float2* dGi = reinterpret_cast<const float2*>(a.dG + (size_t)i * 256) + lane;   // this lane's channels
  const float2 Di0 = dGi[0], Di1 = dGi[32], Di2 = dGi[64], Di3 = dGi[96];
  float fx = 0.f, fy = 0.f, fz = 0.f;
  double w = 0.0;
  for (int t = 0; t < a.ntype; ++t) {
    const bool own = t == ti;
    EmbLane L;
    bool loaded = false;
    for (int base = 0; base < n; base += 32) {
      const int k = base + lane;
      const uint32_t ent = k < n ? row[k] : 0u;
      const int tj = (int)((ent >> 27) & 7);
      const bool sel = k < n && (own || tj == t);
      const unsigned mask = __ballot_sync(0xffffffffu, sel);
      if (!mask) continue;   // warp-uniform
      if (!loaded) { emb_lane_load(W + kEmbBlock * t, lane, r_rc, L); loaded = true; }
      const int m = __popc(mask);
      if (sel) {
        const int rk = __popc(mask & ((1u << lane) - 1u));
        const int j = ent & NNPE_J_MASK;
        const float4 xj = a.pos[j];
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float rsq = dx * dx + dy * dy + dz * dz;
        const float r = sqrtf(rsq);
        const float cf = r - a.rc, den = 1.f + cf * cf;
        const int s = (int)(ent >> 30);
        su[rk] = r * r_rc;
        scf[rk] = a.scale * (1.f - 1.f / den);
        sdcf[rk] = a.scale * (2.f * cf / (den * den));
        sdx[rk] = dx; sdy[rk] = dy; sdz[rk] = dz; srsq[rk] = rsq; sr[rk] = r;
        sjo[rk] = own ? owner_of(j, a.N, a.gowner) * 256 + s * 64 : 0;
        sfl[rk] = s | ((own && tj == ti) ? 4 : 0) | (own ? 8 : 0);
      }
      __syncwarp();
      for (int g0 = 0; g0 < m; g0 += kForceGroup) {   // groups of up to 16 of the chunk's pairs
        const int mg = min(kForceGroup, m - g0);
        for (int p = 0; p < mg; ++p) {
          const float h = tanh_fast(fmaf(L.w1, su[g0 + p], L.b1));
          hb[p * 32 + lane] = h;
          gb[p * 32 + lane] = (1.f - h * h) * L.w1r;
        }
        __syncwarp();
        for (int p = 0; p < mg; ++p) {
          const int fl = sfl[g0 + p];
          float2 D = make_float2(0.f, 0.f);
          if (fl & 8) D = *reinterpret_cast<const float2*>(a.dG + sjo[g0 + p] + 2 * lane);
          if (!(fl & 8) || (fl & 4)) {
            const int sc = fl & 3;
            const float2 d = sc == 0 ? Di0 : sc == 1 ? Di1 : sc == 2 ? Di2 : Di3;
            D.x += d.x;
            D.y += d.y;
          }
          float z0 = L.b2a, z1 = L.b2b, k0 = 0.f, k1 = 0.f;
          emb_row(L, hb + p * 32, z0, z1);
          emb_row(L, gb + p * 32, k0, k1);
          const float y0 = tanh_fast(z0), y1 = tanh_fast(z1);
          const float c = scf[g0 + p], dc = sdcf[g0 + p];
          vb[p * 33 + lane] = D.x * fmaf(c * (1.f - y0 * y0), k0, dc * y0) + D.y * fmaf(c * (1.f - y1 * y1), k1, dc * y1);
        }
        __syncwarp();
        if (lane < mg) {
          const int q = g0 + lane;
          float T = 0.f;
#pragma unroll 8
          for (int l = 0; l < 32; ++l) T += vb[lane * 33 + l];
          const float fpair = -T / sr[q];
          fx += sdx[q] * fpair;
          fy += sdy[q] * fpair;
          fz += sdz[q] * fpair;
          if (EV) w += 0.5 * (double)(fpair * srsq[q]);
        }
        __syncwarp();
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
    if (EV) w += __shfl_xor_sync(0xffffffffu, w, o);
  }
  if (lane == 0) {
    const float4 f = a.frc[i];
    a.frc[i] = make_float4(f.x + fx, f.y + fy, f.z + fz, f.w);
    if (EV) a.watom[i] += w;
  }
}

// ---- fitting network (FP32): C[rows] = epi(A[rows] x B), 32 rows x 128 columns per block,
// 256 threads with 4x4 outputs each, K staged through shared memory in chunks of 32.
enum FitEpi { EPI_L1 = 0, EPI_L2 = 1, EPI_B2 = 2, EPI_B1 = 3 };
struct FitArgs {
  const float* A;      // [M x K] rows in species order (or gathered through idx)
  const int* idx;      // row -> atom (gather/scatter), or null for direct rows
  const float* B;      // weights
  bool transB;         // B element (k,n) = transB ? B[n*K + k] : B[k*N + n]
  int M, K, N;
  const float* bias;   // [N]
  const float* a3;     // L2: output weights [N]
  const float* c3;     // L2: output bias
  const float* aux;    // B2: H1 rows (for 1-h^2)
  float* C;            // output rows
  double* enet;        // L2: per-atom energy (indexed through idx)
  bool gatherA, scatterC;
};

template <int EPI>
__global__ void __launch_bounds__(256) k_fit_gemm(FitArgs f) {
  __shared__ float As[32][33];
  __shared__ float Bs[32][128 + 4];
  const int t = threadIdx.x;
  const int tr = t >> 5, tc = t & 31;       // rows tr*4..+4, cols tc*4..+4
  const int row0 = blockIdx.x * 32, col0 = blockIdx.y * 128;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < f.K; k0 += 32) {
    for (int e = t; e < 32 * 32; e += 256) {
      const int r = e >> 5, k = e & 31;
      const int gr = row0 + r;
      float v = 0.f;
      if (gr < f.M && k0 + k < f.K) {
        const int src = f.gatherA ? f.idx[gr] : gr;
        v = f.A[(size_t)src * f.K + k0 + k];
      }
      As[r][k] = v;
    }
    for (int e = t; e < 32 * 128; e += 256) {
      const int k = e >> 7, n = e & 127;
      float v = 0.f;
      if (k0 + k < f.K && col0 + n < f.N)
        v = f.transB ? f.B[(size_t)(col0 + n) * f.K + k0 + k] : f.B[(size_t)(k0 + k) * f.N + col0 + n];
      Bs[k][n] = v;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      float av[4], bv[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) { av[q] = As[tr * 4 + q][k]; bv[q] = Bs[k][tc * 4 + q]; }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int p = 0; p < 4; ++p) acc[q][p] += av[q] * bv[p];
    }
    __syncthreads();
  }
  float epart[4] = {0, 0, 0, 0};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int gr = row0 + tr * 4 + q;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int gc = col0 + tc * 4 + p;
      if (gr >= f.M || gc >= f.N) continue;
      float v = acc[q][p];
      if (EPI == EPI_L1) {
        v = tanhf(v + f.bias[gc]);
        f.C[(size_t)gr * f.N + gc] = v;
      } else if (EPI == EPI_L2) {
        const float h = tanhf(v + f.bias[gc]);
        epart[q] += h * f.a3[gc];
        f.C[(size_t)gr * f.N + gc] = f.a3[gc] * (1.f - h * h);
      } else if (EPI == EPI_B2) {
        const float h = f.aux[(size_t)gr * f.N + gc];
        f.C[(size_t)gr * f.N + gc] = v * (1.f - h * h);
      } else {
        f.C[(size_t)f.idx[gr] * f.N + gc] = v;
      }
    }
  }
  if (EPI == EPI_L2) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float v = epart[q];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      const int gr = row0 + tr * 4 + q;
      if (tc == 0 && gr < f.M) f.enet[f.idx[gr]] = (double)v + (double)f.c3[0];
    }
  }
}

// The same four GEMMs with a 64-row x 128-column block tile for K and N multiples of 4 (B row-major
// [K][N]; the backward's transposed weights are kept as their own row-major copies). 256 threads,
// each 8 rows x 4 columns; the A tile stays row-major in shared memory and every thread reads 4 k of
// one row as a 16-byte broadcast (its warp shares its rows), the B tile 4 columns as one 16-byte
// load: 12 shared-memory loads per 128 FMAs. The next K chunk is loaded into registers while the
// current one is multiplied.
constexpr int kFgRows = 64, kFgK = 32, kFgAStride = kFgK + 4, kFgBStride = 128 + 4;
template <int EPI>
__global__ void __launch_bounds__(256, 2) k_fit_gemm64(FitArgs f) {
  __shared__ __align__(16) float As[kFgRows * kFgAStride];
  __shared__ __align__(16) float Bs[kFgK * kFgBStride];
  const int t = threadIdx.x, tr = t >> 5, tc = t & 31;   // rows 8 tr .. 8 tr + 7, columns 4 tc .. 4 tc + 3
  const int row0 = blockIdx.x * kFgRows, col0 = blockIdx.y * 128;
  // loaders: A as 2 float4 per thread (row e / 8, k quad e % 8), B as 4 float4 (k e / 32, column quad e % 32)
  int asrc[2];
  bool aval[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int gr = row0 + (t >> 3) + 32 * u;
    aval[u] = gr < f.M;
    asrc[u] = aval[u] ? (f.gatherA ? f.idx[gr] : gr) : 0;
  }
  const int akq = (t & 7) * 4, bn = (t & 31) * 4;
  const bool bval = col0 + bn < f.N;
  float4 ra[2], rb[4];
  auto load = [&](int k0) {
#pragma unroll
    for (int u = 0; u < 2; ++u)
      ra[u] = (aval[u] && k0 + akq < f.K) ? *reinterpret_cast<const float4*>(f.A + (size_t)asrc[u] * f.K + k0 + akq)
                                          : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = (t >> 5) + 8 * u;
      rb[u] = (bval && k0 + k < f.K) ? *reinterpret_cast<const float4*>(f.B + (size_t)(k0 + k) * f.N + col0 + bn)
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  float acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  load(0);
  for (int k0 = 0; k0 < f.K; k0 += kFgK) {
#pragma unroll
    for (int u = 0; u < 2; ++u) *reinterpret_cast<float4*>(As + ((t >> 3) + 32 * u) * kFgAStride + akq) = ra[u];
#pragma unroll
    for (int u = 0; u < 4; ++u) *reinterpret_cast<float4*>(Bs + ((t >> 5) + 8 * u) * kFgBStride + bn) = rb[u];
    __syncthreads();
    if (k0 + kFgK < f.K) load(k0 + kFgK);
    const int kn = min(kFgK, f.K - k0);
    for (int k = 0; k < kn; k += 4) {
      float4 a4[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a4[i] = *reinterpret_cast<const float4*>(As + (tr * 8 + i) * kFgAStride + k);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const float4 b = *reinterpret_cast<const float4*>(Bs + (k + kk) * kFgBStride + tc * 4);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float av = kk == 0 ? a4[i].x : kk == 1 ? a4[i].y : kk == 2 ? a4[i].z : a4[i].w;
          acc[i][0] = fmaf(av, b.x, acc[i][0]);
          acc[i][1] = fmaf(av, b.y, acc[i][1]);
          acc[i][2] = fmaf(av, b.z, acc[i][2]);
          acc[i][3] = fmaf(av, b.w, acc[i][3]);
        }
      }
    }
    __syncthreads();
  }
  const int gc = col0 + tc * 4;
  const bool cval = gc < f.N;
  float4 bias = make_float4(0.f, 0.f, 0.f, 0.f), a3 = bias;
  if (cval && (EPI == EPI_L1 || EPI == EPI_L2)) bias = *reinterpret_cast<const float4*>(f.bias + gc);
  if (cval && EPI == EPI_L2) a3 = *reinterpret_cast<const float4*>(f.a3 + gc);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gr = row0 + tr * 8 + i;
    float v[4] = {acc[i][0], acc[i][1], acc[i][2], acc[i][3]};
    float epart = 0.f;
    if (gr < f.M && cval) {
      if (EPI == EPI_L1) {
        v[0] = tanhf(v[0] + bias.x); v[1] = tanhf(v[1] + bias.y); v[2] = tanhf(v[2] + bias.z); v[3] = tanhf(v[3] + bias.w);
        *reinterpret_cast<float4*>(f.C + (size_t)gr * f.N + gc) = make_float4(v[0], v[1], v[2], v[3]);
      } else if (EPI == EPI_L2) {
        const float h0 = tanhf(v[0] + bias.x), h1 = tanhf(v[1] + bias.y), h2 = tanhf(v[2] + bias.z), h3 = tanhf(v[3] + bias.w);
        epart = h0 * a3.x + h1 * a3.y + h2 * a3.z + h3 * a3.w;
        *reinterpret_cast<float4*>(f.C + (size_t)gr * f.N + gc) =
            make_float4(a3.x * (1.f - h0 * h0), a3.y * (1.f - h1 * h1), a3.z * (1.f - h2 * h2), a3.w * (1.f - h3 * h3));
      } else if (EPI == EPI_B2) {
        const float4 h = *reinterpret_cast<const float4*>(f.aux + (size_t)gr * f.N + gc);
        *reinterpret_cast<float4*>(f.C + (size_t)gr * f.N + gc) =
            make_float4(v[0] * (1.f - h.x * h.x), v[1] * (1.f - h.y * h.y), v[2] * (1.f - h.z * h.z), v[3] * (1.f - h.w * h.w));
      } else {
        *reinterpret_cast<float4*>(f.C + (size_t)f.idx[gr] * f.N + gc) = make_float4(v[0], v[1], v[2], v[3]);
      }
    }
    if (EPI == EPI_L2) {   // the warp holds row gr's 128 columns: energy in a fixed shuffle order
      for (int o = 16; o > 0; o >>= 1) epart += __shfl_xor_sync(0xffffffffu, epart, o);
      if (tc == 0 && gr < f.M) f.enet[f.idx[gr]] = (double)epart + (double)f.c3[0];
    }
  }
}

}  // namespace

static int nnp_set_smem_attrs(nnpe_ctx* c, int smem_desc, int smem_force) {
  static_assert(kEmbWarps == kEmbWarpsHost && kDescScratch == kDescScratchHost && kForceScratch == kForceScratchHost,
                "shared-memory layout of the FP32 embedding kernels");
  NNPE_CUDA(c, cudaFuncSetAttribute(k_emb_desc_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_desc));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_emb_force_f32<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_force));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_emb_force_f32<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_force));
  return 0;
}

static NnpArgs make_args(nnpe_ctx* c) {
  NnpModel* m = c->nnp;
  NnpArgs a;
  a.pos = c->d_pos; a.info = c->d_info; a.pairtype = c->d_pairtype; a.gowner = c->d_gowner; a.list6 = m->d_list6;
  a.n6 = m->d_n6; a.cap6 = m->cap6; a.ntype = c->ntype; a.N = c->natom; a.nbin = m->nbin;
  a.r_dr = m->kind == 0 ? (float)m->nbin / m->rc : 0.f;
  a.rc = m->rc; a.scale = m->scale; a.e2 = m->e2; a.tdesc = m->d_tdesc; a.tpair = m->d_tpair; a.embw = m->d_embw;
  a.G = m->d_G; a.dG = m->d_dG; a.frc = c->d_frc; a.eatom = c->d_eatom; a.watom = c->d_watom;
  return a;
}

// Fitting network forward + backward: per species, 4 GEMMs (L1, L2 with energy, B2, B1).
static int fit_f32_enqueue(nnpe_ctx* c) {
  NnpModel* m = c->nnp;
  const size_t fb = fit_block(m->din, m->h1, m->h2);
  const bool wide = m->din % 4 == 0 && m->h1 % 4 == 0 && m->h2 % 4 == 0 && m->h2 <= 128;
  auto up4 = [](size_t n) { return (n + 3) & ~(size_t)3; };
  for (int t = 0; t < c->ntype; ++t) {
    const int M = m->soff[t + 1] - m->soff[t];
    if (!M) continue;
    const float* w = m->d_fitw + fb * t;
    const float *A1 = w, *c1 = A1 + (size_t)m->din * m->h1, *A2 = c1 + m->h1, *c2 = A2 + (size_t)m->h1 * m->h2;
    const float *A3 = c2 + m->h2, *c3 = A3 + m->h2;
    const int* idx = m->d_sidx + m->soff[t];
    float* H1 = m->d_H1 + (size_t)m->soff[t] * m->h1;
    float* G2 = m->d_G2 + (size_t)m->soff[t] * m->h2;
    float* G1 = m->d_G1 + (size_t)m->soff[t] * m->h1;
    FitArgs f{};
    f.idx = idx; f.M = M; f.c3 = c3; f.enet = m->d_enet;
    if (wide) {
      const float* g = m->d_fitg + m->fitg_block * t;
      const size_t o2 = up4((size_t)m->din * m->h1), o2t = o2 + up4((size_t)m->h1 * m->h2),
                   o1t = o2t + up4((size_t)m->h2 * m->h1), oc1 = o1t + up4((size_t)m->h1 * m->din),
                   oc2 = oc1 + up4(m->h1), oa3 = oc2 + up4(m->h2);
      const int gm = nblocks(M, kFgRows);
      f.A = m->d_G; f.K = m->din; f.B = g; f.N = m->h1; f.bias = g + oc1; f.C = H1; f.gatherA = true;
      k_fit_gemm64<EPI_L1><<<dim3(gm, nblocks(m->h1, 128)), 256, 0, c->stream>>>(f);
      f.A = H1; f.K = m->h1; f.B = g + o2; f.N = m->h2; f.bias = g + oc2; f.C = G2; f.gatherA = false; f.a3 = g + oa3;
      k_fit_gemm64<EPI_L2><<<dim3(gm, 1), 256, 0, c->stream>>>(f);
      f.A = G2; f.K = m->h2; f.B = g + o2t; f.N = m->h1; f.aux = H1; f.C = G1;
      k_fit_gemm64<EPI_B2><<<dim3(gm, nblocks(m->h1, 128)), 256, 0, c->stream>>>(f);
      f.A = G1; f.K = m->h1; f.B = g + o1t; f.N = m->din; f.C = m->d_dG;
      k_fit_gemm64<EPI_B1><<<dim3(gm, nblocks(m->din, 128)), 256, 0, c->stream>>>(f);
      continue;
    }
    dim3 g1(nblocks(M, 32), nblocks(m->h1, 128));
    f.A = m->d_G; f.K = m->din; f.B = A1; f.N = m->h1; f.bias = c1; f.C = H1; f.gatherA = true; f.transB = false;
    k_fit_gemm<EPI_L1><<<g1, 256, 0, c->stream>>>(f);
    dim3 g2(nblocks(M, 32), nblocks(m->h2, 128));
    f.A = H1; f.K = m->h1; f.B = A2; f.N = m->h2; f.bias = c2; f.C = G2; f.gatherA = false; f.a3 = A3;
    k_fit_gemm<EPI_L2><<<g2, 256, 0, c->stream>>>(f);
    dim3 g3(nblocks(M, 32), nblocks(m->h1, 128));
    f.A = G2; f.K = m->h2; f.B = A2; f.N = m->h1; f.transB = true; f.aux = H1; f.C = G1;
    k_fit_gemm<EPI_B2><<<g3, 256, 0, c->stream>>>(f);
    dim3 g4(nblocks(M, 32), nblocks(m->din, 128));
    f.A = G1; f.K = m->h1; f.B = A1; f.N = m->din; f.transB = true; f.C = m->d_dG;
    k_fit_gemm<EPI_B1><<<g4, 256, 0, c->stream>>>(f);
  }
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int nnp_species_enqueue(nnpe_ctx* c) {
  NnpModel* m = c->nnp;
  k_species<<<nblocks(c->natom, 256), 256, 0, c->stream>>>(c->d_info, m->d_sidx, m->d_scount, m->d_soff_dev, c->natom,
                                                          c->ntype, c->d_ctrl);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int nnp_forces_enqueue(nnpe_ctx* c, bool ev, bool filter6) {
  NnpModel* m = c->nnp;
  const int N = c->natom;
  cudaStream_t st = c->stream;
  const float cs = m->rc * m->rc;
  if (filter6)   // else the pair kernel of this step has filled the list (forces.cu)
    k_filter6<<<nblocks((long)N * 32, 128), 128, 0, st>>>(c->d_pos, force_list(c), force_count(c), c->cap, m->d_list6, m->d_n6,
                                                        m->cap6, cs, N, c->d_ctrl);
  if (int rc = nnp_species_enqueue(c)) return rc;
  NnpArgs a = make_args(c);
  if (m->bf16) return nnp_tc_forces_enqueue(c, ev);
  m->g_bf16 = false;
  if (m->kind == 0) {
    k_gauss_desc<<<nblocks((long)N * 32, 128), 128, 0, st>>>(a);
  } else {
    const size_t smem = sizeof(float) * ((size_t)kEmbBlock * c->ntype + kEmbWarps * kDescScratch);
    k_emb_desc_f32<<<nblocks(N, kEmbWarps), kEmbWarps * 32, smem, st>>>(a);
  }
  if (int rc = fit_f32_enqueue(c)) return rc;
  if (m->kind == 0) {
    if (ev) k_gauss_force<true><<<nblocks((long)N * 32, 128), 128, 0, st>>>(a);
    else k_gauss_force<false><<<nblocks((long)N * 32, 128), 128, 0, st>>>(a);
  } else {
    const size_t smem = sizeof(float) * ((size_t)kEmbBlock * c->ntype + kEmbWarps * kForceScratch);
    if (ev) k_emb_force_f32<true><<<nblocks(N, kEmbWarps), kEmbWarps * 32, smem, st>>>(a);
    else k_emb_force_f32<false><<<nblocks(N, kEmbWarps), kEmbWarps * 32, smem, st>>>(a);
  }
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int nnpe_nnp_get(nnpe_ctx* c, float* G, float* dG, double* e_atom) {
  if (!c || !c->nnp) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_get: no network");
  NnpModel* m = c->nnp;
  const int N = c->natom, D = m->din;
  std::vector<int> aid(N);
  std::vector<float> g((size_t)N * D), d((size_t)N * D);
  std::vector<double> e(N);
  NNPE_CUDA(c, cudaMemcpyAsync(aid.data(), c->d_atom_id, sizeof(int) * N, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(g.data(), m->d_G, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(d.data(), m->d_dG, sizeof(float) * d.size(), cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(e.data(), m->d_enet, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  if (m->g_bf16) {   // BF16 rows in the first half of the buffer: widen (exact) from the top down
    const uint16_t* h = reinterpret_cast<const uint16_t*>(g.data());
    for (size_t k = g.size(); k-- > 0;) {
      const uint32_t u = (uint32_t)h[k] << 16;
      std::memcpy(&g[k], &u, 4);
    }
  }
  for (int i = 0; i < N; ++i) {
    const int a = aid[i];
    if (G) std::memcpy(G + (size_t)a * D, g.data() + (size_t)i * D, sizeof(float) * D);
    if (dG) std::memcpy(dG + (size_t)a * D, d.data() + (size_t)i * D, sizeof(float) * D);
    if (e_atom) e_atom[a] = e[i];
  }
  return NNPE_OK;
}

int nnpe_sync_errors(nnpe_ctx* c);

// Grid autotuning of the tensor-core kernels on the context's current state (the list is built
// first when it is stale, and one force evaluation fills the network's pair and species lists).
// The force array is left holding partial sums: the next force evaluation rewrites it.
int nnpe_nnp_autotune(nnpe_ctx* c, int reps, int use_cache, int* grid_desc, int* grid_force) {
  if (!c || !c->have_setup || !c->nnp) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_autotune: no network set up");
  cudaSetDevice(c->device);
  if (int rc = rebuild_enqueue(c, true)) return rc;
  if (int rc = ghost_update_enqueue(c, true)) return rc;
  if (int rc = forces_enqueue(c, false)) return rc;
  if (int rc = nnpe_sync_errors(c)) return rc;
  return nnp_tc_autotune(c, reps, use_cache != 0, grid_desc, grid_force);
}

int nnpe_nnp_grids(nnpe_ctx* c, int grid_desc, int grid_force) {
  if (!c) return NNPE_EARG;
  return nnp_tc_set_grids(c, grid_desc, grid_force);
}

int nnpe_nnp_get_grids(nnpe_ctx* c, int* grid_desc, int* grid_force) {
  if (!c) return NNPE_EARG;
  return nnp_tc_get_grids(c, grid_desc, grid_force);
}

int nnpe_nnp_info(nnpe_ctx* c, int* din, int* kind) {
  if (!c || !c->nnp) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_info: no network");
  if (din) *din = c->nnp->din;
  if (kind) *kind = c->nnp->kind;
  return NNPE_OK;
}

// NNPOTENTIAL_TBL constructor inputs (pair_nnp.cpp:457-519): the paramfile's first token names
// the model file (here an NNPE model: text header up to "end", then float32 weights); the weight
// file holds bond/angle/dihedral coefficients in their raw form (setParam() doubles the 2a/2c
// entries and scales the dihedral ones, bond.cpp:57-64 etc.), then coef_p, coef_w, coef_d, coef_r.
int nnpe_nnp_load(nnpe_ctx* c, double cutoff, int nbin, const char* paramfile, const char* wtfile) {
  if (!c || !c->have_setup || !paramfile || !wtfile) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_load");
  char model[512];
  FILE* fp = fopen(paramfile, "r");
  if (!fp) return nnpe_fail(c, NNPE_EFILE, std::string("cannot open ") + paramfile);
  const int got = fscanf(fp, "%511s", model);
  fclose(fp);
  if (got != 1) return nnpe_fail(c, NNPE_EFILE, "paramfile: read error");
  fp = fopen(model, "rb");
  if (!fp) return nnpe_fail(c, NNPE_EFILE, std::string("cannot open model ") + model);
  char line[512];
  std::string desc;
  int e1 = 32, e2 = 64, h1 = 0, h2 = 0, ntype = 0, ngauss = 20;
  float scale = 1.f;
  while (fgets(line, sizeof line, fp)) {
    char key[64];
    if (sscanf(line, "%63s", key) != 1) continue;
    const std::string k(key);
    if (k == "end") break;
    if (k == "descriptor") {
      char d[64];
      int n = sscanf(line, "%*s %63s", d);
      if (n != 1) { fclose(fp); return nnpe_fail(c, NNPE_EFILE, "model: descriptor line"); }
      desc = d;
      if (desc == "embed") sscanf(line, "%*s %*s %d %d %f", &e1, &e2, &scale);
      else sscanf(line, "%*s %*s %d", &ngauss);
    } else if (k == "fitting") sscanf(line, "%*s %d %d", &h1, &h2);
    else if (k == "ntype") sscanf(line, "%*s %d", &ntype);
  }
  if ((desc != "embed" && desc != "gauss") || ntype != c->ntype || h1 <= 0 || h2 <= 0 || (desc == "gauss" && ngauss != 20)) {
    fclose(fp);
    return nnpe_fail(c, NNPE_EFILE, "model: unsupported header (descriptor embed|gauss 20, fitting h1 h2, ntype)");
  }
  const int kind = desc == "embed" ? 1 : 0;
  const int din = kind ? 4 * e2 : 20;
  const size_t eb = (size_t)e1 + e1 + (size_t)e1 * e2 + e2;
  std::vector<float> embw(kind ? eb * ntype : 0), fitw(fit_block(din, h1, h2) * ntype);
  if ((kind && fread(embw.data(), sizeof(float), embw.size(), fp) != embw.size()) ||
      fread(fitw.data(), sizeof(float), fitw.size(), fp) != fitw.size()) {
    fclose(fp);
    return nnpe_fail(c, NNPE_EFILE, "model: truncated weights");
  }
  fclose(fp);
  fp = fopen(wtfile, "rb");
  if (!fp) return nnpe_fail(c, NNPE_EFILE, std::string("cannot open ") + wtfile);
  const int P = c->npair;
  std::vector<float> bc((size_t)c->nbtyp * 4), ac((size_t)c->natyp * 4), dc((size_t)c->ndtyp * 4), cp((size_t)P * 24),
      cw((size_t)P * 80), cd((size_t)P * 80), cr((size_t)P * 80);
  bool ok = fread(bc.data(), 4, bc.size(), fp) == bc.size() && fread(ac.data(), 4, ac.size(), fp) == ac.size() &&
            fread(dc.data(), 4, dc.size(), fp) == dc.size() && fread(cp.data(), 4, cp.size(), fp) == cp.size() &&
            fread(cw.data(), 4, cw.size(), fp) == cw.size() && fread(cd.data(), 4, cd.size(), fp) == cd.size() &&
            fread(cr.data(), 4, cr.size(), fp) == cr.size();
  fclose(fp);
  if (!ok) return nnpe_fail(c, NNPE_EFILE, "weight file: truncated");
  for (int i = 0; i < c->nbtyp; ++i) { bc[4 * i + 1] *= 2; bc[4 * i + 3] *= 2; }   // BOND::setParam()
  for (int i = 0; i < c->natyp; ++i) { ac[4 * i + 1] *= 2; ac[4 * i + 3] *= 2; }   // ANGLE::setParam()
  for (int i = 0; i < c->ndtyp; ++i) { dc[4 * i + 2] *= 2; dc[4 * i + 3] *= 3; }   // DIHEDRAL::setParam()
  if (int rc = nnpe_bonded_coefs(c, bc.data(), ac.data(), dc.data())) return rc;
  return nnpe_nnp_set(c, kind, cutoff, nbin, scale, e1, e2, h1, h2, cp.data(), cw.data(), cd.data(), cr.data(),
                      kind ? embw.data() : nullptr, fitw.data());
}

// Total pairs inside the network cutoff in the last evaluation (sum of the compact list counts).
int64_t nnpe_nnp_pairs(nnpe_ctx* c) {
  if (!c || !c->nnp) return -1;
  std::vector<int> n(c->natom);
  if (cudaMemcpyAsync(n.data(), c->nnp->d_n6, sizeof(int) * c->natom, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return -1;
  int64_t s = 0;
  for (int v : n) s += v;
  return s;
}
