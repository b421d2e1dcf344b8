// g(r) histogram (GR, grsq.cpp:28-219) and its sine transform S(q) (SQ, grsq.cpp:258-322).
//
// Counts are exact integers: each block privatises a uint32 histogram in shared memory and
// flushes it once into the uint64 global histogram (integer atomics, order independent, so the
// result is bit-identical run to run and to the reference's per-thread int sums). The
// normalisation and the transform run in FP64.
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace {

constexpr int kGrThreads = 256;

// Cell-based tally to gr_cutoff (grsq.cpp:151-205) or list-based to the pair cutoff
// (grsq.cpp:94-149): +1 per ordered (real atom, neighbour) pair, which reproduces the reference's
// +2 per real pair counted once and +1 per image pair counted from each side.
template <bool LIST>
__global__ void __launch_bounds__(kGrThreads) k_gr_tally(const float4* __restrict__ pos, const int2* __restrict__ info,
                                                         const int* __restrict__ cell, const int* __restrict__ cstart,
                                                         const int* __restrict__ cend, const int* __restrict__ gcstart,
                                                         const int* __restrict__ gcend, const int4* __restrict__ rows,
                                                         const int* __restrict__ nrows, int maxrows,
                                                         const uint32_t* __restrict__ list, const int* __restrict__ ncount,
                                                         int cap, const int* __restrict__ pairtype, int ntype, int npair,
                                                         int nbin, float rmaxsq, float r_dr,
                                                         unsigned long long* __restrict__ out, int N) {
  extern __shared__ uint32_t hist[];
  const int H = npair * nbin;
  for (int k = threadIdx.x; k < H; k += blockDim.x) hist[k] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int per_block = (N + gridDim.x - 1) / gridDim.x;
  const int a0 = blockIdx.x * per_block, a1 = min(N, a0 + per_block);
  for (int i = a0 + wib; i < a1; i += nw) {
    const float4 xi = pos[i];
    const int* ptrow = pairtype + (info[i].y & 0xFF) * ntype;
    if (LIST) {
      const uint32_t* row = list + (size_t)i * cap;
      const int n = ncount[i];
      for (int k = lane; k < n; k += 32) {
        const uint32_t e = row[k];
        const float4 xj = pos[e & NNPE_J_MASK];
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float rsq = dx * dx + dy * dy + dz * dz;
        if (rsq < rmaxsq) {
          const int bin = (int)(sqrtf(rsq) * r_dr);
          if (bin < nbin) atomicAdd(&hist[ptrow[(e >> 27) & 7] * nbin + bin], 1u);
        }
      }
    } else {
      const int ci = cell[i];
      const int nr = nrows[ci];
      const int4* R = rows + (size_t)ci * maxrows;
      for (int pass = 0; pass < 2; ++pass)
        for (int r = 0; r < nr; ++r) {
          const int4 rw = R[r];
          const int j0 = pass ? gcstart[rw.x] : cstart[rw.x];
          const int j1 = pass ? gcend[rw.y] : cend[rw.y];
          for (int j = j0 + lane; j < j1; j += 32) {
            if (!pass && j == i) continue;
            const float4 xj = pos[j];
            const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            const float rsq = dx * dx + dy * dy + dz * dz;
            if (rsq < rmaxsq) {
              const int bin = (int)(sqrtf(rsq) * r_dr);
              if (bin < nbin) atomicAdd(&hist[ptrow[info[j].y & 0xFF] * nbin + bin], 1u);
            }
          }
        }
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < H; k += blockDim.x)
    if (hist[k]) atomicAdd(out + k, (unsigned long long)hist[k]);
}

// g(r)-1 = counts*norm - 1 with the GR normaliser (grsq.cpp:56-70) in FP64.
__global__ void k_gr_norm(const unsigned long long* __restrict__ counts, const double* __restrict__ normg, double* gr,
                          int npair, int nbin) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npair * nbin) return;
  const int p = k / nbin, b = k % nbin;
  gr[k] = (double)counts[k] * (normg[p] / (b * (b + 1.0) + 1.0 / 3.0)) - 1.0;
}

// S_p(q_i) = sum_r sin(q_i r) 4 pi rho dr r / q_i * (g_p(r)-1), q_i=(i+.5) qmax/nq (grsq.cpp:270-279).
__global__ void k_sq(const double* __restrict__ gr, double* __restrict__ sq, double* __restrict__ qq, int npair, int nbin,
                     int nq, double dr, double dq, double four_pi_rho_dr) {
  __shared__ double sh[256];
  const int iq = blockIdx.x;
  const double q = (iq + 0.5) * dq;
  if (threadIdx.x == 0) qq[iq] = q;
  for (int p = 0; p < npair; ++p) {
    double acc = 0;
    for (int j = threadIdx.x; j < nbin; j += blockDim.x) {
      const double r = (j + 0.5) * dr;
      acc += sin(q * r) * four_pi_rho_dr * r / q * gr[(size_t)p * nbin + j];
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) sq[(size_t)p * nq + iq] = sh[0];
    __syncthreads();
  }
}

}  // namespace

static int dalloc_u64(nnpe_ctx* c, unsigned long long** p, size_t n) {
  if (*p) dev_free(*p);
  *p = nullptr;
  NNPE_CUDA(c, dev_malloc(c, (void**)p, std::max<size_t>(n, 1) * sizeof(unsigned long long)));
  return 0;
}
static int dalloc_f64(nnpe_ctx* c, double** p, size_t n) {
  if (*p) dev_free(*p);
  *p = nullptr;
  NNPE_CUDA(c, dev_malloc(c, (void**)p, std::max<size_t>(n, 1) * sizeof(double)));
  return 0;
}

extern "C" int nnpe_gr_setup(nnpe_ctx* c, int nbin_inner, int nq, double qmax, int gr_interval, int gr_interval_long) {
  if (!c || !c->have_setup || nbin_inner <= 0 || nq <= 0) return nnpe_fail(c, NNPE_EARG, "nnpe_gr_setup");
  cudaSetDevice(c->device);
  // GR(nbi, r_max=gr_cutoff, r_max_inner=pair_cutoff) in float (grsq.cpp:38-47)
  const float r_inner = c->pair_cutoff, r_max = c->gr_cutoff;
  if (r_max < r_inner) return nnpe_fail(c, NNPE_EARG, "r_max_inner larger than r_max");
  c->gr_nbin_inner = nbin_inner;
  c->gr_dr = r_inner / nbin_inner;
  c->gr_r_dr = nbin_inner / r_inner;
  c->gr_rmaxsq_inner = r_inner * r_inner;
  c->gr_nbin = (int)(r_max * c->gr_r_dr);
  {
    float t = c->gr_nbin * c->gr_dr;
    c->gr_rmaxsq = t * t;
  }
  c->gr_nq = nq;
  c->gr_qmax = qmax;
  c->gr_interval = gr_interval;
  c->gr_interval_long = gr_interval_long;
  const int P = c->npair;
  if (int rc = dalloc_u64(c, &c->d_gr_counts, (size_t)P * c->gr_nbin)) return rc;
  if (int rc = dalloc_u64(c, &c->d_gr_counts_inner, (size_t)P * nbin_inner)) return rc;
  if (int rc = dalloc_f64(c, &c->d_gr, (size_t)P * c->gr_nbin)) return rc;
  if (int rc = dalloc_f64(c, &c->d_sq, (size_t)P * nq)) return rc;
  if (int rc = dalloc_f64(c, &c->d_gr_norm, P)) return rc;
  if (int rc = dalloc_f64(c, &c->d_qq, nq)) return rc;
  // normaliser per pair in FP64 (the reference's int product overflows above 2^31, grsq.cpp:63)
  std::vector<long long> cnt(c->ntype, 0);
  for (int t : c->h_typ) ++cnt[t];
  const double bl_rdr = (double)c->grid.bl * (double)c->gr_r_dr;
  const double rc_dr3 = bl_rdr * bl_rdr * bl_rdr / (4 * M_PI);
  std::vector<double> ng(P);
  for (int i = 0, p = 0; i < c->ntype; ++i)
    for (int j = i; j < c->ntype; ++j, ++p)
      ng[p] = rc_dr3 / ((double)cnt[i] * (i == j ? (double)(cnt[j] - 1) : 2.0 * cnt[j]));
  NNPE_CUDA(c, cudaMemcpy(c->d_gr_norm, ng.data(), sizeof(double) * P, cudaMemcpyHostToDevice));
  const int smem = (int)(sizeof(uint32_t) * P * std::max(c->gr_nbin, nbin_inner));
  if (smem > 200 * 1024) return nnpe_fail(c, NNPE_EOVERFLOW, "g(r) histogram does not fit in shared memory");
  NNPE_CUDA(c, cudaFuncSetAttribute(k_gr_tally<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_gr_tally<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

int gr_tally_enqueue(nnpe_ctx* c, int inner) {
  const int P = c->npair;
  const int nbin = inner ? c->gr_nbin_inner : c->gr_nbin;
  unsigned long long* out = inner ? c->d_gr_counts_inner : c->d_gr_counts;
  NNPE_CUDA(c, cudaMemsetAsync(out, 0, sizeof(unsigned long long) * P * nbin, c->stream));
  const size_t smem = sizeof(uint32_t) * P * nbin;
  if (smem > 200 * 1024) return nnpe_fail(c, NNPE_EOVERFLOW, "g(r) histogram does not fit in shared memory");
  const int blocks = std::min(nnpe_sm_count(c->device) * 4, std::max(1, c->natom / 8));
  if (inner) {
    k_gr_tally<true><<<blocks, kGrThreads, smem, c->stream>>>(
        c->d_pos, c->d_info, c->d_cell, c->d_cstart, c->d_cend, c->d_gcstart, c->d_gcend, nullptr, nullptr, 0, c->d_list,
        c->d_ncount, c->cap, c->d_pairtype, c->ntype, P, nbin, c->gr_rmaxsq_inner, c->gr_r_dr, out, c->natom);
  } else {
    k_gr_tally<false><<<blocks, kGrThreads, smem, c->stream>>>(
        c->d_pos, c->d_info, c->d_cell, c->d_cstart, c->d_cend, c->d_gcstart, c->d_gcend, c->st_gr.rows, c->st_gr.nrows,
        c->st_gr.maxrows, nullptr, nullptr, c->cap, c->d_pairtype, c->ntype, P, nbin, c->gr_rmaxsq, c->gr_r_dr, out,
        c->natom);
  }
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

// GR::tally<true> clears and fills only the first nbin_r_inner bins of the per-thread counts
// (grsq.cpp:96-105); the bins beyond keep the last cell-based tally, and reduce_local/SQ::compute
// read all nbin_r bins (grsq.cpp:207-219, 299-322). The list-based counts are therefore copied
// over the first bins of the full-range counts, which then hold exactly the reference's sums.
static int merge_inner_enqueue(nnpe_ctx* c) {
  const size_t w = sizeof(unsigned long long);
  NNPE_CUDA(c, cudaMemcpy2DAsync(c->d_gr_counts, w * c->gr_nbin, c->d_gr_counts_inner, w * c->gr_nbin_inner,
                                 w * c->gr_nbin_inner, c->npair, cudaMemcpyDeviceToDevice, c->stream));
  return 0;
}

// g(r) over the full range and S(q) from it (SQ::compute uses gr->nbin_r bins, grsq.cpp:282).
static int sq_enqueue(nnpe_ctx* c) {
  const int P = c->npair, nbin = c->gr_nbin;
  k_gr_norm<<<nblocks((long)P * nbin, 256), 256, 0, c->stream>>>(c->d_gr_counts, c->d_gr_norm, c->d_gr, P, nbin);
  const double dr = (double)c->gr_dr;
  const double rho = (double)c->natom / std::pow((double)c->grid.bl, 3);
  k_sq<<<c->gr_nq, 256, 0, c->stream>>>(c->d_gr, c->d_sq, c->d_qq, P, nbin, c->gr_nq, dr, c->gr_qmax / c->gr_nq,
                                        4 * M_PI * rho * dr);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int rmdf_step_enqueue(nnpe_ctx* c, bool potential);

// One g(r) step of the loop (run.cpp:286-299): tally, g(r), S(q), then the RMDF table update.
int gr_step_enqueue(nnpe_ctx* c, bool long_tally, bool rmdf_potential) {
  const int inner = long_tally ? 0 : 1;
  if (int rc = gr_tally_enqueue(c, inner)) return rc;
  if (inner)
    if (int rc = merge_inner_enqueue(c)) return rc;
  c->gr_tallied = inner;
  if (int rc = sq_enqueue(c)) return rc;
  return rmdf_step_enqueue(c, rmdf_potential);
}

int nnpe_sync_errors(nnpe_ctx* c);

extern "C" int nnpe_gr_tally(nnpe_ctx* c, int inner) {
  if (!c || !c->have_setup || !c->d_gr_counts) return nnpe_fail(c, NNPE_EARG, "nnpe_gr_tally: no g(r) set up");
  cudaSetDevice(c->device);
  if (int rc = gr_tally_enqueue(c, inner ? 1 : 0)) return rc;
  if (inner)
    if (int rc = merge_inner_enqueue(c)) return rc;
  c->gr_tallied = inner ? 1 : 0;
  return nnpe_sync_errors(c);
}

extern "C" int nnpe_gr_nbin(const nnpe_ctx* c, int inner) { return c ? (inner ? c->gr_nbin_inner : c->gr_nbin) : 0; }

extern "C" int nnpe_gr_get(nnpe_ctx* c, int inner, uint64_t* counts, double* gr) {
  if (!c || !c->d_gr_counts) return nnpe_fail(c, NNPE_EARG, "nnpe_gr_get: no g(r) set up");
  const int P = c->npair, nbin = inner ? c->gr_nbin_inner : c->gr_nbin;
  if (counts)
    NNPE_CUDA(c, cudaMemcpyAsync(counts, inner ? c->d_gr_counts_inner : c->d_gr_counts, sizeof(uint64_t) * P * nbin,
                                 cudaMemcpyDeviceToHost, c->stream));
  if (gr) {
    k_gr_norm<<<nblocks((long)P * nbin, 256), 256, 0, c->stream>>>(inner ? c->d_gr_counts_inner : c->d_gr_counts,
                                                                    c->d_gr_norm, c->d_gr, P, nbin);
    NNPE_CUDA(c, cudaMemcpyAsync(gr, c->d_gr, sizeof(double) * P * nbin, cudaMemcpyDeviceToHost, c->stream));
  }
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  return NNPE_OK;
}

extern "C" int nnpe_sq_compute(nnpe_ctx* c, int inner, double* sq, double* q) {
  if (!c || !c->d_gr_counts) return nnpe_fail(c, NNPE_EARG, "nnpe_sq_compute: no g(r) set up");
  cudaSetDevice(c->device);
  (void)inner;   // S(q) always spans the full g(r) range, as SQ::compute
  if (int rc = sq_enqueue(c)) return rc;
  if (sq) NNPE_CUDA(c, cudaMemcpyAsync(sq, c->d_sq, sizeof(double) * c->npair * c->gr_nq, cudaMemcpyDeviceToHost, c->stream));
  if (q) NNPE_CUDA(c, cudaMemcpyAsync(q, c->d_qq, sizeof(double) * c->gr_nq, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  return NNPE_OK;
}
