// Direct S(q): the structure factor summed over reciprocal lattice vectors, SQD (grsq.cpp:362-608).
//
// The reference's G set: G = (2 pi / L) (i, j, k) over the half space (k > 0; k = 0, j > 0;
// k = j = 0, i > 0) with i^2 + j^2 + k^2 <= (int)(q_max / g)^2, |G| binned on the q grid
// i * q_max / nq (the last bin takes the rest up to q_max). Per G and atom type t,
// S_t = sum_a sin(G.x_a) and C_t = sum_a cos(G.x_a); per bin and type pair (t1 <= t2),
// sq = mean over the bin's G of (S_t1 S_t2 + C_t1 C_t2) * N / (n_t1 n_t2), minus N / n_t1 when
// t1 == t2. The set membership, |G| and the bin edges use the reference's float arithmetic, so that
// every bin holds the same vectors.
//
// On the device the G set is cut into runs of up to 16 vectors that are consecutive along one
// axis. One thread owns a run. The CTA stages the atoms (FP64 fractional coordinates, type, and
// the unit phasor e^{2 pi i u} along each axis) in shared memory, and every thread walks them in
// the same order: per atom one sincospi of the run's first phase, reduced to [-1/2, 1/2) turns in
// FP64, then one complex multiplication by the axis phasor per further vector. The sums
// over atoms are FP32 per thread (the reference sums in float too); the products per bin are summed
// in FP64 by one warp per bin over its vectors in a fixed order, so results are deterministic.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "internal.cuh"

namespace {

constexpr int kRunLen = 16;
constexpr int kSqdThreads = 128;

}  // namespace

struct SqdState {
  int nq = 0;
  float qmax = 0.f;
  int ngv = 0, nrun = 0, npair = 0, ntype = 0;
  std::vector<double> q;        // mean |G| per bin
  std::vector<int> count;       // vectors per bin
  std::vector<double> sq;       // [nq][npair], last compute
  bool have = false;            // a compute has run since set-up
  int4* d_runs = nullptr;       // (i, j, k) of the first vector, (axis << 8) | length
  int* d_rstart = nullptr;      // index of the run's first vector
  float2* d_sc = nullptr;       // [ngv][ntype] (S, C)
  int* d_bstart = nullptr;      // [nq + 1] CSR over d_bg
  int* d_bg = nullptr;          // vector indices of each bin, ascending
  double* d_fb = nullptr;       // [2][npair] factor, base
  double* d_sq = nullptr;       // [nq][npair]
};

namespace {

void sqd_release(SqdState* s) {
  if (!s) return;
  for (void* p : {(void*)s->d_runs, (void*)s->d_rstart, (void*)s->d_sc, (void*)s->d_bstart, (void*)s->d_bg,
                  (void*)s->d_fb, (void*)s->d_sq})
    if (p) dev_free(p);
  s->d_runs = nullptr; s->d_rstart = nullptr; s->d_sc = nullptr; s->d_bstart = nullptr; s->d_bg = nullptr;
  s->d_fb = nullptr; s->d_sq = nullptr;
}

// Per-thread S/C sums of its run over all atoms of type t. Every thread reads the same staged atom
// at the same time, so the type test is uniform across the CTA.
__global__ void __launch_bounds__(kSqdThreads) k_sqd_runs(const double4* __restrict__ xd, const int2* __restrict__ info,
                                                          int N, double inv_l, const int4* __restrict__ runs,
                                                          const int* __restrict__ rstart, int nrun, int ntype,
                                                          float2* __restrict__ sc) {
  __shared__ double su[kSqdThreads], sv[kSqdThreads], sw[kSqdThreads];
  __shared__ float2 ph[3][kSqdThreads];
  __shared__ int st[kSqdThreads];
  const int r = blockIdx.x * kSqdThreads + threadIdx.x;
  const bool valid = r < nrun;
  const int4 run = valid ? runs[r] : make_int4(0, 0, 0, 0);
  const int axis = (run.w >> 8) & 3, len = run.w & 0xFF;
  const double ki = run.x, kj = run.y, kk = run.z;
  for (int t = 0; t < ntype; ++t) {
    float s[kRunLen], c[kRunLen];
#pragma unroll
    for (int k = 0; k < kRunLen; ++k) s[k] = c[k] = 0.f;
    for (int a0 = 0; a0 < N; a0 += kSqdThreads) {
      __syncthreads();
      const int a = a0 + threadIdx.x;
      if (a < N) {
        const double4 x = xd[a];
        const double u = x.x * inv_l, v = x.y * inv_l, w = x.z * inv_l;
        su[threadIdx.x] = u; sv[threadIdx.x] = v; sw[threadIdx.x] = w;
        st[threadIdx.x] = info_type(info[a]);
        float sn, cs;
        sincospif((float)(2.0 * (u - rint(u))), &sn, &cs); ph[0][threadIdx.x] = make_float2(cs, sn);
        sincospif((float)(2.0 * (v - rint(v))), &sn, &cs); ph[1][threadIdx.x] = make_float2(cs, sn);
        sincospif((float)(2.0 * (w - rint(w))), &sn, &cs); ph[2][threadIdx.x] = make_float2(cs, sn);
      }
      __syncthreads();
      const int n = min(kSqdThreads, N - a0);
      if (!valid) continue;
      for (int j = 0; j < n; ++j) {
        if (st[j] != t) continue;
        double turns = fma(ki, su[j], fma(kj, sv[j], kk * sw[j]));
        turns -= rint(turns);
        float sn, cs;
        sincospif((float)(2.0 * turns), &sn, &cs);
        const float2 e = ph[axis][j];
        // every run steps the full length (a shorter run's extra sums are never stored), so the
        // inner loop carries no predicates: two adds and one complex multiply per vector
#pragma unroll
        for (int k = 0; k < kRunLen; ++k) {
          s[k] += sn;
          c[k] += cs;
          const float c2 = fmaf(cs, e.x, -sn * e.y), s2 = fmaf(sn, e.x, cs * e.y);
          cs = c2;
          sn = s2;
        }
      }
    }
    if (valid) {
      const int g0 = rstart[r];
#pragma unroll
      for (int k = 0; k < kRunLen; ++k)
        if (k < len) sc[(size_t)(g0 + k) * ntype + t] = make_float2(s[k], c[k]);
    }
  }
}

// One warp per bin: sum over its vectors of S1 S2 + C1 C2 per type pair in FP64 (lane-strided,
// then a fixed shuffle tree), normalised as SQD::compute does (grsq.cpp:566-570).
__global__ void k_sqd_bins(const float2* __restrict__ sc, const int* __restrict__ bstart, const int* __restrict__ bg,
                           int ntype, int npair, const double* __restrict__ fb, double* __restrict__ sq) {
  const int b = blockIdx.x, lane = threadIdx.x;
  const int g0 = bstart[b], g1 = bstart[b + 1], n = g1 - g0;
  int p = 0;
  for (int t1 = 0; t1 < ntype; ++t1)
    for (int t2 = t1; t2 < ntype; ++t2, ++p) {
      double acc = 0.0;
      for (int k = g0 + lane; k < g1; k += 32) {
        const int g = bg[k];
        const float2 a = sc[(size_t)g * ntype + t1], c = sc[(size_t)g * ntype + t2];
        acc += (double)a.x * (double)c.x + (double)a.y * (double)c.y;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) sq[(size_t)b * npair + p] = n > 0 ? acc / n * fb[p] - fb[npair + p] : 0.0;
    }
}

template <typename T>
int upload(nnpe_ctx* c, T** d, const std::vector<T>& h) {
  NNPE_CUDA(c, dev_malloc(c, (void**)d, sizeof(T) * std::max<size_t>(h.size(), 1)));
  if (!h.empty()) NNPE_CUDA(c, cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return 0;
}

}  // namespace

void sqd_free(nnpe_ctx* c) {
  if (!c || !c->sqd) return;
  sqd_release(c->sqd);
  delete c->sqd;
  c->sqd = nullptr;
}

// SQD::SQD (grsq.cpp:362-489): the G set, its bins, the mean |G| per bin and the pair factors.
int nnpe_sqd_setup(nnpe_ctx* c, int nq, double qmax, int* ngv_out) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_sqd_setup: not set up");
  if (nq <= 0 || !(qmax > 0)) return nnpe_fail(c, NNPE_EARG, "nnpe_sqd_setup: bad q grid");
  cudaSetDevice(c->device);
  sqd_free(c);
  auto* s = new SqdState();
  c->sqd = s;
  s->nq = nq;
  s->qmax = (float)qmax;
  s->ntype = c->ntype;
  s->npair = c->ntype * (c->ntype + 1) / 2;
  // ENVIRON::two_pi / ENVIRON::bl and the cutoffs in float, as numtype is
  const float two_pi = (float)(2.0 * 3.14159265358979323846);
  const float g = two_pi / c->grid.bl;
  const float ratio = s->qmax / g;
  const int kc = (int)ratio;
  const int cut = (int)(ratio * ratio);
  const float dq = s->qmax / (float)nq;
  std::vector<int4> runs;
  std::vector<int> rstart, gbin;
  std::vector<double> gsum(nq, 0.0);
  s->count.assign(nq, 0);
  auto add_vector = [&](int i, int j, int k) {
    const int n2 = i * i + j * j + k * k;
    const float gscl = std::sqrt((float)n2) * g;
    int b = std::min(nq - 1, std::max(0, (int)(gscl / dq)));
    while (b + 1 < nq && !(gscl < (float)(b + 1) * dq)) ++b;   // largest b with b*dq <= |G|
    while (b > 0 && gscl < (float)b * dq) --b;
    gbin.push_back(b);
    gsum[b] += gscl;
    s->count[b] += 1;
  };
  auto add_run = [&](int i, int j, int k, int axis, int len) {
    rstart.push_back((int)gbin.size());
    runs.push_back(make_int4(i, j, k, (axis << 8) | len));
    for (int q = 0; q < len; ++q) add_vector(i + (axis == 0 ? q : 0), j + (axis == 1 ? q : 0), k + (axis == 2 ? q : 0));
  };
  for (int i = -kc; i <= kc; ++i)          // k > 0: runs along k
    for (int j = -kc; j <= kc; ++j) {
      int kmax = 0;
      while (i * i + j * j + (kmax + 1) * (kmax + 1) <= cut) ++kmax;
      for (int k = 1; k <= kmax; k += kRunLen) add_run(i, j, k, 2, std::min(kRunLen, kmax - k + 1));
    }
  for (int i = -kc; i <= kc; ++i) {        // k = 0, j > 0: runs along j
    int jmax = 0;
    while (i * i + (jmax + 1) * (jmax + 1) <= cut) ++jmax;
    for (int j = 1; j <= jmax; j += kRunLen) add_run(i, j, 0, 1, std::min(kRunLen, jmax - j + 1));
  }
  {                                        // k = j = 0, i > 0: runs along i
    int imax = 0;
    while ((imax + 1) * (imax + 1) <= cut) ++imax;
    for (int i = 1; i <= imax; i += kRunLen) add_run(i, 0, 0, 0, std::min(kRunLen, imax - i + 1));
  }
  s->ngv = (int)gbin.size();
  s->nrun = (int)runs.size();
  const size_t sc_bytes = (size_t)s->ngv * s->ntype * sizeof(float2);
  if (sc_bytes > (size_t)4 << 30)
    return nnpe_fail(c, NNPE_EOVERFLOW, "nnpe_sqd_setup: " + std::to_string(s->ngv) +
                                            " G vectors need more than 4 GB of per-vector sums; lower q_max");
  s->q.assign(nq, 0.0);
  for (int b = 0; b < nq; ++b) s->q[b] = s->count[b] ? gsum[b] / s->count[b] : 0.0;
  std::vector<int> bstart(nq + 1, 0), fill(nq, 0), bg(s->ngv);
  for (int b = 0; b < nq; ++b) bstart[b + 1] = bstart[b] + s->count[b];
  for (int v = 0; v < s->ngv; ++v) bg[bstart[gbin[v]] + fill[gbin[v]]++] = v;
  // factor N/(n_i n_j) and base N/n_j on the diagonal (grsq.cpp:474-482)
  std::vector<int> n(c->ntype, 0);
  for (int t : c->h_typ) n[t] += 1;
  std::vector<double> fb(2 * s->npair, 0.0);
  int p = 0;
  for (int i = 0; i < c->ntype; ++i)
    for (int j = i; j < c->ntype; ++j, ++p) {
      const double N = c->natom;
      fb[p] = (n[i] && n[j]) ? N / ((double)n[i] * n[j]) : 0.0;
      fb[s->npair + p] = (i == j && n[j]) ? N / n[j] : 0.0;
    }
  if (int rc = upload(c, &s->d_runs, runs)) return rc;
  if (int rc = upload(c, &s->d_rstart, rstart)) return rc;
  if (int rc = upload(c, &s->d_bstart, bstart)) return rc;
  if (int rc = upload(c, &s->d_bg, bg)) return rc;
  if (int rc = upload(c, &s->d_fb, fb)) return rc;
  NNPE_CUDA(c, dev_malloc(c, (void**)&s->d_sc, std::max<size_t>(sc_bytes, 16)));
  NNPE_CUDA(c, dev_malloc(c, (void**)&s->d_sq, sizeof(double) * std::max(1, nq * s->npair)));
  s->sq.assign((size_t)nq * s->npair, 0.0);
  if (ngv_out) *ngv_out = s->ngv;
  return NNPE_OK;
}

// SQD::compute (grsq.cpp:542-573) on the current positions.
int nnpe_sqd_compute(nnpe_ctx* c) {
  if (!c || !c->sqd) return nnpe_fail(c, NNPE_EARG, "nnpe_sqd_compute: no nnpe_sqd_setup");
  SqdState* s = c->sqd;
  cudaSetDevice(c->device);
  const double inv_l = 1.0 / (double)c->grid.bl;
  if (s->nrun > 0)
    k_sqd_runs<<<(s->nrun + kSqdThreads - 1) / kSqdThreads, kSqdThreads, 0, c->stream>>>(
        c->d_xd, c->d_info, c->natom, inv_l, s->d_runs, s->d_rstart, s->nrun, s->ntype, s->d_sc);
  k_sqd_bins<<<s->nq, 32, 0, c->stream>>>(s->d_sc, s->d_bstart, s->d_bg, s->ntype, s->npair, s->d_fb, s->d_sq);
  NNPE_CHECK_LAUNCH(c);
  NNPE_CUDA(c, cudaMemcpyAsync(s->sq.data(), s->d_sq, sizeof(double) * s->sq.size(), cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  s->have = true;
  return NNPE_OK;
}

int nnpe_sqd_get(nnpe_ctx* c, double* q, double* sq, int* count) {
  if (!c || !c->sqd) return nnpe_fail(c, NNPE_EARG, "nnpe_sqd_get: no nnpe_sqd_setup");
  SqdState* s = c->sqd;
  if (q) std::copy(s->q.begin(), s->q.end(), q);
  if (sq) std::copy(s->sq.begin(), s->sq.end(), sq);
  if (count) std::copy(s->count.begin(), s->count.end(), count);
  return NNPE_OK;
}

// SQD::dump (grsq.cpp:575-608): "# num" then, for each non-empty bin, q and one column per type
// pair; with append, the file's previous columns are averaged in with weight 1 - 1/num, num capped
// at 100 (MAXACC, grsq.cpp:25).
int nnpe_sqd_dump(nnpe_ctx* c, const char* fname, int append) {
  if (!c || !c->sqd || !fname) return nnpe_fail(c, NNPE_EARG, "nnpe_sqd_dump");
  SqdState* s = c->sqd;
  if (!s->have) return nnpe_fail(c, NNPE_EARG, "nnpe_sqd_dump: no nnpe_sqd_compute yet");
  std::vector<double> out = s->sq;
  int num = 1;
  FILE* fp = nullptr;
  if (append && (fp = fopen(fname, "r"))) {
    if (fscanf(fp, "# %d ", &num) != 1) num = 0;
    num = std::min(num + 1, 100);
    const double factor = 1.0 / num, cofactor = 1 - factor;
    for (int i = 0; i < s->nq; ++i) {
      if (!s->count[i]) continue;
      double v;
      if (fscanf(fp, "%lf ", &v) != 1) break;
      if (std::fabs(v - s->q[i]) > 1e-5) fprintf(stderr, "warning: large diff: %g %g\n", v, s->q[i]);
      for (int p = 0; p < s->npair; ++p) {
        if (fscanf(fp, "%lf ", &v) != 1) break;
        out[(size_t)i * s->npair + p] = out[(size_t)i * s->npair + p] * factor + cofactor * v;
      }
    }
    fclose(fp);
  }
  fp = fopen(fname, "w");
  if (!fp) return nnpe_fail(c, NNPE_EFILE, std::string("nnpe_sqd_dump: cannot write ") + fname);
  fprintf(fp, "# %d\n", num);
  for (int i = 0; i < s->nq; ++i) {
    if (!s->count[i]) continue;
    fprintf(fp, "%.15e", s->q[i]);
    for (int p = 0; p < s->npair; ++p) fprintf(fp, " %.15e", out[(size_t)i * s->npair + p]);
    fprintf(fp, "\n");
  }
  fclose(fp);
  return NNPE_OK;
}
