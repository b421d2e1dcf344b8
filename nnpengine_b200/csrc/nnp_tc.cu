// BF16 tensor-core (tcgen05) path of the radial-embedding network.
//
// Three kernels per force evaluation, each issuing its GEMMs as tcgen05.mma from one thread with
// operands in shared memory (no-swizzle K-major canonical layout, see tc_util.cuh) and FP32
// accumulators in tensor memory, read back row-per-thread for the epilogues:
//
//  k_tc_desc   one atom per 128-row tile (rows = the atom's pairs inside rc): each thread builds its
//              pair's first embedding layer h1 = tanh(W1*u + b1) into the A tile, block-diagonal
//              over neighbour species (K = ntype*32), so one MMA chain A x [W2_0; W2_1]^T gives the
//              second layer for every row whatever its species; epilogue y = tanh(z + b2) * cff,
//              then a fixed-order column reduction per special class into G_i (no atomics).
//  k_tc_fit    128 atoms of one species per tile: G -> h1 -> h2 -> E forward and the hand-written
//              backward dE/dG = ((A3 (1-h2^2)) A2^T (1-h1^2)) A1^T as four MMA chains (N = 128, 128,
//              128, 256); every activation stays in shared memory between the chains.
//  k_tc_force  one atom per tile again: recompute z2 (MMA 1), form g_c = a_c cff (1-y_c^2) with
//              a_c = scale*(dE/dG_i + dE/dG_j) (MMA 2 back through W2), finish dE/dr on the CUDA
//              cores and reduce fpair*(x_i-x_j) over the tile's rows in a fixed order.
//
// Every wait on the MMA-completion mbarrier is bounded; on time-out the kernel records
// NNPE_DEV_TIMEOUT, stops issuing work, frees its tensor memory and returns.
#include <cstring>
#include <vector>

#include "nnp.cuh"
#include "tc_util.cuh"

#define NNPE_DEV_TIMEOUT 32

struct NnpTc {
  int Kd = 0;                        // ntype*32: block-diagonal K of the embedding's second layer
  unsigned char* d_wdesc = nullptr;  // B image, N=64 (channel) x K=Kd: W2_t[q][c] at k=t*32+q
  unsigned char* d_wblk = nullptr;   // B image, N=Kd x K=64: W2_t[q][c] at n=t*32+q, k=c
  unsigned char* d_fit = nullptr;    // per species: L1 (N128,K256) L2 (128,128) B2 (128,128) B1 (256,128)
  size_t fit_stride = 0;
  float* d_emb_small = nullptr;      // per species: W1[32] b1[32] b2[64]
  float* d_fit_small = nullptr;      // per species: c1[128] c2[128] A3[128] c3 (stride 388)
  int* d_tile_sp = nullptr;          // fitting tiles: species, first row
  int* d_tile_row = nullptr;
  int ntiles = 0;
  int* d_soff = nullptr;
};

namespace {

constexpr int kFitSmallStride = 388;
constexpr size_t kImgL1 = 128 * 256 * 2, kImgL2 = 128 * 128 * 2, kImgB2 = 128 * 128 * 2, kImgB1 = 256 * 128 * 2;

__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

struct TcArgs {
  const float4* pos;
  const uint32_t* list6;
  const int* n6;
  const int* gowner;
  const unsigned char* wdesc;
  const unsigned char* wblk;
  const float* emb_small;
  float* G;
  const float* dG;
  float4* frc;
  double* watom;
  int* ctrl;
  int cap6, N, Kd;
  float rc, scale;
};

__device__ __forceinline__ void copy_image(unsigned char* dst, const unsigned char* src, int bytes, int t, int nt) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(dst);
  for (int k = t; k < bytes / 16; k += nt) d[k] = __ldg(s + k);
}

// Pair row of a tile: geometry, species, first embedding layer into the A tile (block tj).
struct PairRow {
  float dx, dy, dz, rsq, r, cff, dcff;
  int s, tj, jo;
  bool valid;
};

__device__ __forceinline__ PairRow load_pair(const TcArgs& a, int i, float4 xi, int k, int n) {
  PairRow p;
  p.valid = k < n;
  p.s = 0; p.tj = 0; p.jo = 0; p.dx = p.dy = p.dz = 0.f; p.rsq = 1.f; p.r = 1.f; p.cff = 0.f; p.dcff = 0.f;
  if (p.valid) {
    const uint32_t ent = a.list6[(size_t)i * a.cap6 + k];
    const int j = ent & NNPE_J_MASK;
    const float4 xj = a.pos[j];
    p.dx = xi.x - xj.x; p.dy = xi.y - xj.y; p.dz = xi.z - xj.z;
    p.rsq = p.dx * p.dx + p.dy * p.dy + p.dz * p.dz;
    p.r = sqrtf(p.rsq);
    const float cf = p.r - a.rc, den = 1.f + cf * cf;
    p.cff = 1.f - 1.f / den;
    p.dcff = 2.f * cf / (den * den);
    p.s = ent >> 30;
    p.tj = (ent >> 27) & 7;
    p.jo = j < a.N ? j : a.gowner[j - a.N];
  }
  return p;
}

__device__ __forceinline__ void write_h1_row(unsigned char* sA, int row, int Kd, const PairRow& p, const float* h) {
  const uint4 zero = make_uint4(0, 0, 0, 0);
  for (int kb = 0; kb < Kd / 8; ++kb) {
    uint4 v = zero;
    if (p.valid && (kb >> 2) == p.tj) v = tc::pack8(h + (kb & 3) * 8);
    *reinterpret_cast<uint4*>(sA + tc::kmajor_off(row, kb * 8, Kd)) = v;
  }
}

// -------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_tc_desc(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int Kd = a.Kd;
  unsigned char* sW = sm;
  unsigned char* sA = sW + 64 * Kd * 2;
  float* sY = reinterpret_cast<float*>(sA + 128 * Kd * 2);   // [128][65]
  int* sS = reinterpret_cast<int*>(sY + 128 * 65);
  const int t = threadIdx.x, w = t >> 5;
  if (w == 0) tc::tmem_alloc(&tmem_base, 64);
  if (t == 0) tc::mbar_init(&bar, 1);
  copy_image(sW, a.wdesc, 64 * Kd * 2, t, 128);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t taddr = tmem + ((uint32_t)(w * 32) << 16);
  const uint32_t idesc = tc::idesc_bf16(128, 64);
  const uint32_t aA = tc::smem_u32(sA), aW = tc::smem_u32(sW);
  const int col = t & 63, half = t >> 6;
  const float r_rc = 1.f / a.rc;
  uint32_t phase = 0;
  bool alive = true;
  const int per = (a.N + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(a.N, i0 + per);
  for (int i = i0; i < i1 && alive; ++i) {
    const float4 xi = a.pos[i];
    const int n = a.n6[i];
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int base = 0; base < n && alive; base += 128) {
      const PairRow p = load_pair(a, i, xi, base + t, n);
      float h[32];
      const float* es = a.emb_small + p.tj * 128;
      const float u = p.r * r_rc;
#pragma unroll
      for (int q = 0; q < 32; ++q) h[q] = tanh_fast(es[q] * u + es[32 + q]);
      write_h1_row(sA, t, Kd, p, h);
      sS[t] = p.s;
      tc::fence_async_smem();
      tc::fence_before();
      __syncthreads();
      tc::fence_after();
      if (t == 0) {
        for (int kk = 0; kk < Kd / 16; ++kk)
          tc::mma_bf16(tmem, tc::tile_desc(aA, Kd, kk), tc::tile_desc(aW, Kd, kk), idesc, kk > 0);
        tc::mma_commit(&bar);
      }
      {
        const bool got = tc::mbar_wait(&bar, phase);
        alive = __syncthreads_and(got) != 0;   // CTA-uniform: every thread takes the same path
        if (!got && (t & 31) == 0) atomicOr(a.ctrl + CTRL_ERR, NNPE_DEV_TIMEOUT);
      }
      phase ^= 1;
      tc::fence_after();
      if (alive) {
        const float cs = p.valid ? a.scale * p.cff : 0.f;
#pragma unroll
        for (int c0 = 0; c0 < 64; c0 += 16) {
          float v[16];
          tc::tmem_ld16(taddr + c0, v);
#pragma unroll
          for (int q = 0; q < 16; ++q) sY[t * 65 + c0 + q] = tanh_fast(v[q] + es[64 + c0 + q]) * cs;
        }
      }
      tc::fence_before();
      __syncthreads();
      const int rows = min(128, n - base);
      for (int rr = 0; rr < 64; ++rr) {
        const int row = half * 64 + rr;
        if (row >= rows) break;
        const float v = sY[row * 65 + col];
        const int sc = sS[row];
        acc[0] += sc == 0 ? v : 0.f;
        acc[1] += sc == 1 ? v : 0.f;
        acc[2] += sc == 2 ? v : 0.f;
        acc[3] += sc == 3 ? v : 0.f;
      }
      __syncthreads();
    }
    // combine the two row halves and store G_i[s*64+c]
#pragma unroll
    for (int sc = 0; sc < 4; ++sc) sY[(half * 4 + sc) * 64 + col] = acc[sc];
    __syncthreads();
    for (int e = t; e < 256; e += 128) a.G[(size_t)i * 256 + e] = sY[e] + sY[256 + e];
    __syncthreads();
  }
  tc::fence_before();
  __syncthreads();
  if (w == 0) tc::tmem_dealloc(tmem, 64);
}

// -------------------------------------------------------------------------------------------
template <bool EV>
__global__ void __launch_bounds__(128) k_tc_force(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  __shared__ float sRed[4][4];
  const int Kd = a.Kd;
  unsigned char* sW1 = sm;                          // N=64 x K=Kd
  unsigned char* sW2 = sW1 + 64 * Kd * 2;           // N=Kd x K=64
  unsigned char* sA = sW2 + Kd * 64 * 2;            // 128 x Kd
  unsigned char* sA2 = sA + 128 * Kd * 2;           // 128 x 64
  float* sdGi = reinterpret_cast<float*>(sA2 + 128 * 64 * 2);   // 256
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const uint32_t ncols = 64 + Kd <= 128 ? 128 : 256;
  if (w == 0) tc::tmem_alloc(&tmem_base, ncols);
  if (t == 0) tc::mbar_init(&bar, 1);
  copy_image(sW1, a.wdesc, 64 * Kd * 2, t, 128);
  copy_image(sW2, a.wblk, Kd * 64 * 2, t, 128);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t taddr = tmem + ((uint32_t)(w * 32) << 16);
  const uint32_t id1 = tc::idesc_bf16(128, 64), id2 = tc::idesc_bf16(128, Kd);
  const uint32_t aA = tc::smem_u32(sA), aA2 = tc::smem_u32(sA2), aW1 = tc::smem_u32(sW1), aW2 = tc::smem_u32(sW2);
  const float r_rc = 1.f / a.rc;
  uint32_t phase = 0;
  bool alive = true;
  const int per = (a.N + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(a.N, i0 + per);
  for (int i = i0; i < i1 && alive; ++i) {
    const float4 xi = a.pos[i];
    const int n = a.n6[i];
    for (int e = t; e < 256; e += 128) sdGi[e] = a.dG[(size_t)i * 256 + e];
    float fx = 0.f, fy = 0.f, fz = 0.f, vir = 0.f;
    for (int base = 0; base < n && alive; base += 128) {
      const PairRow p = load_pair(a, i, xi, base + t, n);
      float h[32];
      const float* es = a.emb_small + p.tj * 128;
      const float u = p.r * r_rc;
#pragma unroll
      for (int q = 0; q < 32; ++q) h[q] = tanh_fast(es[q] * u + es[32 + q]);
      write_h1_row(sA, t, Kd, p, h);
      tc::fence_async_smem();
      tc::fence_before();
      __syncthreads();
      tc::fence_after();
      if (t == 0) {
        for (int kk = 0; kk < Kd / 16; ++kk)
          tc::mma_bf16(tmem, tc::tile_desc(aA, Kd, kk), tc::tile_desc(aW1, Kd, kk), id1, kk > 0);
        tc::mma_commit(&bar);
      }
      {
        const bool got = tc::mbar_wait(&bar, phase);
        alive = __syncthreads_and(got) != 0;
        if (!got && lane == 0) atomicOr(a.ctrl + CTRL_ERR, NNPE_DEV_TIMEOUT);
      }
      phase ^= 1;
      tc::fence_after();
      float dEdr = 0.f;
      if (alive) {
        const float* dGj = a.dG + (size_t)p.jo * 256 + p.s * 64;
        const float* dGi = sdGi + p.s * 64;
#pragma unroll
        for (int c0 = 0; c0 < 64; c0 += 16) {
          float v[16], g[16];
          tc::tmem_ld16(taddr + c0, v);
#pragma unroll
          for (int q = 0; q < 16; q += 4) {
            float4 dj = make_float4(0.f, 0.f, 0.f, 0.f);
            if (p.valid) dj = *reinterpret_cast<const float4*>(dGj + c0 + q);
            const float dd[4] = {dj.x, dj.y, dj.z, dj.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int c = c0 + q + e;
              const float y = tanh_fast(v[q + e] + es[64 + c]);
              const float ac = a.scale * (dGi[c] + dd[e]);
              dEdr += ac * y * p.dcff;
              g[q + e] = p.valid ? ac * p.cff * (1.f - y * y) : 0.f;
            }
          }
          *reinterpret_cast<uint4*>(sA2 + tc::kmajor_off(t, c0, 64)) = tc::pack8(g);
          *reinterpret_cast<uint4*>(sA2 + tc::kmajor_off(t, c0 + 8, 64)) = tc::pack8(g + 8);
        }
      }
      tc::fence_async_smem();
      tc::fence_before();
      __syncthreads();
      tc::fence_after();
      if (alive && t == 0) {
        for (int kk = 0; kk < 4; ++kk)
          tc::mma_bf16(tmem + 64, tc::tile_desc(aA2, 64, kk), tc::tile_desc(aW2, 64, kk), id2, kk > 0);
        tc::mma_commit(&bar);
      }
      if (alive) {
        const bool got = tc::mbar_wait(&bar, phase);
        alive = __syncthreads_and(got) != 0;
        if (!got && lane == 0) atomicOr(a.ctrl + CTRL_ERR, NNPE_DEV_TIMEOUT);
      }
      phase ^= 1;
      tc::fence_after();
      if (alive) {
        for (int k16 = 0; k16 < Kd / 16; ++k16) {
          float v[16];
          tc::tmem_ld16(taddr + 64 + k16 * 16, v);
          if ((k16 >> 1) == p.tj) {
#pragma unroll
            for (int q = 0; q < 16; ++q) {
              const int qq = (k16 & 1) * 16 + q;
              dEdr += v[q] * (1.f - h[qq] * h[qq]) * es[qq] * r_rc;
            }
          }
        }
        if (p.valid) {
          const float fpair = -dEdr / p.r;
          fx += p.dx * fpair; fy += p.dy * fpair; fz += p.dz * fpair;
          if (EV) vir += 0.5f * fpair * p.rsq;
        }
      }
      tc::fence_before();
      __syncthreads();
    }
    for (int o = 16; o > 0; o >>= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, o);
      fy += __shfl_xor_sync(0xffffffffu, fy, o);
      fz += __shfl_xor_sync(0xffffffffu, fz, o);
      vir += __shfl_xor_sync(0xffffffffu, vir, o);
    }
    if (lane == 0) { sRed[w][0] = fx; sRed[w][1] = fy; sRed[w][2] = fz; sRed[w][3] = vir; }
    __syncthreads();
    if (t == 0) {
      const float4 f = a.frc[i];
      a.frc[i] = make_float4(f.x + ((sRed[0][0] + sRed[1][0]) + (sRed[2][0] + sRed[3][0])),
                             f.y + ((sRed[0][1] + sRed[1][1]) + (sRed[2][1] + sRed[3][1])),
                             f.z + ((sRed[0][2] + sRed[1][2]) + (sRed[2][2] + sRed[3][2])), f.w);
      if (EV) a.watom[i] += (double)((sRed[0][3] + sRed[1][3]) + (sRed[2][3] + sRed[3][3]));
    }
    __syncthreads();
  }
  tc::fence_before();
  __syncthreads();
  if (w == 0) tc::tmem_dealloc(tmem, ncols);
}

// -------------------------------------------------------------------------------------------
struct FitTcArgs {
  const int* sidx;
  const int* soff;
  const int* tile_sp;
  const int* tile_row;
  const float* G;
  const unsigned char* fit;
  size_t fit_stride;
  const float* small;
  float* dG;
  double* enet;
  int* ctrl;
};

__device__ __forceinline__ bool fit_mma(uint32_t tmem, uint32_t aA, int KA, uint32_t aB, int N, uint64_t* bar, uint32_t phase,
                                        int t, int* ctrl) {
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (t == 0) {
    const uint32_t id = tc::idesc_bf16(128, N);
    for (int kk = 0; kk < KA / 16; ++kk) tc::mma_bf16(tmem, tc::tile_desc(aA, KA, kk), tc::tile_desc(aB, KA, kk), id, kk > 0);
    tc::mma_commit(bar);
  }
  const bool got = tc::mbar_wait(bar, phase);
  const bool ok = __syncthreads_and(got) != 0;
  if (!got && (t & 31) == 0) atomicOr(ctrl + CTRL_ERR, NNPE_DEV_TIMEOUT);
  tc::fence_after();
  return ok;
}

__device__ __forceinline__ void sync_image(unsigned char* sW, const unsigned char* src, int bytes, int t) {
  tc::fence_before();
  __syncthreads();
  copy_image(sW, src, bytes, t, 128);
}

__global__ void __launch_bounds__(128) k_tc_fit(FitTcArgs f) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  unsigned char* sAct = sm;                 // 128 x 256 (G), later 128 x 128 (g2)
  unsigned char* sH1 = sm + 128 * 256 * 2;  // 128 x 128 (h1, later g1)
  unsigned char* sW = sH1 + 128 * 128 * 2;  // up to 64 KB
  const int t = threadIdx.x, w = t >> 5;
  const int sp = f.tile_sp[blockIdx.x], row0 = f.tile_row[blockIdx.x];
  const int M = f.soff[sp + 1] - f.soff[sp];
  const bool valid = row0 + t < M;
  const int atom = valid ? f.sidx[f.soff[sp] + row0 + t] : 0;
  const unsigned char* img = f.fit + f.fit_stride * sp;
  const float* sm_c1 = f.small + kFitSmallStride * sp;
  const float *sm_c2 = sm_c1 + 128, *sm_a3 = sm_c1 + 256, *sm_c3 = sm_c1 + 384;
  if (w == 0) tc::tmem_alloc(&tmem_base, 256);
  if (t == 0) tc::mbar_init(&bar, 1);
  // G row -> bf16 A tile (K=256)
  for (int k = 0; k < 256; k += 8) {
    float g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (valid) {
      const float4 u = *reinterpret_cast<const float4*>(f.G + (size_t)atom * 256 + k);
      const float4 v = *reinterpret_cast<const float4*>(f.G + (size_t)atom * 256 + k + 4);
      g[0] = u.x; g[1] = u.y; g[2] = u.z; g[3] = u.w; g[4] = v.x; g[5] = v.y; g[6] = v.z; g[7] = v.w;
    }
    *reinterpret_cast<uint4*>(sAct + tc::kmajor_off(t, k, 256)) = tc::pack8(g);
  }
  copy_image(sW, img, (int)kImgL1, t, 128);
  const uint32_t tmem = tmem_base;
  const uint32_t taddr = tmem + ((uint32_t)(w * 32) << 16);
  const uint32_t aAct = tc::smem_u32(sAct), aH1 = tc::smem_u32(sH1), aW = tc::smem_u32(sW);
  bool ok = true;
  // L1: z1 = G A1 (+c1), h1 = tanh
  ok = fit_mma(tmem, aAct, 256, aW, 128, &bar, 0, t, f.ctrl);
  if (ok) {
    for (int c0 = 0; c0 < 128; c0 += 16) {
      float v[16];
      tc::tmem_ld16(taddr + c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = tanh_fast(v[q] + sm_c1[c0 + q]);
      *reinterpret_cast<uint4*>(sH1 + tc::kmajor_off(t, c0, 128)) = tc::pack8(v);
      *reinterpret_cast<uint4*>(sH1 + tc::kmajor_off(t, c0 + 8, 128)) = tc::pack8(v + 8);
    }
  }
  sync_image(sW, img + kImgL1, (int)kImgL2, t);
  // L2: z2 = h1 A2 (+c2), h2 = tanh, E = h2 A3 + c3, g2 = A3 (1-h2^2)
  if (ok) ok = fit_mma(tmem + 128, aH1, 128, aW, 128, &bar, 1, t, f.ctrl);
  if (ok) {
    float e = 0.f;
    for (int c0 = 0; c0 < 128; c0 += 16) {
      float v[16];
      tc::tmem_ld16(taddr + 128 + c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float h2 = tanh_fast(v[q] + sm_c2[c0 + q]);
        e += h2 * sm_a3[c0 + q];
        v[q] = sm_a3[c0 + q] * (1.f - h2 * h2);
      }
      *reinterpret_cast<uint4*>(sAct + tc::kmajor_off(t, c0, 128)) = tc::pack8(v);
      *reinterpret_cast<uint4*>(sAct + tc::kmajor_off(t, c0 + 8, 128)) = tc::pack8(v + 8);
    }
    if (valid) f.enet[atom] = (double)e + (double)sm_c3[0];
  }
  sync_image(sW, img + kImgL1 + kImgL2, (int)kImgB2, t);
  // B2: u = g2 A2^T, g1 = u (1-h1^2)
  if (ok) ok = fit_mma(tmem, aAct, 128, aW, 128, &bar, 0, t, f.ctrl);
  if (ok) {
    for (int c0 = 0; c0 < 128; c0 += 16) {
      float v[16];
      tc::tmem_ld16(taddr + c0, v);
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        uint4* pchunk = reinterpret_cast<uint4*>(sH1 + tc::kmajor_off(t, c0 + 8 * hh, 128));
        const uint4 hv = *pchunk;
        const __nv_bfloat162* hb = reinterpret_cast<const __nv_bfloat162*>(&hv);
        float gg[8];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float2 hf = __bfloat1622float2(hb[e]);
          gg[2 * e] = v[8 * hh + 2 * e] * (1.f - hf.x * hf.x);
          gg[2 * e + 1] = v[8 * hh + 2 * e + 1] * (1.f - hf.y * hf.y);
        }
        *pchunk = tc::pack8(gg);
      }
    }
  }
  sync_image(sW, img + kImgL1 + kImgL2 + kImgB2, (int)kImgB1, t);
  // B1: dE/dG = g1 A1^T (N = 256)
  if (ok) ok = fit_mma(tmem, aH1, 128, aW, 256, &bar, 1, t, f.ctrl);
  if (ok) {
    for (int c0 = 0; c0 < 256; c0 += 16) {
      float v[16];
      tc::tmem_ld16(taddr + c0, v);   // warp-collective: every lane loads, valid rows store
      if (valid) {
        float4* dst = reinterpret_cast<float4*>(f.dG + (size_t)atom * 256 + c0);
        dst[0] = make_float4(v[0], v[1], v[2], v[3]); dst[1] = make_float4(v[4], v[5], v[6], v[7]);
        dst[2] = make_float4(v[8], v[9], v[10], v[11]); dst[3] = make_float4(v[12], v[13], v[14], v[15]);
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (w == 0) tc::tmem_dealloc(tmem, 256);
}

uint16_t f2bf(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
// byte-image of an N x K K-major no-swizzle bf16 tile, val(n,k)
template <typename F>
void put_image(std::vector<uint16_t>& img, size_t base, int N, int K, F&& val) {
  for (int n = 0; n < N; ++n)
    for (int k = 0; k < K; ++k) {
      const size_t off = ((size_t)(((n >> 3) * (K >> 3) + (k >> 3)) << 7) + ((n & 7) << 4) + ((k & 7) << 1)) / 2;
      img[base + off] = f2bf(val(n, k));
    }
}

}  // namespace

void nnp_tc_free(NnpModel* m) {
  NnpTc* t = m->tc;
  if (!t) return;
  for (void* p : {(void*)t->d_wdesc, (void*)t->d_wblk, (void*)t->d_fit, (void*)t->d_emb_small, (void*)t->d_fit_small,
                  (void*)t->d_tile_sp, (void*)t->d_tile_row, (void*)t->d_soff})
    if (p) cudaFree(p);
  delete t;
  m->tc = nullptr;
}

// Weight images and tile tables for the tensor-core path (embedding 1->32->64, fitting 256->128->128).
int nnp_tc_setup(nnpe_ctx* c) {
  NnpModel* m = c->nnp;
  if (m->kind != 1 || m->e1 != 32 || m->e2 != 64 || m->h1 != 128 || m->h2 != 128) return 0;   // FP32 only
  auto* t = new NnpTc();
  m->tc = t;
  const int T = c->ntype, Kd = 32 * T;
  t->Kd = Kd;
  const size_t eb = 32 + 32 + 32 * 64 + 64;
  const float* E = m->h_embw.data();
  std::vector<uint16_t> wdesc((size_t)64 * Kd), wblk((size_t)Kd * 64);
  put_image(wdesc, 0, 64, Kd, [&](int n, int k) { return E[eb * (k / 32) + 64 + (k % 32) * 64 + n]; });
  put_image(wblk, 0, Kd, 64, [&](int n, int k) { return E[eb * (n / 32) + 64 + (n % 32) * 64 + k]; });
  std::vector<float> emb_small((size_t)T * 128);
  for (int s = 0; s < T; ++s)
    for (int q = 0; q < 32; ++q) {
      emb_small[s * 128 + q] = E[eb * s + q];
      emb_small[s * 128 + 32 + q] = E[eb * s + 32 + q];
      emb_small[s * 128 + 64 + q] = E[eb * s + 64 + 32 * 64 + q];
      emb_small[s * 128 + 96 + q] = E[eb * s + 64 + 32 * 64 + 32 + q];
    }
  const size_t fb = (size_t)256 * 128 + 128 + 128 * 128 + 128 + 128 + 1;
  const size_t stride_el = (kImgL1 + kImgL2 + kImgB2 + kImgB1) / 2;
  std::vector<uint16_t> fit(stride_el * T);
  std::vector<float> fit_small((size_t)kFitSmallStride * T, 0.f);
  for (int s = 0; s < T; ++s) {
    const float* W = m->h_fitw.data() + fb * s;
    const float *A1 = W, *c1 = A1 + 256 * 128, *A2 = c1 + 128, *c2 = A2 + 128 * 128, *A3 = c2 + 128, *c3 = A3 + 128;
    const size_t b = stride_el * s;
    put_image(fit, b, 128, 256, [&](int n, int k) { return A1[k * 128 + n]; });                                  // L1
    put_image(fit, b + kImgL1 / 2, 128, 128, [&](int n, int k) { return A2[k * 128 + n]; });                     // L2
    put_image(fit, b + (kImgL1 + kImgL2) / 2, 128, 128, [&](int n, int k) { return A2[n * 128 + k]; });          // B2
    put_image(fit, b + (kImgL1 + kImgL2 + kImgB2) / 2, 256, 128, [&](int n, int k) { return A1[n * 128 + k]; }); // B1
    for (int q = 0; q < 128; ++q) {
      fit_small[kFitSmallStride * s + q] = c1[q];
      fit_small[kFitSmallStride * s + 128 + q] = c2[q];
      fit_small[kFitSmallStride * s + 256 + q] = A3[q];
    }
    fit_small[kFitSmallStride * s + 384] = c3[0];
  }
  std::vector<int> tsp, trow;
  for (int s = 0; s < T; ++s)
    for (int r = 0; r < m->soff[s + 1] - m->soff[s]; r += 128) { tsp.push_back(s); trow.push_back(r); }
  t->ntiles = (int)tsp.size();
  t->fit_stride = stride_el * 2;
  auto up = [&](void** d, const void* h, size_t bytes) -> int {
    NNPE_CUDA(c, cudaMalloc(d, std::max<size_t>(bytes, 16)));
    if (bytes) NNPE_CUDA(c, cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice));
    return 0;
  };
  if (int rc = up((void**)&t->d_wdesc, wdesc.data(), wdesc.size() * 2)) return rc;
  if (int rc = up((void**)&t->d_wblk, wblk.data(), wblk.size() * 2)) return rc;
  if (int rc = up((void**)&t->d_fit, fit.data(), fit.size() * 2)) return rc;
  if (int rc = up((void**)&t->d_emb_small, emb_small.data(), emb_small.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_fit_small, fit_small.data(), fit_small.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_tile_sp, tsp.data(), tsp.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_tile_row, trow.data(), trow.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_soff, m->soff.data(), m->soff.size() * 4)) return rc;
  const int smem_desc = 64 * Kd * 2 + 128 * Kd * 2 + 128 * 65 * 4 + 128 * 4;
  const int smem_force = 64 * Kd * 2 + Kd * 64 * 2 + 128 * Kd * 2 + 128 * 64 * 2 + 256 * 4;
  const int smem_fit = 128 * 256 * 2 + 128 * 128 * 2 + 256 * 128 * 2;
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_desc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_desc));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_force<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_force));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_force<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_force));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_fit, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_fit));
  return 0;
}

int nnp_tc_forces_enqueue(nnpe_ctx* c, bool ev) {
  NnpModel* m = c->nnp;
  NnpTc* t = m->tc;
  if (!t) return nnpe_fail(c, NNPE_EARG, "BF16 tensor-core path needs the 1->32->64 / 256->128->128 network");
  const int Kd = t->Kd;
  TcArgs a;
  a.pos = c->d_pos; a.list6 = m->d_list6; a.n6 = m->d_n6; a.gowner = c->d_gowner; a.wdesc = t->d_wdesc; a.wblk = t->d_wblk;
  a.emb_small = t->d_emb_small; a.G = m->d_G; a.dG = m->d_dG; a.frc = c->d_frc; a.watom = c->d_watom; a.ctrl = c->d_ctrl;
  a.cap6 = m->cap6; a.N = c->natom; a.Kd = Kd; a.rc = m->rc; a.scale = m->scale;
  const int sms = nnpe_sm_count(c->device);
  const int smem_desc = 64 * Kd * 2 + 128 * Kd * 2 + 128 * 65 * 4 + 128 * 4;
  const int smem_force = 64 * Kd * 2 + Kd * 64 * 2 + 128 * Kd * 2 + 128 * 64 * 2 + 256 * 4;
  const int smem_fit = 128 * 256 * 2 + 128 * 128 * 2 + 256 * 128 * 2;
  k_tc_desc<<<std::min(c->natom, sms * 3), 128, smem_desc, c->stream>>>(a);
  FitTcArgs f;
  f.sidx = m->d_sidx; f.soff = t->d_soff; f.tile_sp = t->d_tile_sp; f.tile_row = t->d_tile_row; f.G = m->d_G;
  f.fit = t->d_fit; f.fit_stride = t->fit_stride; f.small = t->d_fit_small; f.dG = m->d_dG; f.enet = m->d_enet;
  f.ctrl = c->d_ctrl;
  k_tc_fit<<<t->ntiles, 128, smem_fit, c->stream>>>(f);
  if (ev) k_tc_force<true><<<std::min(c->natom, sms * 4), 128, smem_force, c->stream>>>(a);
  else k_tc_force<false><<<std::min(c->natom, sms * 4), 128, smem_force, c->stream>>>(a);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

namespace {
// One CTA: D[128][N] = bf16(A[128][K]) x bf16(B[N][K])^T with FP32 accumulation in TMEM.
__global__ void __launch_bounds__(128) k_tc_selftest(const float* __restrict__ A, const float* __restrict__ B,
                                                     float* __restrict__ D, int N, int K, int ncols, int* err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int t = threadIdx.x, w = t >> 5;
  unsigned char* sA = smraw;
  unsigned char* sB = smraw + 128 * K * 2;
  if (w == 0) tc::tmem_alloc(&tmem_base, ncols);
  if (t == 0) tc::mbar_init(&bar, 1);
  for (int k = 0; k < K; k += 8) {
    float f[8];
    for (int q = 0; q < 8; ++q) f[q] = A[t * K + k + q];
    *reinterpret_cast<uint4*>(sA + tc::kmajor_off(t, k, K)) = tc::pack8(f);
  }
  for (int r = t; r < N; r += 128)
    for (int k = 0; k < K; k += 8) {
      float f[8];
      for (int q = 0; q < 8; ++q) f[q] = B[r * K + k + q];
      *reinterpret_cast<uint4*>(sB + tc::kmajor_off(r, k, K)) = tc::pack8(f);
    }
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tbase = tmem_base;
  if (t == 0) {
    const uint32_t idesc = tc::idesc_bf16(128, N);
    for (int kk = 0; kk < K / 16; ++kk)
      tc::mma_bf16(tbase, tc::tile_desc(tc::smem_u32(sA), K, kk), tc::tile_desc(tc::smem_u32(sB), K, kk), idesc, kk > 0);
    tc::mma_commit(&bar);
  }
  const bool ok = tc::mbar_wait(&bar, 0);
  if (!ok && (t & 31) == 0) atomicOr(err, 1);
  tc::fence_after();
  if (ok) {
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tbase + ((uint32_t)(w * 32) << 16) + c0, v);
      for (int q = 0; q < 16; ++q) D[(size_t)t * N + c0 + q] = v[q];
    }
  }
  tc::fence_before();
  __syncthreads();
  if (w == 0) tc::tmem_dealloc(tbase, ncols);
}
}  // namespace

// Self-test of the tcgen05 tile path: D[128][N] = A[128][K] x B[N][K]^T with BF16 operands.
extern "C" int nnpe_tc_selftest(int device, int N, int K, const float* A, const float* B, float* D) {
  if (N < 16 || N > 256 || N % 16 || K < 16 || K > 128 || K % 16 || !A || !B || !D) return NNPE_EARG;
  if (cudaSetDevice(device) != cudaSuccess) return NNPE_ECUDA;
  float *dA, *dB, *dD;
  int* derr;
  int ncols = 32;
  while (ncols < N) ncols <<= 1;
  if (cudaMalloc(&dA, sizeof(float) * 128 * K) || cudaMalloc(&dB, sizeof(float) * N * K) ||
      cudaMalloc(&dD, sizeof(float) * 128 * N) || cudaMalloc(&derr, sizeof(int)))
    return NNPE_ECUDA;
  cudaMemcpy(dA, A, sizeof(float) * 128 * K, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, B, sizeof(float) * N * K, cudaMemcpyHostToDevice);
  cudaMemset(derr, 0, sizeof(int));
  const int smem = (128 + N) * K * 2;
  cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  k_tc_selftest<<<1, 128, smem>>>(dA, dB, dD, N, K, ncols, derr);
  cudaError_t e = cudaDeviceSynchronize();
  int herr = 0;
  cudaMemcpy(D, dD, sizeof(float) * 128 * N, cudaMemcpyDeviceToHost);
  cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(dA); cudaFree(dB); cudaFree(dD); cudaFree(derr);
  if (e != cudaSuccess) return NNPE_ECUDA;
  return herr ? NNPE_ETIMEOUT : NNPE_OK;
}
