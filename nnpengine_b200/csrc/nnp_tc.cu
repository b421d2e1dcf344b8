// BF16 tensor-core (tcgen05) path of the radial-embedding network.
//
// Three kernels per force evaluation, each issuing its GEMMs as tcgen05.mma from one thread with
// operands in shared memory (no-swizzle canonical layouts, see tc_util.cuh) and FP32 accumulators
// in tensor memory, read back row-per-thread for the epilogues. Tiles of the two pair kernels hold
// up to 128 pairs of one atom, one pair per MMA row (TMEM lane):
//
//  k_tc_desc   first layer h1 = tanh(W1 u + b1) per pair into the A tile, block-diagonal over the
//              neighbour species (plus a one-hot bias slice) so one MMA chain gives every row the
//              second layer of its own net; epilogue y = scale cff tanh(z); the sum over pairs
//              into G_i by special class is a second MMA with a one-hot A (no shuffles, no atomics).
//  k_tc_fit    128 atoms of one species per tile: G -> h1 -> h2 -> E forward and the hand-written
//              backward dE/dG = ((A3 (1-h2^2)) A2^T (1-h1^2)) A1^T as four MMA chains (N = 128, 128,
//              128, 256); every activation stays in shared memory between the chains.
//  k_tc_force  second layer and its r-derivative per directed pair (two MMAs), the contraction with
//              the centre's dE/dG_i on the CUDA cores, and the pair force applied to both atoms in
//              64-bit fixed point (order-independent sums); k_facc_apply adds it to the forces.
//
// Every wait on the MMA-completion mbarrier is bounded; on time-out the kernel records
// NNPE_DEV_TIMEOUT, stops issuing work, frees its tensor memory and returns.
#include <cstring>
#include <vector>

#include "nnp.cuh"
#include "tc_util.cuh"

#define NNPE_DEV_TIMEOUT 32

struct NnpTc {
  int Kd = 0;                        // ntype*32
  unsigned char* d_wdesc = nullptr;  // B image N=64 (channel) x K=80: W2_t[q][c] at k=t*32+q, b2_t[c] at k=64+t
  unsigned long long* d_facc = nullptr;   // network forces [natom][3], fixed point (2^-32) for order-free sums
  unsigned char* d_fit = nullptr;    // per species: L1 (N128,K256) L2 (128,128) B2 (128,128) B1 (256,128)
  size_t fit_stride = 0;
  float* d_emb_small = nullptr;      // per species: W1[32] b1[32] b2[64]
  float* d_fit_small = nullptr;      // per species: c1[128] c2[128] A3[128] c3 (stride 388)
  int* d_tile_sp = nullptr;          // fitting tiles: species, first row
  int* d_tile_row = nullptr;
  int ntiles = 0;
  int* d_soff = nullptr;
  int ctas_desc = 1, ctas_force = 1;   // resident CTAs per SM (shared memory, registers, tensor memory)
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
  const int2* info;
  const uint32_t* list6;
  const int* n6;
  const int* gowner;
  const unsigned char* wdesc;
  unsigned long long* facc;
  const float* emb_small;
  float* G;
  const float* dG;
  float4* frc;
  double* watom;
  int* ctrl;
  int cap6, N, Kd, ntype, npos;
  float rc, scale;
};

__device__ __forceinline__ void copy_image(unsigned char* dst, const unsigned char* src, int bytes, int t, int nt) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(dst);
  for (int k = t; k < bytes / 16; k += nt) d[k] = __ldg(s + k);
}

// Wait for the MMA chain committed to bar: thread 0 polls the mbarrier (bounded) while the other
// threads block on the CTA barrier, so waiting warps take no issue slots from other CTAs. Returns
// false on every thread when the wait timed out, after recording NNPE_DEV_TIMEOUT.
__device__ __forceinline__ bool cta_wait_mma(uint64_t* bar, uint32_t phase, int* ctrl) {
  bool got = true;
  if (threadIdx.x == 0) {
    got = tc::mbar_wait(bar, phase);
    if (!got) atomicOr(ctrl + CTRL_ERR, NNPE_DEV_TIMEOUT);
  }
  const bool ok = __syncthreads_and(got) != 0;
  tc::fence_after();
  return ok;
}

// Pair of a tile: geometry, species, cutoff factor and its derivative.
struct PairRow {
  float dx, dy, dz, rsq, r, cff, dcff;
  int s, tj, jo;
  bool valid;
};

// list entry -> position index, kept inside the position array for entries past the atom's
// count (those rows are fetched ahead of time and discarded)
__device__ __forceinline__ int entry_j(uint32_t ent, int npos) {
  const int j = ent & NNPE_J_MASK;
  return j < npos ? j : 0;
}

__device__ __forceinline__ PairRow make_pair(const TcArgs& a, float3 xi, uint32_t ent, float3 xj, bool valid) {
  PairRow p;
  p.valid = valid;
  p.s = 0; p.tj = 0; p.jo = 0; p.dx = p.dy = p.dz = 0.f; p.rsq = 1.f; p.r = 1.f; p.cff = 0.f; p.dcff = 0.f;
  if (valid) {
    const int j = ent & NNPE_J_MASK;
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

// Per-species embedding constants in shared memory, row stride 129 floats so that the two
// species' rows fall in different banks: W1 [0,32), b1 [32,64), b2 [64,128).
constexpr int kEmbStride = 129;
__device__ __forceinline__ void load_emb(float* sE, const float* emb_small, int ntype, int t, int nt) {
  for (int k = t; k < 2 * 128; k += nt) sE[(k >> 7) * kEmbStride + (k & 127)] = (k >> 7) < ntype ? emb_small[k] : 0.f;
}

// 16 first-layer units [q0, q0+16) of species sp's net at u = r/rc: h = tanh(W1 u + b1), and
// v = dh/dr = (1 - h^2) W1 / rc when V.
template <bool V>
__device__ __forceinline__ void first_layer16(const float* sE, int sp, float u, float r_rc, int q0, bool on, float* h,
                                              float* v) {
  const float* e = sE + sp * kEmbStride;
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const float w1 = e[q0 + q];
    const float hq = on ? tanh_fast(w1 * u + e[32 + q0 + q]) : 0.f;
    h[q] = hq;
    if (V) v[q] = on ? (1.f - hq * hq) * w1 * r_rc : 0.f;
  }
}

constexpr int kTile = 128;   // pairs per tile (MMA rows)
// K of the embedding's second-layer MMAs: the first layer in the block of the pair's species
// ([0, 32) species 0, [32, 64) species 1) and a one-hot bias slice [64, 80) that adds b2_t.
constexpr int kKE = 80;

// Tile walk of the pair kernels: a CTA owns atoms [i0, i1) and visits their pairs in tiles of up
// to kTile (one atom per tile). Row p's list entry and neighbour position for the next tile are
// fetched while the current tile computes.
struct TileCursor {
  int i, base, n;
  float3 xi;
  uint32_t ent;
  float3 xj;
};
__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ void cursor_next(const TcArgs& a, const TileCursor& c, int i1, int p, TileCursor& nx,
                                            bool& more) {
  nx.i = c.i; nx.base = c.base + kTile; nx.n = c.n; nx.xi = c.xi;
  if (nx.base >= c.n) { nx.i = c.i + 1; nx.base = 0; }
  more = nx.i < i1;
  nx.ent = 0;
  if (more) {
    nx.ent = a.list6[(size_t)nx.i * a.cap6 + nx.base + p];
    if (nx.i != c.i) { nx.n = a.n6[nx.i]; nx.xi = xyz(a.pos[nx.i]); }
  }
}
__device__ __forceinline__ void cursor_first(const TcArgs& a, int i0, int p, TileCursor& c) {
  c.i = i0; c.base = 0; c.n = a.n6[i0]; c.xi = xyz(a.pos[i0]);
  c.ent = a.list6[(size_t)i0 * a.cap6 + p];
  c.xj = xyz(a.pos[entry_j(c.ent, a.npos)]);
}

// Row p of an A tile [128 x kKE]: 16 values at k0 of the species block sp, zeros at the same
// offset of the other block; with bias, the one-hot of sp in the bias slice (else zeros).
__device__ __forceinline__ void put_row16(unsigned char* tile, int p, int sp, int k0, const float* v) {
  *reinterpret_cast<uint4*>(tile + tc::kmajor_off(p, 32 * sp + k0, kKE)) = tc::pack8(v);
  *reinterpret_cast<uint4*>(tile + tc::kmajor_off(p, 32 * sp + k0 + 8, kKE)) = tc::pack8(v + 8);
  const uint4 z = make_uint4(0, 0, 0, 0);
  *reinterpret_cast<uint4*>(tile + tc::kmajor_off(p, 32 * (1 - sp) + k0, kKE)) = z;
  *reinterpret_cast<uint4*>(tile + tc::kmajor_off(p, 32 * (1 - sp) + k0 + 8, kKE)) = z;
}
__device__ __forceinline__ void put_bias(unsigned char* tile, int p, int sp, bool one) {
  uint4 u = make_uint4(0, 0, 0, 0);
  if (one) {   // bf16 1.0 in element sp of the first 8
    const uint32_t v = 0x3F80u << (16 * (sp & 1));
    if (sp < 2) u.x = v; else u.y = v;
  }
  *reinterpret_cast<uint4*>(tile + tc::kmajor_off(p, 64, kKE)) = u;
  *reinterpret_cast<uint4*>(tile + tc::kmajor_off(p, 72, kKE)) = make_uint4(0, 0, 0, 0);
}

// -------------------------------------------------------------------------------------------
// Descriptor. Tile = up to 128 pairs of one atom i, pair p in MMA row / TMEM lane p = thread p.
//  MMA 1: Z = H1 W2s + b2, H1 [128 x 80] holding each pair's first layer in the block of its
//         neighbour species plus the one-hot bias slice, W2s = [W2_0; W2_1; b2] (K = 80, N = 64):
//         row p of Z is the second-layer input of the net of t_p.
//  epilogue: Y[p][c] = scale cff_p tanh(Z[p][c]), rounded to BF16, written over the H1 tile
//         (which MMA 1 has consumed).
//  MMA 2: G_i[s][c] = sum_p S[s][p] Y[p][c], S the one-hot of the pair's special class: A = S
//         (8 rows, read with zero row-group stride so every 8-row group of the M = 128 tile
//         repeats it), B = Y (MN-major), K = the tile's pairs. Lanes 0..3 of the accumulator
//         then hold G_i by class, in FP32.
// Rows past the atom's pairs are neither computed nor read (H1 rows past the count only feed
// unread accumulator rows; Y rows up to the 16-pair MMA granule are written as zeros).
constexpr int kSmemDesc = 64 * kKE * 2 + kTile * kKE * 2 + 8 * kTile * 2 + 2 * kEmbStride * 4;
__global__ void __launch_bounds__(128, 8) k_tc_desc(TcArgs a) {
  extern __shared__ __align__(128) unsigned char sm[];   // no-swizzle operands need 16-byte alignment
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  unsigned char* sW = sm;                        // B of MMA 1: N = 64 channels x K = 80
  unsigned char* sHY = sW + 64 * kKE * 2;        // A of MMA 1 (128 pairs x K = 80), then B of MMA 2
  unsigned char* sS = sHY + kTile * kKE * 2;     // A of MMA 2: 8 classes x K = 128 pairs
  float* sE = reinterpret_cast<float*>(sS + 8 * kTile * 2);   // embedding constants (8 CTAs per SM fit)
  const int t = threadIdx.x, w = t >> 5, lane = t & 31, p = t;
  if (w == 0) tc::tmem_alloc(&tmem_base, 64);
  if (t == 0) tc::mbar_init(&bar, 1);
  copy_image(sW, a.wdesc, 64 * kKE * 2, t, 128);
  load_emb(sE, a.emb_small, a.ntype, t, 128);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t taddr = tmem + ((uint32_t)(w * 32) << 16);
  const uint32_t aW = tc::smem_u32(sW), aHY = tc::smem_u32(sHY), aS = tc::smem_u32(sS);
  const float r_rc = 1.f / a.rc;
  uint32_t phase = 0;
  bool alive = true;
  const int per = (a.N + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(a.N, i0 + per);
  TileCursor cur;
  if (i0 < i1) cursor_first(a, i0, p, cur);
  bool more = i0 < i1;
  while (more && alive) {
    TileCursor nx;
    cursor_next(a, cur, i1, p, nx, more);
    const int cnt = max(0, min(kTile, cur.n - cur.base)), NK = (cnt + 15) & ~15;
    const PairRow pr = make_pair(a, cur.xi, cur.ent, cur.xj, p < cnt);
    if (pr.valid) {
      const float u = pr.r * r_rc;
#pragma unroll
      for (int hq = 0; hq < 2; ++hq) {
        float h[16];
        first_layer16<false>(sE, pr.tj, u, r_rc, 16 * hq, true, h, nullptr);
        put_row16(sHY, p, pr.tj, 16 * hq, h);
      }
      put_bias(sHY, p, pr.tj, true);
    }
    if (p < NK) {
      const uint16_t one = 0x3F80u;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        *reinterpret_cast<uint16_t*>(sS + tc::kmajor_off(c, p, kTile)) = (pr.valid && pr.s == c) ? one : (uint16_t)0;
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (t == 0) {
      const uint32_t id = tc::idesc_bf16(128, 64);
      for (int kk = 0; kk < kKE / 16; ++kk)
        tc::mma_bf16(tmem, tc::tile_desc(aHY, kKE, kk), tc::tile_desc(aW, kKE, kk), id, kk > 0);
      tc::mma_commit(&bar);
    }
    alive = cta_wait_mma(&bar, phase, a.ctrl);
    phase ^= 1;
    nx.xj = more ? xyz(a.pos[entry_j(nx.ent, a.npos)]) : make_float3(0.f, 0.f, 0.f);
    if (alive && 32 * w < NK) {   // warp-uniform
      const float cs = a.scale * pr.cff;   // 0 for rows past the atom's pairs
#pragma unroll
      for (int c0 = 0; c0 < 64; c0 += 32) {
        float z[16], z2[16];
        tc::tmem_ld16x2(taddr + c0, taddr + c0 + 16, z, z2);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          z[q] = pr.valid ? tanh_fast(z[q]) * cs : 0.f;
          z2[q] = pr.valid ? tanh_fast(z2[q]) * cs : 0.f;
        }
        if (p < NK) {
          *reinterpret_cast<uint4*>(sHY + tc::mnmajor_off(c0, p, 64)) = tc::pack8(z);
          *reinterpret_cast<uint4*>(sHY + tc::mnmajor_off(c0 + 8, p, 64)) = tc::pack8(z + 8);
          *reinterpret_cast<uint4*>(sHY + tc::mnmajor_off(c0 + 16, p, 64)) = tc::pack8(z2);
          *reinterpret_cast<uint4*>(sHY + tc::mnmajor_off(c0 + 24, p, 64)) = tc::pack8(z2 + 8);
        }
      }
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    float* Gi = a.G + (size_t)cur.i * 256;
    if (NK > 0) {   // CTA-uniform
      if (alive && t == 0) {
        const uint32_t id = tc::idesc_bf16(128, 64, true);
        for (int kk = 0; kk < NK / 16; ++kk)
          tc::mma_bf16(tmem, tc::tile_desc_bcast(aS, kTile, kk), tc::tile_desc_mn(aHY, 64, kk), id, kk > 0);
        tc::mma_commit(&bar);
      }
      if (alive) alive = cta_wait_mma(&bar, phase, a.ctrl);
      phase ^= 1;
      if (alive && w == 0) {   // lanes 0..3 hold G_i by special class
#pragma unroll
        for (int c0 = 0; c0 < 64; c0 += 32) {
          float g[16], g2[16];
          tc::tmem_ld16x2(tmem + c0, tmem + c0 + 16, g, g2);
          if (lane < 4) {
            float4* dst = reinterpret_cast<float4*>(Gi + lane * 64 + c0);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              const float* src = q < 4 ? g + 4 * q : g2 + 4 * (q - 4);
              float4 v = make_float4(src[0], src[1], src[2], src[3]);
              if (cur.base > 0) {
                const float4 o = dst[q];
                v.x += o.x; v.y += o.y; v.z += o.z; v.w += o.w;
              }
              dst[q] = v;
            }
          }
        }
      }
    } else if (cur.base == 0) {
      for (int e = t; e < 256; e += 128) Gi[e] = 0.f;   // an atom without pairs
    }
    tc::fence_before();
    __syncthreads();
    cur = nx;
  }
  tc::fence_before();
  __syncthreads();
  if (w == 0) tc::tmem_dealloc(tmem, 64);
}

// -------------------------------------------------------------------------------------------
// Force. The pair (i, j) enters G_i through the net of t_j and G_j through the net of t_i, so
// dE/dr_ij = T(i->j) + T(j->i) with T(i->j) = scale sum_c dE/dG_i[s*64+c] d(y_c cff)/dr, y the
// net of t_j. Each directed pair of the full list computes its own T from the centre's dE/dG_i
// (one net per pair, no gather of dE/dG_j) and applies fpair = -T/r with opposite signs to i and
// to j's owner; the reverse visit supplies the other half. Forces are summed in 64-bit fixed
// point (2^-32), whose integer additions give the same bits in any order, and added to the
// FP32 forces by k_facc_apply.
//  MMA 1: Z = H W2s + b2 (as in the descriptor), MMA 2: K = V W2s, V = dh1/dr in the same
//  block layout with a zero bias slice, so K[p][c] = dz2_c/dr.
//  epilogue: thread (p, half) takes 32 channels: with a = dE/dG_i[s][c] and y = tanh(z),
//  d(y cff)/dr = y dcff + cff (1 - y^2) kappa, so T = scale (dcff sum a y + cff sum a kappa (1 - y^2)).
// The per-atom virial gets -T r for each of the atom's directed pairs.
// Tensor memory: Z in columns [0, 64), K in [64, 128).
constexpr int kSmemForce = 64 * kKE * 2 + 2 * kTile * kKE * 2 + 256 * 4 + 2 * kTile * 4 + 2 * kEmbStride * 4;
constexpr float kFix = 4294967296.f;   // fixed-point scale of the network forces

__device__ __forceinline__ void fix_add(unsigned long long* dst, float v) {
  atomicAdd(dst, (unsigned long long)__float2ll_rn(v * kFix));
}

template <bool EV>
__global__ void __launch_bounds__(256, 4) k_tc_force(TcArgs a) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  __shared__ float sRed[4][3];
  __shared__ double sVir[4];
  unsigned char* sW = sm;                                        // B: N = 64 x K = 80
  unsigned char* sH = sW + 64 * kKE * 2;                         // A of MMA 1
  unsigned char* sV = sH + kTile * kKE * 2;                      // A of MMA 2
  float* sdGi = reinterpret_cast<float*>(sV + kTile * kKE * 2);  // dE/dG_i [256]
  float* sAcc = sdGi + 256;                                      // [2][128]: per-half sums
  float* sE = sAcc + 2 * kTile;
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int p = ((w & 3) << 5) | lane, half = w >> 2;   // pair row, channel half of this thread
  if (w == 0) tc::tmem_alloc(&tmem_base, 128);
  if (t == 0) tc::mbar_init(&bar, 1);
  copy_image(sW, a.wdesc, 64 * kKE * 2, t, 256);
  load_emb(sE, a.emb_small, a.ntype, t, 256);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t taddr = tmem + ((uint32_t)((w & 3) * 32) << 16);
  const uint32_t aW = tc::smem_u32(sW), aH = tc::smem_u32(sH), aV = tc::smem_u32(sV);
  const float r_rc = 1.f / a.rc;
  uint32_t phase = 0;
  bool alive = true;
  const int per = (a.N + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(a.N, i0 + per);
  TileCursor cur;
  if (i0 < i1) cursor_first(a, i0, p, cur);
  bool more = i0 < i1;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  double vir = 0.0;
  while (more && alive) {
    TileCursor nx;
    cursor_next(a, cur, i1, p, nx, more);
    if (cur.base == 0) sdGi[t] = a.dG[(size_t)cur.i * 256 + t];
    const int cnt = max(0, min(kTile, cur.n - cur.base));
    const PairRow pr = make_pair(a, cur.xi, cur.ent, cur.xj, p < cnt);
    if (pr.valid) {
      float h[16], v[16];
      first_layer16<true>(sE, pr.tj, pr.r * r_rc, r_rc, 16 * half, true, h, v);
      put_row16(sH, p, pr.tj, 16 * half, h);
      put_row16(sV, p, pr.tj, 16 * half, v);
      if (half == 0) { put_bias(sH, p, pr.tj, true); put_bias(sV, p, pr.tj, false); }
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (t == 0) {
      const uint32_t id = tc::idesc_bf16(128, 64);
      for (int kk = 0; kk < kKE / 16; ++kk)
        tc::mma_bf16(tmem, tc::tile_desc(aH, kKE, kk), tc::tile_desc(aW, kKE, kk), id, kk > 0);
      for (int kk = 0; kk < kKE / 16; ++kk)
        tc::mma_bf16(tmem + 64, tc::tile_desc(aV, kKE, kk), tc::tile_desc(aW, kKE, kk), id, kk > 0);
      tc::mma_commit(&bar);
    }
    alive = cta_wait_mma(&bar, phase, a.ctrl);
    phase ^= 1;
    nx.xj = more ? xyz(a.pos[entry_j(nx.ent, a.npos)]) : make_float3(0.f, 0.f, 0.f);
    float sy = 0.f, sk = 0.f;
    if (alive && 32 * (w & 3) < cnt) {   // warp-uniform: the loads below are warp-collective
      const float* ag = sdGi + pr.s * 64 + 32 * half;
#pragma unroll
      for (int c0 = 0; c0 < 32; c0 += 16) {
        float z[16], kap[16];
        tc::tmem_ld16x2(taddr + 32 * half + c0, taddr + 64 + 32 * half + c0, z, kap);
#pragma unroll
        for (int q = 0; q < 16; q += 4) {
          const float4 a4 = *reinterpret_cast<const float4*>(ag + c0 + q);
          const float av[4] = {a4.x, a4.y, a4.z, a4.w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float y = tanh_fast(z[q + e]);
            sy = fmaf(av[e], y, sy);
            sk = fmaf(av[e] * kap[q + e], fmaf(-y, y, 1.f), sk);
          }
        }
      }
    }
    sAcc[half * kTile + p] = pr.valid ? a.scale * (pr.dcff * sy + pr.cff * sk) : 0.f;
    __syncthreads();
    if (half == 0 && pr.valid) {
      const float fpair = -(sAcc[p] + sAcc[kTile + p]) / pr.r;
      const float gx = pr.dx * fpair, gy = pr.dy * fpair, gz = pr.dz * fpair;
      fx += gx; fy += gy; fz += gz;
      unsigned long long* fj = a.facc + 3 * (size_t)pr.jo;
      fix_add(fj, -gx); fix_add(fj + 1, -gy); fix_add(fj + 2, -gz);
      if (EV) vir += (double)(fpair * pr.rsq);
    }
    if (!more || nx.i != cur.i) {   // CTA-uniform: last tile of atom cur.i
      if (w < 4) {
        for (int o = 16; o > 0; o >>= 1) {
          fx += __shfl_xor_sync(0xffffffffu, fx, o);
          fy += __shfl_xor_sync(0xffffffffu, fy, o);
          fz += __shfl_xor_sync(0xffffffffu, fz, o);
          if (EV) vir += __shfl_xor_sync(0xffffffffu, vir, o);
        }
        if (lane == 0) { sRed[w][0] = fx; sRed[w][1] = fy; sRed[w][2] = fz; sVir[w] = vir; }
      }
      __syncthreads();
      if (t == 0 && cur.n > 0) {
        unsigned long long* fi = a.facc + 3 * (size_t)cur.i;
        fix_add(fi, (sRed[0][0] + sRed[1][0]) + (sRed[2][0] + sRed[3][0]));
        fix_add(fi + 1, (sRed[0][1] + sRed[1][1]) + (sRed[2][1] + sRed[3][1]));
        fix_add(fi + 2, (sRed[0][2] + sRed[1][2]) + (sRed[2][2] + sRed[3][2]));
        if (EV) a.watom[cur.i] += (sVir[0] + sVir[1]) + (sVir[2] + sVir[3]);
      }
      fx = fy = fz = 0.f;
      vir = 0.0;
    }
    tc::fence_before();
    __syncthreads();
    cur = nx;
  }
  tc::fence_before();
  __syncthreads();
  if (w == 0) tc::tmem_dealloc(tmem, 128);
}

// frc[i] += fixed-point network force of atom i
__global__ void k_facc_apply(const unsigned long long* __restrict__ facc, float4* __restrict__ frc, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double s = 1.0 / kFix;
  float4 f = frc[i];
  f.x += (float)((double)(long long)facc[3 * i] * s);
  f.y += (float)((double)(long long)facc[3 * i + 1] * s);
  f.z += (float)((double)(long long)facc[3 * i + 2] * s);
  frc[i] = f;
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
  return cta_wait_mma(bar, phase, ctrl);
}

__device__ __forceinline__ void sync_image(unsigned char* sW, const unsigned char* src, int bytes, int t) {
  tc::fence_before();
  __syncthreads();
  copy_image(sW, src, bytes, t, 128);
}

__global__ void __launch_bounds__(128) k_tc_fit(FitTcArgs f) {
  extern __shared__ __align__(128) unsigned char sm[];
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
  for (void* p : {(void*)t->d_wdesc, (void*)t->d_facc, (void*)t->d_fit, (void*)t->d_emb_small, (void*)t->d_fit_small,
                  (void*)t->d_tile_sp, (void*)t->d_tile_row, (void*)t->d_soff})
    if (p) dev_free(p);
  delete t;
  m->tc = nullptr;
}

// Weight images and tile tables for the tensor-core path (embedding 1->32->64, fitting 256->128->128).
int nnp_tc_setup(nnpe_ctx* c) {
  NnpModel* m = c->nnp;
  // the tensor-core kernels hold every species' net side by side in K = 64 / N = 128: at most 2 species
  if (m->kind != 1 || m->e1 != 32 || m->e2 != 64 || m->h1 != 128 || m->h2 != 128 || c->ntype > 2) return 0;
  auto* t = new NnpTc();
  m->tc = t;
  const int T = c->ntype, Kd = 32 * T;
  t->Kd = Kd;
  const size_t eb = 32 + 32 + 32 * 64 + 64;
  const float* E = m->h_embw.data();
  std::vector<uint16_t> wdesc((size_t)64 * kKE);
  put_image(wdesc, 0, 64, kKE, [&](int n, int k) {
    if (k < 64) return k / 32 < T ? E[eb * (k / 32) + 64 + (k % 32) * 64 + n] : 0.f;
    return k - 64 < T ? E[eb * (k - 64) + 64 + 32 * 64 + n] : 0.f;   // bias rows b2_t
  });
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
    NNPE_CUDA(c, dev_malloc(c, d, std::max<size_t>(bytes, 16)));
    if (bytes) NNPE_CUDA(c, cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice));
    return 0;
  };
  if (int rc = up((void**)&t->d_wdesc, wdesc.data(), wdesc.size() * 2)) return rc;
  NNPE_CUDA(c, dev_malloc(c, (void**)&t->d_facc, sizeof(unsigned long long) * 3 * std::max(c->natom, 1)));
  if (int rc = up((void**)&t->d_fit, fit.data(), fit.size() * 2)) return rc;
  if (int rc = up((void**)&t->d_emb_small, emb_small.data(), emb_small.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_fit_small, fit_small.data(), fit_small.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_tile_sp, tsp.data(), tsp.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_tile_row, trow.data(), trow.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_soff, m->soff.data(), m->soff.size() * 4)) return rc;
  const int smem_desc = kSmemDesc, smem_force = kSmemForce;
  const int smem_fit = 128 * 256 * 2 + 128 * 128 * 2 + 256 * 128 * 2;
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_desc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_desc));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_force<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_force));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_force<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_force));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_fit, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_fit));
  // one wave of resident CTAs: a grid larger than what fits leaves a partial second wave
  int od = 0, of = 0;
  NNPE_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&od, k_tc_desc, 128, smem_desc));
  NNPE_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&of, k_tc_force<true>, 256, smem_force));
  t->ctas_desc = std::max(1, std::min(od, 512 / 64));
  t->ctas_force = std::max(1, std::min(of, 512 / 128));
  return 0;
}

int nnp_tc_forces_enqueue(nnpe_ctx* c, bool ev) {
  NnpModel* m = c->nnp;
  NnpTc* t = m->tc;
  if (!t) return nnpe_fail(c, NNPE_EARG, "BF16 tensor-core path needs the 1->32->64 / 256->128->128 network");
  const int Kd = t->Kd;
  TcArgs a;
  a.pos = c->d_pos; a.info = c->d_info; a.list6 = m->d_list6; a.n6 = m->d_n6; a.gowner = c->d_gowner; a.wdesc = t->d_wdesc; a.facc = t->d_facc;
  a.emb_small = t->d_emb_small; a.G = m->d_G; a.dG = m->d_dG; a.frc = c->d_frc; a.watom = c->d_watom; a.ctrl = c->d_ctrl;
  a.cap6 = m->cap6; a.N = c->natom; a.Kd = Kd; a.ntype = c->ntype; a.npos = c->natom + c->Gcap; a.rc = m->rc; a.scale = m->scale;
  const int sms = nnpe_sm_count(c->device);
  const int smem_fit = 128 * 256 * 2 + 128 * 128 * 2 + 256 * 128 * 2;
  k_tc_desc<<<std::min(c->natom, sms * t->ctas_desc), 128, kSmemDesc, c->stream>>>(a);
  FitTcArgs f;
  f.sidx = m->d_sidx; f.soff = t->d_soff; f.tile_sp = t->d_tile_sp; f.tile_row = t->d_tile_row; f.G = m->d_G;
  f.fit = t->d_fit; f.fit_stride = t->fit_stride; f.small = t->d_fit_small; f.dG = m->d_dG; f.enet = m->d_enet;
  f.ctrl = c->d_ctrl;
  k_tc_fit<<<t->ntiles, 128, smem_fit, c->stream>>>(f);
  NNPE_CUDA(c, cudaMemsetAsync(t->d_facc, 0, sizeof(unsigned long long) * 3 * c->natom, c->stream));
  const int gforce = std::min(c->natom, sms * t->ctas_force);
  if (ev) k_tc_force<true><<<gforce, 256, kSmemForce, c->stream>>>(a);
  else k_tc_force<false><<<gforce, 256, kSmemForce, c->stream>>>(a);
  k_facc_apply<<<(c->natom + 255) / 256, 256, 0, c->stream>>>(t->d_facc, c->d_frc, c->natom);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

namespace {
// One CTA: D[128][N] = bf16(A[128][K]) x bf16(B[N][K])^T with FP32 accumulation in TMEM.
// mode 0: A, B K-major; mode 1: B MN-major; mode 2: A row-broadcast (rows repeat every 8, SBO=0).
__global__ void __launch_bounds__(128) k_tc_selftest(const float* __restrict__ A, const float* __restrict__ B,
                                                     float* __restrict__ D, int N, int K, int ncols, int mode, int* err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int t = threadIdx.x, w = t >> 5;
  unsigned char* sA = smraw;
  unsigned char* sB = smraw + 128 * K * 2;
  if (w == 0) tc::tmem_alloc(&tmem_base, ncols);
  if (t == 0) tc::mbar_init(&bar, 1);
  const bool a_bcast = mode == 2 || mode == 3, b_mn = mode == 1 || mode == 3;
  if (!a_bcast || t < 8)
    for (int k = 0; k < K; k += 8) {
      float f[8];
      for (int q = 0; q < 8; ++q) f[q] = A[t * K + k + q];
      *reinterpret_cast<uint4*>(sA + tc::kmajor_off(t, k, K)) = tc::pack8(f);
    }
  if (b_mn) {
    // MN-major: thread handles (k, 8 consecutive n) chunks
    for (int e = t; e < K * (N / 8); e += 128) {
      const int k = e / (N / 8), n0 = (e % (N / 8)) * 8;
      float f[8];
      for (int q = 0; q < 8; ++q) f[q] = B[(n0 + q) * K + k];
      *reinterpret_cast<uint4*>(sB + tc::mnmajor_off(n0, k, N)) = tc::pack8(f);
    }
  } else {
    for (int r = t; r < N; r += 128)
      for (int k = 0; k < K; k += 8) {
        float f[8];
        for (int q = 0; q < 8; ++q) f[q] = B[r * K + k + q];
        *reinterpret_cast<uint4*>(sB + tc::kmajor_off(r, k, K)) = tc::pack8(f);
      }
  }
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tbase = tmem_base;
  if (t == 0) {
    const uint32_t idesc = tc::idesc_bf16(128, N, b_mn);
    for (int kk = 0; kk < K / 16; ++kk) {
      const uint64_t ad = a_bcast ? tc::tile_desc_bcast(tc::smem_u32(sA), K, kk) : tc::tile_desc(tc::smem_u32(sA), K, kk);
      const uint64_t bd = b_mn ? tc::tile_desc_mn(tc::smem_u32(sB), N, kk) : tc::tile_desc(tc::smem_u32(sB), K, kk);
      tc::mma_bf16(tbase, ad, bd, idesc, kk > 0);
    }
    tc::mma_commit(&bar);
  }
  const bool ok = tc::mbar_wait(&bar, 0);
  if (!ok && (t & 31) == 0) atomicOr(err, 1);
  tc::fence_after();
  if (__syncthreads_and(ok)) {
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
extern "C" int nnpe_tc_selftest(int device, int mode, int N, int K, const float* A, const float* B, float* D) {
  if (N < 16 || N > 256 || N % 16 || K < 16 || K > 128 || K % 16 || !A || !B || !D || mode < 0 || mode > 3) return NNPE_EARG;
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
  k_tc_selftest<<<1, 128, smem>>>(dA, dB, dD, N, K, ncols, mode, derr);
  cudaError_t e = cudaDeviceSynchronize();
  int herr = 0;
  cudaMemcpy(D, dD, sizeof(float) * 128 * N, cudaMemcpyDeviceToHost);
  cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(dA); cudaFree(dB); cudaFree(dD); cudaFree(derr);
  if (e != cudaSuccess) return NNPE_ECUDA;
  return herr ? NNPE_ETIMEOUT : NNPE_OK;
}
