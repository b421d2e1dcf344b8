// BF16 tensor-core (tcgen05) path of the radial-embedding network.
//
// Three kernels per force evaluation, each issuing its GEMMs as tcgen05.mma from one thread with
// operands in shared memory (no-swizzle canonical layouts, see tc_util.cuh) and FP32 accumulators
// in tensor memory, read back row-per-thread for the epilogues. The two pair kernels walk a CTA's
// atoms as packed tiles of up to 128 pairs (one pair per MMA row / TMEM lane) holding at most two
// atom segments, and pipeline them: the first layer of the next tile is built while the tensor core
// runs the current one.
//
//  k_tc_desc2   first layer h1 = tanh(W1 u + b1) per pair into the A tile, block-diagonal over the
//               neighbour species, so one MMA chain gives every row the second layer of its own
//               net (b2 enters the same chain as a one-hot K slice); epilogue y = scale cff
//               tanh(z + b2) (BF16 pairs); the sum over pairs into G by
//               atom segment and special class is a second MMA with a one-hot A (no atomics); G is
//               stored as BF16 rows, the fitting kernel's operand type.
//  k_tc_fit     128 atoms of one species per tile (G rows fetched by cp.async straight into the
//               K-major A tile): G -> h1 -> h2 -> E forward and the hand-written
//               backward dE/dG = ((A3 (1-h2^2)) A2^T (1-h1^2)) A1^T as four MMA chains (N = 128, 128,
//               128, 256); activations stay in shared memory; the backward reads the forward's
//               weight images as MN-major (transposed) tiles.
//  k_tc_force2  second layer and its r-derivative per directed pair (two MMAs), the contraction with
//               the centre's dE/dG on the CUDA cores, and the pair force applied to both atoms in
//               64-bit fixed point (order-independent sums); k_facc_apply4 adds it to the forces.
//
// Every wait on an MMA-completion mbarrier is bounded; on time-out the kernel records
// NNPE_DEV_TIMEOUT, stops issuing work, frees its tensor memory and returns.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "nnp.cuh"
#include "tc_util.cuh"

struct NnpTc {
  unsigned long long* d_facc = nullptr;   // network forces and virial [natom][4], fixed point (2^-32)
  unsigned char* d_fit = nullptr;    // per species: L1 (N128,K256) and L2 (128,128) images
  size_t fit_stride = 0;
  float* d_emb_small = nullptr;      // per species: W1[32] b1[32] b2[64]
  float* d_fit_small = nullptr;      // per species: c1[128] c2[128] A3[128] c3 (stride 388)
  int* d_tile_sp = nullptr;          // fitting tiles: species, first row
  int* d_tile_row = nullptr;
  int ntiles = 0;
  int* d_soff = nullptr;
  int ctas_desc = 4, ctas_force = 2;   // CTAs per SM in the grid (shared and tensor memory bound)
  int grid_desc = 0, grid_force = 0;   // grid sizes chosen by the autotuner or the caller (0: default)
  unsigned char* d_wdesc64 = nullptr;  // B image N=64 x K=64: W2_t[q][c] at k=t*32+q (b2 added in the epilogue)
};

namespace {

constexpr int kFitSmallStride = 388;
constexpr size_t kImgL1 = 128 * 256 * 2, kImgL2 = 128 * 128 * 2;

__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Two FP32 values rounded to BF16 and packed (lo in the low half, as __floats2bfloat162_rn does).
__device__ __forceinline__ uint32_t pack_bf2(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
// (w0 u + b0, w1 u + b1) on the packed FP32 pipe, rounded to BF16 and packed.
__device__ __forceinline__ uint32_t pack_fma2(float w0, float w1, float2 u2, float b0, float b1) {
  const float2 v = __ffma2_rn(make_float2(w0, w1), u2, make_float2(b0, b1));
  return pack_bf2(v.x, v.y);
}
// tanh of two packed BF16 values (one transcendental-unit operation for both).
__device__ __forceinline__ uint32_t tanh_bf2(uint32_t x) {
  uint32_t y;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(y) : "r"(x));
  return y;
}
__device__ __forceinline__ uint32_t mul_bf2(uint32_t a, uint32_t b) {
  uint32_t y;
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(y) : "r"(a), "r"(b));
  return y;
}
__device__ __forceinline__ uint32_t fma_bf2(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

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

constexpr int kTile = 128;   // rows of an MMA tile (pairs)

constexpr float kFix = 4294967296.f;   // fixed-point scale of the network forces (2^-32)

// 64-bit fixed-point accumulation: integer additions give the same bits in any order.
__device__ __forceinline__ void fix_add(unsigned long long* dst, float v) {
  atomicAdd(dst, (unsigned long long)__float2ll_rn(v * kFix));
}

// -------------------------------------------------------------------------------------------
// Descriptor, pipelined over packed tiles.
//
// A CTA owns a contiguous range of atoms. Its pairs (per-atom counts n6) are cut into tiles of at most 128 rows holding at most two atom segments:
// the rest of atom a (la = 0) and, when that ends inside the tile, the start of atom a+1 (la = 1),
// so the 8-row one-hot reduction of the descriptor (rows 4 la + s) covers every tile. A
// segment that runs past the tile end is carried in shared memory to the next tile, and an atom's
// G is stored once, when its last segment is reduced, so no two CTAs or tiles write it.
//
// Per tile t the CTA's 128 threads (row p = thread p) run, in order:
//   (0) wait for MMA 2 of tile t-1 (its operand buffer and TMEM buffer become free),
//   (1) all warps: G of tile t-1 out of TMEM[(t-1) % 2] (16 channels each); first layer of tile t+1 into operand
//       buffer A[(t+1) % 2], loads of tile t+2 issued,
//   (2) barrier, after which MMA 1 of tile t is complete,
//   (3) MMA 1 of tile t+1 into TMEM[(t+1) % 2] (Z = H W2s, K = 64 block-diagonal over the neighbour
//       species; b2 is added in the epilogue),
//   (4) epilogue of tile t: y = scale cff tanh(z) -> Y (BF16, MN-major) over A[t % 2], and the
//       one-hot S of the (la, s) rows,
//   (5) barrier; MMA 2 of tile t: TMEM[t % 2] = S Y.
// MMA 1 of tile t+1 runs during the epilogue of tile t and MMA 2 of tile t during the next
// iteration's wait; two operand and two TMEM buffers keep every buffer out of reach of the MMA that
// reads it, and four CTAs per SM overlap each other's waits. The activations are BF16 operands of the next MMA, so their tanh is evaluated on
// BF16 pairs (one transcendental-unit operation per two values).
constexpr int kK64 = 64;
constexpr int kEmbStride4 = 148;   // 16-byte aligned rows of the per-species constants: W1[32] b1[32] b2[64], 4 unused, WR[16]
constexpr int kWrOff = 132;        // WR: w/rc of the first layer as BF16 pairs (the force kernel's r-derivative)
constexpr int kDescStages = 2;
// The second layer's bias b2 enters MMA 1 as a fifth K=16 slice: A = the row's one-hot species
// (column tj of a [128 x 16] tile whose columns 8..15 stay zero), B = b2 of each species (BF16), so
// Z = H W2 + b2 leaves TMEM with the bias already added.
constexpr int kWImg = 64 * kK64 * 2;            // B of MMA 1: [W2_0; W2_1], N = 64 x K = 64
constexpr int kWBiasImg = 64 * 16 * 2;          // B of the bias slice: N = 64 x K = 16, column s = b2 of species s
constexpr int kBiasA = kTile * 16 * 2;          // A of the bias slice, one per operand stage
__device__ __forceinline__ uint32_t bias_a_off(int p) { return tc::kmajor_off(p, 0, 16); }
// one-hot row chunk (k = 0..7) of species tj in BF16
__device__ __forceinline__ uint4 onehot8(int tj) {
  uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int k = 0; k < 4; ++k) w[k] = (tj == 2 * k ? 0x3F80u : 0u) | (tj == 2 * k + 1 ? 0x3F800000u : 0u);
  return make_uint4(w[0], w[1], w[2], w[3]);
}
constexpr int kSmemDesc2 = kWImg + kWBiasImg + kDescStages * kTile * kK64 * 2 + 8 * kTile * 2 + kDescStages * kBiasA +
                           2 * kEmbStride4 * 4 + 256 * 4;

struct DescArgs {
  const float4* pos;
  const uint32_t* list6;
  const int* n6;
  const int* gowner;
  const unsigned char* wdesc;   // B of MMA 1: N = 64 channels x K = 64, [W2_0; W2_1]; then the bias slice's B
  const float* emb_small;       // per species W1[32] b1[32] b2[64] (stride 128)
  uint32_t* G2;                 // descriptor rows [N][256] BF16, two per word (the fitting kernel's operand)
  int* ctrl;
  int cap6, N, ntype, npos;
  float rc, scale, r_rc;   // r_rc = 1/rc
};

struct TileSeg { int a, k0, na, nb; };

// Next tile of the CTA's range from cursor (a, k0); atoms without pairs are skipped (and get G = 0
// here when G2 is given).
__device__ __forceinline__ bool next_tile_n6(const int* n6, uint32_t* G2, int& a, int& k0, int i1, TileSeg& s, int t, int nt) {
  while (a < i1 && __ldg(n6 + a) == 0) {
    if (G2)
      for (int e = t; e < 128; e += nt) G2[(size_t)a * 128 + e] = 0u;
    ++a;
    k0 = 0;
  }
  if (a >= i1) return false;
  const int rem = __ldg(n6 + a) - k0;
  s.a = a; s.k0 = k0; s.na = min(rem, kTile); s.nb = 0;
  if (s.na == rem) {
    const int b = a + 1;
    const int nbt = b < i1 ? __ldg(n6 + b) : 0;
    if (s.na < kTile && nbt > 0) {
      s.nb = min(nbt, kTile - s.na);
      if (s.nb == nbt) { a = b + 1; k0 = 0; } else { a = b; k0 = s.nb; }
    } else {
      a += 1; k0 = 0;
    }
  } else {
    k0 += s.na;
  }
  return true;
}
__device__ __forceinline__ bool next_tile(const DescArgs& d, int& a, int& k0, int i1, TileSeg& s, int t) {
  return next_tile_n6(d.n6, d.G2, a, k0, i1, s, t, 128);
}

// Row p of a tile: its atom, la, list entry and the two positions (loaded ahead of use).
struct RowFetch {
  int atom, la, jo;
  bool valid;
  uint32_t ent;
  float4 xi, xj;
};
__device__ __forceinline__ void fetch_entry(const DescArgs& d, const TileSeg& s, bool have, int p, RowFetch& f) {
  f.valid = have && p < s.na + s.nb;
  f.la = p < s.na ? 0 : 1;
  f.atom = f.la ? s.a + 1 : s.a;
  f.ent = 0;
  if (f.valid) {
    const int slot = f.la ? p - s.na : s.k0 + p;
    f.ent = __ldg(d.list6 + (size_t)f.atom * d.cap6 + slot);
    f.xi = __ldg(d.pos + f.atom);
  }
}
__device__ __forceinline__ void fetch_xj(const DescArgs& d, RowFetch& f, bool owner = false) {
  f.jo = 0;
  if (f.valid) {
    const int j = f.ent & NNPE_J_MASK;
    f.xj = __ldg(d.pos + (j < d.npos ? j : 0));
    if (owner) f.jo = j < d.N ? j : __ldg(d.gowner + (j - d.N < d.npos - d.N ? j - d.N : 0));
  }
}

struct DescRow {
  float cs;     // scale * cff(r), 0 for rows past the tile's pairs
  int tj, s, la;
  bool valid;
};

// First layer of one row into A (block of species tj, zeros in the other block); returns the
// row's epilogue data.
__device__ __forceinline__ DescRow desc_first_layer(const DescArgs& d, const RowFetch& f, const float* sE,
                                                    unsigned char* A, unsigned char* AB, int p) {
  DescRow r;
  r.valid = f.valid; r.cs = 0.f; r.tj = 0; r.s = 0; r.la = f.la;
  if (!f.valid) return r;
  const float dx = f.xi.x - f.xj.x, dy = f.xi.y - f.xj.y, dz = f.xi.z - f.xj.z;
  // approximate square root and reciprocal (the hardware rsqrt / rcp units): a few ulp, far below
  // the BF16 rounding of the operands they feed; cff = 1 - 1/(1+cf^2) = cf^2/(1+cf^2)
  const float rsq = dx * dx + dy * dy + dz * dz;
  const float rr = rsq * rsqrtf(rsq);
  const float cf = rr - d.rc;
  r.cs = d.scale * __fdividef(cf * cf, 1.f + cf * cf);
  r.s = f.ent >> 30;
  r.tj = (f.ent >> 27) & 7;
  const float u = rr * d.r_rc;
  const float2 u2 = make_float2(u, u);
  *reinterpret_cast<uint4*>(AB + bias_a_off(p)) = onehot8(r.tj);
  const float4* W1 = reinterpret_cast<const float4*>(sE + r.tj * kEmbStride4);
  const float4* B1 = reinterpret_cast<const float4*>(sE + r.tj * kEmbStride4 + 32);
#pragma unroll
  for (int g = 0; g < 4; ++g) {   // 8 units per 16-byte chunk, tanh on BF16 pairs (h is a BF16 operand)
    const float4 w0 = W1[2 * g], w1 = W1[2 * g + 1], b0 = B1[2 * g], b1 = B1[2 * g + 1];
    uint4 h;
    h.x = tanh_bf2(pack_fma2(w0.x, w0.y, u2, b0.x, b0.y));
    h.y = tanh_bf2(pack_fma2(w0.z, w0.w, u2, b0.z, b0.w));
    h.z = tanh_bf2(pack_fma2(w1.x, w1.y, u2, b1.x, b1.y));
    h.w = tanh_bf2(pack_fma2(w1.z, w1.w, u2, b1.z, b1.w));
    *reinterpret_cast<uint4*>(A + tc::kmajor_off(p, 32 * r.tj + 8 * g, kK64)) = h;
    *reinterpret_cast<uint4*>(A + tc::kmajor_off(p, 32 * (1 - r.tj) + 8 * g, kK64)) = make_uint4(0, 0, 0, 0);
  }
  return r;
}

// Channels [c0, c0 + 16) of the G rows (la, s) = lanes 4 la + s of this warp's quarter of the MMA 2
// accumulator (S repeats every 8 rows, so every quarter holds them) at taddr, added to the carried
// partial of a segment that began in an earlier tile; stored when the atom's last pair was in this
// tile, else carried. Each of the CTA's four warps takes one 16-channel slice.
__device__ __forceinline__ void desc_readout(const DescArgs& d, uint32_t taddr, const TileSeg& sg, float* sCarry, int lane,
                                             int c0) {
  float g[16];
  tc::tmem_ld16(taddr, g);
  const int la = lane >> 2, sc = lane & 3;
  const bool mine = lane < 8 && (la == 0 || sg.nb > 0);
  const int atom = sg.a + la;
  const int nrow = la ? sg.nb : sg.na, start = la ? 0 : sg.k0;
  const bool done = mine && start + nrow == __ldg(d.n6 + atom);
  if (mine && la == 0 && start > 0) {
#pragma unroll
    for (int c = 0; c < 16; ++c) g[c] += sCarry[sc * 64 + c0 + c];
  }
  __syncwarp();
  if (mine) {
    if (done) {   // BF16 (round to nearest), the rounding the fitting kernel's operand takes
      uint4* dst = reinterpret_cast<uint4*>(d.G2 + (size_t)atom * 128 + sc * 32 + c0 / 2);
      dst[0] = tc::pack8(g);
      dst[1] = tc::pack8(g + 8);
    } else {
#pragma unroll
      for (int c = 0; c < 16; ++c) sCarry[sc * 64 + c0 + c] = g[c];
    }
  }
  __syncwarp();
}

__global__ void __launch_bounds__(128, 4) k_tc_desc2(DescArgs d) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t bar_z[2], bar_g;
  __shared__ uint32_t tmem_base;
  __shared__ int s_range[2];
  unsigned char* sW = sm;                                       // B of MMA 1 (64 x 64), then the bias slice's B
  unsigned char* sA = sW + kWImg + kWBiasImg;                   // 2 x [128 x 64]: H of MMA 1, then Y of MMA 2
  unsigned char* sS = sA + kDescStages * kTile * kK64 * 2;      // A of MMA 2 (8 x 128, MN-major)
  unsigned char* sAB = sS + 8 * kTile * 2;                      // 2 x [128 x 16]: A of the bias slice
  float* sE = reinterpret_cast<float*>(sAB + kDescStages * kBiasA);   // per species W1 b1 b2 (stride 148)
  float* sCarry = sE + 2 * kEmbStride4;                         // partial G of a segment cut by a tile end
  const int t = threadIdx.x, w = t >> 5, lane = t & 31, p = t;
  if (w == 0) tc::tmem_alloc(&tmem_base, 128);
  if (t == 0) {
    tc::mbar_init(&bar_z[0], 1);
    tc::mbar_init(&bar_z[1], 1);
    tc::mbar_init(&bar_g, 1);
    // atom range of this CTA (equal atom counts; the tiles below adapt to the pair counts)
    int r[2];
    for (int e = 0; e < 2; ++e) r[e] = (int)((long long)d.N * (blockIdx.x + e) / gridDim.x);
    s_range[0] = r[0];
    s_range[1] = r[1];
  }
  copy_image(sW, d.wdesc, kWImg + kWBiasImg, t, 128);
  // operand stages and bias slices start zeroed (rows past a tile's pairs must read finite values)
  for (int k = t; k < kDescStages * kTile * kK64 * 2 / 16; k += 128) reinterpret_cast<uint4*>(sA)[k] = make_uint4(0, 0, 0, 0);
  for (int k = t; k < kDescStages * kBiasA / 16; k += 128) reinterpret_cast<uint4*>(sAB)[k] = make_uint4(0, 0, 0, 0);
  for (int k = t; k < 2 * 128; k += 128) sE[(k >> 7) * kEmbStride4 + (k & 127)] = (k >> 7) < d.ntype ? d.emb_small[k] : 0.f;
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t lane_off = (uint32_t)(w * 32) << 16;
  const uint32_t aW = tc::smem_u32(sW), aS = tc::smem_u32(sS), aWB = aW + kWImg, aAB = tc::smem_u32(sAB);
  const int i1 = s_range[1];
  int ca = s_range[0], ck0 = 0;
  uint32_t ph_z[2] = {0, 0}, ph_g = 0;
  bool alive = true;

  // prologue: tile 0 built, its MMA 1 issued; tile 1 fetched
  TileSeg seg0{0, 0, 0, 0}, seg1{0, 0, 0, 0}, seg2{0, 0, 0, 0}, segp{0, 0, 0, 0};
  bool have0 = next_tile(d, ca, ck0, i1, seg0, t);
  RowFetch f0, f1, f2;
  fetch_entry(d, seg0, have0, p, f0);
  fetch_xj(d, f0);
  bool have1 = have0 && next_tile(d, ca, ck0, i1, seg1, t);
  fetch_entry(d, seg1, have1, p, f1);
  DescRow row0 = desc_first_layer(d, f0, sE, sA, sAB, p);
  fetch_xj(d, f1);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (have0 && t == 0) {
    const uint32_t id = tc::idesc_bf16(128, 64);
    for (int kk = 0; kk < kK64 / 16; ++kk) tc::mma_bf16(tmem, tc::tile_desc(tc::smem_u32(sA), kK64, kk), tc::tile_desc(aW, kK64, kk), id, kk > 0);
    tc::mma_bf16(tmem, tc::tile_desc(aAB, 16, 0), tc::tile_desc(aWB, 16, 0), id, 1);
    tc::mma_commit(&bar_z[0]);
  }
  bool havep = false;
  int last_buf = 0;
  DescRow row1 = row0;
  for (int it = 0; have0 && alive; ++it) {
    const int b0 = it & 1, b1 = b0 ^ 1;
    unsigned char* A0 = sA + (size_t)b0 * kTile * kK64 * 2;
    unsigned char* A1 = sA + (size_t)b1 * kTile * kK64 * 2;
    // (0) MMA 2 of tile it-1 complete: A[b1] (its Y) free, its G ready in TMEM[b1]
    if (havep) {
      alive = cta_wait_mma(&bar_g, ph_g, d.ctrl);
      ph_g ^= 1;
      if (!alive) break;
    }
    // (1) all warps: G of tile it-1 (16 channels each), first layer of tile it+1 into A[b1], loads of tile it+2
    if (havep) desc_readout(d, tmem + 64 * b1 + lane_off + 16 * w, segp, sCarry, lane, 16 * w);
    bool have2 = false;
    seg2 = TileSeg{0, 0, 0, 0};
    if (have1) {
      row1 = desc_first_layer(d, f1, sE, A1, sAB + b1 * kBiasA, p);
      have2 = next_tile(d, ca, ck0, i1, seg2, t);
    }
    fetch_entry(d, seg2, have2, p, f2);
    // (2) barrier: A[b1] written, TMEM[b1] read out, MMA 1 of tile it complete
    tc::fence_async_smem();
    tc::fence_before();
    {
      bool ok = true;
      if (t == 0) {
        ok = tc::mbar_wait(&bar_z[b0], ph_z[b0]);
        if (!ok) atomicOr(d.ctrl + CTRL_ERR, NNPE_DEV_TIMEOUT);
      }
      alive = __syncthreads_and(ok) != 0;
    }
    tc::fence_after();
    ph_z[b0] ^= 1;
    if (!alive) break;
    // (3) MMA 1 of tile it+1 into TMEM[b1]
    if (have1 && t == 0) {
      const uint32_t id = tc::idesc_bf16(128, 64);
      const uint32_t aA = tc::smem_u32(A1);
      for (int kk = 0; kk < kK64 / 16; ++kk) tc::mma_bf16(tmem + 64 * b1, tc::tile_desc(aA, kK64, kk), tc::tile_desc(aW, kK64, kk), id, kk > 0);
      tc::mma_bf16(tmem + 64 * b1, tc::tile_desc(aAB + b1 * kBiasA, 16, 0), tc::tile_desc(aWB, 16, 0), id, 1);
      tc::mma_commit(&bar_z[b1]);
    }
    // (4) epilogue of tile it: y = scale cff tanh(z) (z includes b2), on BF16 pairs (Y is a BF16 operand)
    const int nrows = seg0.na + seg0.nb, NK = (nrows + 15) & ~15;
    if (32 * w < NK) {   // warp-uniform
      const float csv = row0.valid ? row0.cs : 0.f;
      const uint32_t cs2 = pack_bf2(csv, csv);
#pragma unroll
      for (int c0 = 0; c0 < 64; c0 += 32) {
        float z[32];
        tc::tmem_ld16x2(tmem + 64 * b0 + lane_off + c0, tmem + 64 * b0 + lane_off + c0 + 16, z, z + 16);
        uint32_t y[16];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          y[2 * q] = mul_bf2(tanh_bf2(pack_bf2(z[4 * q], z[4 * q + 1])), cs2);
          y[2 * q + 1] = mul_bf2(tanh_bf2(pack_bf2(z[4 * q + 2], z[4 * q + 3])), cs2);
        }
        // Rows past the tile's pairs carry y = 0 (cs = 0) and a zero S column. Their Z is finite:
        // the operand stages start zeroed and afterwards hold earlier tiles' first layers, so
        // 0 x Y adds exact zeros to G.
        if (p < NK) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            *reinterpret_cast<uint4*>(A0 + tc::mnmajor_off(c0 + 8 * q, p, 64)) = make_uint4(y[4 * q], y[4 * q + 1], y[4 * q + 2], y[4 * q + 3]);
        }
      }
      // S is held MN-major (row p of the pair dimension = 8 contiguous classes (la, s)): one 16-byte
      // one-hot per row
      if (p < NK) *reinterpret_cast<uint4*>(sS + 16 * p) = onehot8(row0.valid ? 4 * row0.la + row0.s : 8);
    }
    fetch_xj(d, f2);
    // (5) MMA 2 of tile it
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (t == 0) {
      const uint32_t id = tc::idesc_bf16(128, 64, true, true);
      const uint32_t aY = tc::smem_u32(A0);
      for (int kk = 0; kk < NK / 16; ++kk)
        tc::mma_bf16(tmem + 64 * b0, tc::tile_desc_bcast_mn(aS, kk), tc::tile_desc_mn(aY, 64, kk), id, kk > 0);
      tc::mma_commit(&bar_g);
    }
    segp = seg0; havep = true; last_buf = b0;
    seg0 = seg1; have0 = have1; row0 = row1;
    seg1 = seg2; have1 = have2; f1 = f2;
  }
  // G of the last tile
  if (havep && alive) {
    alive = cta_wait_mma(&bar_g, ph_g, d.ctrl);
    if (alive) desc_readout(d, tmem + 64 * last_buf + lane_off + 16 * w, segp, sCarry, lane, 16 * w);
  }
  tc::fence_before();
  __syncthreads();
  if (w == 0) tc::tmem_dealloc(tmem, 128);
}

// -------------------------------------------------------------------------------------------
// Force, pipelined over the packed tiles of the descriptor kernel (up to two atom segments per
// tile). 256 threads: row p = t % 128, half h = t / 128 takes hidden units [16h, 16h+16) of the
// first layer and channels [32h, 32h+32) of the epilogue (warps w and w+4 read the same TMEM
// lanes). Per tile t:
//   (1) first layer of tile t+1: H and V = dH/dr into A stage (t+1) % 2, dE/dG of its atoms into
//       shared memory; loads of tile t+2 issued,
//   (2) barrier, after which MMA of tile t is complete,
//   (3) MMA of tile t+1: Z = H W2s and K = V W2s into TMEM stage (t+1) % 2 (128 columns),
//   (4) epilogue of tile t: each half's share of T = scale (dcff sum_c a_c y_c + cff sum_c a_c
//       kappa_c (1 - y_c^2)), y = tanh(z + b2) (b2 added by the H MMA's bias slice), a = dE/dG_i[s*64 + c],
//   (5) barrier; half 0: fpair = -T/r applied to j's owner (64-bit fixed-point atomics) and summed
//       per atom segment over each warp (one atomic per segment and warp) for i; the virial the same.
constexpr int kSmemForce2 = kWImg + kWBiasImg + 2 * 2 * kTile * kK64 * 2 + 2 * kBiasA + 2 * 2 * 256 * 4 + 2 * kEmbStride4 * 4 +
                            2 * kTile * 4;

struct ForceArgs {
  const float4* pos;
  const uint32_t* list6;
  const int* n6;
  const int* gowner;
  const unsigned char* wdesc;
  const float* emb_small;
  const float* dG;
  unsigned long long* facc;   // [N][4]: force x, y, z and virial, fixed point (2^-32)
  int* ctrl;
  int cap6, N, ntype, npos;
  float rc, scale, r_rc;   // r_rc = 1/rc
};

struct ForceRow {
  float dx, dy, dz, rinv, rsq, cff, dcff;
  int s, tj, la, jo;
  bool valid;
};

__device__ __forceinline__ ForceRow force_first_layer(const ForceArgs& a, const RowFetch& f, const float* sE,
                                                      unsigned char* AH, unsigned char* AV, unsigned char* AB, int p,
                                                      int half) {
  ForceRow r;
  r.valid = f.valid; r.la = f.la; r.s = 0; r.tj = 0; r.jo = 0;
  r.dx = r.dy = r.dz = 0.f; r.rinv = 1.f; r.rsq = 1.f; r.cff = 0.f; r.dcff = 0.f;
  if (!f.valid) return r;
  r.dx = f.xi.x - f.xj.x; r.dy = f.xi.y - f.xj.y; r.dz = f.xi.z - f.xj.z;
  r.rsq = r.dx * r.dx + r.dy * r.dy + r.dz * r.dz;
  // approximate rsqrt / rcp (a few ulp, below the BF16 rounding of the operands they feed);
  // cff = cf^2/(1+cf^2), dcff = 2 cf/(1+cf^2)^2
  r.rinv = rsqrtf(r.rsq);
  const float rr = r.rsq * r.rinv;
  const float cf = rr - a.rc, rd = __fdividef(1.f, 1.f + cf * cf);
  r.cff = cf * cf * rd;
  r.dcff = 2.f * cf * rd * rd;
  r.s = f.ent >> 30;
  r.tj = (f.ent >> 27) & 7;
  r.jo = f.jo;
  const float u = rr * a.r_rc;
  const float2 u2 = make_float2(u, u);
  if (half == 0) *reinterpret_cast<uint4*>(AB + bias_a_off(p)) = onehot8(r.tj);   // b2 enters the H MMA only
  const float4* W1 = reinterpret_cast<const float4*>(sE + r.tj * kEmbStride4);
  const float4* B1 = reinterpret_cast<const float4*>(sE + r.tj * kEmbStride4 + 32);
  const uint4* WR = reinterpret_cast<const uint4*>(sE + r.tj * kEmbStride4 + kWrOff);
  const uint32_t one2 = 0x3F803F80u;   // (1, 1) in BF16
#pragma unroll
  for (int gg = 0; gg < 2; ++gg) {
    const int g = 2 * half + gg;   // 8-unit chunk
    const float4 w0 = W1[2 * g], w1 = W1[2 * g + 1], b0 = B1[2 * g], b1 = B1[2 * g + 1];
    // h on BF16 pairs (it is a BF16 operand), and V = (1 - h^2) w / rc from it on BF16 pairs: one
    // transcendental-unit operation per two units, the derivative without conversions
    uint4 h, v;
    h.x = tanh_bf2(pack_fma2(w0.x, w0.y, u2, b0.x, b0.y));
    h.y = tanh_bf2(pack_fma2(w0.z, w0.w, u2, b0.z, b0.w));
    h.z = tanh_bf2(pack_fma2(w1.x, w1.y, u2, b1.x, b1.y));
    h.w = tanh_bf2(pack_fma2(w1.z, w1.w, u2, b1.z, b1.w));
    const uint4 wr = WR[g];
    v.x = mul_bf2(fma_bf2(h.x ^ 0x80008000u, h.x, one2), wr.x);
    v.y = mul_bf2(fma_bf2(h.y ^ 0x80008000u, h.y, one2), wr.y);
    v.z = mul_bf2(fma_bf2(h.z ^ 0x80008000u, h.z, one2), wr.z);
    v.w = mul_bf2(fma_bf2(h.w ^ 0x80008000u, h.w, one2), wr.w);
    *reinterpret_cast<uint4*>(AH + tc::kmajor_off(p, 32 * r.tj + 8 * g, kK64)) = h;
    *reinterpret_cast<uint4*>(AV + tc::kmajor_off(p, 32 * r.tj + 8 * g, kK64)) = v;
    *reinterpret_cast<uint4*>(AH + tc::kmajor_off(p, 32 * (1 - r.tj) + 8 * g, kK64)) = make_uint4(0, 0, 0, 0);
    *reinterpret_cast<uint4*>(AV + tc::kmajor_off(p, 32 * (1 - r.tj) + 8 * g, kK64)) = make_uint4(0, 0, 0, 0);
  }
  return r;
}

// dE/dG of the tile's atoms (1 or 2): two values per thread, loaded a tile ahead into registers and
// stored into sdG[2][256] when the tile is built.
__device__ __forceinline__ float2 fetch_tile_dG(const ForceArgs& a, const TileSeg& sg, bool have, int t) {
  float2 v = make_float2(0.f, 0.f);
  if (!have) return v;
  v.x = __ldg(a.dG + (size_t)sg.a * 256 + t);   // k = t: atom 0, column t (t < 256)
  if (sg.nb > 0) v.y = __ldg(a.dG + (size_t)(sg.a + 1) * 256 + t);
  return v;
}
__device__ __forceinline__ void store_tile_dG(float2 v, float* sdG, int t) {
  sdG[t] = v.x;
  sdG[256 + t] = v.y;
}

__device__ __forceinline__ float seg_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <bool EV>
__global__ void __launch_bounds__(256, 2) k_tc_force2(ForceArgs a) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t bar[2];
  __shared__ uint32_t tmem_base;
  unsigned char* sW = sm;                                          // 64 x 64, then the bias slice's B
  unsigned char* sAH = sW + kWImg + kWBiasImg;                     // 2 stages x [H | V], 32 KB each
  unsigned char* sAB = sAH + 2 * 2 * kTile * kK64 * 2;             // 2 stages x [128 x 16]: A of the bias slice
  float* sdG = reinterpret_cast<float*>(sAB + 2 * kBiasA);         // 2 stages x [2][256]
  float* sE = sdG + 2 * 512;
  float* sAcc = sE + 2 * kEmbStride4;                              // [2][128] per-half partial T
  const int t = threadIdx.x, w = t >> 5, lane = t & 31, p = t & 127, half = t >> 7;
  if (w == 0) tc::tmem_alloc(&tmem_base, 256);
  if (t == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
  }
  copy_image(sW, a.wdesc, kWImg + kWBiasImg, t, 256);
  for (int k = t; k < 2 * kBiasA / 16; k += 256) reinterpret_cast<uint4*>(sAB)[k] = make_uint4(0, 0, 0, 0);
  for (int k = t; k < 2 * 128; k += 256) sE[(k >> 7) * kEmbStride4 + (k & 127)] = (k >> 7) < a.ntype ? a.emb_small[k] : 0.f;
  for (int k = t; k < 2 * 16; k += 256) {
    const int sp = k >> 4, q = k & 15;
    const float r_rc = a.r_rc;
    const float w0 = sp < a.ntype ? a.emb_small[sp * 128 + 2 * q] : 0.f, w1 = sp < a.ntype ? a.emb_small[sp * 128 + 2 * q + 1] : 0.f;
    reinterpret_cast<uint32_t*>(sE)[sp * kEmbStride4 + kWrOff + q] = pack_bf2(w0 * r_rc, w1 * r_rc);
  }
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t lane_off = (uint32_t)((w & 3) * 32) << 16;
  const uint32_t aW = tc::smem_u32(sW), aWB = aW + kWImg, aAB = tc::smem_u32(sAB);
  const int i0 = (int)((long long)a.N * blockIdx.x / gridDim.x), i1 = (int)((long long)a.N * (blockIdx.x + 1) / gridDim.x);
  int ca = i0, ck0 = 0;
  uint32_t ph[2] = {0, 0};
  bool alive = true;
  // RowFetch reads list6/pos through a DescArgs view of the same arrays
  DescArgs dv;
  dv.pos = a.pos; dv.list6 = a.list6; dv.n6 = a.n6; dv.gowner = a.gowner; dv.cap6 = a.cap6; dv.N = a.N; dv.npos = a.npos;
  TileSeg seg0{0, 0, 0, 0}, seg1{0, 0, 0, 0}, seg2{0, 0, 0, 0};
  RowFetch f0, f1, f2;
  bool have0 = next_tile_n6(a.n6, nullptr, ca, ck0, i1, seg0, t, 256);
  fetch_entry(dv, seg0, have0, p, f0);
  fetch_xj(dv, f0, true);
  const float2 g0 = fetch_tile_dG(a, seg0, have0, t);
  bool have1 = have0 && next_tile_n6(a.n6, nullptr, ca, ck0, i1, seg1, t, 256);
  fetch_entry(dv, seg1, have1, p, f1);
  float2 g1 = fetch_tile_dG(a, seg1, have1, t);
  ForceRow row0 = force_first_layer(a, f0, sE, sAH, sAH + kTile * kK64 * 2, sAB, p, half);
  if (have0) store_tile_dG(g0, sdG, t);
  fetch_xj(dv, f1, true);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (have0 && t == 0) {
    const uint32_t id = tc::idesc_bf16(128, 64);
    const uint32_t aH = tc::smem_u32(sAH), aV = aH + kTile * kK64 * 2;
    for (int kk = 0; kk < kK64 / 16; ++kk) tc::mma_bf16(tmem, tc::tile_desc(aH, kK64, kk), tc::tile_desc(aW, kK64, kk), id, kk > 0);
    tc::mma_bf16(tmem, tc::tile_desc(aAB, 16, 0), tc::tile_desc(aWB, 16, 0), id, 1);
    for (int kk = 0; kk < kK64 / 16; ++kk) tc::mma_bf16(tmem + 64, tc::tile_desc(aV, kK64, kk), tc::tile_desc(aW, kK64, kk), id, kk > 0);
    tc::mma_commit(&bar[0]);
  }
  ForceRow row1 = row0;
  for (int it = 0; have0 && alive; ++it) {
    const int b0 = it & 1, b1 = b0 ^ 1;
    unsigned char* AH1 = sAH + (size_t)b1 * 2 * kTile * kK64 * 2;
    // (1) first layer and dE/dG of tile it+1; loads of tile it+2
    bool have2 = false;
    seg2 = TileSeg{0, 0, 0, 0};
    float2 g2 = make_float2(0.f, 0.f);
    if (have1) {
      row1 = force_first_layer(a, f1, sE, AH1, AH1 + kTile * kK64 * 2, sAB + b1 * kBiasA, p, half);
      store_tile_dG(g1, sdG + 512 * b1, t);
      have2 = next_tile_n6(a.n6, nullptr, ca, ck0, i1, seg2, t, 256);
    }
    fetch_entry(dv, seg2, have2, p, f2);
    g2 = fetch_tile_dG(a, seg2, have2, t);
    // (2) barrier: MMA of tile it complete, stage it+1 written
    tc::fence_async_smem();
    tc::fence_before();
    {
      bool ok = true;
      if (t == 0) {
        ok = tc::mbar_wait(&bar[b0], ph[b0]);
        if (!ok) atomicOr(a.ctrl + CTRL_ERR, NNPE_DEV_TIMEOUT);
      }
      alive = __syncthreads_and(ok) != 0;
    }
    tc::fence_after();
    ph[b0] ^= 1;
    if (!alive) break;
    // (3) MMA of tile it+1
    if (have1 && t == 0) {
      const uint32_t id = tc::idesc_bf16(128, 64);
      const uint32_t aH = tc::smem_u32(AH1), aV = aH + kTile * kK64 * 2;
      const uint32_t td = tmem + 128 * b1;
      for (int kk = 0; kk < kK64 / 16; ++kk) tc::mma_bf16(td, tc::tile_desc(aH, kK64, kk), tc::tile_desc(aW, kK64, kk), id, kk > 0);
      tc::mma_bf16(td, tc::tile_desc(aAB + b1 * kBiasA, 16, 0), tc::tile_desc(aWB, 16, 0), id, 1);
      for (int kk = 0; kk < kK64 / 16; ++kk) tc::mma_bf16(td + 64, tc::tile_desc(aV, kK64, kk), tc::tile_desc(aW, kK64, kk), id, kk > 0);
      tc::mma_commit(&bar[b1]);
    }
    // (4) epilogue of tile it: this half's share of T
    const int nrows = seg0.na + seg0.nb;
    float part = 0.f;
    if (32 * (w & 3) < nrows) {   // warp-uniform: the loads below are warp-collective
      const float* ag = sdG + 512 * b0 + row0.la * 256 + row0.s * 64 + 32 * half;
      // channel pairs on the packed FP32 pipe (two lanes of arithmetic per instruction)
      float2 sy2 = make_float2(0.f, 0.f), sk2 = make_float2(0.f, 0.f);
      const float2 one2f = make_float2(1.f, 1.f);
#pragma unroll
      for (int c0 = 0; c0 < 32; c0 += 16) {
        float z[16], kap[16];
        tc::tmem_ld16x2(tmem + 128 * b0 + lane_off + 32 * half + c0, tmem + 128 * b0 + lane_off + 64 + 32 * half + c0, z, kap);
#pragma unroll
        for (int q = 0; q < 16; q += 4) {
          const float4 a4 = *reinterpret_cast<const float4*>(ag + c0 + q);
          const float2 av[2] = {make_float2(a4.x, a4.y), make_float2(a4.z, a4.w)};
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const float2 y = make_float2(tanh_fast(z[q + 2 * e]), tanh_fast(z[q + 2 * e + 1]));   // z includes b2
            sy2 = __ffma2_rn(av[e], y, sy2);
            const float2 u = __ffma2_rn(make_float2(-y.x, -y.y), y, one2f);
            sk2 = __ffma2_rn(__fmul2_rn(av[e], make_float2(kap[q + 2 * e], kap[q + 2 * e + 1])), u, sk2);
          }
        }
      }
      if (row0.valid) part = a.scale * (row0.dcff * (sy2.x + sy2.y) + row0.cff * (sk2.x + sk2.y));
    }
    sAcc[half * kTile + p] = part;
    fetch_xj(dv, f2, true);
    __syncthreads();
    // (5) both halves form the row's pair force: half 0 applies it to j's owner, half 1 sums it per
    // atom segment for the atoms of the tile
    {
      float gx = 0.f, gy = 0.f, gz = 0.f, vr = 0.f;
      if (row0.valid) {
        const float fpair = -(sAcc[p] + sAcc[kTile + p]) * row0.rinv;
        gx = row0.dx * fpair; gy = row0.dy * fpair; gz = row0.dz * fpair;
        if (EV) vr = fpair * row0.rsq;
      }
      if (half == 0) {
        if (row0.valid) {
          unsigned long long* fj = a.facc + 4 * (size_t)row0.jo;
          fix_add(fj, -gx); fix_add(fj + 1, -gy); fix_add(fj + 2, -gz);
        }
      } else {
      const unsigned in0 = __ballot_sync(0xffffffffu, row0.valid && row0.la == 0);
      const unsigned in1 = __ballot_sync(0xffffffffu, row0.valid && row0.la == 1);
#pragma unroll
      for (int sgm = 0; sgm < 2; ++sgm) {
        const unsigned in = sgm ? in1 : in0;
        if (!in) continue;   // warp-uniform
        const bool mine = row0.valid && row0.la == sgm;
        const float sx = seg_sum(mine ? gx : 0.f), sy2 = seg_sum(mine ? gy : 0.f), sz = seg_sum(mine ? gz : 0.f);
        const float sv = EV ? seg_sum(mine ? vr : 0.f) : 0.f;
        if (lane == 0) {
          unsigned long long* fi = a.facc + 4 * (size_t)(seg0.a + sgm);
          fix_add(fi, sx); fix_add(fi + 1, sy2); fix_add(fi + 2, sz);
          if (EV) fix_add(fi + 3, sv);
        }
      }
      }
    }
    seg0 = seg1; have0 = have1; row0 = row1;
    seg1 = seg2; have1 = have2; f1 = f2; g1 = g2;
  }
  tc::fence_before();
  __syncthreads();
  if (w == 0) tc::tmem_dealloc(tmem, 256);
}

// frc[i] += network force of atom i, watom[i] += its virial (EV), from the [N][4] fixed-point sums,
// which are left zeroed for the next force kernel (the buffer starts zeroed at set-up).
template <bool EV>
__global__ void k_facc_apply4(unsigned long long* __restrict__ facc, float4* __restrict__ frc, double* watom, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double s = 1.0 / kFix;
  ulonglong2* q = reinterpret_cast<ulonglong2*>(facc + 4 * (size_t)i);
  const ulonglong2 a = q[0], b = q[1];
  q[0] = make_ulonglong2(0ull, 0ull);
  q[1] = make_ulonglong2(0ull, 0ull);
  float4 f = frc[i];
  f.x += (float)((double)(long long)a.x * s);
  f.y += (float)((double)(long long)a.y * s);
  f.z += (float)((double)(long long)b.x * s);
  frc[i] = f;
  if (EV) watom[i] += (double)(long long)b.y * s;
}

// -------------------------------------------------------------------------------------------
struct FitTcArgs {
  const int* sidx;
  const int* soff;
  const int* tile_sp;
  const int* tile_row;
  const uint16_t* G16;   // descriptor rows [N][256] BF16
  const unsigned char* fit;
  size_t fit_stride;
  const float* small;
  float* dG;
  double* enet;
  int* ctrl;
};

// One MMA chain of the fitting kernel: thread 0 waits for the weight image's bulk copy (wbar,
// wphase), issues the chain and waits for its completion; false (and NNPE_DEV_TIMEOUT) when either
// bounded wait gave up. b_mn: the B image is read as an MN-major tile (the transpose of the
// K-major image of the forward layer: the backward's A^T without a second image).
__device__ __forceinline__ bool fit_mma(uint32_t tmem, uint32_t aA, int KA, uint32_t aB, int N, uint64_t* bar, uint32_t phase,
                                        uint64_t* wbar, uint32_t wphase, int t, int* ctrl, bool b_mn = false) {
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  bool got = true;
  if (t == 0) {
    got = tc::mbar_wait(wbar, wphase);
    if (got) {
      const uint32_t id = tc::idesc_bf16(128, N, b_mn);
      for (int kk = 0; kk < KA / 16; ++kk)
        tc::mma_bf16(tmem, tc::tile_desc(aA, KA, kk), b_mn ? tc::tile_desc_mn(aB, N, kk) : tc::tile_desc(aB, KA, kk), id, kk > 0);
      tc::mma_commit(bar);
      got = tc::mbar_wait(bar, phase);
    }
    if (!got) atomicOr(ctrl + CTRL_ERR, NNPE_DEV_TIMEOUT);
  }
  const bool ok = __syncthreads_and(got) != 0;
  tc::fence_after();
  return ok;
}

// Weight image -> shared memory: thread 0 arms the buffer's barrier with the image size and issues
// bulk copies of at most 32 KB (the tensor core is the only reader, so no proxy fence is needed).
__device__ __forceinline__ void load_image(unsigned char* dst, const unsigned char* src, uint32_t bytes, uint64_t* bar) {
  tc::mbar_arrive_expect_tx(bar, bytes);
  for (uint32_t off = 0; off < bytes; off += 32768u)
    tc::bulk_g2s(dst + off, src + off, min(32768u, bytes - off), bar);
}

// 128 atoms of one species per CTA; the two weight images (A1 and A2, K-major) arrive by bulk
// copies (one barrier each) that overlap the G fetch and the first MMA chain. The backward chains
// read the same images as MN-major tiles, which are A1^T and A2^T, so no transposed copy is
// loaded. 256 threads: row p = t % 128 (TMEM lane), half h = t / 128 takes half of each
// epilogue's columns.
__global__ void __launch_bounds__(256) k_tc_fit(FitTcArgs f) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t bar, bar_w[2];
  __shared__ uint32_t tmem_base;
  __shared__ float sEn[2][128];             // per-half partial energies
  __shared__ __align__(16) float sSmall[kFitSmallStride];   // this species' c1, c2, a3, c3
  unsigned char* sAct = sm;                 // 128 x 256 (G), later 128 x 128 (g2)
  unsigned char* sH1 = sm + 128 * 256 * 2;  // 128 x 128 (h1, later g1)
  unsigned char* sW0 = sH1 + 128 * 128 * 2; // L1 image (K-major A1; MN-major it is A1^T for B1)
  unsigned char* sW1 = sW0 + 128 * 256 * 2; // L2 image (K-major A2; MN-major it is A2^T for B2)
  const int t = threadIdx.x, w = t >> 5, p = t & 127, half = t >> 7;
  const int sp = f.tile_sp[blockIdx.x], row0 = f.tile_row[blockIdx.x];
  const int M = f.soff[sp + 1] - f.soff[sp];
  const bool valid = row0 + p < M;
  const int atom = valid ? f.sidx[f.soff[sp] + row0 + p] : 0;
  const unsigned char* img = f.fit + f.fit_stride * sp;
  for (int k = t; k < kFitSmallStride; k += 256) sSmall[k] = __ldg(f.small + kFitSmallStride * sp + k);
  const float* sm_c1 = sSmall;   // read after the barrier below
  const float *sm_c2 = sm_c1 + 128, *sm_c3 = sm_c1 + 384, *sm_a3 = sm_c1 + 256;
  int issued0 = 0, issued1 = 0;             // bulk loads per buffer (thread 0)
  if (w == 0) tc::tmem_alloc(&tmem_base, 256);
  if (t == 0) {
    tc::mbar_init(&bar, 1);
    tc::mbar_init(&bar_w[0], 1);
    tc::mbar_init(&bar_w[1], 1);
    load_image(sW0, img, (uint32_t)kImgL1, &bar_w[0]);            // buffer 0, phase 0: L1
    load_image(sW1, img + kImgL1, (uint32_t)kImgL2, &bar_w[1]);   // buffer 1, phase 0: L2
    issued0 = issued1 = 1;
  }
  // this half of the BF16 G row -> A tile (K=256), 16-byte core-matrix rows straight from global
  for (int k = 128 * half; k < 128 * half + 128; k += 8) {
    if (valid) tc::cp_async16(sAct + tc::kmajor_off(p, k, 256), f.G16 + (size_t)atom * 256 + k);
    else *reinterpret_cast<uint4*>(sAct + tc::kmajor_off(p, k, 256)) = make_uint4(0, 0, 0, 0);
  }
  tc::cp_async_commit();
  tc::cp_async_wait<0>();   // G landed
  // The TMEM address that warp 0's alloc wrote is read only after a barrier: the alloc blocks while
  // CTAs of other kernels on this SM (other streams) hold the columns, and a thread reading the
  // slot before it is written would take a stale address.
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  const uint32_t taddr = tmem + ((uint32_t)((w & 3) * 32) << 16);
  const uint32_t aAct = tc::smem_u32(sAct), aH1 = tc::smem_u32(sH1), aW0 = tc::smem_u32(sW0), aW1 = tc::smem_u32(sW1);
  bool ok = true;
  // L1: z1 = G A1 (+c1), h1 = tanh
  ok = fit_mma(tmem, aAct, 256, aW0, 128, &bar, 0, &bar_w[0], 0, t, f.ctrl);
  if (ok) {
    for (int c0 = 64 * half; c0 < 64 * half + 64; c0 += 32) {   // two 16-column loads behind one wait
      float v[32];
      tc::tmem_ld16x2(taddr + c0, taddr + c0 + 16, v, v + 16);
#pragma unroll
      for (int q = 0; q < 32; ++q) v[q] = tanh_fast(v[q] + sm_c1[c0 + q]);
#pragma unroll
      for (int k = 0; k < 4; ++k) *reinterpret_cast<uint4*>(sH1 + tc::kmajor_off(p, c0 + 8 * k, 128)) = tc::pack8(v + 8 * k);
    }
  }
  // L2: z2 = h1 A2 (+c2), h2 = tanh, E = h2 A3 + c3, g2 = A3 (1-h2^2)
  if (ok) ok = fit_mma(tmem + 128, aH1, 128, aW1, 128, &bar, 1, &bar_w[1], 0, t, f.ctrl);
  if (ok) {
    float e = 0.f;
    for (int c0 = 64 * half; c0 < 64 * half + 64; c0 += 32) {
      float v[32];
      tc::tmem_ld16x2(taddr + 128 + c0, taddr + 128 + c0 + 16, v, v + 16);
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const float h2 = tanh_fast(v[q] + sm_c2[c0 + q]);
        e += h2 * sm_a3[c0 + q];
        v[q] = sm_a3[c0 + q] * (1.f - h2 * h2);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) *reinterpret_cast<uint4*>(sAct + tc::kmajor_off(p, c0 + 8 * k, 128)) = tc::pack8(v + 8 * k);
    }
    sEn[half][p] = e;
  }
  // B2: u = g2 A2^T, g1 = u (1-h1^2)
  if (ok) ok = fit_mma(tmem, aAct, 128, aW1, 128, &bar, 0, &bar_w[1], 0, t, f.ctrl, true);
  if (ok && half == 0 && valid) f.enet[atom] = (double)(sEn[0][p] + sEn[1][p]) + (double)sm_c3[0];
  if (ok) {
    for (int c0 = 64 * half; c0 < 64 * half + 64; c0 += 16) {
      float v[16];
      tc::tmem_ld16(taddr + c0, v);
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        uint4* pchunk = reinterpret_cast<uint4*>(sH1 + tc::kmajor_off(p, c0 + 8 * hh, 128));
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
  // B1: dE/dG = g1 A1^T (N = 256)
  if (ok) ok = fit_mma(tmem, aH1, 128, aW0, 256, &bar, 1, &bar_w[0], 0, t, f.ctrl, true);
  if (ok) {
    for (int c0 = 128 * half; c0 < 128 * half + 128; c0 += 32) {
      float v[32];
      tc::tmem_ld16x2(taddr + c0, taddr + c0 + 16, v, v + 16);   // warp-collective: every lane loads, valid rows store
      if (valid) {
        float4* dst = reinterpret_cast<float4*>(f.dG + (size_t)atom * 256 + c0);
#pragma unroll
        for (int k = 0; k < 8; ++k) dst[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
      }
    }
  }
  if (!ok && t == 0) {
    // a wait gave up: let the bulk loads still in flight land (bounded) before the CTA exits. A
    // buffer's phases complete in order, so waiting for the parity of its last load covers both.
    // If that wait gives up too, copies may still land in shared memory that the SM hands to the
    // next CTA: the context is poisoned and the host refuses further work on it.
    bool drained = true;
    if (issued0) drained = tc::mbar_wait(&bar_w[0], (uint32_t)((issued0 - 1) & 1), 200000000ll) && drained;
    if (issued1) drained = tc::mbar_wait(&bar_w[1], (uint32_t)((issued1 - 1) & 1), 200000000ll) && drained;
    if (!drained) atomicOr(f.ctrl + CTRL_ERR, NNPE_DEV_POISONED);
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
  for (void* p : {(void*)t->d_wdesc64, (void*)t->d_facc, (void*)t->d_fit, (void*)t->d_emb_small, (void*)t->d_fit_small,
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
  const int T = c->ntype;
  const size_t eb = 32 + 32 + 32 * 64 + 64;
  const float* E = m->h_embw.data();
  std::vector<uint16_t> wdesc64((size_t)(kWImg + kWBiasImg) / 2);
  put_image(wdesc64, 0, 64, kK64, [&](int n, int k) { return k / 32 < T ? E[eb * (k / 32) + 64 + (k % 32) * 64 + n] : 0.f; });
  // the bias slice's B: column s = b2 of species s (the A slice is the row's one-hot species)
  put_image(wdesc64, kWImg / 2, 64, 16, [&](int n, int k) { return k < T ? E[eb * k + 64 + 32 * 64 + n] : 0.f; });
  std::vector<float> emb_small((size_t)T * 128);
  for (int s = 0; s < T; ++s)
    for (int q = 0; q < 32; ++q) {
      emb_small[s * 128 + q] = E[eb * s + q];
      emb_small[s * 128 + 32 + q] = E[eb * s + 32 + q];
      emb_small[s * 128 + 64 + q] = E[eb * s + 64 + 32 * 64 + q];
      emb_small[s * 128 + 96 + q] = E[eb * s + 64 + 32 * 64 + 32 + q];
    }
  const size_t fb = (size_t)256 * 128 + 128 + 128 * 128 + 128 + 128 + 1;
  const size_t stride_el = (kImgL1 + kImgL2) / 2;
  std::vector<uint16_t> fit(stride_el * T);
  std::vector<float> fit_small((size_t)kFitSmallStride * T, 0.f);
  for (int s = 0; s < T; ++s) {
    const float* W = m->h_fitw.data() + fb * s;
    const float *A1 = W, *c1 = A1 + 256 * 128, *A2 = c1 + 128, *c2 = A2 + 128 * 128, *A3 = c2 + 128, *c3 = A3 + 128;
    const size_t b = stride_el * s;
    put_image(fit, b, 128, 256, [&](int n, int k) { return A1[k * 128 + n]; });                                  // L1
    put_image(fit, b + kImgL1 / 2, 128, 128, [&](int n, int k) { return A2[k * 128 + n]; });                     // L2
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
  if (int rc = up((void**)&t->d_wdesc64, wdesc64.data(), wdesc64.size() * 2)) return rc;
  NNPE_CUDA(c, dev_malloc(c, (void**)&t->d_facc, sizeof(unsigned long long) * 4 * std::max(c->natom, 1)));
  NNPE_CUDA(c, cudaMemset(t->d_facc, 0, sizeof(unsigned long long) * 4 * std::max(c->natom, 1)));   // the apply re-zeroes it
  if (int rc = up((void**)&t->d_fit, fit.data(), fit.size() * 2)) return rc;
  if (int rc = up((void**)&t->d_emb_small, emb_small.data(), emb_small.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_fit_small, fit_small.data(), fit_small.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_tile_sp, tsp.data(), tsp.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_tile_row, trow.data(), trow.size() * 4)) return rc;
  if (int rc = up((void**)&t->d_soff, m->soff.data(), m->soff.size() * 4)) return rc;
  const int smem_fit = 128 * 256 * 2 + 128 * 128 * 2 + kImgL1 + kImgL2;
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_desc2, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemDesc2));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_force2<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemForce2));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_force2<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemForce2));
  NNPE_CUDA(c, cudaFuncSetAttribute(k_tc_fit, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_fit));
  return 0;
}

int nnp_tc_forces_enqueue(nnpe_ctx* c, bool ev) {
  NnpModel* m = c->nnp;
  NnpTc* t = m->tc;
  if (!t) return nnpe_fail(c, NNPE_EARG, "BF16 tensor-core path needs the 1->32->64 / 256->128->128 network");
  const int sms = nnpe_sm_count(c->device);
  const int smem_fit = 128 * 256 * 2 + 128 * 128 * 2 + kImgL1 + kImgL2;
  DescArgs dd;
  dd.pos = c->d_pos; dd.list6 = m->d_list6; dd.n6 = m->d_n6; dd.gowner = c->d_gowner;
  dd.wdesc = t->d_wdesc64; dd.emb_small = t->d_emb_small; dd.G2 = reinterpret_cast<uint32_t*>(m->d_G); dd.ctrl = c->d_ctrl;
  dd.cap6 = m->cap6; dd.N = c->natom; dd.ntype = c->ntype; dd.npos = c->natom + c->Gcap; dd.rc = m->rc; dd.scale = m->scale;
  dd.r_rc = 1.f / m->rc;
  const int gdesc = t->grid_desc > 0 ? t->grid_desc : std::max(1, std::min(c->natom, sms * t->ctas_desc));
  k_tc_desc2<<<gdesc, 128, kSmemDesc2, c->stream>>>(dd);
  m->g_bf16 = true;
  FitTcArgs f;
  f.sidx = m->d_sidx; f.soff = t->d_soff; f.tile_sp = t->d_tile_sp; f.tile_row = t->d_tile_row;
  f.G16 = reinterpret_cast<const uint16_t*>(m->d_G);
  f.fit = t->d_fit; f.fit_stride = t->fit_stride; f.small = t->d_fit_small; f.dG = m->d_dG; f.enet = m->d_enet;
  f.ctrl = c->d_ctrl;
  k_tc_fit<<<t->ntiles, 256, smem_fit, c->stream>>>(f);
  ForceArgs fa;
  fa.pos = c->d_pos; fa.list6 = m->d_list6; fa.n6 = m->d_n6; fa.gowner = c->d_gowner; fa.wdesc = t->d_wdesc64;
  fa.emb_small = t->d_emb_small; fa.dG = m->d_dG; fa.facc = t->d_facc; fa.ctrl = c->d_ctrl;
  fa.cap6 = m->cap6; fa.N = c->natom; fa.ntype = c->ntype; fa.npos = c->natom + c->Gcap; fa.rc = m->rc; fa.scale = m->scale;
  fa.r_rc = 1.f / m->rc;
  const int gforce = t->grid_force > 0 ? t->grid_force : std::max(1, std::min(c->natom, sms * t->ctas_force));
  const int gapply = (c->natom + 255) / 256;
  if (ev) {
    k_tc_force2<true><<<gforce, 256, kSmemForce2, c->stream>>>(fa);
    k_facc_apply4<true><<<gapply, 256, 0, c->stream>>>(t->d_facc, c->d_frc, c->d_watom, c->natom);
  } else {
    k_tc_force2<false><<<gforce, 256, kSmemForce2, c->stream>>>(fa);
    k_facc_apply4<false><<<gapply, 256, 0, c->stream>>>(t->d_facc, c->d_frc, c->d_watom, c->natom);
  }
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

// Grid autotuner of the two pair kernels. The packed tiles follow each CTA's atom range, so the
// grid size sets both the load balance and the number of partially filled tiles; the best size
// depends on the atom count, the pair density and what else shares the device. Candidates: 1-4
// CTAs per SM for the descriptor kernel (its occupancy limit), 1-2 for the force kernel, and
// fractions of one wave for small systems; each is timed over `reps` network evaluations of the
// context's current list with CUDA events, the descriptor grid first with the force grid at its
// default, then the force grid. A result is cached per (device, species, half-octave of the atom
// count) for the process, so that replicas of a similar size reuse it. The choice fixes how a
// CTA's pairs are cut into tiles, so results with different grids agree to FP32 rounding of the
// descriptor sums, and two runs with the same grid are bit-identical.
namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, std::pair<int, int>> g_tune_cache;

std::vector<int> grid_candidates(int natom, int sms, int max_per_sm) {
  std::vector<int> v;
  for (int k = max_per_sm; k >= 1; --k) v.push_back(sms * k);
  v.push_back(sms / 2);
  v.push_back(sms / 4);
  for (int& g : v) g = std::max(1, std::min(natom, g));
  std::vector<int> u;
  for (int g : v)
    if (std::find(u.begin(), u.end(), g) == u.end()) u.push_back(g);
  return u;
}
}  // namespace

int nnpe_sync_errors(nnpe_ctx* c);

int nnp_tc_autotune(nnpe_ctx* c, int reps, bool use_cache, int* grid_desc, int* grid_force) {
  NnpModel* m = c->nnp;
  NnpTc* t = m ? m->tc : nullptr;
  if (!t || !m->bf16) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_autotune: the BF16 tensor-core network is not active");
  const int sms = nnpe_sm_count(c->device);
  const auto key = std::make_tuple(c->device, c->ntype, (int)std::floor(2.0 * std::log2((double)std::max(c->natom, 1))));
  if (use_cache) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      t->grid_desc = std::min(it->second.first, c->natom);
      t->grid_force = std::min(it->second.second, c->natom);
      c->graph_valid = false;
      c->fs_valid = false;
      if (grid_desc) *grid_desc = t->grid_desc;
      if (grid_force) *grid_force = t->grid_force;
      return NNPE_OK;
    }
  }
  reps = std::max(1, reps);
  cudaEvent_t a, b;
  NNPE_CUDA(c, cudaEventCreate(&a));
  NNPE_CUDA(c, cudaEventCreate(&b));
  auto time_now = [&](float* ms) -> int {
    if (int rc = nnp_tc_forces_enqueue(c, false)) return rc;   // warm
    NNPE_CUDA(c, cudaEventRecord(a, c->stream));
    for (int r = 0; r < reps; ++r)
      if (int rc = nnp_tc_forces_enqueue(c, false)) return rc;
    NNPE_CUDA(c, cudaEventRecord(b, c->stream));
    NNPE_CUDA(c, cudaEventSynchronize(b));
    NNPE_CUDA(c, cudaEventElapsedTime(ms, a, b));
    return 0;
  };
  int rc = 0;
  int best_d = 0, best_f = 0;
  float best = 1e30f, ms = 0.f;
  t->grid_force = 0;
  for (int g : grid_candidates(c->natom, sms, t->ctas_desc)) {
    t->grid_desc = g;
    if ((rc = time_now(&ms))) break;
    if (ms < best) { best = ms; best_d = g; }
  }
  if (!rc) {
    t->grid_desc = best_d;
    best = 1e30f;
    for (int g : grid_candidates(c->natom, sms, t->ctas_force)) {
      t->grid_force = g;
      if ((rc = time_now(&ms))) break;
      if (ms < best) { best = ms; best_f = g; }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) {
    t->grid_desc = t->grid_force = 0;
    return rc;
  }
  t->grid_force = best_f;
  c->graph_valid = false;
  c->fs_valid = false;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = {best_d, best_f};
  }
  if (grid_desc) *grid_desc = best_d;
  if (grid_force) *grid_force = best_f;
  return nnpe_sync_errors(c);
}

int nnp_tc_set_grids(nnpe_ctx* c, int grid_desc, int grid_force) {
  NnpTc* t = c->nnp ? c->nnp->tc : nullptr;
  if (!t) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_grids: no tensor-core network");
  if (grid_desc < 0 || grid_force < 0) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_grids: negative grid");
  t->grid_desc = grid_desc > 0 ? std::min(grid_desc, std::max(c->natom, 1)) : 0;
  t->grid_force = grid_force > 0 ? std::min(grid_force, std::max(c->natom, 1)) : 0;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

int nnp_tc_get_grids(nnpe_ctx* c, int* grid_desc, int* grid_force) {
  NnpTc* t = c->nnp ? c->nnp->tc : nullptr;
  if (!t) return nnpe_fail(c, NNPE_EARG, "nnpe_nnp_grids: no tensor-core network");
  const int sms = nnpe_sm_count(c->device);
  if (grid_desc) *grid_desc = t->grid_desc > 0 ? t->grid_desc : std::max(1, std::min(c->natom, sms * t->ctas_desc));
  if (grid_force) *grid_force = t->grid_force > 0 ? t->grid_force : std::max(1, std::min(c->natom, sms * t->ctas_force));
  return NNPE_OK;
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
