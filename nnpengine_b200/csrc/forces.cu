// Pair forces (LJTableCoulDSF, pair.cpp:289-419) and bonded terms (bond.cpp:108-137,
// angle.cpp:245-294, dihedral.cpp:403-460), plus the deterministic FP64 energy reduction.
//
// Compiled with -fmad=false: every float expression below evaluates in the order the reference
// spells it, without contraction, so a pair's fpair is the reference's bit for bit; only the
// summation order over neighbours differs (full list, warp gather instead of the half list).
#include "internal.cuh"

namespace {

__constant__ float c_special_lj[4] = {1.f, 0.f, 0.f, 0.5f};
__constant__ float c_special_coul[4] = {1.f, 0.f, 0.f, (float)(5 / 6.)};
constexpr float kElectricK = 332.06371f;

struct PairParams {
  const float4* pos;
  const uint32_t* list;     // the full list
  const int* ncount;
  // the pruned copy (nullptr: pruning off). The pass reads it, or, when CTRL_PRUNE is set at its
  // start, reads the full list and remakes it (entries with rsq < prunesq, in list order) with the
  // positions of this pass.
  uint32_t* plist;
  int* pcount;
  float4* xprune;
  float prunesq;
  const int2* info;
  const float2* table;
  const int* pairtype;
  float4* frc;
  double* eatom;
  double* watom;
  int N, cap, ntype, nbin;
  float cutoff, cutsq, r_dr, vc, fc;
  // energy/virial steps: entries with float rsq >= evgatesq skip the FP64 evaluation. The gate
  // lies 0.2 % beyond rc^2, far outside the few-ulp rounding of the float rsq, so the FP64 test
  // rsq < rc^2 on the same two positions still decides which pairs count.
  float evgatesq;
  double rc64, vc64, fc64;   // cutoff, -1/rc and -1/rc^2 in double (pair.cpp:191-193)
  bool accumulate;
  // the network term's pair list, filtered here from the same distances (nullptr: not wanted)
  uint32_t* list6;
  int* n6;
  int cap6;
  float cut6sq;
  int* ctrl;
};

// 1/sqrt(a) in double with neither a division nor a square root: the single-precision hardware
// estimate refined by two Newton-Raphson steps for f(y) = 1/y^2 - a, y <- y + y (1 - a y^2) / 2.
// Each step squares the relative error (times 1.5): below 2^-22 for the estimate, below 2^-43
// after one step, and at double rounding after the second.
__device__ __forceinline__ double rsqrt64(double a) {
  double y = (double)rsqrtf((float)a);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double t = fma(-(a * y), y, 1.0);
    y = fma(0.5 * y, t, y);
  }
  return y;
}

// FP64 pair energy and fpair*rsq of one pair at double separation: the energy/virial reductions of
// ev steps (pair.cpp:365-410) evaluated in double so that cancellation in the Coulomb sum does not
// leave FP32 rounding in the total. 1/r, 1/r^3 and fc/r come from one double 1/sqrt(rsq).
__device__ __forceinline__ void pair_energy64(const PairParams& p, const float2* tab0, int s, double qq, double rsq,
                                              double* e, double* w) {
  const double rc = p.rc64;
  if (!(rsq < rc * rc)) return;
  const double rinv = rsqrt64(rsq);
  const double r = rsq * rinv;
  double u = r * (double)p.r_dr - 0.5;
  const int t1 = (int)u;
  const double w2 = u - t1, w1 = 1 - w2;
  const float2 a = tab0[t1], b = tab0[t1 + 1];
  const double slj = c_special_lj[s], sco = s == 3 ? 5.0 / 6.0 : (double)c_special_coul[s];
  const double vc = p.vc64, fc = p.fc64;
  const double fpair = ((double)a.x * w1 + (double)b.x * w2) * slj + qq * (rinv * rinv * rinv + fc * rinv) * sco;
  const double ue = ((double)a.y * w1 + (double)b.y * w2) * slj + qq * (rinv + vc + fc * (rc - r)) * sco;
  *e += 0.5 * ue;
  *w += 0.5 * fpair * rsq;
}

// One warp per atom: lanes stride over the atom's list row (coalesced 128-byte reads), gather
// neighbour positions, and reduce with shuffles; the warp writes the atom's force once (no
// atomics, deterministic). With list6 set, the entries inside the network cutoff (the same float
// rsq, the reference's `rsq < cutsq` of pair_nnp.cpp:656) are compacted in list order into the
// network's pair list on the way, so the list is read once per step.
// EXACT=true evaluates fpair with the reference's float sequence (IEEE sqrt and divisions, no
// contraction), bit-identical per pair. EXACT=false keeps the same cutoff test (so the same pairs
// interact) but uses rsqrt and fused multiply-adds: ~1 ulp per pair, forces within 1e-6 relative.
template <bool EV, bool EXACT>
__device__ __forceinline__ void pair_row(const PairParams& p, int i, int lane, bool reprune) {
  const float4 xi = p.pos[i];
  const int ti = p.info[i].y & 0xFF;
  const int* ptrow = p.pairtype + ti * p.ntype;
  const bool full = reprune || !p.plist;
  const uint32_t* row = (full ? p.list : p.plist) + (size_t)i * p.cap;
  const int n = full ? p.ncount[i] : p.pcount[i];
  float fx = 0.f, fy = 0.f, fz = 0.f;
  double e = 0.0, w = 0.0;
  uint32_t* out6 = p.list6 ? p.list6 + (size_t)i * p.cap6 : nullptr;
  int cnt6 = 0;
  uint32_t* outp = reprune ? p.plist + (size_t)i * p.cap : nullptr;
  int cntp = 0;
  // software pipeline over 32-entry chunks: the list entries two chunks ahead and the neighbour
  // positions one chunk ahead are in flight while a chunk is evaluated
  uint32_t e_nx = lane < n ? __ldg(row + lane) : 0u;
  uint32_t e_nx2 = lane + 32 < n ? __ldg(row + lane + 32) : 0u;
  float4 x_nx = lane < n ? __ldg(p.pos + (e_nx & NNPE_J_MASK)) : xi;
  for (int base = 0; base < n; base += 32) {
    const int k = base + lane;
    const bool in = k < n;
    const uint32_t ent = e_nx;
    const float4 xj = x_nx;
    e_nx = e_nx2;
    x_nx = k + 32 < n ? __ldg(p.pos + (e_nx & NNPE_J_MASK)) : xi;
    e_nx2 = k + 64 < n ? __ldg(row + k + 64) : 0u;
    float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    const float rsq = dx * dx + dy * dy + dz * dz;
    if (out6) {   // warp-uniform
      const bool ok6 = in && rsq < p.cut6sq;
      const unsigned b6 = __ballot_sync(0xffffffffu, ok6);
      if (ok6) {
        const int idx = cnt6 + __popc(b6 & ((1u << lane) - 1));
        if (idx < p.cap6) out6[idx] = ent;
      }
      cnt6 += __popc(b6);
    }
    if (outp) {   // warp-uniform
      const bool kp = in && rsq < p.prunesq;
      const unsigned bp = __ballot_sync(0xffffffffu, kp);
      if (kp) outp[cntp + __popc(bp & ((1u << lane) - 1))] = ent;
      cntp += __popc(bp);
    }
    if (!in) continue;
    if (rsq < p.cutsq) {
      const int tj = (ent >> 27) & 7, s = ent >> 30;
      const float2* tab = p.table + (size_t)ptrow[tj] * (p.nbin + 1);
      float fpair;
      if (EXACT) {
        const float r = sqrtf(rsq);
        float ipw1 = r * p.r_dr - 0.5F;
        const int t1 = (int)ipw1;
        const float ipw2 = ipw1 - (float)t1;
        ipw1 = 1 - ipw2;
        const float2 a = __ldg(tab + t1), b = __ldg(tab + t1 + 1);
        fpair = (a.x * ipw1 + b.x * ipw2) * c_special_lj[s];
        const float qq = xi.w * xj.w * kElectricK;
        fpair += qq * (1 / (r * rsq) + p.fc / r) * c_special_coul[s];
      } else {
        const float rinv = rsqrtf(rsq);
        const float r = rsq * rinv;
        const float u = fmaf(r, p.r_dr, -0.5F);
        const int t1 = (int)u;
        const float w2 = u - (float)t1;
        const float2 a = __ldg(tab + t1), b = __ldg(tab + t1 + 1);
        const float flj = fmaf(b.x - a.x, w2, a.x);
        const float qq = xi.w * xj.w * kElectricK;
        const float fco = qq * rinv * fmaf(rinv, rinv, p.fc);
        fpair = fmaf(flj, c_special_lj[s], fco * c_special_coul[s]);
      }
      fx = fmaf(dx, fpair, fx); fy = fmaf(dy, fpair, fy); fz = fmaf(dz, fpair, fz);
    }
    if (EV && rsq < p.evgatesq) {
      // the separation of the two float positions the forces use, exact in double
      const double ddx = (double)xi.x - (double)xj.x, ddy = (double)xi.y - (double)xj.y, ddz = (double)xi.z - (double)xj.z;
      const int tj = (ent >> 27) & 7, s = ent >> 30;
      pair_energy64(p, p.table + (size_t)ptrow[tj] * (p.nbin + 1), s, (double)xi.w * (double)xj.w * 332.06371,
                    ddx * ddx + ddy * ddy + ddz * ddz, &e, &w);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
    if (EV) {
      e += __shfl_xor_sync(0xffffffffu, e, o);
      w += __shfl_xor_sync(0xffffffffu, w, o);
    }
  }
  if (out6 && lane == 0) {
    p.n6[i] = min(cnt6, p.cap6);
    if (cnt6 > p.cap6) atomicOr(p.ctrl + CTRL_ERR, NNPE_DEV_LIST_OVERFLOW);
  }
  if (outp && lane == 0) {
    p.pcount[i] = cntp;
    p.xprune[i] = xi;
  }
  if (lane == 0) {
    if (p.accumulate) {
      float4 f = p.frc[i];
      p.frc[i] = make_float4(f.x + fx, f.y + fy, f.z + fz, 0.f);
    } else {
      p.frc[i] = make_float4(fx, fy, fz, 0.f);
    }
    if (EV) {
      p.eatom[i] = p.accumulate ? p.eatom[i] + e : e;
      p.watom[i] = p.accumulate ? p.watom[i] + w : w;
    }
  }
}

// With pruning on, the pass reads the pruned copy of the list; on the steps that asked for a new
// copy (a rebuild, or an atom displaced prune_delta/2 since the last copy) it reads the full list
// instead and remakes the copy from the distances it computes anyway.
template <bool EV, bool EXACT>
__global__ void __launch_bounds__(128) k_pair(PairParams p) {
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const bool reprune = p.plist && *reinterpret_cast<volatile int*>(p.ctrl + CTRL_PRUNE) != 0;   // grid-uniform
  if (i < p.N) pair_row<EV, EXACT>(p, i, lane, reprune);
  if (reprune) prune_pass_done(p.ctrl);
}

__global__ void k_zero_forces(float4* frc, double* eatom, double* watom, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  frc[i] = make_float4(0, 0, 0, 0);
  eatom[i] = 0;
  watom[i] = 0;
}

struct BondedParams {
  const float4* pos;
  const int* sorted_of_id;
  const int* molshift;
  const int* terms;        // per molecule [bond, angle, dih] starts
  const int4* bond;
  const int4* angle;
  const int* dih;
  const float4* bcoef;
  const float4* acoef;
  const float4* dcoef;
  float4* frc;
  double* emol;
  double* wmol;
  int nmol;
  GridParams g;
};

// x_mol (environ.h:38-40): the real atom or the periodic image of it that lies within half a box
// of its molecule's representative, recomputed as x + shift every step like the image itself.
__device__ __forceinline__ float3 xmol(const BondedParams& p, int a, int* si) {
  const int s = p.sorted_of_id[a];
  *si = s;
  const float4 x = p.pos[s];
  float sh[3];
  shift_of(p.g, p.molshift[a], sh);
  return make_float3(x.x + sh[0], x.y + sh[1], x.z + sh[2]);
}
__device__ __forceinline__ void addf(float4* frc, int s, float fx, float fy, float fz) {
  float4 f = frc[s];
  frc[s] = make_float4(f.x + fx, f.y + fy, f.z + fz, f.w);
}

__device__ __forceinline__ double3 xmol64(const BondedParams& p, int a) {
  const float4 x = p.pos[p.sorted_of_id[a]];
  float sh[3];
  shift_of(p.g, p.molshift[a], sh);
  return make_double3((double)x.x + sh[0], (double)x.y + sh[1], (double)x.z + sh[2]);
}

// One thread per molecule evaluates all of its bonded terms (molecules never share atoms, so
// the read-modify-write of the atoms' forces is race free).
template <bool EV>
__global__ void k_bonded(BondedParams p) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= p.nmol) return;
  double e = 0.0, w = 0.0;
  const int b0 = p.terms[3 * m], b1 = p.terms[3 * m + 3];
  for (int t = b0; t < b1; ++t) {
    const int4 b = p.bond[t];
    const float4 c = p.bcoef[b.x];
    int si, sj;
    const float3 xi = xmol(p, b.y, &si), xj = xmol(p, b.z, &sj);
    float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
    float rr = sqrtf(dx * dx + dy * dy + dz * dz);
    const float dr = rr - c.x;
    const float bdr = c.z - dr;
    const float ff = dr * (c.w + c.y * bdr * (bdr - dr)) / rr;
    dx *= ff; dy *= ff; dz *= ff;
    addf(p.frc, si, -dx, -dy, -dz);
    addf(p.frc, sj, dx, dy, dz);
    if (EV) {   // bond.cpp:131-135 in FP64
      const double3 a = xmol64(p, b.y), bb = xmol64(p, b.z);
      const double ex = a.x - bb.x, ey = a.y - bb.y, ez = a.z - bb.z;
      const double r = sqrt(ex * ex + ey * ey + ez * ez);
      const double d = r - c.x, bd = c.z - d;
      e += 0.5 * d * d * (c.y * bd * bd + c.w);
      w -= d * (c.w + c.y * bd * (bd - d)) / r * r * r;
    }
  }
  const int a0 = p.terms[3 * m + 1], a1 = p.terms[3 * m + 4];
  for (int t = a0; t < a1; ++t) {
    const int4 a4 = p.angle[t];
    const float4 c = p.acoef[a4.x];
    int si, sj, sk;
    const float3 xi = xmol(p, a4.y, &si), xj = xmol(p, a4.z, &sj), xk = xmol(p, a4.w, &sk);
    float dx1 = xi.x - xj.x, dy1 = xi.y - xj.y, dz1 = xi.z - xj.z;
    float dx2 = xk.x - xj.x, dy2 = xk.y - xj.y, dz2 = xk.z - xj.z;
    const float r_r1 = 1 / sqrtf(dx1 * dx1 + dy1 * dy1 + dz1 * dz1);
    const float r_r2 = 1 / sqrtf(dx2 * dx2 + dy2 * dy2 + dz2 * dz2);
    dx1 *= r_r1; dy1 *= r_r1; dz1 *= r_r1;
    dx2 *= r_r2; dy2 *= r_r2; dz2 *= r_r2;
    const float cq = dx1 * dx2 + dy1 * dy2 + dz1 * dz2;
    const float dcq = cq - c.x;
    const float b_dcq = c.z - dcq;
    const float fe = dcq * (c.w + c.y * b_dcq * (b_dcq - dcq));
    float ff = fe * r_r1;
    float fx = ff * (cq * dx1 - dx2), fy = ff * (cq * dy1 - dy2), fz = ff * (cq * dz1 - dz2);
    addf(p.frc, si, fx, fy, fz);
    addf(p.frc, sj, -fx, -fy, -fz);
    ff = fe * r_r2;
    fx = ff * (dx1 - cq * dx2); fy = ff * (dy1 - cq * dy2); fz = ff * (dz1 - cq * dz2);
    addf(p.frc, sk, -fx, -fy, -fz);
    addf(p.frc, sj, fx, fy, fz);
    if (EV) {   // angle.cpp:289-292 in FP64
      const double3 a = xmol64(p, a4.y), bb = xmol64(p, a4.z), cc = xmol64(p, a4.w);
      const double u1x = a.x - bb.x, u1y = a.y - bb.y, u1z = a.z - bb.z, u2x = cc.x - bb.x, u2y = cc.y - bb.y, u2z = cc.z - bb.z;
      const double cqd = (u1x * u2x + u1y * u2y + u1z * u2z) /
                         sqrt((u1x * u1x + u1y * u1y + u1z * u1z) * (u2x * u2x + u2y * u2y + u2z * u2z));
      const double d = cqd - c.x, bd = c.z - d;
      e += 0.5 * d * d * (c.y * bd * bd + c.w);
    }
  }
  const int d0 = p.terms[3 * m + 2], d1 = p.terms[3 * m + 5];
  for (int t = d0; t < d1; ++t) {
    const int* d = p.dih + 5 * t;
    const float4 c = p.dcoef[d[0]];
    int si, sj, sk, sl;
    const float3 xi = xmol(p, d[1], &si), xj = xmol(p, d[2], &sj), xk = xmol(p, d[3], &sk), xl = xmol(p, d[4], &sl);
    float dx1 = xi.x - xj.x, dy1 = xi.y - xj.y, dz1 = xi.z - xj.z;
    float dx2 = xk.x - xj.x, dy2 = xk.y - xj.y, dz2 = xk.z - xj.z;
    float dx3 = xl.x - xk.x, dy3 = xl.y - xk.y, dz3 = xl.z - xk.z;
    const float r_rsq2 = 1 / (dx2 * dx2 + dy2 * dy2 + dz2 * dz2);
    const float dot12 = (dx1 * dx2 + dy1 * dy2 + dz1 * dz2) * r_rsq2;
    const float dot32 = (dx3 * dx2 + dy3 * dy2 + dz3 * dz2) * r_rsq2;
    dx1 -= dx2 * dot12; dy1 -= dy2 * dot12; dz1 -= dz2 * dot12;
    dx3 -= dx2 * dot32; dy3 -= dy2 * dot32; dz3 -= dz2 * dot32;
    float r_r1 = 1 / sqrtf(dx1 * dx1 + dy1 * dy1 + dz1 * dz1);
    float r_r3 = 1 / sqrtf(dx3 * dx3 + dy3 * dy3 + dz3 * dz3);
    dx1 *= r_r1; dy1 *= r_r1; dz1 *= r_r1;
    dx3 *= r_r3; dy3 *= r_r3; dz3 *= r_r3;
    const float cq = dx1 * dx3 + dy1 * dy3 + dz1 * dz3;
    const float ff = (c.w * cq + c.z) * cq + c.y;
    r_r1 *= ff; r_r3 *= ff;
    const float f1x = r_r1 * (cq * dx1 - dx3), f1y = r_r1 * (cq * dy1 - dy3), f1z = r_r1 * (cq * dz1 - dz3);
    const float f3x = r_r3 * (cq * dx3 - dx1), f3y = r_r3 * (cq * dy3 - dy1), f3z = r_r3 * (cq * dz3 - dz1);
    const float f2x = f1x * dot12 + f3x * dot32, f2y = f1y * dot12 + f3y * dot32, f2z = f1z * dot12 + f3z * dot32;
    addf(p.frc, si, f1x, f1y, f1z);
    addf(p.frc, sl, f3x, f3y, f3z);
    addf(p.frc, sj, f2x - f1x, f2y - f1y, f2z - f1z);
    addf(p.frc, sk, -(f2x + f3x), -(f2y + f3y), -(f2z + f3z));
    if (EV) {   // dihedral.cpp:454-458 in FP64
      const double3 a = xmol64(p, d[1]), bb = xmol64(p, d[2]), cc = xmol64(p, d[3]), dd = xmol64(p, d[4]);
      double v1x = a.x - bb.x, v1y = a.y - bb.y, v1z = a.z - bb.z;
      const double v2x = cc.x - bb.x, v2y = cc.y - bb.y, v2z = cc.z - bb.z;
      double v3x = dd.x - cc.x, v3y = dd.y - cc.y, v3z = dd.z - cc.z;
      const double r2 = 1 / (v2x * v2x + v2y * v2y + v2z * v2z);
      const double d12 = (v1x * v2x + v1y * v2y + v1z * v2z) * r2, d32 = (v3x * v2x + v3y * v2y + v3z * v2z) * r2;
      v1x -= v2x * d12; v1y -= v2y * d12; v1z -= v2z * d12;
      v3x -= v2x * d32; v3y -= v2y * d32; v3z -= v2z * d32;
      const double cqd = (v1x * v3x + v1y * v3y + v1z * v3z) /
                         sqrt((v1x * v1x + v1y * v1y + v1z * v1z) * (v3x * v3x + v3y * v3y + v3z * v3z));
      e += (((double)c.w / 3 * cqd + (double)c.z / 2) * cqd + c.y) * cqd + c.x;
    }
  }
  if (EV) {
    p.emol[m] = e;
    p.wmol[m] = w;
  }
}

// Deterministic FP64 reduction of per-atom / per-molecule partials into d_red:
// [0] pair+bonded energy, [1] virial, [2] kinetic energy, [3] network energy.
__device__ double block_sum(double v, double* sh) {
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s) sh[t] += sh[t + s];
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}

// Deterministic two-pass reduction: kReduceBlocks blocks each sum a fixed contiguous share of the
// per-atom / per-molecule partials in a fixed order, then one block sums the block partials in
// block order (the same bits on every run).
constexpr int kReduceBlocks = 256;
constexpr int kReduceThreads = 256;

__global__ void __launch_bounds__(kReduceThreads) k_reduce_part(const double* eatom, const double* watom, const double* kin,
                                                                 const double* emol, const double* wmol, const double* enet,
                                                                 int N, int nmol, int nnet, bool with_kin, double* part) {
  __shared__ double sh[kReduceThreads];
  const int t = threadIdx.x, b = blockIdx.x, B = gridDim.x;
  double e = 0, w = 0, k = 0, en = 0;
  {
    const int a0 = (int)((long long)N * b / B), a1 = (int)((long long)N * (b + 1) / B);
    for (int i = a0 + t; i < a1; i += kReduceThreads) { e += eatom[i]; w += watom[i]; if (with_kin) k += kin[i]; }
    const int m0 = (int)((long long)nmol * b / B), m1 = (int)((long long)nmol * (b + 1) / B);
    for (int m = m0 + t; m < m1; m += kReduceThreads) { e += emol[m]; w += wmol[m]; }
    const int n0 = (int)((long long)nnet * b / B), n1 = (int)((long long)nnet * (b + 1) / B);
    for (int m = n0 + t; m < n1; m += kReduceThreads) en += enet[m];
  }
  e = block_sum(e, sh);
  w = block_sum(w, sh);
  k = block_sum(k, sh);
  en = block_sum(en, sh);
  if (t == 0) {
    part[4 * b] = e; part[4 * b + 1] = w; part[4 * b + 2] = k; part[4 * b + 3] = en;
  }
}

__global__ void __launch_bounds__(kReduceBlocks) k_reduce_final(const double* part, bool with_kin, double* red, LogRec* log,
                                                                int log_cap, int* ctrl, bool write_log) {
  __shared__ double sh[kReduceBlocks];
  const int t = threadIdx.x;
  const double e = block_sum(part[4 * t], sh), w = block_sum(part[4 * t + 1], sh);
  const double k = block_sum(part[4 * t + 2], sh), en = block_sum(part[4 * t + 3], sh);
  if (t == 0) {
    red[0] = e + en; red[1] = w; red[3] = en;
    if (with_kin) red[2] = k;
    if (write_log) {
      const int slot = ctrl[CTRL_NLOG];
      if (slot < log_cap) {
        LogRec r;
        r.erg = e + en; r.virial = w; r.ekin = with_kin ? k : red[2]; r.erg_nnp = en; r.erg_exp = red[4];
        r.step = ctrl[CTRL_STEP]; r.nbuild = ctrl[CTRL_NBUILD]; r.pad0 = r.pad1 = 0;
        log[slot] = r;
      }
      ctrl[CTRL_NLOG] = slot + 1;
    }
  }
}

}  // namespace

const double* nnp_atom_energy_ptr(nnpe_ctx* c);   // nnp.cu
bool nnp_enabled(nnpe_ctx* c);
float nnp_cutoff(nnpe_ctx* c);

bool nnp_list6(nnpe_ctx* c, uint32_t** list6, int** n6, int* cap6, float* cut6);   // nnp.cu

int pair_enqueue(nnpe_ctx* c, bool ev, bool filter6) {
  const int N = c->natom;
  PairParams p;
  p.pos = c->d_pos; p.list = c->d_list; p.ncount = c->d_ncount; p.info = c->d_info; p.table = c->d_table;
  const bool pr = prune_in_pair(c);
  p.plist = pr ? c->d_plist : nullptr; p.pcount = pr ? c->d_pcount : nullptr; p.xprune = pr ? c->d_xprune : nullptr;
  p.prunesq = pr ? prune_cutsq(c) : 0.f;
  p.pairtype = c->d_pairtype; p.frc = c->d_frc; p.eatom = c->d_eatom; p.watom = c->d_watom;
  p.N = N; p.cap = c->cap; p.ntype = c->ntype; p.nbin = c->nbin;
  p.cutoff = c->pair_cutoff; p.cutsq = c->pair_cutoff * c->pair_cutoff;
  p.r_dr = (float)c->nbin / c->pair_cutoff;   // LJTableCoulDSF ctor (pair.cpp:176-177)
  p.vc = -1 / p.cutoff; p.fc = p.vc / p.cutoff;  // pair.cpp:191-193 (erfc disabled)
  p.rc64 = p.cutoff; p.vc64 = -1 / p.rc64; p.fc64 = p.vc64 / p.rc64;
  p.evgatesq = p.cutsq * 1.002f;
  p.accumulate = false;
  p.list6 = nullptr; p.n6 = nullptr; p.cap6 = 0; p.cut6sq = 0.f; p.ctrl = c->d_ctrl;
  if (filter6) {
    float cut6 = 0.f;
    nnp_list6(c, &p.list6, &p.n6, &p.cap6, &cut6);
    p.cut6sq = cut6 * cut6;
  }
  const int blocks = nblocks((long)N * 32, 128);
  if (c->exact_forces) {
    if (ev) k_pair<true, true><<<blocks, 128, 0, c->stream>>>(p);
    else k_pair<false, true><<<blocks, 128, 0, c->stream>>>(p);
  } else {
    if (ev) k_pair<true, false><<<blocks, 128, 0, c->stream>>>(p);
    else k_pair<false, false><<<blocks, 128, 0, c->stream>>>(p);
  }
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int bonded_enqueue(nnpe_ctx* c, bool ev) {
  cudaStream_t st = c->stream;
  if (c->d_mol_terms && (c->nbond + c->nangle + c->ndih) > 0) {
    BondedParams b;
    b.pos = c->d_pos; b.sorted_of_id = c->d_sorted_of_id; b.molshift = c->d_molshift; b.terms = c->d_mol_terms;
    b.bond = c->d_bond; b.angle = c->d_angle; b.dih = c->d_dih; b.bcoef = c->d_bcoef; b.acoef = c->d_acoef;
    b.dcoef = c->d_dcoef; b.frc = c->d_frc; b.emol = c->d_emol; b.wmol = c->d_wmol; b.nmol = c->nmol; b.g = c->grid;
    if (ev) k_bonded<true><<<nblocks(c->nmol, 128), 128, 0, st>>>(b);
    else k_bonded<false><<<nblocks(c->nmol, 128), 128, 0, st>>>(b);
  } else if (ev) {
    NNPE_CUDA(c, cudaMemsetAsync(c->d_emol, 0, sizeof(double) * c->nmol, st));
    NNPE_CUDA(c, cudaMemsetAsync(c->d_wmol, 0, sizeof(double) * c->nmol, st));
  }
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

// The force block: pair (writes the forces), network term (adds), bonded terms (add).
// The pair kernel filters the network's pairs when both terms run and the network cutoff lies
// inside the list.
bool pair_filters_list6(nnpe_ctx* c) {
  return c->nnp && nnp_enabled(c) && c->pair_on && c->d_table && nnp_cutoff(c) <= c->pair_cutoff + c->skin;
}

int forces_enqueue(nnpe_ctx* c, bool ev) {
  const bool net = c->nnp && nnp_enabled(c);
  const bool fused = pair_filters_list6(c);
  if (c->pair_on && c->d_table) {
    if (int rc = pair_enqueue(c, ev, fused)) return rc;
  } else {
    k_zero_forces<<<nblocks(c->natom, 256), 256, 0, c->stream>>>(c->d_frc, c->d_eatom, c->d_watom, c->natom);
  }
  if (net)
    if (int rc = nnp_forces_enqueue(c, ev, !fused)) return rc;
  if (int rc = bonded_enqueue(c, ev)) return rc;
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int energy_reduce_enqueue(nnpe_ctx* c, int mode) {
  // mode 0: energies only; 1: energies + kinetic into the log; 2: kinetic only (no log);
  // 3: energies into the log with the kinetic energy of the last thermostat step
  const double* enet = c->nnp ? nnp_atom_energy_ptr(c) : nullptr;
  const int nnet = enet ? c->natom : 0;
  const bool bonded = c->d_mol_terms && (c->nbond + c->nangle + c->ndih) > 0;
  const bool with_kin = mode == 1 || mode == 2;
  k_reduce_part<<<kReduceBlocks, kReduceThreads, 0, c->stream>>>(c->d_eatom, c->d_watom, c->d_kin, c->d_emol, c->d_wmol,
                                                                  enet, c->natom, bonded || mode >= 0 ? c->nmol : 0, nnet,
                                                                  with_kin, c->d_red_part);
  k_reduce_final<<<1, kReduceBlocks, 0, c->stream>>>(c->d_red_part, with_kin, c->d_red, c->d_log, c->log_cap, c->d_ctrl,
                                                     mode == 1 || mode == 3);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int nnpe_sync_errors(nnpe_ctx* c);
int check_valid_enqueue(nnpe_ctx* c);

namespace {
// positions in atom-id order (host layout) -> sorted master/FP32 coordinates
__global__ void k_scatter_positions(const float* __restrict__ x, const int* __restrict__ aid, double4* __restrict__ xd,
                                    float4* __restrict__ pos, int N, double bl, bool fp64) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const int a = aid[k];
  const float px = x[3 * a], py = x[3 * a + 1], pz = x[3 * a + 2];
  // the periodic image of the host's position nearest the stored one: the rebuild folds the stored
  // coordinates into the box and the host's own coordinates need not follow (or may be folded at
  // other times), so positions stay continuous between list builds
  const double4 o = xd[k];
  const double rbl = 1.0 / bl;
  const double sx = rint((o.x - (double)px) * rbl) * bl, sy = rint((o.y - (double)py) * rbl) * bl,
               sz = rint((o.z - (double)pz) * rbl) * bl;
  double4 n;   // no shift (the usual case) stores the host's coordinates unchanged
  if (fp64) {
    n = make_double4((double)px + sx, (double)py + sy, (double)pz + sz, 0);
  } else {   // FP32 state: the float arithmetic of the fold, x - m*bl
    n = make_double4(__fadd_rn(px, (float)sx), __fadd_rn(py, (float)sy), __fadd_rn(pz, (float)sz), 0);
  }
  xd[k] = n;
  pos[k] = make_float4((float)n.x, (float)n.y, (float)n.z, pos[k].w);
}
// sorted forces -> atom-id order
__global__ void k_gather_forces(const float4* __restrict__ frc, const int* __restrict__ aid, float* __restrict__ f, int N) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const int a = aid[k];
  const float4 v = frc[k];
  f[3 * a] = v.x; f[3 * a + 1] = v.y; f[3 * a + 2] = v.z;
}
__global__ void k_qm_to_pos(const float2* __restrict__ qm, float4* __restrict__ pos, int N) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) pos[k].w = qm[k].x;
}
}  // namespace

// Force evaluation at caller-owned host positions: the drop-in call a host-side run loop makes
// (positions in, forces and energy out, in atom-id order). The list is checked and rebuilt on the
// device as needed (run.cpp:236-283), then the force block runs (run.cpp:302-342).
int refuse_if_poisoned(nnpe_ctx* c) {
  if (c->poisoned)
    return nnpe_fail(c, NNPE_ETIMEOUT, "a device wait gave up with copies in flight: the context refuses work until nnpe_setup");
  return 0;
}

// The device part of the host-owned force step, between the positions' copy in and the forces' copy
// out: positions into the sorted state, list check and (device-conditional) rebuild, images, forces,
// optional energy reduction, forces gathered back into atom-id order.
static int force_step_body(nnpe_ctx* c, bool ev, float* xstage, float* fstage) {
  const int N = c->natom;
  k_scatter_positions<<<nblocks(N, 256), 256, 0, c->stream>>>(xstage, c->d_atom_id, c->d_xd, c->d_pos, N, (double)c->grid.bl, c->fp64_state);
  if (int rc = check_valid_enqueue(c)) return rc;
  if (int rc = rebuild_enqueue(c, true)) return rc;
  if (int rc = ghost_update_enqueue(c, true)) return rc;
  if (int rc = forces_enqueue(c, ev)) return rc;
  if (ev)
    if (int rc = energy_reduce_enqueue(c, 0)) return rc;
  k_gather_forces<<<nblocks(N, 256), 256, 0, c->stream>>>(c->d_frc, c->d_atom_id, fstage, N);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

// The body runs as one CUDA graph launch (about thirty kernels, most of them tiny or exiting at once
// when no rebuild is due, which a host would otherwise launch one by one at a few microseconds
// each). The graph is captured on first use per (energies, staging) and dropped whenever the
// context's step graphs are (any change of the set-up, tables, network or grids).
static int force_step_launch(nnpe_ctx* c, bool ev, float* xstage, float* fstage) {
  if (!c->fs_valid) {
    for (auto& g : c->fs_graph)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    c->fs_valid = true;
  }
  const int v = ev ? 1 : 0;
  if (c->fs_graph[v] && c->fs_xstage[v] != xstage) {
    cudaGraphExecDestroy(c->fs_graph[v]);
    c->fs_graph[v] = nullptr;
  }
  if (!c->fs_graph[v]) {
    cudaGraph_t g;
    NNPE_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = force_step_body(c, ev, xstage, fstage);
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return nnpe_fail(c, NNPE_ECUDA, std::string("force step capture: ") + cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&c->fs_graph[v], g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      c->fs_graph[v] = nullptr;
      return nnpe_fail(c, NNPE_ECUDA, std::string("force step graph: ") + cudaGetErrorString(ei));
    }
    c->fs_xstage[v] = xstage;
  }
  NNPE_CUDA(c, cudaGraphLaunch(c->fs_graph[v], c->stream));
  return 0;
}

int force_step_staged(nnpe_ctx* c, const float* x_host, float* f_host, double* erg, double* virial, float* xstage,
                      float* fstage, bool graph) {
  if (int rc = refuse_if_poisoned(c)) return rc;
  const int N = c->natom;
  if (!c->first_step_done && !c->force_step_init) {
    k_qm_to_pos<<<nblocks(N, 256), 256, 0, c->stream>>>(c->d_qm, c->d_pos, N);
    c->force_step_init = true;
  }
  const bool ev = erg || virial;
  NNPE_CUDA(c, cudaMemcpyAsync(xstage, x_host, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, c->stream));
  if (int rc = graph ? force_step_launch(c, ev, xstage, fstage) : force_step_body(c, ev, xstage, fstage)) return rc;
  if (ev) NNPE_CUDA(c, cudaMemcpyAsync(c->h_red, c->d_red, sizeof(double) * 2, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(f_host, fstage, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  if (ev) {
    if (erg) *erg = c->h_red[0];
    if (virial) *virial = c->h_red[1];
  }
  return NNPE_OK;
}

extern "C" int nnpe_force_step(nnpe_ctx* c, const float* x_host, float* f_host, double* erg, double* virial) {
  if (!c || !c->have_setup || !x_host || !f_host) return nnpe_fail(c, NNPE_EARG, "nnpe_force_step");
  cudaSetDevice(c->device);
  const int N = c->natom;
  if (!c->d_xstage) {
    NNPE_CUDA(c, dev_malloc(c, (void**)&c->d_xstage, sizeof(float) * 3 * N));
    NNPE_CUDA(c, dev_malloc(c, (void**)&c->d_fstage, sizeof(float) * 3 * N));
  }
  return force_step_staged(c, x_host, f_host, erg, virial, c->d_xstage, c->d_fstage, true);
}

extern "C" int nnpe_compute_forces(nnpe_ctx* c, int ev, double* erg, double* virial) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_compute_forces: not set up");
  if (int rc = refuse_if_poisoned(c)) return rc;
  cudaSetDevice(c->device);
  if (int rc = forces_enqueue(c, ev != 0)) return rc;
  if (ev) {
    if (int rc = energy_reduce_enqueue(c, 0)) return rc;
    NNPE_CUDA(c, cudaMemcpyAsync(c->h_red, c->d_red, sizeof(double) * 16, cudaMemcpyDeviceToHost, c->stream));
  }
  if (int rc = nnpe_sync_errors(c)) return rc;
  if (ev) {
    if (erg) *erg = c->h_red[0];
    if (virial) *virial = c->h_red[1];
  }
  return NNPE_OK;
}
