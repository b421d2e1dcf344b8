// List rebuild on the device: refold + cell binning, stable counting sort by cell, explicit
// periodic images, image sort, molecule images for the bonded terms, and the full Verlet list.
//
// Every kernel takes the device rebuild flag and returns at once when it is clear, so that one
// step is a fixed launch sequence (capturable in a CUDA graph) and the decision "is the list
// still valid" (NEIGHLIST::isvalid, neighlist.cpp:178-187) never round-trips to the host.
#include <algorithm>

#include "internal.cuh"

namespace {

__device__ __forceinline__ bool skip(const int* ctrl, bool cond) { return cond && ctrl[CTRL_REBUILD] == 0; }

__global__ void k_zero_counts(int* a, int* b, int n, const int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) { a[i] = 0; b[i] = 0; }
}

// LOCAL::refold_and_tag (environ.cpp:234-262): wrap x -= nearbyint(x*r_bl)*bl and bin.
__global__ void k_refold_bin(double4* __restrict__ xd, int* __restrict__ ctmp, int* __restrict__ slot,
                             int* __restrict__ ccount, int N, GridParams g, bool fp64, int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double4 x = xd[i];
  float xf, yf, zf;
  if (fp64) {
    const double bl = (double)g.bl, rbl = 1.0 / bl;
    x.x -= rint(x.x * rbl) * bl;
    x.y -= rint(x.y * rbl) * bl;
    x.z -= rint(x.z * rbl) * bl;
    xf = (float)x.x; yf = (float)x.y; zf = (float)x.z;
  } else {
    xf = (float)x.x; yf = (float)x.y; zf = (float)x.z;
    xf = fsub(xf, fmul(rintf(fmul(xf, g.r_bl)), g.bl));
    yf = fsub(yf, fmul(rintf(fmul(yf, g.r_bl)), g.bl));
    zf = fsub(zf, fmul(rintf(fmul(zf, g.r_bl)), g.bl));
    x.x = xf; x.y = yf; x.z = zf;
  }
  xd[i] = x;
  int c = cell_of(g, xf, yf, zf, ctrl + CTRL_ERR);
  ctmp[i] = c;
  slot[i] = atomicAdd(&ccount[c], 1);
}

// Exclusive scan of n counts by one block: start[k] = offset + sum(in[<k]), end[k] = start[k] + in[k].
__global__ void __launch_bounds__(1024) k_scan(const int* __restrict__ in, int n, int* __restrict__ start,
                                               int* __restrict__ end, int offset, int* total, const int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  // One block of 1024 threads over segments of 8192 values: each segment is loaded into shared
  // memory with coalesced reads, every thread scans 8 consecutive values there, the 1024 thread
  // totals are scanned with warp shuffles, and the results go back out with coalesced writes.
  constexpr int kPer = 8, kSeg = 1024 * kPer;
  __shared__ __align__(16) int buf[kSeg];
  __shared__ int warp_sums[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  int carry = offset;
  for (int seg = 0; seg < n; seg += kSeg) {
    const int m = min(kSeg, n - seg);
    for (int k = t; k < kSeg; k += 1024) buf[k] = k < m ? in[seg + k] : 0;
    __syncthreads();
    int4* mine = reinterpret_cast<int4*>(buf + t * kPer);
    const int4 a = mine[0], b = mine[1];
    const int local = a.x + a.y + a.z + a.w + b.x + b.y + b.z + b.w;
    int v = local;   // inclusive scan over the warp
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    if (lane == 31) warp_sums[w] = v;
    __syncthreads();
    if (w == 0) {
      int x = warp_sums[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += u;
      }
      warp_sums[lane] = x;
    }
    __syncthreads();
    int p0 = carry + v - local + (w ? warp_sums[w - 1] : 0);   // exclusive prefix of this thread's 8
    const int seg_total = warp_sums[31];
    int4 sa, sb;
    sa.x = p0; p0 += a.x; sa.y = p0; p0 += a.y; sa.z = p0; p0 += a.z; sa.w = p0; p0 += a.w;
    sb.x = p0; p0 += b.x; sb.y = p0; p0 += b.y; sb.z = p0; p0 += b.z; sb.w = p0;
    mine[0] = sa;
    mine[1] = sb;
    __syncthreads();
    for (int k = t; k < m; k += 1024) {
      const int sv = buf[k];
      start[seg + k] = sv;
      if (end) end[seg + k] = sv + in[seg + k];
    }
    carry += seg_total;
    __syncthreads();   // buf and warp_sums are reused by the next segment
  }
  if (t == 0 && total) *total = carry;
}

__global__ void k_scatter(const int* __restrict__ ctmp, const int* __restrict__ slot, const int* __restrict__ cstart,
                          int* __restrict__ perm, int N, int base, const int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  perm[cstart[ctmp[i]] - base + slot[i]] = i;
}

__global__ void k_gscatter(const int* __restrict__ gcell, const int* __restrict__ gslot, const int* __restrict__ gcstart,
                           int* __restrict__ perm, int Gcap, int base, const int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  const int ng = min(ctrl[CTRL_NGHOST], Gcap);
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  perm[gcstart[gcell[g]] - base + gslot[g]] = g;
}

// Within each cell, order entries by their previous index: together with the counting sort this
// is the stable sort of ENVIRON::sort / sort_ghost (environ.cpp:332-346, 384-389).
constexpr int kSortWarps = 4, kSortCap = 1024;
__global__ void __launch_bounds__(kSortWarps * 32) k_cell_sort(int* __restrict__ perm, const int* __restrict__ cstart,
                                                               const int* __restrict__ cend, int ncell, int base,
                                                               int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  __shared__ int buf[kSortWarps][kSortCap];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cidx = blockIdx.x * kSortWarps + w;
  if (cidx >= ncell) return;
  const int s = cstart[cidx] - base, n = cend[cidx] - cstart[cidx];
  if (n <= 1) return;
  if (n > kSortCap) {
    if (lane == 0) atomicOr(ctrl + CTRL_ERR, NNPE_DEV_CELL_OVERFLOW);
    return;
  }
  int* b = buf[w];
  for (int k = lane; k < n; k += 32) b[k] = perm[s + k];
  __syncwarp();
  for (int k = lane; k < n; k += 32) {
    const int v = b[k];
    int r = 0;
    for (int m = 0; m < n; ++m) r += b[m] < v;
    perm[s + r] = v;
  }
}

// Gather the per-atom arrays into the new order (scratch), then copy back with derived fields.
__global__ void k_gather(const int* __restrict__ perm, const double4* __restrict__ xd, const double4* __restrict__ vd,
                         const float4* __restrict__ acc, const int2* __restrict__ info, const int* __restrict__ aid,
                         const float2* __restrict__ qm, const int* __restrict__ ctmp, double4* __restrict__ sxd,
                         double4* __restrict__ svd, float4* __restrict__ sacc, int2* __restrict__ sinfo,
                         int* __restrict__ satom, float2* __restrict__ sqm, int* __restrict__ cell, int N,
                         const int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const int j = perm[k];
  sxd[k] = xd[j]; svd[k] = vd[j]; sacc[k] = acc[j]; sinfo[k] = info[j]; satom[k] = aid[j]; sqm[k] = qm[j];
  cell[k] = ctmp[j];
}

__global__ void k_copyback(const double4* __restrict__ sxd, const double4* __restrict__ svd, const float4* __restrict__ sacc,
                           const int2* __restrict__ sinfo, const int* __restrict__ satom, const float2* __restrict__ sqm,
                           double4* __restrict__ xd, double4* __restrict__ vd, float4* __restrict__ acc,
                           int2* __restrict__ info, int* __restrict__ aid, float2* __restrict__ qm,
                           float4* __restrict__ pos, int* __restrict__ sorted_of_id, int* __restrict__ molshift,
                           int* __restrict__ gcnt, int N, GridParams g, const int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const double4 x = sxd[k];
  const int a = satom[k];
  const float2 qq = sqm[k];
  xd[k] = x; vd[k] = svd[k]; acc[k] = sacc[k]; info[k] = sinfo[k]; aid[k] = a; qm[k] = qq;
  const float xf = (float)x.x, yf = (float)x.y, zf = (float)x.z;
  pos[k] = make_float4(xf, yf, zf, qq.x);
  sorted_of_id[a] = k;
  molshift[a] = 13;
  // number of periodic images of this atom (LOCAL::generate_ghost, environ.cpp:410-439)
  const int xs = xf > g.ghost_lim ? -1 : 0, xe = xf < -g.ghost_lim ? 1 : 0;
  const int ys = yf > g.ghost_lim ? -1 : 0, ye = yf < -g.ghost_lim ? 1 : 0;
  const int zs = zf > g.ghost_lim ? -1 : 0, ze = zf < -g.ghost_lim ? 1 : 0;
  int n = 0;
  if (xs != xe || ys != ye || zs != ze) n = (xe - xs + 1) * (ye - ys + 1) * (ze - zs + 1) - 1;
  gcnt[k] = n;
}

// Images in (owner, shift-loop) order, i.e. the order tidyup_ghost concatenates them
// (environ.cpp:157-176 over threads owning ascending index ranges), with their cells.
__global__ void k_ghost_emit(const float4* __restrict__ pos, const int* __restrict__ goff, int* __restrict__ gowner,
                             int* __restrict__ gshift, int* __restrict__ gcell, int* __restrict__ gslot,
                             int* __restrict__ gccount, int N, int Gcap, GridParams g, int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0 && ctrl[CTRL_NGHOST] > Gcap) atomicOr(ctrl + CTRL_ERR, NNPE_DEV_GHOST_OVERFLOW);
  if (k >= N) return;
  const float4 p = pos[k];
  const int xs = p.x > g.ghost_lim ? -1 : 0, xe = p.x < -g.ghost_lim ? 1 : 0;
  const int ys = p.y > g.ghost_lim ? -1 : 0, ye = p.y < -g.ghost_lim ? 1 : 0;
  const int zs = p.z > g.ghost_lim ? -1 : 0, ze = p.z < -g.ghost_lim ? 1 : 0;
  if (xs == xe && ys == ye && zs == ze) return;
  int o = goff[k];
  for (int ix = xs; ix <= xe; ++ix)
    for (int iy = ys; iy <= ye; ++iy)
      for (int iz = zs; iz <= ze; ++iz) {
        if (!ix && !iy && !iz) continue;
        const int gg = o++;
        if (gg >= Gcap) continue;
        const int code = (ix + 1) * 9 + (iy + 1) * 3 + (iz + 1);
        float s[3];
        shift_of(g, code, s);
        // ghost position x_owner + shift (environ.cpp:505-507)
        const int c = cell_of(g, fadd(p.x, s[0]), fadd(p.y, s[1]), fadd(p.z, s[2]), ctrl + CTRL_ERR);
        gowner[gg] = k;
        gshift[gg] = code;
        gcell[gg] = c;
        gslot[gg] = atomicAdd(&gccount[c], 1);
      }
}

// Sorted images: position, info, owner; molecule images for the bonded terms
// (update_ghost_and_info, environ.cpp:444-470).
__global__ void k_ghost_gather(const int* __restrict__ perm, const int* __restrict__ tgowner, const int* __restrict__ tgshift,
                               const int* __restrict__ tgcell, int* __restrict__ gowner, int* __restrict__ gshift,
                               float4* __restrict__ pos, int2* __restrict__ info, int* __restrict__ cell,
                               const int* __restrict__ aid, const int* __restrict__ sorted_of_id,
                               const int* __restrict__ mol_rep, int* __restrict__ molshift, int N, int Gcap,
                               GridParams g, const int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  const int ng = min(ctrl[CTRL_NGHOST], Gcap);
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ng) return;
  const int src = perm[k];
  const int owner = tgowner[src], code = tgshift[src];
  gowner[k] = owner;
  gshift[k] = code;
  float s[3];
  shift_of(g, code, s);
  const float4 p = pos[owner];
  const float4 q = make_float4(fadd(p.x, s[0]), fadd(p.y, s[1]), fadd(p.z, s[2]), p.w);
  pos[N + k] = q;
  const int2 inf = info[owner];
  info[N + k] = inf;
  cell[N + k] = tgcell[src];
  if (info_intra(inf) != 0) {
    const int rep = sorted_of_id[mol_rep[inf.x]];
    const float4 r = pos[rep];
    if (fabsf(fsub(q.x, r.x)) < g.h_bl && fabsf(fsub(q.y, r.y)) < g.h_bl && fabsf(fsub(q.z, r.z)) < g.h_bl)
      molshift[aid[owner]] = code;
  }
}

// NEIGHLIST::build<true> (neighlist.cpp:190-331). The atoms of one cell share its stencil rows, so
// one warp takes a group of up to kBuildGroup atoms of a cell, reads each candidate of the rows
// (cell, position, type) once, and tests it against every atom of the group. Each atom's row is
// appended exactly as a warp of its own would: real cells, then image cells, in stencil-row order
// and index order, ballot-compacted. A candidate is accepted without a distance test when its cell
// carries the no-check bit (NEGH_USE_INNERCUT; the candidate's cell is read only in rows that have
// such cells), else when rsq < (cutoff+skin)^2 in the reference's float sequence.
// kBuildWarpsPerCell warps share a cell's groups (group g goes to warp g mod that); at 6 Å cells
// (half of cutoff + skin) a cell holds about 22 atoms of water, so its groups usually run at once,
// and the register cap keeps 8 CTAs per SM.
constexpr int kBuildGroup = 4;
constexpr int kBuildWarpsPerCell = 6;
__global__ void __launch_bounds__(128, 8) k_build_list(const float4* __restrict__ pos, const int2* __restrict__ info,
                                                    const int* __restrict__ cell, const int* __restrict__ cstart,
                                                    const int* __restrict__ cend, const int* __restrict__ gcstart,
                                                    const int* __restrict__ gcend, const int4* __restrict__ rows,
                                                    const int* __restrict__ nrows, int maxrows,
                                                    const int* __restrict__ special, int nmax,
                                                    uint32_t* __restrict__ list, int* __restrict__ ncount,
                                                    float4* __restrict__ xbuild, int ncell, int cap, float cutsq,
                                                    int* ctrl, bool cond) {
  if (skip(ctrl, cond)) return;
  const int lane = threadIdx.x & 31;
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int ci = wid / kBuildWarpsPerCell;
  if (ci >= ncell) return;
  const int a0 = cstart[ci], a1 = cend[ci];
  const int nr = nrows[ci];
  const int4* R = rows + (size_t)ci * maxrows;
  const unsigned below = (1u << lane) - 1;
  for (int g0 = a0 + (wid % kBuildWarpsPerCell) * kBuildGroup; g0 < a1; g0 += kBuildWarpsPerCell * kBuildGroup) {
    const int na = min(kBuildGroup, a1 - g0);
    float xi[kBuildGroup], yi[kBuildGroup], zi[kBuildGroup];
    int mol[kBuildGroup], spo[kBuildGroup], cnt[kBuildGroup];
#pragma unroll
    for (int k = 0; k < kBuildGroup; ++k) {
      const int i = g0 + min(k, na - 1);
      const float4 x = pos[i];
      const int2 inf = info[i];
      xi[k] = x.x; yi[k] = x.y; zi[k] = x.z;
      mol[k] = inf.x;
      spo[k] = (info_moltype(inf) * nmax + info_intra(inf)) * nmax;
      cnt[k] = 0;
    }
    for (int pass = 0; pass < 2; ++pass) {
      for (int r = 0; r < nr; ++r) {
        const int4 row = R[r];
        const int j0 = pass ? gcstart[row.x] : cstart[row.x];
        const int j1 = pass ? gcend[row.y] : cend[row.y];
        for (int base = j0; base < j1; base += 32) {
          const int j = base + lane;
          const bool inr = j < j1;
          float4 xj = make_float4(0.f, 0.f, 0.f, 0.f);
          int2 infj = make_int2(-1, 0);
          bool nochk = false;
          if (inr) {
            if (row.z) nochk = (row.z >> (cell[j] - row.x)) & 1;
            xj = pos[j];
            infj = info[j];
          }
          const uint32_t ent = (uint32_t)j | ((uint32_t)info_type(infj) << 27);
#pragma unroll
          for (int k = 0; k < kBuildGroup; ++k) {
            if (k < na) {
              const bool ok = inr && (pass || j != g0 + k) &&
                              (nochk || rsq3(fsub(xi[k], xj.x), fsub(yi[k], xj.y), fsub(zi[k], xj.z)) < cutsq);
              const unsigned b = __ballot_sync(0xffffffffu, ok);
              if (ok) {
                const int sp = infj.x == mol[k] ? special[spo[k] + info_intra(infj)] : 0;
                const int idx = cnt[k] + __popc(b & below);
                if (idx < cap) list[(size_t)(g0 + k) * cap + idx] = ent | ((uint32_t)sp << 30);
              }
              cnt[k] += __popc(b);
            }
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kBuildGroup; ++k) {
      if (k < na && lane == 0) {
        ncount[g0 + k] = min(cnt[k], cap);
        xbuild[g0 + k] = make_float4(xi[k], yi[k], zi[k], pos[g0 + k].w);
        if (cnt[k] >= cap) atomicOr(ctrl + CTRL_ERR, NNPE_DEV_LIST_OVERFLOW);
      }
    }
  }
}

// update_ghost_pos<false> (environ.cpp:515-520) every step; after a rebuild it recomputes the
// same values. Thread 0 also retires the rebuild flag and counts the build (NEIGHLIST::nbuild).
__global__ void k_ghost_update(float4* __restrict__ pos, const int* __restrict__ gowner, const int* __restrict__ gshift,
                               int N, int Gcap, GridParams g, int* ctrl) {
  const int ng = min(ctrl[CTRL_NGHOST], Gcap);
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < ng) {
    float s[3];
    shift_of(g, gshift[k], s);
    const float4 p = pos[gowner[k]];
    pos[N + k] = make_float4(fadd(p.x, s[0]), fadd(p.y, s[1]), fadd(p.z, s[2]), p.w);
  }
}

__global__ void k_finish_rebuild(int* ctrl) {
  if (ctrl[CTRL_REBUILD]) {
    ctrl[CTRL_REBUILD] = 0;
    ctrl[CTRL_NBUILD] += 1;
    ctrl[CTRL_PRUNE] = 1;   // a new list: the pruned copy is made from it before the forces
    ctrl[CTRL_RESORT] = 1;  // a new order: the network's species lists follow it
  }
}

// isvalid: any atom displaced more than skin/2 since the last build (neighlist.cpp:178-187); with
// xprune, also more than prune_delta/2 since the last prune (the pruned copy is then stale).
__global__ void k_check_valid(const float4* __restrict__ pos, const float4* __restrict__ xbuild,
                              const float4* __restrict__ xprune, int N, float dx2, float pdx2, int* ctrl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float4 a = pos[i], b = xbuild[i];
  if (rsq3(fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)) > dx2) ctrl[CTRL_REBUILD] = 1;
  if (xprune) {
    const float4 p = xprune[i];
    if (rsq3(fsub(a.x, p.x), fsub(a.y, p.y), fsub(a.z, p.z)) > pdx2) ctrl[CTRL_PRUNE] = 1;
  }
}

// Dynamic pruning. The Verlet list holds every pair within cutoff + skin of the last build; most
// of its outer shell is beyond the force cutoff at any one step, yet the pair kernel evaluates
// every entry. When CTRL_PRUNE is set (a rebuild, or an atom displaced more than delta/2 since the
// last prune), this kernel copies each atom's row keeping the entries within cutoff + delta at the
// current positions, in list order, and records those positions. Until an atom moves delta/2, a
// pair beyond cutoff + delta then cannot come within the cutoff (each of its atoms moved less than
// delta/2), so the copy holds every pair the forces need. One warp per atom (grid-stride); without
// the flag every block returns at once. The last block to finish clears the flag, after every block
// has read it.
__global__ void __launch_bounds__(256) k_prune(const float4* __restrict__ pos, const uint32_t* __restrict__ list,
                                               const int* __restrict__ ncount, int cap, uint32_t* __restrict__ plist,
                                               int* __restrict__ pcount, float4* __restrict__ xprune, int N, float cutsq,
                                               int* ctrl) {
  if (*reinterpret_cast<volatile int*>(ctrl + CTRL_PRUNE) == 0) return;   // block-uniform
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += nw) {   // warp-uniform
    const float4 xi = pos[i];
    const uint32_t* row = list + (size_t)i * cap;
    uint32_t* out = plist + (size_t)i * cap;
    const int n = ncount[i];
    int cnt = 0;
    // software pipeline over 32-entry chunks: entries two chunks ahead and neighbour positions one
    // chunk ahead are in flight while a chunk is tested
    uint32_t e_nx = lane < n ? __ldg(row + lane) : 0u;
    uint32_t e_nx2 = lane + 32 < n ? __ldg(row + lane + 32) : 0u;
    float4 x_nx = lane < n ? __ldg(pos + (e_nx & NNPE_J_MASK)) : xi;
    for (int base = 0; base < n; base += 32) {
      const int k = base + lane;
      const uint32_t e = e_nx;
      const float4 xj = x_nx;
      e_nx = e_nx2;
      x_nx = k + 32 < n ? __ldg(pos + (e_nx & NNPE_J_MASK)) : xi;
      e_nx2 = k + 64 < n ? __ldg(row + k + 64) : 0u;
      const bool keep = k < n && rsq3(fsub(xi.x, xj.x), fsub(xi.y, xj.y), fsub(xi.z, xj.z)) < cutsq;
      const unsigned b = __ballot_sync(0xffffffffu, keep);
      if (keep) out[cnt + __popc(b & ((1u << lane) - 1))] = e;
      cnt += __popc(b);
    }
    if (lane == 0) {
      pcount[i] = cnt;
      xprune[i] = xi;
    }
  }
  prune_pass_done(ctrl);
}

}  // namespace

int rebuild_enqueue(nnpe_ctx* c, bool cond) {
  const int N = c->natom, G = c->Gcap, NG = c->grid.num_grid;
  cudaStream_t st = c->stream;
  const GridParams g = c->grid;
  int* ctrl = c->d_ctrl;
  const int T = 256;
  k_zero_counts<<<nblocks(NG, T), T, 0, st>>>(c->d_ccount, c->d_gccount, NG, ctrl, cond);
  k_refold_bin<<<nblocks(N, T), T, 0, st>>>(c->d_xd, c->d_ctmp, c->d_slot, c->d_ccount, N, g, c->fp64_state, ctrl, cond);
  k_scan<<<1, 1024, 0, st>>>(c->d_ccount, NG, c->d_cstart, c->d_cend, 0, nullptr, ctrl, cond);
  k_scatter<<<nblocks(N, T), T, 0, st>>>(c->d_ctmp, c->d_slot, c->d_cstart, c->d_perm, N, 0, ctrl, cond);
  k_cell_sort<<<nblocks(NG, kSortWarps), kSortWarps * 32, 0, st>>>(c->d_perm, c->d_cstart, c->d_cend, NG, 0, ctrl, cond);
  k_gather<<<nblocks(N, T), T, 0, st>>>(c->d_perm, c->d_xd, c->d_vd, c->d_acc, c->d_info, c->d_atom_id, c->d_qm, c->d_ctmp,
                                        c->d_sxd, c->d_svd, c->d_sacc, c->d_sinfo, c->d_satom, c->d_sqm, c->d_cell, N, ctrl, cond);
  k_copyback<<<nblocks(N, T), T, 0, st>>>(c->d_sxd, c->d_svd, c->d_sacc, c->d_sinfo, c->d_satom, c->d_sqm, c->d_xd, c->d_vd,
                                          c->d_acc, c->d_info, c->d_atom_id, c->d_qm, c->d_pos, c->d_sorted_of_id,
                                          c->d_molshift, c->d_gcnt, N, g, ctrl, cond);
  k_scan<<<1, 1024, 0, st>>>(c->d_gcnt, N, c->d_goff, nullptr, 0, ctrl + CTRL_NGHOST, ctrl, cond);
  k_ghost_emit<<<nblocks(N, T), T, 0, st>>>(c->d_pos, c->d_goff, c->d_gtmp_owner, c->d_gtmp_shift, c->d_gtmp_cell,
                                            c->d_gtmp_slot, c->d_gccount, N, G, g, ctrl, cond);
  k_scan<<<1, 1024, 0, st>>>(c->d_gccount, NG, c->d_gcstart, c->d_gcend, N, nullptr, ctrl, cond);
  k_gscatter<<<nblocks(G, T), T, 0, st>>>(c->d_gtmp_cell, c->d_gtmp_slot, c->d_gcstart, c->d_perm, G, N, ctrl, cond);
  k_cell_sort<<<nblocks(NG, kSortWarps), kSortWarps * 32, 0, st>>>(c->d_perm, c->d_gcstart, c->d_gcend, NG, N, ctrl, cond);
  k_ghost_gather<<<nblocks(G, T), T, 0, st>>>(c->d_perm, c->d_gtmp_owner, c->d_gtmp_shift, c->d_gtmp_cell, c->d_gowner,
                                              c->d_gshift, c->d_pos, c->d_info, c->d_cell, c->d_atom_id, c->d_sorted_of_id,
                                              c->d_mol_rep, c->d_molshift, N, G, g, ctrl, cond);
  const float cs = c->pair_cutoff + c->skin;
  k_build_list<<<nblocks((long)NG * kBuildWarpsPerCell * 32, 128), 128, 0, st>>>(
      c->d_pos, c->d_info, c->d_cell, c->d_cstart, c->d_cend, c->d_gcstart, c->d_gcend, c->st_pair.rows, c->st_pair.nrows,
      c->st_pair.maxrows, c->d_special, c->nmax, c->d_list, c->d_ncount, c->d_xbuild, NG, c->cap, cs * cs, ctrl, cond);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

bool prune_active(const nnpe_ctx* c) { return c->d_plist && c->prune_delta > 0.f && c->prune_delta < c->skin; }
const uint32_t* force_list(const nnpe_ctx* c) { return prune_active(c) ? c->d_plist : c->d_list; }
const int* force_count(const nnpe_ctx* c) { return prune_active(c) ? c->d_pcount : c->d_ncount; }
float prune_dx2(const nnpe_ctx* c) {
  const float h = 0.5f * c->prune_delta;
  return h * h;
}
float nnp_cutoff(nnpe_ctx* c);   // nnp.cu
float prune_cutsq(const nnpe_ctx* c) {
  const float rc = std::max(c->pair_cutoff, c->nnp ? nnp_cutoff(const_cast<nnpe_ctx*>(c)) : 0.f) + c->prune_delta;
  return rc * rc;
}
bool prune_in_pair(const nnpe_ctx* c) { return prune_active(c) && c->pair_on && c->d_table; }

// With pruning on, the pruned copy of the list, remade on the device when CTRL_PRUNE is set. It
// follows every ghost update (the images must hold this step's positions), so that every force
// evaluation reads a current copy; when the pair kernel runs in the force evaluation, that kernel
// remakes the copy in its own pass over the full list instead (prune_in_pair).
static void prune_enqueue(nnpe_ctx* c) {
  if (!prune_active(c) || prune_in_pair(c)) return;
  const int blocks = std::max(1, std::min(nblocks((long)c->natom * 32, 256), 8 * nnpe_sm_count(c->device)));
  k_prune<<<blocks, 256, 0, c->stream>>>(c->d_pos, c->d_list, c->d_ncount, c->cap, c->d_plist, c->d_pcount, c->d_xprune,
                                         c->natom, prune_cutsq(c), c->d_ctrl);
}

// The ghost images of this step's positions, the end of a rebuild and the pruned copy of the list.
int ghost_update_enqueue(nnpe_ctx* c, bool) {
  k_ghost_update<<<nblocks(c->Gcap, 256), 256, 0, c->stream>>>(c->d_pos, c->d_gowner, c->d_gshift, c->natom, c->Gcap,
                                                               c->grid, c->d_ctrl);
  k_finish_rebuild<<<1, 1, 0, c->stream>>>(c->d_ctrl);
  prune_enqueue(c);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int check_valid_enqueue(nnpe_ctx* c) {
  const float h = c->skin / 2;
  k_check_valid<<<nblocks(c->natom, 256), 256, 0, c->stream>>>(c->d_pos, c->d_xbuild, prune_active(c) ? c->d_xprune : nullptr,
                                                               c->natom, h * h, prune_dx2(c), c->d_ctrl);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

static int sync_errors(nnpe_ctx* c) {
  NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  const int e = c->h_ctrl[CTRL_ERR];
  if (e & NNPE_DEV_POISONED) c->poisoned = true;
  if (c->poisoned)
    return nnpe_fail(c, NNPE_ETIMEOUT, "a device wait gave up with copies in flight: the context refuses work until nnpe_setup");
  if (e & NNPE_DEV_TIMEOUT) return nnpe_fail(c, NNPE_ETIMEOUT, "a bounded device wait gave up");
  if (e & NNPE_DEV_LIST_OVERFLOW) return nnpe_fail(c, NNPE_EOVERFLOW, "nei_list overflow");
  if (e & NNPE_DEV_GHOST_OVERFLOW) return nnpe_fail(c, NNPE_EOVERFLOW, "ghost overflow");
  if (e & NNPE_DEV_CELL_OVERFLOW) return nnpe_fail(c, NNPE_EOVERFLOW, "cell overflow in sort");
  if (e & NNPE_DEV_CELL_RANGE) return nnpe_fail(c, NNPE_ERANGE, "atom outside the cell grid");
  return 0;
}

int nnpe_sync_errors(nnpe_ctx* c) { return sync_errors(c); }

extern "C" int nnpe_list_build(nnpe_ctx* c) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_list_build: not set up");
  cudaSetDevice(c->device);
  int one = 1;
  NNPE_CUDA(c, cudaMemcpyAsync(c->d_ctrl + CTRL_REBUILD, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  if (int rc = rebuild_enqueue(c, true)) return rc;
  if (int rc = ghost_update_enqueue(c, true)) return rc;
  return sync_errors(c);
}

extern "C" int nnpe_list_isvalid(nnpe_ctx* c, int* valid) {
  if (!c || !c->have_setup || !valid) return nnpe_fail(c, NNPE_EARG, "nnpe_list_isvalid");
  cudaSetDevice(c->device);
  NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  if (c->h_ctrl[CTRL_REBUILD]) { *valid = 0; return NNPE_OK; }
  if (int rc = check_valid_enqueue(c)) return rc;
  NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  *valid = c->h_ctrl[CTRL_REBUILD] ? 0 : 1;
  return NNPE_OK;
}

extern "C" int nnpe_ghost_update(nnpe_ctx* c) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_ghost_update");
  k_ghost_update<<<nblocks(c->Gcap, 256), 256, 0, c->stream>>>(c->d_pos, c->d_gowner, c->d_gshift, c->natom, c->Gcap,
                                                               c->grid, c->d_ctrl);
  prune_enqueue(c);
  NNPE_CHECK_LAUNCH(c);
  return NNPE_OK;
}

// ENVIRON::verify_grid (environ.cpp:638-683) on host copies of a cell sort: the real atoms fill
// the cells in cell order from index 0 and the images from index natom, each cell's range starts
// where the previous one ends, and every entry's stored cell is both the cell whose range holds it
// and the cell of its position in the reference's float arithmetic ((int)((g_offset + x) * g_rdx)
// per axis, environ.cpp:252-260). Returns NNPE_ERANGE at the first violation, with its cell or
// entry index in *bad and a code in *what (1 bounds, 2 contiguity, 3 reversed range, 4 stored cell,
// 5 position's cell).
extern "C" int nnpe_verify_grid_arrays(int natom, int nimage, int num_gx, float g_offset, float g_rdx,
                                       const int* cstart, const int* cend, const int* gcstart, const int* gcend,
                                       const int* cell, const float* pos4, int64_t* bad, int* what) {
  if (natom <= 0 || nimage < 0 || num_gx <= 0 || !cstart || !cend || !gcstart || !gcend || !cell || !pos4)
    return NNPE_EARG;
  const int NG = num_gx * num_gx * num_gx, ntot = natom + nimage;
  auto fail = [&](int code, int64_t idx) {
    if (bad) *bad = idx;
    if (what) *what = code;
    return (int)NNPE_ERANGE;
  };
  auto axis = [&](float x) {
    const float s = g_offset + x;   // rounded, then multiplied and rounded: the device's fadd, fmul
    return (int)(s * g_rdx);
  };
  if (cstart[0] != 0 || gcstart[0] != natom || cend[NG - 1] != natom || gcend[NG - 1] != ntot) return fail(1, 0);
  for (int i = 1; i < NG; ++i)
    if (cstart[i] != cend[i - 1] || gcstart[i] != gcend[i - 1]) return fail(2, i);
  for (int i = 0; i < NG; ++i) {
    for (int pass = 0; pass < 2; ++pass) {
      const int j0 = pass ? gcstart[i] : cstart[i], j1 = pass ? gcend[i] : cend[i];
      if (j0 > j1 || j0 < 0 || j1 > ntot) return fail(3, i);
      for (int j = j0; j < j1; ++j) {
        if (cell[j] != i) return fail(4, j);
        const float* x = pos4 + 4 * (size_t)j;
        if (axis(x[0]) * num_gx * num_gx + axis(x[1]) * num_gx + axis(x[2]) != i) return fail(5, j);
      }
    }
  }
  if (bad) *bad = -1;
  if (what) *what = 0;
  return NNPE_OK;
}

// The same check on the context's own cell sort (copied from the device; synchronises its stream).
// Positions move between list builds, so it is meaningful right after a build (nnpe_list_build).
extern "C" int nnpe_verify_grid(nnpe_ctx* c) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_verify_grid: not set up");
  if (int rc = sync_errors(c)) return rc;
  const int N = c->natom, NG = c->grid.num_grid;
  NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  const int ng = std::min(c->h_ctrl[CTRL_NGHOST], c->Gcap), ntot = N + ng;
  std::vector<int> cs(NG), ce(NG), gs(NG), ge(NG), cell(ntot);
  std::vector<float4> pos(ntot);
  NNPE_CUDA(c, cudaMemcpyAsync(cs.data(), c->d_cstart, sizeof(int) * NG, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(ce.data(), c->d_cend, sizeof(int) * NG, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(gs.data(), c->d_gcstart, sizeof(int) * NG, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(ge.data(), c->d_gcend, sizeof(int) * NG, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(cell.data(), c->d_cell, sizeof(int) * ntot, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaMemcpyAsync(pos.data(), c->d_pos, sizeof(float4) * ntot, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  int64_t bad = -1;
  int what = 0;
  const int rc = nnpe_verify_grid_arrays(N, ng, c->grid.num_gx, c->grid.g_offset, c->grid.g_rdx, cs.data(), ce.data(),
                                         gs.data(), ge.data(), cell.data(), reinterpret_cast<const float*>(pos.data()),
                                         &bad, &what);
  if (rc) return nnpe_fail(c, rc, "nnpe_verify_grid: violation " + std::to_string(what) + " at " + std::to_string(bad));
  return NNPE_OK;
}
