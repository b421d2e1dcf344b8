// Internal definitions of libnnpe.so: the per-system context resident in HBM and the device
// helpers shared by the kernels.
//
// HBM layout of one system (sorted order = real atoms sorted by cell, then periodic images
// sorted by cell, as ENVIRON::sort/sort_ghost leave them, environ.cpp:303-399):
//   pos   float4 [N+Gcap]  x, y, z (FP32 force-field coordinates) and charge q
//   info  int2   [N+Gcap]  molecule id, packed (type | intra<<8 | moltype<<16)
//   cell  int    [N+Gcap]  grid cell of the entry
//   xd,vd double4[N]       master position/velocity (FP64; float-exact in FP32 mode)
//   acc   float4 [N]       acceleration (VERLET's f after updateV), frc float4 [N] forces
//   list  uint32 [N*cap]   full Verlet list, row per atom: j | type_j<<27 | special<<30
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/nnpe.h"

#define NNPE_MAX_TYPES 8
#define NNPE_J_MASK 0x07FFFFFFu
#define NNPE_MAX_ROW 32

// control words in device memory (ctx->d_ctrl)
enum {
  CTRL_NGHOST = 0,
  CTRL_REBUILD = 1,
  CTRL_ERR = 2,
  CTRL_NBUILD = 3,
  CTRL_STEP = 4,
  CTRL_NLOG = 5,
  CTRL_PRUNE = 6,        // the pruned list is stale: set by a rebuild or a displacement past delta/2
  CTRL_PRUNE_DONE = 7,   // blocks of k_prune that finished (the last one clears CTRL_PRUNE)
  CTRL_NPRUNE = 8,       // prunes so far
  CTRL_RESORT = 9,       // the sorted order changed (a rebuild, or a new network): species lists are stale
  CTRL_RESORT_DONE = 10, // blocks of k_species that finished (the last one clears CTRL_RESORT)
  CTRL_WORDS = 12
};

struct GridParams {
  float bl, r_bl, h_bl, m_bl;       // ENVIRON::set_bl (environ.h:105)
  float g_dx, g_rdx, g_offset;      // ENVIRON::init_grid (environ.cpp:143-155)
  float ghost_lim;                  // LOCAL::set_ghost_lim (environ.h:142)
  int num_gx, num_gxsq, num_grid;
};

struct Stencil {
  int4* rows = nullptr;   // [num_grid*maxrows] (first cell, last cell, no-check bits, 0)
  int* nrows = nullptr;   // [num_grid]
  int maxrows = 0;
  float cut = 0;          // cutoff+skin it was built for
};

struct LogRec {
  double erg, virial, ekin, erg_nnp, erg_exp;
  int step, nbuild, pad0, pad1;
};

struct NnpModel;   // network term (nnp.cu)
struct RmdfState;  // structure-factor refinement (rmdf.cu)
struct SqdState;   // direct S(q) over reciprocal lattice vectors (sqd.cu)

struct nnpe_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  // ---- system (host copies, atom-id order) ----
  int natom = 0, ntype = 0, npair = 0, nmol = 0, nmoltype = 0, nmax = 0;
  double bl = 0;
  std::vector<int> h_typ, h_mol_id, h_intra, h_amoltype, h_special, h_mol_rep;
  std::vector<float> h_mass, h_q;
  std::vector<int> top_bonds, top_angles, top_dihs;   // expanded topology read with the system
  // ---- setup ----
  bool have_system = false, have_setup = false, first_step_done = false;
  bool poisoned = false;   // NNPE_DEV_POISONED seen: no further work until nnpe_setup
  float pair_cutoff = 10, skin = 2, gr_cutoff = 10, comm_cutoff = 12;
  int cap = 2048;
  GridParams grid{};
  Stencil st_pair, st_gr;
  // ---- pair table ----
  int nbin = 0;
  bool pair_on = true;
  bool exact_forces = false;   // pair fpair in the reference's exact float sequence
  float2* d_table = nullptr;   // [npair][nbin+1] (F/r, U)
  // ---- bonded ----
  int nbond = 0, nangle = 0, ndih = 0;
  int nbtyp = 0, natyp = 0, ndtyp = 0;
  int4* d_bond = nullptr;      // per term: type, atoms (atom ids)
  int4* d_angle = nullptr;
  int* d_dih = nullptr;        // 5 ints per term
  float4* d_bcoef = nullptr;
  float4* d_acoef = nullptr;
  float4* d_dcoef = nullptr;
  int* d_mol_terms = nullptr;  // per molecule: [bond start, angle start, dih start] (nmol+1)*3
  int* d_mol_atoms = nullptr;  // per molecule: first atom id, count (atom ids contiguous per molecule)
  // ---- verlet / thermostat ----
  double dt = 1.0;
  bool fp64_state = true;
  int thermo_kind = 0, thermo_interval = 0;
  double t_start = 300, t_end = 300, thermo_frac = 0.1;
  uint64_t seed = 1;
  int total_steps_hint = 0;
  // ---- device state ----
  int Gcap = 0;
  double4 *d_xd = nullptr, *d_vd = nullptr;
  float4 *d_acc = nullptr, *d_frc = nullptr, *d_pos = nullptr, *d_xbuild = nullptr;
  int2* d_info = nullptr;
  int* d_cell = nullptr;
  int* d_atom_id = nullptr;
  int* d_sorted_of_id = nullptr;
  float2* d_qm = nullptr;      // (q, 1/m) per sorted atom
  int *d_gowner = nullptr, *d_gshift = nullptr;
  int* d_molshift = nullptr;   // by atom id
  int* d_mol_rep = nullptr;    // by molecule: atom id of the representative
  int* d_special = nullptr;
  int* d_pairtype = nullptr;
  // cells
  int *d_ccount = nullptr, *d_cstart = nullptr, *d_cend = nullptr;
  int *d_gccount = nullptr, *d_gcstart = nullptr, *d_gcend = nullptr;
  // rebuild scratch
  int *d_slot = nullptr, *d_ctmp = nullptr, *d_perm = nullptr, *d_gcnt = nullptr, *d_goff = nullptr;
  int *d_gtmp_owner = nullptr, *d_gtmp_shift = nullptr, *d_gtmp_cell = nullptr, *d_gtmp_slot = nullptr;
  double4 *d_sxd = nullptr, *d_svd = nullptr;
  float4* d_sacc = nullptr;
  int2* d_sinfo = nullptr;
  int* d_satom = nullptr;
  float2* d_sqm = nullptr;
  // list
  uint32_t* d_list = nullptr;
  int* d_ncount = nullptr;
  // dynamically pruned copy of the list (the pairs within the force cutoff + prune_delta at the
  // last prune) and the positions at that prune; the pair and network kernels read it while no
  // atom has moved prune_delta/2 since (prune_delta <= 0 or >= skin: off, they read the full list)
  uint32_t* d_plist = nullptr;
  int* d_pcount = nullptr;
  float4* d_xprune = nullptr;
  float prune_delta = 0.5f;
  // energies
  double *d_eatom = nullptr, *d_watom = nullptr, *d_kin = nullptr;   // per atom
  double *d_emol = nullptr, *d_wmol = nullptr;                         // per molecule
  double* d_red = nullptr;       // reduction outputs [8]
  double* d_red_part = nullptr;  // per-block partial sums of the energy reduction [256][4]
  LogRec* d_log = nullptr;
  int log_cap = 0;
  int* d_ctrl = nullptr;
  int* h_ctrl = nullptr;         // pinned
  double* h_red = nullptr;       // pinned
  // g(r)
  int gr_nbin_inner = 0, gr_nbin = 0, gr_nq = 0, gr_interval = 0, gr_interval_long = 0;
  float gr_dr = 0, gr_r_dr = 0, gr_rmaxsq = 0, gr_rmaxsq_inner = 0;
  double gr_qmax = 0;
  unsigned long long *d_gr_counts = nullptr, *d_gr_counts_inner = nullptr;
  double *d_gr = nullptr, *d_sq = nullptr, *d_gr_norm = nullptr, *d_qq = nullptr;
  int gr_tallied = -1;           // 0/1 = which tally is current
  // host-buffer force evaluation staging
  float *d_xstage = nullptr, *d_fstage = nullptr;
  bool force_step_init = false;
  // network term
  NnpModel* nnp = nullptr;
  // RMDF refinement of the pair table (d_red[4] holds the last erg_exp)
  RmdfState* rmdf = nullptr;
  SqdState* sqd = nullptr;
  // device bytes held by this context (dev_malloc / dev_free)
  int64_t dev_bytes = 0;
  // CUDA graphs of the step variants
  cudaGraphExec_t graph_exec[16] = {};
  bool graph_valid = false;
  // CUDA graphs of the host-owned force step (without / with energies), keyed by their staging
  float* fs_xstage[2] = {};
  cudaGraphExec_t fs_graph[2] = {};
  bool fs_valid = false;
};

// ---------------------------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------------------------
int nnpe_fail(nnpe_ctx* c, int code, const std::string& msg);
#define NNPE_CUDA(ctx, call)                                                                      \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return nnpe_fail((ctx), NNPE_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)
#define NNPE_CHECK_LAUNCH(ctx) NNPE_CUDA(ctx, cudaGetLastError())

// ---------------------------------------------------------------------------------------------
// exact single-precision arithmetic (no contraction), the reference's float sequences
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
// sqr(a)+sqr(b)+sqr(c) evaluated left to right without FMA (mathlib.h:4; neighlist.cpp:260)
__device__ __forceinline__ float rsq3(float dx, float dy, float dz) {
  return fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
}
// cell index of environ.cpp:252-260: (int)((g_offset + x) * g_rdx) per axis
__device__ __forceinline__ int cell_axis(const GridParams& g, float x) {
  return __float2int_rz(fmul(fadd(g.g_offset, x), g.g_rdx));
}
__device__ __forceinline__ int cell_of(const GridParams& g, float x, float y, float z, int* err) {
  int ix = cell_axis(g, x), iy = cell_axis(g, y), iz = cell_axis(g, z);
  if (ix < 0 || iy < 0 || iz < 0 || ix >= g.num_gx || iy >= g.num_gx || iz >= g.num_gx) {
    atomicOr(err, NNPE_DEV_CELL_RANGE);
    ix = min(max(ix, 0), g.num_gx - 1);
    iy = min(max(iy, 0), g.num_gx - 1);
    iz = min(max(iz, 0), g.num_gx - 1);
  }
  return ix * g.num_gxsq + iy * g.num_gx + iz;
}
__device__ __forceinline__ void shift_of(const GridParams& g, int code, float* s) {
  int c0 = code / 9 - 1, c1 = (code / 3) % 3 - 1, c2 = code % 3 - 1;
  s[0] = c0 == 0 ? 0.f : (c0 > 0 ? g.bl : g.m_bl);
  s[1] = c1 == 0 ? 0.f : (c1 > 0 ? g.bl : g.m_bl);
  s[2] = c2 == 0 ? 0.f : (c2 > 0 ? g.bl : g.m_bl);
}
__device__ __forceinline__ int info_type(int2 info) { return info.y & 0xFF; }
__device__ __forceinline__ int info_intra(int2 info) { return (info.y >> 8) & 0xFF; }
__device__ __forceinline__ int info_moltype(int2 info) { return info.y >> 16; }

// ---------------------------------------------------------------------------------------------
// host-side launch helpers shared across translation units
// ---------------------------------------------------------------------------------------------
static inline int nblocks(long n, int threads) { return (int)((n + threads - 1) / threads); }
int nnpe_sm_count(int device);

// internal entry points implemented in the kernel files
int rebuild_enqueue(nnpe_ctx* c, bool conditional);
int ghost_update_enqueue(nnpe_ctx* c, bool conditional);
int forces_enqueue(nnpe_ctx* c, bool ev);
int energy_reduce_enqueue(nnpe_ctx* c, int nlog_slot_from_device);
int verlet_x_enqueue(nnpe_ctx* c, double dt_override, bool check_valid);
int verlet_v_enqueue(nnpe_ctx* c, bool kinetic);
int thermostat_enqueue(nnpe_ctx* c);
int gr_tally_enqueue(nnpe_ctx* c, int inner);
int alloc_state(nnpe_ctx* c);
int build_stencil_host(nnpe_ctx* c, float cutoff, int max_nbin, Stencil* out);
int nnp_forces_enqueue(nnpe_ctx* c, bool ev, bool filter6 = true);
// Dynamic pruning of the list (rebuild.cu). The pair and network kernels read force_list() /
// force_count(): the pruned copy while pruning is on, else the full list.
bool prune_active(const nnpe_ctx* c);
const uint32_t* force_list(const nnpe_ctx* c);
const int* force_count(const nnpe_ctx* c);
float prune_dx2(const nnpe_ctx* c);     // (prune_delta/2)^2, the displacement that makes the copy stale
float prune_cutsq(const nnpe_ctx* c);   // (max(pair, network cutoff) + prune_delta)^2, what the copy keeps
// The pair kernel remakes the copy itself in the pass that reads the full list (when it runs in
// the force evaluation); else a separate pass after the ghost update does.
bool prune_in_pair(const nnpe_ctx* c);
// End of a pass that remade the pruned copy (CTRL_PRUNE was set at its start, block-uniformly):
// the last block to finish clears the request, after every block has read it.
static __device__ __forceinline__ void prune_pass_done(int* ctrl) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(reinterpret_cast<unsigned*>(ctrl + CTRL_PRUNE_DONE), 1u) == gridDim.x - 1) {
      ctrl[CTRL_PRUNE] = 0;
      ctrl[CTRL_PRUNE_DONE] = 0;
      ctrl[CTRL_NPRUNE] += 1;
    }
  }
}
// The host-positions force step (nnpe_force_step) with its staging buffers given by the caller:
// xstage and fstage hold at least 3 * natom floats each on the context's device. graph: launch the
// device part as the context's cached CUDA graph (else kernel by kernel).
int force_step_staged(nnpe_ctx* c, const float* x_host, float* f_host, double* erg, double* virial, float* xstage,
                      float* fstage, bool graph);
// Resolves the device address of the allocation-free step's static staging on c's device (loading
// the module that holds it); nnpe_setup calls it so that later steps load and reserve nothing.
int noalloc_stage_prepare(nnpe_ctx* c);
// A context that saw NNPE_DEV_POISONED refuses work until nnpe_setup.
int refuse_if_poisoned(nnpe_ctx* c);
int nnpe_bonded_coefs(nnpe_ctx* c, const float* bcoef, const float* acoef, const float* dcoef);
void nnp_free(nnpe_ctx* c);
// Device allocations of a context go through these two, which keep the context's byte count
// (nnpe_ctx::dev_bytes) for the serving loop's memory ledger.
cudaError_t dev_malloc(nnpe_ctx* c, void** p, size_t bytes);
void dev_free(void* p);
void rmdf_free(nnpe_ctx* c);
void sqd_free(nnpe_ctx* c);
