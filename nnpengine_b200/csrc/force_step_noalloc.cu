// Allocation-free force step: nnpe_force_step with its host <-> device staging of positions and
// forces in a statically reserved device array instead of buffers that the library allocates on
// first use. It has no counterpart in the reference (whose force step runs on host memory).
//
// Who needs it: a host run loop whose process reserves the device's memory up front for its own
// allocator, where an allocation by the library fails or escapes that allocator's accounting; and
// a loop that keeps other streams busy, where the implicit synchronisation that a device memory
// allocation brings between streams is not acceptable. Such a caller cannot let the first force
// step call cudaMalloc, so this entry point never allocates: the staging lives in g_stage below,
// which every GPU that loads the library holds until the process exits.
//
// The first call on a device looks up the device address of g_stage (cudaGetSymbolAddress, with
// that device current) and keeps it; make that first call before any stream capture. All
// contexts on one device share g_stage, so calls that overlap in time race on it.
#include <mutex>

#include "internal.cuh"

int check_valid_enqueue(nnpe_ctx* c);

namespace {

// Largest system the static staging holds: positions in and forces out, 3 floats per atom each,
// 3 MiB in all.
constexpr int kStageMaxAtoms = 131072;
__device__ __align__(256) float g_stage[2 * 3 * kStageMaxAtoms];

constexpr int kMaxDevices = 64;
std::mutex g_stage_mu;
float* g_stage_addr[kMaxDevices] = {};

// Device address of g_stage on c's device (current when called), looked up once per device.
int stage_address(nnpe_ctx* c, float** out) {
  if (c->device < 0 || c->device >= kMaxDevices)
    return nnpe_fail(c, NNPE_EARG, "nnpe_force_step_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_stage_mu);
  if (!g_stage_addr[c->device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_stage);
    if (e != cudaSuccess)
      return nnpe_fail(c, NNPE_ECUDA, std::string("nnpe_force_step_noalloc: cudaGetSymbolAddress: ") +
                                          cudaGetErrorString(e));
    g_stage_addr[c->device] = static_cast<float*>(p);
  }
  *out = g_stage_addr[c->device];
  return NNPE_OK;
}

// positions in atom-id order (host layout, staged) -> sorted master/FP32 coordinates
__global__ void k_stage_scatter_positions(const float* __restrict__ x, const int* __restrict__ aid, double4* __restrict__ xd,
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
// sorted forces -> atom-id order (staged)
__global__ void k_stage_gather_forces(const float4* __restrict__ frc, const int* __restrict__ aid,
                                      float* __restrict__ f, int N) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const int a = aid[k];
  const float4 v = frc[k];
  f[3 * a] = v.x; f[3 * a + 1] = v.y; f[3 * a + 2] = v.z;
}
__global__ void k_stage_charges(const float2* __restrict__ qm, float4* __restrict__ pos, int N) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) pos[k].w = qm[k].x;
}

}  // namespace

// The same step as nnpe_force_step (list check and rebuild on the device, forces, optional FP64
// energy and virial), with positions staged in g_stage[0, 3N) and forces in g_stage[3N', ...).
// Nothing in g_stage has to start at zero: every call overwrites the 3N floats of each half that
// it reads (the positions by the host copy, the forces by the gather, aid being a permutation).
extern "C" int nnpe_force_step_noalloc(nnpe_ctx* c, const float* x_host, float* f_host, double* erg,
                                       double* virial) {
  if (!c) return NNPE_EARG;
  if (c->natom > kStageMaxAtoms)
    return nnpe_fail(c, NNPE_EARG, "nnpe_force_step_noalloc: " + std::to_string(c->natom) +
                                       " atoms exceed the static staging limit of " +
                                       std::to_string(kStageMaxAtoms) + " atoms");
  if (!c->have_setup || !x_host || !f_host) return nnpe_fail(c, NNPE_EARG, "nnpe_force_step_noalloc");
  NNPE_CUDA(c, cudaSetDevice(c->device));
  float* stage = nullptr;
  if (int rc = stage_address(c, &stage)) return rc;
  float* xstage = stage;
  float* fstage = stage + 3 * kStageMaxAtoms;
  const int N = c->natom;
  if (!c->first_step_done && !c->force_step_init) {
    k_stage_charges<<<nblocks(N, 256), 256, 0, c->stream>>>(c->d_qm, c->d_pos, N);
    c->force_step_init = true;
  }
  NNPE_CUDA(c, cudaMemcpyAsync(xstage, x_host, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, c->stream));
  k_stage_scatter_positions<<<nblocks(N, 256), 256, 0, c->stream>>>(xstage, c->d_atom_id, c->d_xd, c->d_pos, N, (double)c->grid.bl, c->fp64_state);
  if (int rc = check_valid_enqueue(c)) return rc;
  if (int rc = rebuild_enqueue(c, true)) return rc;
  if (int rc = ghost_update_enqueue(c, true)) return rc;
  const bool ev = erg || virial;
  if (int rc = forces_enqueue(c, ev)) return rc;
  if (ev) {
    if (int rc = energy_reduce_enqueue(c, 0)) return rc;
    NNPE_CUDA(c, cudaMemcpyAsync(c->h_red, c->d_red, sizeof(double) * 2, cudaMemcpyDeviceToHost, c->stream));
  }
  k_stage_gather_forces<<<nblocks(N, 256), 256, 0, c->stream>>>(c->d_frc, c->d_atom_id, fstage, N);
  NNPE_CUDA(c, cudaMemcpyAsync(f_host, fstage, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  if (ev) {
    if (erg) *erg = c->h_red[0];
    if (virial) *virial = c->h_red[1];
  }
  return NNPE_OK;
}
