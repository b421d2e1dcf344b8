// Allocation-free force step: nnpe_force_step with its host <-> device staging of positions and
// forces in a statically reserved device array instead of buffers that the library allocates on
// first use. It has no counterpart in the reference (whose force step runs on host memory).
//
// Who needs it: a host run loop whose process reserves the device's memory up front for its own
// allocator, where an allocation by the library fails or escapes that allocator's accounting; and
// a loop that keeps other streams busy, where the implicit synchronisation that a device memory
// allocation brings between streams is not acceptable. Such a caller cannot let the force step
// call cudaMalloc, so this entry point never allocates: the staging lives in g_stage below.
//
// g_stage sits in this file's own device module. nnpe_setup resolves its address on the context's
// device (cudaGetSymbolAddress with that device current), which loads the module and reserves the
// 3 MiB there, so that the force step itself loads and reserves nothing, even under lazy module
// loading; the array is then held on that device until the process exits. nnpe_setup refreshes
// the address each time it runs, so a context set up after a device reset does not use a stale
// one; a reset under a context that is already set up is not supported. All contexts on one
// device share g_stage, so calls that overlap in time race on it.
#include <mutex>

#include "internal.cuh"

namespace {

// Largest system the static staging holds: positions in and forces out, 3 floats per atom each,
// 3 MiB in all.
constexpr int kStageMaxAtoms = 131072;
__device__ __align__(256) float g_stage[2 * 3 * kStageMaxAtoms];

constexpr int kMaxDevices = 64;
std::mutex g_stage_mu;
float* g_stage_addr[kMaxDevices] = {};

}  // namespace

int noalloc_stage_prepare(nnpe_ctx* c) {
  if (c->device < 0 || c->device >= kMaxDevices)
    return nnpe_fail(c, NNPE_EARG, "nnpe_setup: device ordinal out of range for the static staging");
  std::lock_guard<std::mutex> lock(g_stage_mu);
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_stage);
  if (e != cudaSuccess)
    return nnpe_fail(c, NNPE_ECUDA, std::string("nnpe_setup: cudaGetSymbolAddress of the static staging: ") +
                                        cudaGetErrorString(e));
  g_stage_addr[c->device] = static_cast<float*>(p);
  return NNPE_OK;
}

// The same step as nnpe_force_step (list check and rebuild on the device, forces, optional FP64
// energy and virial), with positions staged in g_stage[0, 3N) and forces in g_stage[3 kStageMaxAtoms, ...).
// Nothing in g_stage has to start at zero: every call overwrites the 3N floats of each half that
// it reads (the positions by the host copy, the forces by the gather, atom ids being a permutation).
extern "C" int nnpe_force_step_noalloc(nnpe_ctx* c, const float* x_host, float* f_host, double* erg,
                                       double* virial) {
  if (!c) return NNPE_EARG;
  if (c->natom > kStageMaxAtoms)
    return nnpe_fail(c, NNPE_EARG, "nnpe_force_step_noalloc: " + std::to_string(c->natom) +
                                       " atoms exceed the static staging limit of " +
                                       std::to_string(kStageMaxAtoms) + " atoms");
  if (!c->have_setup || !x_host || !f_host) return nnpe_fail(c, NNPE_EARG, "nnpe_force_step_noalloc");
  if (c->device < 0 || c->device >= kMaxDevices) return nnpe_fail(c, NNPE_EARG, "nnpe_force_step_noalloc: device");
  NNPE_CUDA(c, cudaSetDevice(c->device));
  float* stage = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_stage_mu);
    stage = g_stage_addr[c->device];
  }
  if (!stage) return nnpe_fail(c, NNPE_EARG, "nnpe_force_step_noalloc: the static staging was not resolved by nnpe_setup");
  // eager launches: instantiating a graph could allocate, which this entry point promises not to do
  return force_step_staged(c, x_host, f_host, erg, virial, stage, stage + 3 * kStageMaxAtoms, false);
}
