// Velocity Verlet (VERLET, verlet.cpp:29-97), thermostats (run.cpp:348-373, ENVIRON::initV
// environ.cpp:190-205) and the step loop of the classical / nnp_run drivers (run.cpp:204-394,
// 1099-1354), issued as a fixed kernel sequence per step and optionally replayed from CUDA graphs.
#include <cmath>
#include <vector>

#include "internal.cuh"

int check_valid_enqueue(nnpe_ctx* c);
int nnpe_sync_errors(nnpe_ctx* c);
int gr_step_enqueue(nnpe_ctx* c, bool long_tally, bool rmdf_potential);
bool rmdf_potential_on_log(const nnpe_ctx* c);

namespace {

constexpr float kAccelF = 4.184e-4f;            // environ.h:78
constexpr double kEkinF = 1195.0286802753603;   // environ.h:79
constexpr double kKTmSqrt = 0.0009118367518929329;
constexpr double kEkT = 335.47968899917714;
constexpr double kEvGPa = 6.9476954570553735;
constexpr double kKB300 = 0.5961612775922496;

// updateX (verlet.cpp:305-319): x += (v + a*hdt)*dt; the acceleration array doubles as f_prev.
// Also refreshes the FP32 coordinates and flags the list for rebuild when an atom moved more than
// skin/2 since the last build (NEIGHLIST::isvalid, neighlist.cpp:178-187); with xprune, flags the
// pruned copy of the list when an atom moved more than prune_delta/2 since the last prune.
__global__ void k_update_x(double4* __restrict__ xd, const double4* __restrict__ vd, const float4* __restrict__ acc,
                           float4* __restrict__ pos, const float4* __restrict__ xbuild, const float4* __restrict__ xprune,
                           int N, float dt, double dt64, bool fp64, bool check, float dx2, float pdx2, int* ctrl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double4 x = xd[i];
  const double4 v = vd[i];
  const float4 a = acc[i];
  float xf, yf, zf;
  if (fp64) {
    const double h = 0.5 * dt64;
    x.x += (v.x + (double)a.x * h) * dt64;
    x.y += (v.y + (double)a.y * h) * dt64;
    x.z += (v.z + (double)a.z * h) * dt64;
    xf = (float)x.x; yf = (float)x.y; zf = (float)x.z;
  } else {
    const float hdt = dt * .5F;
    xf = (float)x.x + ((float)v.x + a.x * hdt) * dt;
    yf = (float)x.y + ((float)v.y + a.y * hdt) * dt;
    zf = (float)x.z + ((float)v.z + a.z * hdt) * dt;
    x.x = xf; x.y = yf; x.z = zf;
  }
  xd[i] = x;
  const float q = pos[i].w;
  pos[i] = make_float4(xf, yf, zf, q);
  if (check) {
    const float4 b = xbuild[i];
    const float ex = xf - b.x, ey = yf - b.y, ez = zf - b.z;
    if (ex * ex + ey * ey + ez * ez > dx2) ctrl[CTRL_REBUILD] = 1;
    if (xprune) {
      const float4 p = xprune[i];
      const float px = xf - p.x, py = yf - p.y, pz = zf - p.z;
      if (px * px + py * py + pz * pz > pdx2) ctrl[CTRL_PRUNE] = 1;
    }
  }
}

// updateV (verlet.cpp:322-337): a = f*(r_m*accelF); v += (a_prev + a)*hdt; plus per-atom kinetic
// energy v^2/r_m*ekinF (computeKE, verlet.cpp:87-97) in FP64.
__global__ void k_update_v(double4* __restrict__ vd, float4* __restrict__ acc, const float4* __restrict__ frc,
                           const float2* __restrict__ qm, double* __restrict__ kin, int N, float dt, double dt64,
                           bool fp64, bool kinetic) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float rm = qm[i].y * kAccelF;
  const float4 f = frc[i], ap = acc[i];
  const float ax = f.x * rm, ay = f.y * rm, az = f.z * rm;
  double4 v = vd[i];
  if (fp64) {
    const double h = 0.5 * dt64;
    v.x += ((double)ap.x + (double)ax) * h;
    v.y += ((double)ap.y + (double)ay) * h;
    v.z += ((double)ap.z + (double)az) * h;
  } else {
    const float hdt = dt * .5F;
    v.x = (float)v.x + (ap.x + ax) * hdt;
    v.y = (float)v.y + (ap.y + ay) * hdt;
    v.z = (float)v.z + (ap.z + az) * hdt;
  }
  vd[i] = v;
  acc[i] = make_float4(ax, ay, az, 0.f);
  if (kinetic) kin[i] = (v.x * v.x + v.y * v.y + v.z * v.z) / (double)qm[i].y * kEkinF;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), a counter-based generator: thermostat draws
// depend only on (seed, step, atom id), not on the atom order or the launch shape.
__device__ __forceinline__ uint4 philox(uint4 ctr, uint2 key) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, ctr.x), lo0 = 0xD2511F53u * ctr.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, ctr.z), lo1 = 0xCD9E8D57u * ctr.z;
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += 0x9E3779B9u;
    key.y += 0xBB67AE85u;
  }
  return ctr;
}
__device__ __forceinline__ double u01(uint32_t a) { return ((double)a + 0.5) * (1.0 / 4294967296.0); }

__device__ __forceinline__ double thermo_temp(double t0, double t1, int step, int total) {
  return total > 0 ? t0 + (t1 - t0) * step / total : t0;
}

// Andersen: ENVIRON::initV(T, frac) (environ.cpp:190-205): each atom with probability frac gets
// fresh Maxwell-Boltzmann components of spread sqrt(T*r_m)*kT_m_sqrt.
__global__ void k_andersen(double4* __restrict__ vd, const float2* __restrict__ qm, const int* __restrict__ aid, int N,
                           double t0, double t1, int total, double frac, uint64_t seed, bool fp64, const int* ctrl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int step = ctrl[CTRL_STEP];
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32) ^ (uint32_t)step);
  const uint4 r0 = philox(make_uint4((uint32_t)aid[i], 0u, (uint32_t)step, 0x41u), key);
  if (u01(r0.x) >= frac) return;
  const uint4 r1 = philox(make_uint4((uint32_t)aid[i], 1u, (uint32_t)step, 0x41u), key);
  const double T = thermo_temp(t0, t1, step, total);
  const double fc = sqrt(T * (double)qm[i].y) * kKTmSqrt;
  const double m1 = sqrt(-2 * log(u01(r0.y))), m2 = sqrt(-2 * log(u01(r1.x)));
  const double tw = 6.283185307179586;
  double4 v = make_double4(m1 * cos(tw * u01(r0.z)) * fc, m1 * sin(tw * u01(r0.z)) * fc, m2 * cos(tw * u01(r1.y)) * fc, 0);
  if (!fp64) { v.x = (float)v.x; v.y = (float)v.y; v.z = (float)v.z; }
  vd[i] = v;
}

// CSVR branch (run.cpp:365-372): scale = sqrt(Gamma(ndof/2, kB*300K)*T_rel / ekin); the gamma
// variate by Marsaglia-Tsang (ACM TOMS 26(3), 2000) with a bounded rejection loop.
__global__ void k_csvr_scale(double* red, int ndof, double t0, double t1, int total, uint64_t seed, const int* ctrl) {
  const int step = ctrl[CTRL_STEP];
  const double alpha = 0.5 * ndof, d = alpha - 1.0 / 3, cc = 1 / sqrt(9 * d);
  const uint2 key = make_uint2((uint32_t)seed ^ 0x5bd1e995u, (uint32_t)(seed >> 32) ^ (uint32_t)step);
  double g = alpha;
  for (uint32_t it = 0; it < 64; ++it) {
    const uint4 r = philox(make_uint4(it, 7u, (uint32_t)step, 0x43u), key);
    const double z = sqrt(-2 * log(u01(r.x))) * cos(6.283185307179586 * u01(r.y));
    const double v = 1 + cc * z;
    if (v <= 0) continue;
    const double v3 = v * v * v;
    if (log(u01(r.z)) < 0.5 * z * z + d - d * v3 + d * log(v3)) { g = d * v3; break; }
  }
  const double T = thermo_temp(t0, t1, step, total) / 300.0;
  red[4] = red[2] > 0 ? sqrt(g * kKB300 * T / red[2]) : 1.0;
}

__global__ void k_scale_v(double4* vd, int N, const double* red, bool fp64) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double s = red[4];
  double4 v = vd[i];
  if (fp64) { v.x *= s; v.y *= s; v.z *= s; }
  else { const float sf = (float)s; v.x = (float)v.x * sf; v.y = (float)v.y * sf; v.z = (float)v.z * sf; }
  vd[i] = v;
}

__global__ void k_step_end(int* ctrl) { ctrl[CTRL_STEP] += 1; }

// FP32 coordinates and charges of the unsorted initial state (before the first rebuild).
__global__ void k_init_pos(const double4* __restrict__ xd, const float2* __restrict__ qm, float4* __restrict__ pos, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double4 x = xd[i];
  pos[i] = make_float4((float)x.x, (float)x.y, (float)x.z, qm[i].x);
}

}  // namespace

int verlet_x_enqueue(nnpe_ctx* c, double dt, bool check) {
  const float h = c->skin / 2;
  k_update_x<<<nblocks(c->natom, 256), 256, 0, c->stream>>>(c->d_xd, c->d_vd, c->d_acc, c->d_pos, c->d_xbuild,
                                                            prune_active(c) ? c->d_xprune : nullptr, c->natom, (float)dt,
                                                            dt, c->fp64_state, check, h * h, prune_dx2(c), c->d_ctrl);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int verlet_v_enqueue(nnpe_ctx* c, bool kinetic) {
  k_update_v<<<nblocks(c->natom, 256), 256, 0, c->stream>>>(c->d_vd, c->d_acc, c->d_frc, c->d_qm, c->d_kin, c->natom,
                                                            (float)c->dt, c->dt, c->fp64_state, kinetic);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

int thermostat_enqueue(nnpe_ctx* c) {
  if (c->thermo_kind == 1) {
    k_andersen<<<nblocks(c->natom, 256), 256, 0, c->stream>>>(c->d_vd, c->d_qm, c->d_atom_id, c->natom, c->t_start, c->t_end,
                                                              c->total_steps_hint, c->thermo_frac, c->seed, c->fp64_state,
                                                              c->d_ctrl);
  } else if (c->thermo_kind == 2) {
    k_csvr_scale<<<1, 1, 0, c->stream>>>(c->d_red, 3 * c->natom, c->t_start, c->t_end, c->total_steps_hint, c->seed, c->d_ctrl);
    k_scale_v<<<nblocks(c->natom, 256), 256, 0, c->stream>>>(c->d_vd, c->natom, c->d_red, c->fp64_state);
  }
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

// One step of run.cpp:230-393 with flags decided on the host from md_step (known there).
static int enqueue_step(nnpe_ctx* c, int variant) {
  const bool f_log = variant & 1, thermo = variant & 2, gr = variant & 4, gr_long = variant & 8;
  if (int rc = verlet_x_enqueue(c, c->dt, true)) return rc;
  if (int rc = rebuild_enqueue(c, true)) return rc;
  if (int rc = ghost_update_enqueue(c, true)) return rc;
  if (gr)
    // run.cpp:298: the potential table is refreshed on log steps when gamma != 1
    if (int rc = gr_step_enqueue(c, gr_long, f_log && rmdf_potential_on_log(c))) return rc;
  if (int rc = forces_enqueue(c, f_log)) return rc;
  // The kinetic energy is computed on thermostat steps, before the thermostat acts, and a log step
  // reports the one of the last thermostat step (run.cpp:349-359, 380); without a thermostat every
  // log step computes its own.
  const bool kin_now = thermo || (f_log && c->thermo_kind == 0);
  if (int rc = verlet_v_enqueue(c, kin_now)) return rc;
  if (f_log) {
    if (int rc = energy_reduce_enqueue(c, kin_now ? 1 : 3)) return rc;
  } else if (thermo) {
    if (int rc = energy_reduce_enqueue(c, 2)) return rc;
  }
  if (thermo)
    if (int rc = thermostat_enqueue(c)) return rc;
  k_step_end<<<1, 1, 0, c->stream>>>(c->d_ctrl);
  NNPE_CHECK_LAUNCH(c);
  return 0;
}

static int step_variant(nnpe_ctx* c, int md_step, int log_interval) {
  int v = 0;
  if (log_interval > 0 && md_step % log_interval == 0) v |= 1;
  if (c->thermo_kind && c->thermo_interval > 0 && md_step % c->thermo_interval == 0) v |= 2;
  if (c->gr_interval > 0 && md_step % c->gr_interval == 0) {
    v |= 4;
    // run.cpp:289-290: list-based tally unless md_step is on the long interval
    if (c->gr_interval_long <= 0 || md_step % c->gr_interval_long == 0) v |= 8;
  }
  return v;
}

static int prepare_run(nnpe_ctx* c, int max_log) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_run: not set up");
  if (int rc = refuse_if_poisoned(c)) return rc;
  if (!c->d_table && !c->nnp && c->pair_on) return nnpe_fail(c, NNPE_EARG, "nnpe_run: no pair table");
  cudaSetDevice(c->device);
  if (max_log > c->log_cap) {
    if (c->d_log) dev_free(c->d_log);
    c->d_log = nullptr;
    NNPE_CUDA(c, dev_malloc(c, (void**)&c->d_log, sizeof(LogRec) * max_log));
    c->log_cap = max_log;
    for (auto& g : c->graph_exec)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    c->graph_valid = false;
    c->fs_valid = false;
  }
  NNPE_CUDA(c, cudaMemsetAsync(c->d_ctrl + CTRL_NLOG, 0, sizeof(int), c->stream));
  if (!c->first_step_done) {
    // run.cpp:193, 220-227: clear f (the acceleration), updateX with dt=-dt, then dt back
    NNPE_CUDA(c, cudaMemsetAsync(c->d_acc, 0, sizeof(float4) * c->natom, c->stream));
    if (!c->d_pos) return nnpe_fail(c, NNPE_EARG, "nnpe_run: no state");
    // FP32 coordinates (with the charge slot updateX keeps) of the state as loaded
    k_init_pos<<<nblocks(c->natom, 256), 256, 0, c->stream>>>(c->d_xd, c->d_qm, c->d_pos, c->natom);
    int one = 1;
    NNPE_CUDA(c, cudaMemcpyAsync(c->d_ctrl + CTRL_REBUILD, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    if (int rc = verlet_x_enqueue(c, -c->dt, false)) return rc;
    c->first_step_done = true;
  }
  return 0;
}

// VERLET::updateX (verlet.cpp:29-43) with an explicit dt; the first call also performs what
// run.cpp:220-221 does before its first updateX (clear f) and takes the loaded state as FP32
// coordinates. Marks the list for a rebuild when an atom moved more than skin/2 since the last
// build (the check NEIGHLIST::isvalid reads).
extern "C" int nnpe_verlet_update_x(nnpe_ctx* c, double dt) {
  if (!c || !c->have_setup || !c->d_pos) return nnpe_fail(c, NNPE_EARG, "nnpe_verlet_update_x: not set up");
  cudaSetDevice(c->device);
  if (!c->first_step_done) {
    NNPE_CUDA(c, cudaMemsetAsync(c->d_acc, 0, sizeof(float4) * c->natom, c->stream));
    k_init_pos<<<nblocks(c->natom, 256), 256, 0, c->stream>>>(c->d_xd, c->d_qm, c->d_pos, c->natom);
    int one = 1;
    NNPE_CUDA(c, cudaMemcpyAsync(c->d_ctrl + CTRL_REBUILD, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    c->first_step_done = true;
  }
  if (int rc = verlet_x_enqueue(c, dt, true)) return rc;
  return nnpe_sync_errors(c);
}

// VERLET::updateV (verlet.cpp:46-61) on the forces of the last evaluation, and the kinetic energy
// (VERLET::computeKE, verlet.cpp:87-97, summed over all atoms in FP64) when ekin != NULL.
extern "C" int nnpe_verlet_update_v(nnpe_ctx* c, double* ekin) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_verlet_update_v: not set up");
  cudaSetDevice(c->device);
  if (int rc = verlet_v_enqueue(c, ekin != nullptr)) return rc;
  if (ekin) {
    if (int rc = energy_reduce_enqueue(c, 2)) return rc;
    NNPE_CUDA(c, cudaMemcpyAsync(c->h_red, c->d_red, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->stream));
  }
  if (int rc = nnpe_sync_errors(c)) return rc;
  if (ekin) *ekin = c->h_red[2];
  return NNPE_OK;
}

static int finish_run(nnpe_ctx* c, nnpe_thermo* log, int max_log, int* nlog) {
  if (int rc = nnpe_sync_errors(c)) return rc;
  const int n = std::min(c->h_ctrl[CTRL_NLOG], max_log);
  if (nlog) *nlog = n;
  if (n > 0 && log) {
    std::vector<LogRec> h(n);
    NNPE_CUDA(c, cudaMemcpy(h.data(), c->d_log, sizeof(LogRec) * n, cudaMemcpyDeviceToHost));
    const double vol = std::pow((double)c->grid.bl, 3);
    for (int k = 0; k < n; ++k) {
      nnpe_thermo& t = log[k];
      t.step = h[k].step; t.nbuild = h[k].nbuild; t.erg = h[k].erg; t.virial = h[k].virial; t.ekin = h[k].ekin;
      t.erg_nnp = h[k].erg_nnp;
      t.erg_exp = h[k].erg_exp;
      t.temperature = t.ekin / c->natom * kEkT;                                 // run.cpp:380
      t.pressure = (t.virial + t.ekin * 2) / 3 * kEvGPa / vol;                   // run.cpp:381
    }
  }
  return NNPE_OK;
}

extern "C" int nnpe_run(nnpe_ctx* c, int nsteps, int log_interval, nnpe_thermo* log, int max_log, int* nlog) {
  if (int rc = prepare_run(c, max_log)) return rc;
  NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  const int step0 = c->h_ctrl[CTRL_STEP];
  for (int s = 0; s < nsteps; ++s)
    if (int rc = enqueue_step(c, step_variant(c, step0 + s, log_interval))) return rc;
  return finish_run(c, log, max_log, nlog);
}

// Launch steps step0..step0+nsteps-1 from the per-variant step graphs without waiting for them
// (the serving loop tracks md_step on the host, so nothing is read back here).
int run_graph_launch(nnpe_ctx* c, int step0, int nsteps, int log_interval) {
  if (!c->graph_valid) {
    for (auto& g : c->graph_exec)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    c->graph_valid = true;
  }
  for (int s = 0; s < nsteps; ++s) {
    const int v = step_variant(c, step0 + s, log_interval);
    if (!c->graph_exec[v]) {
      cudaGraph_t g;
      NNPE_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int rc = enqueue_step(c, v);
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      if (rc) return rc;
      if (e != cudaSuccess) return nnpe_fail(c, NNPE_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      NNPE_CUDA(c, cudaGraphInstantiate(&c->graph_exec[v], g, 0));
      cudaGraphDestroy(g);
    }
    NNPE_CUDA(c, cudaGraphLaunch(c->graph_exec[v], c->stream));
  }
  return 0;
}
int run_prepare(nnpe_ctx* c, int max_log) { return prepare_run(c, max_log); }
int run_finish(nnpe_ctx* c, nnpe_thermo* log, int max_log, int* nlog) { return finish_run(c, log, max_log, nlog); }

extern "C" int nnpe_run_graph(nnpe_ctx* c, int nsteps, int log_interval, nnpe_thermo* log, int max_log, int* nlog) {
  if (int rc = prepare_run(c, max_log)) return rc;
  NNPE_CUDA(c, cudaMemcpyAsync(c->h_ctrl, c->d_ctrl, sizeof(int) * CTRL_WORDS, cudaMemcpyDeviceToHost, c->stream));
  NNPE_CUDA(c, cudaStreamSynchronize(c->stream));
  const int step0 = c->h_ctrl[CTRL_STEP];
  if (!c->graph_valid) {
    for (auto& g : c->graph_exec)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    c->graph_valid = true;
  }
  for (int s = 0; s < nsteps; ++s) {
    const int v = step_variant(c, step0 + s, log_interval);
    if (!c->graph_exec[v]) {
      cudaGraph_t g;
      NNPE_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int rc = enqueue_step(c, v);
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      if (rc) return rc;
      if (e != cudaSuccess) return nnpe_fail(c, NNPE_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      NNPE_CUDA(c, cudaGraphInstantiate(&c->graph_exec[v], g, 0));
      cudaGraphDestroy(g);
    }
    NNPE_CUDA(c, cudaGraphLaunch(c->graph_exec[v], c->stream));
  }
  return finish_run(c, log, max_log, nlog);
}

extern "C" int nnpe_set_total_steps(nnpe_ctx* c, int total) {
  if (!c) return NNPE_EARG;
  c->total_steps_hint = total;
  c->graph_valid = false;
  c->fs_valid = false;
  return NNPE_OK;
}

int pair_enqueue(nnpe_ctx* c, bool ev, bool filter6);
bool pair_filters_list6(nnpe_ctx* c);
int bonded_enqueue(nnpe_ctx* c, bool ev);

// Enqueue one kernel class on the context's stream without synchronising, for timing it with
// events: 0 pair force, 1 list rebuild (all rebuild kernels), 2 bonded, 3 network term,
// 4 updateX+updateV, 5 cell-based g(r) tally, 6 list-based g(r) tally.
extern "C" int nnpe_profile_enqueue(nnpe_ctx* c, int which) {
  if (!c || !c->have_setup) return nnpe_fail(c, NNPE_EARG, "nnpe_profile_enqueue: not set up");
  switch (which) {
    case 0: return pair_enqueue(c, false, pair_filters_list6(c));
    case 1: {
      int one = 1;
      NNPE_CUDA(c, cudaMemcpyAsync(c->d_ctrl + CTRL_REBUILD, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
      if (int rc = rebuild_enqueue(c, true)) return rc;
      return ghost_update_enqueue(c, true);
    }
    case 2: return bonded_enqueue(c, false);
    case 3: return c->nnp ? nnp_forces_enqueue(c, false, !pair_filters_list6(c)) : 0;
    case 4: {
      if (int rc = verlet_x_enqueue(c, 0.0, false)) return rc;
      return verlet_v_enqueue(c, false);
    }
    case 5: return c->d_gr_counts ? gr_tally_enqueue(c, 0) : nnpe_fail(c, NNPE_EARG, "no g(r)");
    case 6: return c->d_gr_counts ? gr_tally_enqueue(c, 1) : nnpe_fail(c, NNPE_EARG, "no g(r)");
    case 7: return pair_enqueue(c, true, pair_filters_list6(c));
  }
  return nnpe_fail(c, NNPE_EARG, "nnpe_profile_enqueue: unknown kernel class");
}

// Kernel launches in one plain MD step (no logging/thermostat/g(r)): the nodes of its graph.
extern "C" int nnpe_launches_per_step(nnpe_ctx* c) {
  if (!c || !c->have_setup) return -1;
  cudaGraph_t g;
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1;
  int rc = enqueue_step(c, 0);
  if (cudaStreamEndCapture(c->stream, &g) != cudaSuccess || rc) return -1;
  size_t n = 0;
  cudaGraphGetNodes(g, nullptr, &n);
  std::vector<cudaGraphNode_t> nodes(n);
  cudaGraphGetNodes(g, nodes.data(), &n);
  int k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    cudaGraphNodeGetType(nd, &t);
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  cudaGraphDestroy(g);
  return k;
}
