// Serving: a persistent request loop that runs independent MD replicas side by side on one GPU.
//
// The reference holds one system per process (ENVIRON is a static singleton, environ.h:20-123), so
// a stream of independent MD requests runs there as one run after another. Here a worker thread
// owns every replica: each admitted request becomes a context (its state resident in HBM, its own
// stream), and its MD steps go to the device as CUDA-graph launches of `chunk_steps` steps
// (run_graph_launch). The loop never waits for one replica to let another proceed:
//
//  * admission: a queued request is admitted, in arrival order, as soon as a replica slot is free
//    and its device footprint fits the HBM budget (requests that fit may pass one that does not;
//    the ledger books each resident replica's own allocations, nnpe_device_bytes);
//  * continuous batching: every resident replica has a chunk in flight; when its completion
//    event fires, the next chunk is launched at once, so replicas of very different sizes overlap
//    on the device and new arrivals join while others run;
//  * retirement: a finished replica's positions, velocities and last energies are copied out and
//    its context is parked; parked contexts are destroyed (their memory returned) when admission
//    needs the room or the device is idle, because freeing device memory waits for the whole GPU.
//
// Every kernel of a replica reads only that replica's buffers and sums in a fixed order, so a
// result is the same bits whether the replica ran alone or among others.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.cuh"

int run_graph_launch(nnpe_ctx* c, int step0, int nsteps, int log_interval);
int run_prepare(nnpe_ctx* c, int max_log);
int run_finish(nnpe_ctx* c, nnpe_thermo* log, int max_log, int* nlog);

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  // system (copies of the caller's arrays)
  int natom = 0, nmoltype = 0, nmax = 0, nbond = 0, nangle = 0, ndih = 0, nsteps = 0;
  double bl = 0, temperature = 300;
  uint64_t seed = 1;
  std::vector<int> typ, mol_id, intra, amt, special, bonds, angles, dihs;
  std::vector<float> mass, q, x, v;
  // progress and result
  int status = 0;   // 0 queued, 1 resident, 2 done, <0 failed (-status is the NNPE_E* code)
  std::string err;
  double t_submit = 0, t_admit = 0, t_done = 0;
  int64_t bytes = 0;
  nnpe_thermo last{};
  std::vector<float> x_out, v_out;
};

struct Replica {
  Request* req = nullptr;
  nnpe_ctx* ctx = nullptr;
  cudaEvent_t done = nullptr;
  int step = 0;           // md_step of the next chunk
  int chunk = 0;          // steps in flight
  bool running = false;
  int64_t bytes = 0;
};

}  // namespace

struct nnpe_server {
  nnpe_serve_config cfg{};
  // owned copies of the force field
  std::vector<float> force, potential, bcoef, acoef, dcoef, coef_p, coef_w, coef_d, coef_r, embw, fitw;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::map<int64_t, std::unique_ptr<Request>> all;
  std::vector<std::unique_ptr<Replica>> resident;
  std::vector<std::unique_ptr<Replica>> parked;
  int64_t next_id = 1, ndone = 0, nsubmitted = 0;
  int64_t bytes_in_use = 0, bytes_parked = 0, peak_bytes = 0;
  int peak_resident = 0;
  std::atomic<bool> stop{false};
  std::thread worker;
  Clock::time_point t0;
  std::string err;
  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

void copy_opt(std::vector<float>& dst, const float* src, size_t n) {
  if (src) dst.assign(src, src + n);
  else dst.clear();
}
const float* ptr_or_null(const std::vector<float>& v) { return v.empty() ? nullptr : v.data(); }

// Device bytes of a replica before it exists (the admission test; the measured figure replaces it
// once the replica is set up): the neighbour list and its pruned copy (2 * natom * neigh_cap int32)
// dominate; per-atom
// state and sort scratch (~400 B); periodic images within skin + cutoff of the faces (~64 B each:
// positions, info, cell, owner, shift and sort scratch), which outnumber the atoms in boxes not
// much larger than the cutoff; with the network term its pair list and descriptor buffers; and a
// fixed part (tables, weight images, graphs).
int64_t footprint_estimate(const nnpe_serve_config& c, int natom, double bl) {
  int64_t per_atom = (int64_t)c.neigh_cap * 4 * 2 + 420;   // the list and its pruned copy
  if (c.nnp_kind >= 0) per_atom += 256 * 4 + 2 * 256 * 4 + 64;
  const double comm = c.skin + c.pair_cutoff, g = (bl + 2 * comm) / bl;
  const double images = std::min((double)natom * (g * g * g - 1) * 1.2 + 4096, 26.0 * natom + 4096);
  return (int64_t)natom * per_atom + (int64_t)(images * 64) + (16ll << 20);
}

int setup_replica(nnpe_server* s, Request* r, nnpe_ctx** out) {
  const nnpe_serve_config& c = s->cfg;
  nnpe_ctx* ctx = nullptr;
  int rc = nnpe_create(c.device, &ctx);
  if (rc) return rc;
  *out = ctx;
  if ((rc = nnpe_set_system(ctx, r->natom, c.ntype, r->bl, r->typ.data(), r->mass.data(), r->q.data(), r->x.data(),
                            r->mol_id.data(), r->intra.data(), r->amt.data(), r->nmoltype, r->nmax, r->special.data())))
    return rc;
  if ((rc = nnpe_set_velocities(ctx, r->v.data()))) return rc;
  if ((rc = nnpe_setup(ctx, c.pair_cutoff, c.skin, c.pair_cutoff, c.neigh_cap))) return rc;
  if (!s->force.empty()) {
    if ((rc = nnpe_pair_set_table(ctx, c.nbin, s->force.data(), s->potential.data()))) return rc;
  } else if ((rc = nnpe_pair_enable(ctx, 0))) {
    return rc;
  }
  if ((rc = nnpe_bonded_set(ctx, r->nbond, r->bonds.data(), c.nbtyp, ptr_or_null(s->bcoef), r->nangle, r->angles.data(),
                            c.natyp, ptr_or_null(s->acoef), r->ndih, r->dihs.data(), c.ndtyp, ptr_or_null(s->dcoef))))
    return rc;
  if (c.nnp_kind >= 0) {
    if ((rc = nnpe_nnp_set(ctx, c.nnp_kind, c.nnp_cutoff, c.nnp_nbin, c.nnp_scale, c.e1, c.e2, c.h1, c.h2,
                           ptr_or_null(s->coef_p), ptr_or_null(s->coef_w), ptr_or_null(s->coef_d), ptr_or_null(s->coef_r),
                           ptr_or_null(s->embw), ptr_or_null(s->fitw))))
      return rc;
    if ((rc = nnpe_nnp_precision(ctx, c.nnp_bf16))) return rc;
  }
  if (c.autotune && c.nnp_kind >= 0 && c.nnp_bf16) {
    // before the first chunk is captured; a size class tuned once serves later replicas from the cache
    if ((rc = nnpe_nnp_autotune(ctx, 3, 1, nullptr, nullptr))) return rc;
  }
  if ((rc = nnpe_verlet_setup(ctx, c.dt, c.fp64_state))) return rc;
  if ((rc = nnpe_thermostat(ctx, c.thermostat, r->temperature, r->temperature, c.thermostat ? c.chunk_steps : 0,
                            c.thermo_frac, r->seed)))
    return rc;
  if ((rc = nnpe_set_total_steps(ctx, r->nsteps))) return rc;
  return NNPE_OK;
}

void fail_request(nnpe_server* s, Request* r, int rc, nnpe_ctx* ctx) {
  std::lock_guard<std::mutex> lk(s->mu);
  r->status = -(rc ? rc : NNPE_ECUDA);
  r->err = ctx ? nnpe_last_error(ctx) : "context creation failed";
  r->t_done = s->now();
  ++s->ndone;
  s->cv_done.notify_all();
}

// Destroy parked contexts (returns their memory; cudaFree waits for the device).
void clear_parked(nnpe_server* s) {
  for (auto& p : s->parked) {
    if (p->done) cudaEventDestroy(p->done);
    nnpe_destroy(p->ctx);
  }
  s->parked.clear();
  std::lock_guard<std::mutex> lk(s->mu);
  s->bytes_in_use -= s->bytes_parked;
  s->bytes_parked = 0;
}

bool admit_one(nnpe_server* s) {
  Request* r = nullptr;
  int64_t need = 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if ((int)s->resident.size() >= s->cfg.max_replicas) return false;
    for (auto it = s->queue.begin(); it != s->queue.end();) {
      const int64_t est = footprint_estimate(s->cfg, (*it)->natom, (*it)->bl);
      if (est > s->cfg.hbm_budget) {   // can never fit: fail it instead of holding it forever
        Request* big = *it;
        it = s->queue.erase(it);
        big->status = -NNPE_EOVERFLOW;
        big->err = "request needs more device memory than the server's HBM budget";
        big->t_done = s->now();
        ++s->ndone;
        s->cv_done.notify_all();
        continue;
      }
      if (s->bytes_in_use + est <= s->cfg.hbm_budget) {
        r = *it;
        need = est;
        s->queue.erase(it);
        break;
      }
      ++it;
    }
    if (!r) {
      // nothing fits: room held by parked replicas is reclaimed first
      if (s->bytes_parked > 0 && !s->queue.empty()) need = -1;
      else return false;
    }
  }
  if (!r) {
    clear_parked(s);
    return true;
  }
  nnpe_ctx* ctx = nullptr;
  int rc = setup_replica(s, r, &ctx);
  if (!rc) rc = run_prepare(ctx, 1);
  int64_t held = 0;
  if (!rc) nnpe_device_bytes(ctx, &held);
  if (rc) {
    fail_request(s, r, rc, ctx);
    if (ctx) nnpe_destroy(ctx);
    return true;
  }
  auto rep = std::make_unique<Replica>();
  rep->req = r;
  rep->ctx = ctx;
  cudaEventCreateWithFlags(&rep->done, cudaEventDisableTiming);
  rep->bytes = held > 0 ? held : need;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->status = 1;
    r->t_admit = s->now();
    r->bytes = rep->bytes;
    s->bytes_in_use += rep->bytes;
    s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
    s->resident.push_back(std::move(rep));
    s->peak_resident = std::max(s->peak_resident, (int)s->resident.size());
  }
  return true;
}

int launch_chunk(nnpe_server* s, Replica* p) {
  const int left = p->req->nsteps - p->step;
  const int n = std::min(left, s->cfg.chunk_steps);
  int rc = run_prepare(p->ctx, 1);
  if (!rc) rc = run_graph_launch(p->ctx, p->step, n, s->cfg.chunk_steps);
  if (!rc && cudaEventRecord(p->done, (cudaStream_t)nnpe_stream(p->ctx)) != cudaSuccess) rc = NNPE_ECUDA;
  if (rc) return rc;
  p->chunk = n;
  p->running = true;
  return 0;
}

// A chunk finished: read its log record, retire the replica when its steps are done.
bool complete_chunk(nnpe_server* s, size_t k) {
  Replica* p = s->resident[k].get();
  p->running = false;
  p->step += p->chunk;
  nnpe_thermo rec{};
  int n = 0;
  int rc = run_finish(p->ctx, &rec, 1, &n);
  Request* r = p->req;
  if (!rc && n > 0) r->last = rec;
  if (!rc && p->step < r->nsteps) return false;
  if (!rc) {
    r->x_out.resize((size_t)r->natom * 3);
    r->v_out.resize((size_t)r->natom * 3);
    rc = nnpe_get_positions(p->ctx, r->x_out.data());
    if (!rc) rc = nnpe_get_velocities(p->ctx, r->v_out.data());
  }
  std::unique_ptr<Replica> gone = std::move(s->resident[k]);
  s->resident.erase(s->resident.begin() + k);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (rc) {
      r->status = -rc;
      r->err = nnpe_last_error(gone->ctx);
    } else {
      r->status = 2;
    }
    r->t_done = s->now();
    ++s->ndone;
    s->bytes_parked += gone->bytes;
    s->cv_done.notify_all();
  }
  s->parked.push_back(std::move(gone));
  return true;
}

void worker_main(nnpe_server* s) {
  cudaSetDevice(s->cfg.device);
  while (!s->stop.load()) {
    bool progressed = false;
    // retire / continue replicas whose chunk completed
    for (size_t k = 0; k < s->resident.size();) {
      Replica* p = s->resident[k].get();
      if (p->running) {
        const cudaError_t q = cudaEventQuery(p->done);
        if (q == cudaSuccess) {
          progressed = true;
          if (complete_chunk(s, k)) continue;   // erased: same index holds the next replica
        } else if (q != cudaErrorNotReady) {
          // the chunk failed (a CUDA error in this context): fail the request instead of waiting on it
          Request* r = p->req;
          {
            std::lock_guard<std::mutex> lk(s->mu);
            r->status = -NNPE_ECUDA;
            r->err = std::string("chunk failed: ") + cudaGetErrorString(q);
            r->t_done = s->now();
            ++s->ndone;
            s->bytes_parked += p->bytes;
            s->cv_done.notify_all();
          }
          p->running = false;
          s->parked.push_back(std::move(s->resident[k]));
          s->resident.erase(s->resident.begin() + k);
          progressed = true;
          continue;
        }
      }
      ++k;
    }
    // admit while slots and memory allow
    while (admit_one(s)) progressed = true;
    // keep a chunk in flight on every resident replica
    for (size_t k = 0; k < s->resident.size();) {
      Replica* p = s->resident[k].get();
      if (!p->running) {
        if (int rc = launch_chunk(s, p)) {
          Request* r = p->req;
          {
            std::lock_guard<std::mutex> lk(s->mu);
            r->status = -rc;
            r->err = nnpe_last_error(p->ctx);
            r->t_done = s->now();
            ++s->ndone;
            s->bytes_parked += p->bytes;
            s->cv_done.notify_all();
          }
          s->parked.push_back(std::move(s->resident[k]));
          s->resident.erase(s->resident.begin() + k);
          continue;
        }
        progressed = true;
      }
      ++k;
    }
    bool idle;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      idle = s->resident.empty() && s->queue.empty();
    }
    if (idle) {
      if (!s->parked.empty()) clear_parked(s);   // the device is idle: freeing costs nothing now
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait_for(lk, std::chrono::milliseconds(50), [&] { return s->stop.load() || !s->queue.empty(); });
    } else if (!progressed) {
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
  for (auto& p : s->resident) {
    cudaStreamSynchronize((cudaStream_t)nnpe_stream(p->ctx));
    s->parked.push_back(std::move(p));
  }
  s->resident.clear();
  clear_parked(s);
}

}  // namespace

extern "C" int nnpe_server_create(const nnpe_serve_config* cfg, nnpe_server** out) {
  if (!cfg || !out || cfg->max_replicas <= 0 || cfg->chunk_steps <= 0 || cfg->hbm_budget <= 0 || cfg->ntype <= 0 ||
      cfg->ntype > NNPE_MAX_TYPES || cfg->neigh_cap <= 0)
    return NNPE_EARG;
  if (cudaSetDevice(cfg->device) != cudaSuccess) return NNPE_ECUDA;
  auto* s = new nnpe_server();
  s->cfg = *cfg;
  const int npair = cfg->ntype * (cfg->ntype + 1) / 2;
  if (cfg->force && cfg->potential && cfg->nbin > 0) {
    copy_opt(s->force, cfg->force, (size_t)npair * (cfg->nbin + 1));
    copy_opt(s->potential, cfg->potential, (size_t)npair * (cfg->nbin + 1));
  }
  copy_opt(s->bcoef, cfg->bcoef, (size_t)4 * std::max(cfg->nbtyp, 0));
  copy_opt(s->acoef, cfg->acoef, (size_t)4 * std::max(cfg->natyp, 0));
  copy_opt(s->dcoef, cfg->dcoef, (size_t)4 * std::max(cfg->ndtyp, 0));
  if (cfg->nnp_kind == 0) {
    copy_opt(s->coef_p, cfg->coef_p, (size_t)npair * 24);
    copy_opt(s->coef_w, cfg->coef_w, (size_t)npair * 80);
    copy_opt(s->coef_d, cfg->coef_d, (size_t)npair * 80);
    copy_opt(s->coef_r, cfg->coef_r, (size_t)npair * 80);
  } else if (cfg->nnp_kind == 1) {
    const size_t eb = (size_t)cfg->e1 * 2 + (size_t)cfg->e1 * cfg->e2 + cfg->e2;
    const size_t din = 4 * (size_t)cfg->e2;
    const size_t fb = din * cfg->h1 + cfg->h1 + (size_t)cfg->h1 * cfg->h2 + cfg->h2 + cfg->h2 + 1;
    copy_opt(s->embw, cfg->embw, eb * cfg->ntype);
    copy_opt(s->fitw, cfg->fitw, fb * cfg->ntype);
    if (cfg->coef_p) copy_opt(s->coef_p, cfg->coef_p, (size_t)npair * 24);
  }
  s->cfg.force = s->cfg.potential = nullptr;   // the copies above are used from here on
  s->t0 = Clock::now();
  s->worker = std::thread(worker_main, s);
  *out = s;
  return NNPE_OK;
}

extern "C" int nnpe_server_submit(nnpe_server* s, const nnpe_request* q, int64_t* id) {
  if (!s || !q || q->natom <= 0 || !(q->bl > 0) || !q->typ || !q->mass || !q->q || !q->x || !q->v || !q->mol_id ||
      !q->intra_id || !q->atom_moltype || q->nmoltype <= 0 || q->nmax <= 0 || !q->special || q->nsteps <= 0)
    return NNPE_EARG;
  auto r = std::make_unique<Request>();
  const size_t n = q->natom;
  r->natom = q->natom; r->bl = q->bl; r->nmoltype = q->nmoltype; r->nmax = q->nmax;
  r->typ.assign(q->typ, q->typ + n); r->mass.assign(q->mass, q->mass + n); r->q.assign(q->q, q->q + n);
  r->x.assign(q->x, q->x + 3 * n); r->v.assign(q->v, q->v + 3 * n);
  r->mol_id.assign(q->mol_id, q->mol_id + n); r->intra.assign(q->intra_id, q->intra_id + n);
  r->amt.assign(q->atom_moltype, q->atom_moltype + n);
  r->special.assign(q->special, q->special + (size_t)q->nmoltype * q->nmax * q->nmax);
  r->nbond = std::max(q->nbond, 0); r->nangle = std::max(q->nangle, 0); r->ndih = std::max(q->ndih, 0);
  if (r->nbond) r->bonds.assign(q->bonds, q->bonds + 3 * (size_t)r->nbond);
  if (r->nangle) r->angles.assign(q->angles, q->angles + 4 * (size_t)r->nangle);
  if (r->ndih) r->dihs.assign(q->dihs, q->dihs + 5 * (size_t)r->ndih);
  r->bonds.push_back(0); r->angles.push_back(0); r->dihs.push_back(0);   // valid pointers when empty
  r->nsteps = q->nsteps; r->temperature = q->temperature; r->seed = q->seed;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    r->t_submit = s->now();
    if (id) *id = r->id;
    s->queue.push_back(r.get());
    s->all[r->id] = std::move(r);
    ++s->nsubmitted;
  }
  s->cv_work.notify_one();
  return NNPE_OK;
}

static void fill_stats(const Request* r, nnpe_request_stats* st) {
  st->id = r->id; st->natom = r->natom; st->nsteps = r->nsteps; st->status = r->status;
  st->t_submit = r->t_submit; st->t_admit = r->t_admit; st->t_done = r->t_done; st->bytes = r->bytes;
  st->erg = r->last.erg; st->ekin = r->last.ekin; st->temperature = r->natom ? r->last.temperature : 0;
}

extern "C" int nnpe_server_wait(nnpe_server* s, int64_t id, double timeout_s, nnpe_request_stats* st) {
  if (!s) return NNPE_EARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return NNPE_EARG;
  Request* r = it->second.get();
  const auto pred = [&] { return r->status == 2 || r->status < 0; };
  if (timeout_s < 0) s->cv_done.wait(lk, pred);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return NNPE_ETIMEOUT;
  if (st) fill_stats(r, st);
  if (r->status < 0) {
    s->err = r->err;
    return -r->status;
  }
  return NNPE_OK;
}

extern "C" int nnpe_server_result(nnpe_server* s, int64_t id, float* x, float* v, nnpe_request_stats* st) {
  if (!s) return NNPE_EARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return NNPE_EARG;
  Request* r = it->second.get();
  if (st) fill_stats(r, st);
  if (r->status != 2) return r->status < 0 ? -r->status : NNPE_EARG;
  if (x) std::copy(r->x_out.begin(), r->x_out.end(), x);
  if (v) std::copy(r->v_out.begin(), r->v_out.end(), v);
  return NNPE_OK;
}

extern "C" int nnpe_server_drain(nnpe_server* s, double timeout_s) {
  if (!s) return NNPE_EARG;
  std::unique_lock<std::mutex> lk(s->mu);
  const auto pred = [&] { return s->ndone == s->nsubmitted; };
  if (timeout_s < 0) s->cv_done.wait(lk, pred);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return NNPE_ETIMEOUT;
  return NNPE_OK;
}

extern "C" int nnpe_server_info(nnpe_server* s, int64_t* done, int64_t* queued, int* resident, int64_t* bytes_in_use,
                                int64_t* peak_bytes, int* peak_resident) {
  if (!s) return NNPE_EARG;
  std::lock_guard<std::mutex> lk(s->mu);
  if (done) *done = s->ndone;
  if (queued) *queued = (int64_t)s->queue.size();
  if (resident) *resident = (int)s->resident.size();
  if (bytes_in_use) *bytes_in_use = s->bytes_in_use;
  if (peak_bytes) *peak_bytes = s->peak_bytes;
  if (peak_resident) *peak_resident = s->peak_resident;
  return NNPE_OK;
}

extern "C" int64_t nnpe_server_footprint(nnpe_server* s, int natom, double bl) {
  return s && natom > 0 && bl > 0 ? footprint_estimate(s->cfg, natom, bl) : -1;
}

extern "C" const char* nnpe_server_error(nnpe_server* s) { return s ? s->err.c_str() : "no server"; }

extern "C" void nnpe_server_destroy(nnpe_server* s) {
  if (!s) return;
  s->stop.store(true);
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  delete s;
}
