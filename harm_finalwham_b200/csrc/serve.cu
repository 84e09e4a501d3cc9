// serve.cu -- continuous-batching serving loop over device-resident solves.
//
// Requests (a configuration, its geometry and initial state, an end time)
// arrive at any time through hgpu_server_submit.  hgpu_server_poll is the
// request loop: it admits pending requests first-fit in arrival order while
// their device footprint (hgpu_context_bytes) fits the server's byte budget
// and the active-slot limit, gives every admitted request its own context
// and CUDA stream with the state resident in HBM, keeps a chunk of time
// steps in flight per request as replays of the request's captured step
// graph (so the work of all admitted requests overlaps on the device and
// the host issues one launch per step), notices finished chunks without blocking
// (cudaEventQuery on an event recorded after a progress copy), retires a
// request when its t reached its end time (the step kernels freeze a
// finished context, so a chunk that overruns the end leaves the state
// unchanged) and downloads its result.  A retired request's context goes
// to an idle pool: the next admission of the same allocation shape reuses
// its device memory, pinned progress word and event (no cudaMalloc/cudaFree
// on the request path; cudaFree would also synchronize the whole device);
// idle contexts are destroyed only when an admission needs their bytes.  A
// request's result is exactly what running it alone gives: its kernels
// touch only its own context.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <chrono>
#include <map>
#include <mutex>
#include <vector>

#include "harmgpu.h"

cudaStream_t hg_stream(hgpu_ctx *x);
int hg_progress_async(hgpu_ctx *x, double *dst, cudaEvent_t ev);
extern "C" {
bool hg_same_shape(const hgpu_config *a, const hgpu_config *b);
int hg_reconfigure(hgpu_ctx *x, const hgpu_config *cfg);
}

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

enum { PENDING = 0, ACTIVE = 1, FINISHED = 2, FAILED = 3 };

struct Request {
  long long id = 0;
  hgpu_config cfg;
  std::vector<double> gcov, gcon, gcovpert, gdet, conn, floors, p;
  const double *src[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // borrowed inputs
  double tf = 0.0;
  int state = PENDING;
  size_t bytes = 0;
  hgpu_ctx *ctx = nullptr;
  double *prog = nullptr;  // pinned, one slot per chunk in flight: t, dt, done, steps
  cudaEvent_t ev[2] = {nullptr, nullptr};
  long long issued = 0, noticed = 0;  // chunks issued / seen complete
  long long steps = 0;
  Clock::time_point t_submit, t_admit, t_finish;
  std::vector<double> p_out;
  std::vector<int> pflag_out;
  double t_out = 0.0;
  int rc = 0;
};

// chunks kept in flight per solve: the next one is queued behind the
// running one, so the solve's stream never waits for the host to notice
constexpr int DEPTH = 2;

size_t zone_count(const hgpu_config &c, int ng_ghosts) {
  auto tot = [&](int n) { return (size_t)(n > 1 ? n + 2 * ng_ghosts : 1); };
  return tot(c.n1) * tot(c.n2) * tot(c.n3);
}

size_t geom_count(const hgpu_config &c) {
  auto tot = [&](int n) { return (size_t)(n > 1 ? n + 2 * c.ng + 1 : 1); };
  return tot(c.n1) * tot(c.n2);
}

}  // namespace

// an idle context kept for reuse, with its progress words and events
struct Slot {
  hgpu_ctx *ctx = nullptr;
  double *prog = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  hgpu_config cfg;
  size_t bytes = 0;
};

struct hgpu_server {
  size_t max_bytes = 0, used = 0, idle_bytes = 0;
  int max_active = 0, chunk = 1, active = 0;
  long long next_id = 1;
  std::map<long long, Request *> reqs;  // ordered by id = arrival order
  std::vector<Slot> idle;
  std::mutex m;
};

static void destroy_slot(Slot &q) {
  if (q.ctx) hgpu_destroy(q.ctx);
  for (int e = 0; e < DEPTH; e++)
    if (q.ev[e]) cudaEventDestroy(q.ev[e]);
  if (q.prog) cudaFreeHost(q.prog);
  q.ctx = nullptr;
  q.ev[0] = q.ev[1] = nullptr;
  q.prog = nullptr;
}

static void release_device(hgpu_server *s, Request *r) {
  Slot q;
  q.ctx = r->ctx;
  q.prog = r->prog;
  q.ev[0] = r->ev[0];
  q.ev[1] = r->ev[1];
  destroy_slot(q);
  r->ctx = nullptr;
  r->ev[0] = r->ev[1] = nullptr;
  r->prog = nullptr;
  if (r->state == ACTIVE) {
    s->used -= r->bytes;
    s->active--;
  }
}

// a finished request hands its context to the idle pool
static void park(hgpu_server *s, Request *r) {
  Slot q;
  q.ctx = r->ctx;
  q.prog = r->prog;
  q.ev[0] = r->ev[0];
  q.ev[1] = r->ev[1];
  q.cfg = r->cfg;
  q.bytes = r->bytes;
  r->ctx = nullptr;
  r->prog = nullptr;
  r->ev[0] = r->ev[1] = nullptr;
  s->used -= r->bytes;
  s->active--;
  s->idle.push_back(q);
  s->idle_bytes += q.bytes;
}

static int admit(hgpu_server *s, Request *r) {
  int rc = HGPU_OK;
  // reuse an idle context of the same shape, else make room and create one
  size_t pick = s->idle.size();
  for (size_t q = 0; q < s->idle.size(); q++)
    if (hg_same_shape(&s->idle[q].cfg, &r->cfg)) {
      pick = q;
      break;
    }
  if (pick < s->idle.size()) {
    Slot q = s->idle[pick];
    s->idle.erase(s->idle.begin() + (long)pick);
    s->idle_bytes -= q.bytes;
    r->ctx = q.ctx;
    r->prog = q.prog;
    r->ev[0] = q.ev[0];
    r->ev[1] = q.ev[1];
    rc = hg_reconfigure(r->ctx, &r->cfg);
  } else {
    while (!s->idle.empty() && s->used + s->idle_bytes + r->bytes > s->max_bytes) {
      s->idle_bytes -= s->idle.front().bytes;
      destroy_slot(s->idle.front());
      s->idle.erase(s->idle.begin());
    }
    rc = hgpu_create(&r->cfg, &r->ctx);
    if (!rc && cudaMallocHost(&r->prog, 4 * DEPTH * sizeof(double)) != cudaSuccess) rc = HGPU_E_NOMEM;
    for (int e = 0; e < DEPTH && !rc; e++)
      if (cudaEventCreateWithFlags(&r->ev[e], cudaEventDisableTiming) != cudaSuccess) rc = HGPU_E_CUDA;
  }
  const bool own = r->src[0] == nullptr;
  if (!rc)
    rc = hgpu_upload_geometry(r->ctx, own ? r->gcov.data() : r->src[0], own ? r->gcon.data() : r->src[1],
                              own ? r->gcovpert.data() : r->src[2], own ? r->gdet.data() : r->src[3],
                              own ? r->conn.data() : r->src[4], own ? r->floors.data() : r->src[5]);
  if (!rc) rc = hgpu_upload_state(r->ctx, own ? r->p.data() : r->src[6], nullptr, 0.0, 0.0);
  for (int q = 0; q < 7; q++) r->src[q] = nullptr;
  if (!rc) rc = hgpu_init_dt(r->ctx, nullptr);
  r->state = ACTIVE;
  s->used += r->bytes;
  s->active++;
  r->t_admit = Clock::now();
  // inputs are on the device now; free the host copies
  r->gcov.clear(); r->gcov.shrink_to_fit();
  r->gcon.clear(); r->gcon.shrink_to_fit();
  r->gcovpert.clear(); r->gcovpert.shrink_to_fit();
  r->gdet.clear(); r->gdet.shrink_to_fit();
  r->conn.clear(); r->conn.shrink_to_fit();
  r->floors.clear(); r->floors.shrink_to_fit();
  r->p.clear(); r->p.shrink_to_fit();
  if (rc) {
    r->rc = rc;
    release_device(s, r);
    r->state = FAILED;
    r->t_finish = Clock::now();
  }
  return rc;
}

static void issue_chunk(hgpu_server *s, Request *r) {
  // a chunk is `chunk` replays of the request's captured time step (one graph
  // launch per step instead of one launch per kernel)
  const int slot = (int)(r->issued % DEPTH);
  int rc = hgpu_step_graph(r->ctx, s->chunk, nullptr);
  if (!rc) rc = hg_progress_async(r->ctx, r->prog + 4 * slot, r->ev[slot]);
  if (rc) {
    r->rc = rc;
    release_device(s, r);
    r->state = FAILED;
    r->t_finish = Clock::now();
    return;
  }
  r->issued++;
}

static void retire(hgpu_server *s, Request *r) {
  size_t nz = zone_count(r->cfg, r->cfg.ng);
  r->p_out.resize(nz * 8);
  r->pflag_out.resize(nz);
  double dt;
  int rc = hgpu_download_state(r->ctx, r->p_out.data(), r->pflag_out.data(), &r->t_out, &dt);
  if (rc) release_device(s, r);
  else park(s, r);
  r->rc = rc;
  r->state = rc ? FAILED : FINISHED;
  r->t_finish = Clock::now();
}

extern "C" {

int hgpu_server_create(size_t max_device_bytes, int max_active, int steps_per_chunk, hgpu_server **out) {
  if (!out || max_active < 1 || steps_per_chunk < 1) return HGPU_E_INVALID;
  hgpu_server *s = new hgpu_server();
  s->max_bytes = max_device_bytes;
  s->max_active = max_active;
  s->chunk = steps_per_chunk;
  *out = s;
  return HGPU_OK;
}

void hgpu_server_destroy(hgpu_server *s) {
  if (!s) return;
  for (auto &kv : s->reqs) {
    Request *r = kv.second;
    if (r->ctx) cudaStreamSynchronize(hg_stream(r->ctx));
    release_device(s, r);
    delete r;
  }
  for (Slot &q : s->idle) destroy_slot(q);
  delete s;
}

static int submit_common(hgpu_server *s, const hgpu_config *cfg, const double *gcov, const double *gcon,
                         const double *gcovpert, const double *gdet, const double *conn, const double *floors,
                         const double *p, double tf, long long *id, bool borrow) {
  if (!s || !cfg || !gcov || !gcon || !gcovpert || !gdet || !conn || !floors || !p || !id) return HGPU_E_INVALID;
  size_t bytes = hgpu_context_bytes(cfg);
  if (bytes == 0 || bytes > s->max_bytes) return HGPU_E_INVALID;
  Request *r = new Request();
  r->cfg = *cfg;
  r->cfg.tf = tf;
  r->tf = tf;
  r->bytes = bytes;
  if (borrow) {
    const double *a[7] = {gcov, gcon, gcovpert, gdet, conn, floors, p};
    for (int q = 0; q < 7; q++) r->src[q] = a[q];
  } else {
    size_t nz = zone_count(*cfg, cfg->ng), nij = geom_count(*cfg);
    r->gcov.assign(gcov, gcov + nij * 128);
    r->gcon.assign(gcon, gcon + nij * 128);
    r->gcovpert.assign(gcovpert, gcovpert + nij * 32);
    r->gdet.assign(gdet, gdet + nij * 8);
    r->conn.assign(conn, conn + nij * 64);
    r->floors.assign(floors, floors + nij * 2);
    r->p.assign(p, p + nz * 8);
  }
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> g(s->m);
  r->id = s->next_id++;
  s->reqs[r->id] = r;
  *id = r->id;
  return HGPU_OK;
}

int hgpu_server_submit(hgpu_server *s, const hgpu_config *cfg, const double *gcov, const double *gcon,
                       const double *gcovpert, const double *gdet, const double *conn, const double *floors,
                       const double *p, double tf, long long *id) {
  return submit_common(s, cfg, gcov, gcon, gcovpert, gdet, conn, floors, p, tf, id, false);
}

int hgpu_server_submit_borrowed(hgpu_server *s, const hgpu_config *cfg, const double *gcov, const double *gcon,
                                const double *gcovpert, const double *gdet, const double *conn,
                                const double *floors, const double *p, double tf, long long *id) {
  return submit_common(s, cfg, gcov, gcon, gcovpert, gdet, conn, floors, p, tf, id, true);
}

int hgpu_server_poll(hgpu_server *s, int *pending, int *active, int *finished) {
  if (!s) return HGPU_E_INVALID;
  std::lock_guard<std::mutex> g(s->m);
  // 1. notice finished chunks; retire finished requests, keep the others busy
  for (auto &kv : s->reqs) {
    Request *r = kv.second;
    if (r->state != ACTIVE) continue;
    bool finished = false, failed = false;
    while (r->noticed < r->issued) {
      const int slot = (int)(r->noticed % DEPTH);
      cudaError_t e = cudaEventQuery(r->ev[slot]);
      if (e == cudaErrorNotReady) break;
      if (e != cudaSuccess) {
        failed = true;
        break;
      }
      r->noticed++;
      r->steps = (long long)r->prog[4 * slot + 3];
      if (r->prog[4 * slot + 2] != 0.0) {
        finished = true;
        break;
      }
    }
    if (failed) {
      r->rc = HGPU_E_CUDA;
      release_device(s, r);
      r->state = FAILED;
      r->t_finish = Clock::now();
      continue;
    }
    // a finished solve is frozen: chunks still queued behind leave it as it is
    if (finished) {
      retire(s, r);
      continue;
    }
    while (r->state == ACTIVE && r->issued - r->noticed < DEPTH) issue_chunk(s, r);
  }
  // 2. admit pending requests first-fit in arrival order
  for (auto &kv : s->reqs) {
    Request *r = kv.second;
    if (r->state != PENDING) continue;
    if (s->active >= s->max_active) break;
    if (s->used + r->bytes > s->max_bytes) continue;
    if (admit(s, r) == HGPU_OK)
      while (r->state == ACTIVE && r->issued - r->noticed < DEPTH) issue_chunk(s, r);
  }
  int np = 0, na = 0, nf = 0;
  for (auto &kv : s->reqs) {
    int st = kv.second->state;
    np += st == PENDING;
    na += st == ACTIVE;
    nf += st == FINISHED || st == FAILED;
  }
  if (pending) *pending = np;
  if (active) *active = na;
  if (finished) *finished = nf;
  return HGPU_OK;
}

int hgpu_server_result(hgpu_server *s, long long id, double *p, int *pflag, double *t, long long *steps,
                       double *queue_ms, double *run_ms) {
  if (!s) return HGPU_E_INVALID;
  std::lock_guard<std::mutex> g(s->m);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return HGPU_E_INVALID;
  Request *r = it->second;
  if (r->state == FAILED) return r->rc ? r->rc : HGPU_E_CUDA;
  if (r->state != FINISHED) return HGPU_E_INVALID;
  if (p) memcpy(p, r->p_out.data(), sizeof(double) * r->p_out.size());
  if (pflag) memcpy(pflag, r->pflag_out.data(), sizeof(int) * r->pflag_out.size());
  if (t) *t = r->t_out;
  if (steps) *steps = r->steps;
  if (queue_ms) *queue_ms = ms_between(r->t_submit, r->t_admit);
  if (run_ms) *run_ms = ms_between(r->t_admit, r->t_finish);
  return HGPU_OK;
}

int hgpu_server_release(hgpu_server *s, long long id) {
  if (!s) return HGPU_E_INVALID;
  std::lock_guard<std::mutex> g(s->m);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end() || it->second->state == ACTIVE || it->second->state == PENDING) return HGPU_E_INVALID;
  delete it->second;
  s->reqs.erase(it);
  return HGPU_OK;
}

}  // extern "C"
