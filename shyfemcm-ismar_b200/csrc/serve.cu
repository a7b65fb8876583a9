// serve.cu -- a continuous-batching request loop for forecast runs.
//
// Requests (a basin, its parameters, an initial state and a step count)
// arrive at any time.  A request is admitted as soon as a slot is free and
// its device footprint (shygpu_footprint) fits what is left of the HBM
// budget; its state then stays resident on the device until it finishes.
// Every admitted run is a model of its own with its own CUDA stream and
// CUDA-graph time step, so the runs' kernels overlap on the device.  Each
// call of shygpu_serve_progress enqueues the next quantum of steps of every
// run whose previous quantum has finished, retires finished runs (their
// results are copied to host memory and their device memory is freed) and
// admits queued requests in arrival order.  A run's arithmetic does not
// depend on what else is in flight, so its result is the same alone and in
// the mix.
//
// The loop is a client of the library's own C ABI (shygpu_create,
// shygpu_set_state, shygpu_enqueue, shygpu_get_state, shygpu_destroy).
// There is no counterpart in the reference, which runs one simulation per
// process.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/shygpu.h"

namespace shy {
int external_fail(int code, const char *msg);
}

namespace {

enum ReqState { Q_QUEUED = 0, Q_ACTIVE = 1, Q_DONE = 2, Q_FAILED = 3 };

template <typename T>
void copy_in(std::vector<T> &dst, const T *src, size_t n) {
  if (src) dst.assign(src, src + n);
  else dst.clear();
}
template <typename T>
const T *ptr_or_null(const std::vector<T> &v) { return v.empty() ? nullptr : v.data(); }
template <typename T>
void drop(std::vector<T> &v) { std::vector<T>().swap(v); }

struct Request {
  int64_t id = 0;
  int state = Q_QUEUED;
  int32_t nsteps = 0, enqueued = 0;
  int64_t footprint = 0;
  double t_submit = 0., t_admit = -1., t_done = -1.;
  std::string error;
  // owned copies of the inputs
  shy_basin b{};
  shy_params p{};
  std::vector<int32_t> nen3v, ilhv, ilhkv, bnd;
  std::vector<float> xgv, ygv, hm3v, hlv, hldv, czv, fcorv, visv, difv, taux, tauy, ppv, rqv, tide;
  std::vector<float> z0, u0, v0, t0, s0, c0;
  // device run
  shygpu_model *m = nullptr;
  cudaEvent_t ev = nullptr;
  bool in_flight = false;
  // a preempted run's device arrays (shygpu_checkpoint_save), loaded back
  // when it is admitted again
  std::vector<unsigned char> ckpt;
  int32_t preemptions = 0;
  // results
  std::vector<float> rz, ru, rv, rt, rs, rc;
  shy_step_info info{};
};

}  // namespace

struct shygpu_server {
  int64_t budget = 0, used = 0;
  int32_t max_active = 1, quantum = 1;
  int64_t next_id = 1;
  std::deque<Request *> queue;
  std::vector<Request *> active;
  std::map<int64_t, std::unique_ptr<Request>> all;
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

static int sfail(int code, const char *fmt, ...) {
  char msg[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  return shy::external_fail(code, msg);
}

extern "C" int shygpu_serve_create(int64_t hbm_budget, int32_t max_active, int32_t quantum_steps,
                                   shygpu_server **out) {
  if (!out) return sfail(SHY_EARG, "serve_create: server pointer is NULL");
  *out = nullptr;
  if (hbm_budget <= 0 || max_active < 1 || quantum_steps < 1)
    return sfail(SHY_EARG, "serve_create: budget > 0, max_active >= 1, quantum >= 1");
  shygpu_server *s = new shygpu_server;
  s->budget = hbm_budget;
  s->max_active = max_active;
  s->quantum = quantum_steps;
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return SHY_OK;
}

extern "C" int shygpu_serve_submit(shygpu_server *s, const shy_basin *bs, const shy_params *ps,
                                   const shy_state *init, int32_t nsteps, int64_t *id_out) {
  if (!s || !bs || !ps || !init || nsteps < 1) return sfail(SHY_EARG, "serve_submit: bad arguments");
  const int64_t fp = shygpu_footprint(1, bs, ps);
  if (fp < 0) return sfail(SHY_EARG, "serve_submit: bad basin");
  if (fp > s->budget)
    return sfail(SHY_ECAPACITY, "serve_submit: footprint %lld bytes exceeds the server's budget", (long long)fp);
  std::unique_ptr<Request> r(new Request);
  const size_t nkn = bs->nkn, nel = bs->nel, nlv = bs->nlv;
  copy_in(r->nen3v, bs->nen3v, 3 * nel);
  copy_in(r->xgv, bs->xgv, nkn);
  copy_in(r->ygv, bs->ygv, nkn);
  copy_in(r->hm3v, bs->hm3v, 3 * nel);
  copy_in(r->hlv, bs->hlv, nlv);
  copy_in(r->hldv, bs->hldv, nlv);
  copy_in(r->ilhv, bs->ilhv, nel);
  copy_in(r->ilhkv, bs->ilhkv, nkn);
  copy_in(r->czv, bs->czv, nel);
  copy_in(r->fcorv, bs->fcorv, nel);
  copy_in(r->visv, bs->visv, (nlv + 1) * nkn);
  copy_in(r->difv, bs->difv, (nlv + 1) * nkn);
  copy_in(r->taux, bs->tauxnv, nkn);
  copy_in(r->tauy, bs->tauynv, nkn);
  copy_in(r->ppv, bs->ppv, nkn);
  copy_in(r->rqv, bs->rqv, nkn);
  copy_in(r->bnd, bs->bnd_index, nkn);
  copy_in(r->tide, bs->tide, (size_t)4 * bs->ntide * bs->nbnd);
  r->b = *bs;
  r->b.nen3v = ptr_or_null(r->nen3v); r->b.xgv = ptr_or_null(r->xgv); r->b.ygv = ptr_or_null(r->ygv);
  r->b.hm3v = ptr_or_null(r->hm3v); r->b.hlv = ptr_or_null(r->hlv); r->b.hldv = ptr_or_null(r->hldv);
  r->b.ilhv = ptr_or_null(r->ilhv); r->b.ilhkv = ptr_or_null(r->ilhkv); r->b.czv = ptr_or_null(r->czv);
  r->b.fcorv = ptr_or_null(r->fcorv); r->b.visv = ptr_or_null(r->visv); r->b.difv = ptr_or_null(r->difv);
  r->b.tauxnv = ptr_or_null(r->taux); r->b.tauynv = ptr_or_null(r->tauy); r->b.ppv = ptr_or_null(r->ppv);
  r->b.rqv = ptr_or_null(r->rqv); r->b.bnd_index = ptr_or_null(r->bnd); r->b.tide = ptr_or_null(r->tide);
  r->p = *ps;
  const int ntr = ps->nconz > 0 ? ps->nconz : 0;
  copy_in(r->z0, init->znv, nkn);
  copy_in(r->u0, init->utlnv, nel * nlv);
  copy_in(r->v0, init->vtlnv, nel * nlv);
  copy_in(r->t0, ps->itemp ? init->tempv : nullptr, nkn * nlv);
  copy_in(r->s0, ps->isalt ? init->saltv : nullptr, nkn * nlv);
  copy_in(r->c0, ntr ? init->conzv : nullptr, (size_t)ntr * nkn * nlv);
  r->nsteps = nsteps;
  r->footprint = fp;
  std::lock_guard<std::mutex> lock(s->mu);
  r->id = s->next_id++;
  r->t_submit = s->now();
  if (id_out) *id_out = r->id;
  s->queue.push_back(r.get());
  s->all[r->id] = std::move(r);
  return SHY_OK;
}

static void retire(shygpu_server *s, Request *r, bool ok) {
  if (r->m) {
    if (ok) {
      const size_t nkn = r->b.nkn, nel = r->b.nel, nlv = r->b.nlv;
      r->rz.resize(nkn);
      r->ru.resize(nel * nlv);
      r->rv.resize(nel * nlv);
      shy_state st{};
      st.znv = r->rz.data(); st.utlnv = r->ru.data(); st.vtlnv = r->rv.data();
      if (r->p.itemp) { r->rt.resize(nkn * nlv); st.tempv = r->rt.data(); }
      if (r->p.isalt) { r->rs.resize(nkn * nlv); st.saltv = r->rs.data(); }
      if (r->p.nconz > 0) { r->rc.resize((size_t)r->p.nconz * nkn * nlv); st.conzv = r->rc.data(); }
      if (shygpu_get_state(r->m, 0, &st) != SHY_OK) { ok = false; r->error = shygpu_last_error(); }
      shygpu_step_info(r->m, 0, &r->info);
    }
    shygpu_destroy(r->m);
    r->m = nullptr;
  }
  if (r->ev) { cudaEventDestroy(r->ev); r->ev = nullptr; }
  s->used -= r->footprint;
  r->state = ok ? Q_DONE : Q_FAILED;
  r->t_done = s->now();
  // the inputs are no longer needed
  drop(r->nen3v); drop(r->xgv); drop(r->ygv); drop(r->hm3v); drop(r->visv); drop(r->difv);
  drop(r->z0); drop(r->u0); drop(r->v0); drop(r->t0); drop(r->s0); drop(r->c0);
}

static bool admit(shygpu_server *s, Request *r) {
  if (shygpu_create(1, &r->b, &r->p, &r->m) != SHY_OK) { r->error = shygpu_last_error(); return false; }
  if (!r->ckpt.empty()) {           // a preempted run continues where it stopped
    if (shygpu_checkpoint_load(r->m, r->ckpt.data(), (int64_t)r->ckpt.size()) != SHY_OK) {
      r->error = shygpu_last_error();
      return false;
    }
    std::vector<unsigned char>().swap(r->ckpt);
  } else {
    shy_state st{};
    st.znv = r->z0.empty() ? nullptr : r->z0.data();
    st.utlnv = r->u0.empty() ? nullptr : r->u0.data();
    st.vtlnv = r->v0.empty() ? nullptr : r->v0.data();
    st.tempv = r->t0.empty() ? nullptr : r->t0.data();
    st.saltv = r->s0.empty() ? nullptr : r->s0.data();
    st.conzv = r->c0.empty() ? nullptr : r->c0.data();
    if (shygpu_set_state(r->m, 0, &st) != SHY_OK) { r->error = shygpu_last_error(); return false; }
  }
  if (cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming) != cudaSuccess) {
    r->error = "event creation failed";
    return false;
  }
  r->state = Q_ACTIVE;
  r->t_admit = s->now();
  return true;
}

extern "C" int shygpu_serve_progress(shygpu_server *s, int32_t block, int32_t *n_active, int32_t *n_queued,
                                     int32_t *n_done) {
  if (!s) return sfail(SHY_EARG, "serve_progress: server is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  // optionally wait for the oldest quantum in flight
  if (block) {
    for (Request *r : s->active)
      if (r->in_flight) { cudaEventSynchronize(r->ev); break; }
  }
  int finished = 0;
  // retire or continue the active runs
  for (size_t i = 0; i < s->active.size();) {
    Request *r = s->active[i];
    if (r->in_flight) {
      const cudaError_t q = cudaEventQuery(r->ev);
      if (q == cudaErrorNotReady) { i++; continue; }
      r->in_flight = false;
      if (q != cudaSuccess) { r->error = cudaGetErrorString(q); retire(s, r, false); }
    }
    if (r->state == Q_ACTIVE && r->enqueued >= r->nsteps) {
      const int st = shygpu_sync(r->m);
      if (st != SHY_OK) r->error = shygpu_last_error();
      retire(s, r, st == SHY_OK);
    }
    if (r->state != Q_ACTIVE) {
      s->active.erase(s->active.begin() + i);
      finished++;
      continue;
    }
    const int32_t q = std::min(s->quantum, r->nsteps - r->enqueued);
    int st = shygpu_enqueue(r->m, q);
    if (st == SHY_OK && cudaEventRecord(r->ev, (cudaStream_t)shygpu_model_stream(r->m)) != cudaSuccess) st = SHY_ECUDA;
    if (st != SHY_OK) {
      r->error = shygpu_last_error();
      retire(s, r, false);
      s->active.erase(s->active.begin() + i);
      finished++;
      continue;
    }
    r->enqueued += q;
    r->in_flight = true;
    i++;
  }
  // admit in arrival order while a slot and the budget allow
  while (!s->queue.empty() && (int32_t)s->active.size() < s->max_active &&
         s->used + s->queue.front()->footprint <= s->budget) {
    Request *r = s->queue.front();
    s->queue.pop_front();
    s->used += r->footprint;
    if (!admit(s, r)) {
      retire(s, r, false);
      finished++;
      continue;
    }
    const int32_t q = std::min(s->quantum, r->nsteps - r->enqueued);
    if (shygpu_enqueue(r->m, q) != SHY_OK ||
        cudaEventRecord(r->ev, (cudaStream_t)shygpu_model_stream(r->m)) != cudaSuccess) {
      r->error = shygpu_last_error();
      retire(s, r, false);
      finished++;
      continue;
    }
    r->enqueued += q;
    r->in_flight = true;
    s->active.push_back(r);
  }
  if (n_active) *n_active = (int32_t)s->active.size();
  if (n_queued) *n_queued = (int32_t)s->queue.size();
  if (n_done) *n_done = finished;
  return SHY_OK;
}

// Preemption: an active run is stopped after its quantum in flight, its
// device arrays go to host memory (an exact checkpoint) and its device
// memory is freed, so the requests already waiting are admitted first; it
// queues behind them and, once admitted again, continues bit for bit.
extern "C" int shygpu_serve_preempt(shygpu_server *s, int64_t id) {
  if (!s) return sfail(SHY_EARG, "serve_preempt: server is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return sfail(SHY_EARG, "serve_preempt: unknown request %lld", (long long)id);
  Request *r = it->second.get();
  if (r->state != Q_ACTIVE) return sfail(SHY_ESTATE, "serve_preempt: request %lld is not running", (long long)id);
  if (r->in_flight) {
    cudaEventSynchronize(r->ev);
    r->in_flight = false;
  }
  int st = shygpu_sync(r->m);
  if (st == SHY_OK) {
    const int64_t n = shygpu_checkpoint_bytes(r->m);
    r->ckpt.resize((size_t)n);
    st = shygpu_checkpoint_save(r->m, r->ckpt.data(), n);
  }
  auto pos = std::find(s->active.begin(), s->active.end(), r);
  if (pos != s->active.end()) s->active.erase(pos);
  if (st != SHY_OK) {
    r->error = shygpu_last_error();
    retire(s, r, false);
    return sfail(st, "serve_preempt: request %lld failed: %s", (long long)id, r->error.c_str());
  }
  shygpu_destroy(r->m);
  r->m = nullptr;
  cudaEventDestroy(r->ev);
  r->ev = nullptr;
  s->used -= r->footprint;
  r->state = Q_QUEUED;
  r->preemptions++;
  s->queue.push_back(r);
  return SHY_OK;
}

extern "C" int shygpu_serve_status(shygpu_server *s, int64_t id, int32_t *state, int32_t *steps_enqueued,
                                   double *t_submit, double *t_admit, double *t_done) {
  if (!s) return sfail(SHY_EARG, "serve_status: server is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return sfail(SHY_EARG, "serve_status: unknown request %lld", (long long)id);
  const Request *r = it->second.get();
  if (state) *state = r->state;
  if (steps_enqueued) *steps_enqueued = r->enqueued;
  if (t_submit) *t_submit = r->t_submit;
  if (t_admit) *t_admit = r->t_admit;
  if (t_done) *t_done = r->t_done;
  return SHY_OK;
}

extern "C" int shygpu_serve_result(shygpu_server *s, int64_t id, shy_state *out, shy_step_info *info) {
  if (!s) return sfail(SHY_EARG, "serve_result: server is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return sfail(SHY_EARG, "serve_result: unknown request %lld", (long long)id);
  Request *r = it->second.get();
  if (r->state == Q_FAILED) return sfail(SHY_ESTATE, "serve_result: request failed: %s", r->error.c_str());
  if (r->state != Q_DONE) return sfail(SHY_ESTATE, "serve_result: request %lld not finished", (long long)id);
  if (out) {
    if (out->znv) memcpy(out->znv, r->rz.data(), r->rz.size() * 4);
    if (out->utlnv) memcpy(out->utlnv, r->ru.data(), r->ru.size() * 4);
    if (out->vtlnv) memcpy(out->vtlnv, r->rv.data(), r->rv.size() * 4);
    if (out->tempv && !r->rt.empty()) memcpy(out->tempv, r->rt.data(), r->rt.size() * 4);
    if (out->saltv && !r->rs.empty()) memcpy(out->saltv, r->rs.data(), r->rs.size() * 4);
    if (out->conzv && !r->rc.empty()) memcpy(out->conzv, r->rc.data(), r->rc.size() * 4);
  }
  if (info) *info = r->info;
  return SHY_OK;
}

extern "C" int shygpu_serve_release(shygpu_server *s, int64_t id) {
  if (!s) return sfail(SHY_EARG, "serve_release: server is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return sfail(SHY_EARG, "serve_release: unknown request %lld", (long long)id);
  if (it->second->state == Q_QUEUED || it->second->state == Q_ACTIVE)
    return sfail(SHY_ESTATE, "serve_release: request %lld still queued or running", (long long)id);
  s->all.erase(it);
  return SHY_OK;
}

extern "C" int64_t shygpu_serve_used(shygpu_server *s) { return s ? s->used : -1; }

extern "C" int shygpu_serve_destroy(shygpu_server *s) {
  if (!s) return SHY_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    for (Request *r : s->active) retire(s, r, false);
    s->active.clear();
    s->queue.clear();
    s->all.clear();
  }
  delete s;
  return SHY_OK;
}
