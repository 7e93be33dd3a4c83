// Serving form: a request loop over a stream of assemblies (rbg_server_*).
//
// Requests are validated and queued on submit.  Each worker thread owns a
// device context; it takes every queued request, oldest first, whose device
// memory estimate fits into its share of the HBM budget (budget / workers)
// and runs them as one batch through the batch engine, so requests that
// arrive while others are on the GPU are folded into the next launch; inside
// a batch the copies of later requests overlap the work of earlier ones.
// With two or more workers the batches of different workers also overlap on
// the device (separate streams); one worker is the default.  A worker's device buffers grow to its largest batch
// and stay allocated, so the budget share bounds its footprint.
//
// The plain mode runs one worker and one rbg_bin_graph call per request: the
// unbatched path, for comparisons on the same arrival stream.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "engine_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  rbg_assembly a{};
  rbg_params p{};                       // copy of the caller's parameters
  int64_t est_bytes = 0, pairs = 0;
  Clock::time_point t_submit, t_start, t_done;
  int status = 1;                       // 1: not finished
  std::string err;
  rbg_graph g{};
  int batch_size = 0, worker = -1;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct rbg_server {
  rbg_server_config cfg{};
  rbg_params defaults{};
  int64_t share = 0;                    // bytes per worker batch
  Clock::time_point t_created;
  std::vector<rbg_ctx *> ctxs;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<int64_t, std::shared_ptr<Request>> reqs;
  int64_t next_id = 1;
  bool stop = false;
  std::string err;

  void worker_loop(int w);
  void run_batch_of(int w, std::vector<std::shared_ptr<Request>> &take);
};

void rbg_server::worker_loop(int w) {
  const size_t max_batch = cfg.plain ? 1 : (size_t)cfg.max_batch;
  for (;;) {
    std::vector<std::shared_ptr<Request>> take;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stop || !queue.empty(); });
      if (queue.empty()) return;         // stop requested and nothing left
      int64_t bytes = 0, pairs = 0;
      while (!queue.empty() && take.size() < max_batch) {
        const std::shared_ptr<Request> &r = queue.front();
        if (!take.empty() &&
            (bytes + r->est_bytes > share || pairs + r->pairs > cfg.max_batch_pairs))
          break;
        bytes += r->est_bytes;
        pairs += r->pairs;
        take.push_back(r);
        queue.pop_front();
      }
    }
    const Clock::time_point t0 = Clock::now();
    for (auto &r : take) {
      r->t_start = t0;
      r->worker = w;
      r->batch_size = (int)take.size();
    }
    run_batch_of(w, take);
    {
      std::lock_guard<std::mutex> lk(mu);
      const Clock::time_point t1 = Clock::now();
      for (auto &r : take) r->t_done = t1;
    }
    cv_done.notify_all();
  }
}

void rbg_server::run_batch_of(int w, std::vector<std::shared_ptr<Request>> &take) {
  rbg_ctx *c = ctxs[w];
  const int nb = (int)take.size();
  std::vector<rbg_graph> outs(nb);
  int rc;
  if (cfg.plain) {
    Request &r = *take[0];
    rc = rbg_bin_graph(c, &r.p, r.a.seqcat, r.a.offsets, r.a.n, r.a.depth, r.a.S, &outs[0]);
  } else {
    std::vector<rbg_assembly> asms(nb);
    for (int i = 0; i < nb; ++i) {
      asms[i] = take[i]->a;
      asms[i].params = &take[i]->p;
    }
    rc = rbg_bin_batch(c, &defaults, asms.data(), nb, outs.data(), nullptr);
  }
  std::lock_guard<std::mutex> lk(mu);
  const std::string e = rc == RBG_OK ? std::string() : std::string(rbg_last_error(c));
  for (int i = 0; i < nb; ++i) {
    take[i]->status = rc;
    take[i]->err = e;
    if (rc == RBG_OK) take[i]->g = outs[i];
  }
  if (rc != RBG_OK) err = e;
}

extern "C" {

int rbg_server_create(const rbg_server_config *cfg, const rbg_params *defaults,
                      rbg_server **out) {
  if (!cfg || !out) return RBG_ERR_ARG;
  *out = nullptr;
  auto *s = new (std::nothrow) rbg_server();
  if (!s) return RBG_ERR_NOMEM;
  s->cfg = *cfg;
  if (defaults) s->defaults = *defaults; else rbg_default_params(&s->defaults);
  if (s->cfg.plain) s->cfg.workers = 1;
  if (s->cfg.workers <= 0) s->cfg.workers = 1;
  if (s->cfg.max_batch <= 0) s->cfg.max_batch = 64;
  if (s->cfg.max_batch_pairs <= 0) s->cfg.max_batch_pairs = 2000000000LL;
  s->t_created = Clock::now();
  if (s->cfg.hbm_budget <= 0) s->cfg.hbm_budget = (int64_t)150 << 30;
  size_t freeb = 0, total = 0;
  if (cudaSetDevice(cfg->device) != cudaSuccess || cudaMemGetInfo(&freeb, &total) != cudaSuccess) {
    delete s;
    return RBG_ERR_CUDA;
  }
  // leave room for the library's own allocations (tables, pinned staging)
  const int64_t usable = (int64_t)freeb - ((int64_t)2 << 30);
  s->cfg.hbm_budget = std::min<int64_t>(s->cfg.hbm_budget, std::max<int64_t>(usable, 1));
  s->share = s->cfg.hbm_budget / s->cfg.workers;
  for (int w = 0; w < s->cfg.workers; ++w) {
    rbg_ctx *c = nullptr;
    const int rc = rbg_create(cfg->device, &c);
    if (rc != RBG_OK) {
      for (rbg_ctx *x : s->ctxs) rbg_destroy(x);
      delete s;
      return rc;
    }
    s->ctxs.push_back(c);
  }
  for (int w = 0; w < s->cfg.workers; ++w) s->workers.emplace_back([s, w] { s->worker_loop(w); });
  *out = s;
  return RBG_OK;
}

int rbg_server_submit(rbg_server *s, const rbg_assembly *a, int64_t *request_id) {
  if (!s || !a || !request_id) return RBG_ERR_ARG;
  auto r = std::make_shared<Request>();
  r->a = *a;
  r->p = a->params ? *a->params : s->defaults;
  r->a.params = nullptr;
  try {
    rbg::validate_assembly(r->a, &r->p, "");
    const int64_t nbases = r->a.n > 0 ? r->a.offsets[r->a.n] : 0;
    r->est_bytes = rbg::batch_request_bytes(&r->p, r->a.n, nbases, r->a.S);
    r->pairs = r->a.n * (r->a.n - 1) / 2;
  } catch (const rbg::Error &e) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = e.what();
    return e.code;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    s->err = "the server is shutting down";
    return RBG_ERR_ARG;
  }
  if (r->est_bytes > s->share) {
    s->err = "the request needs " + std::to_string(r->est_bytes) +
             " bytes of device memory, more than a worker's share of the HBM budget (" +
             std::to_string(s->share) + ")";
    return RBG_ERR_NOMEM;
  }
  r->id = s->next_id++;
  r->t_submit = Clock::now();
  s->reqs[r->id] = r;
  s->queue.push_back(r);
  *request_id = r->id;
  s->cv_work.notify_one();
  return RBG_OK;
}

int rbg_server_wait(rbg_server *s, int64_t id, double timeout_s, rbg_graph *out,
                    rbg_request_stats *st) {
  if (!s || !out) return RBG_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) {
    s->err = "unknown request id " + std::to_string(id);
    return RBG_ERR_ARG;
  }
  std::shared_ptr<Request> r = it->second;
  auto done = [&] { return r->status != 1 && r->t_done != Clock::time_point(); };
  if (timeout_s < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    return RBG_ERR_TIMEOUT;
  }
  s->reqs.erase(it);
  if (st) {
    st->queue_ms = ms_between(r->t_submit, r->t_start);
    st->service_ms = ms_between(r->t_start, r->t_done);
    st->latency_ms = ms_between(r->t_submit, r->t_done);
    st->batch_size = r->batch_size;
    st->worker = r->worker;
    st->est_bytes = r->est_bytes;
    st->submit_s = ms_between(s->t_created, r->t_submit) / 1000.0;
    st->done_s = ms_between(s->t_created, r->t_done) / 1000.0;
  }
  if (r->status != RBG_OK) {
    s->err = r->err;
    return r->status;
  }
  *out = r->g;
  return RBG_OK;
}

const char *rbg_server_last_error(rbg_server *s) { return s ? s->err.c_str() : "null server"; }

int rbg_server_destroy(rbg_server *s) {
  if (!s) return RBG_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto &t : s->workers) t.join();
  for (auto &kv : s->reqs)
    if (kv.second->status == RBG_OK) rbg_free_graph(&kv.second->g);
  for (rbg_ctx *c : s->ctxs) rbg_destroy(c);
  delete s;
  return RBG_OK;
}

}  // extern "C"
