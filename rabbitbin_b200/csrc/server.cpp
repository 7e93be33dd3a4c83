// Serving form: a request loop over a stream of assemblies (rbg_server_*).
//
// Requests are validated and queued on submit, in one of two size classes:
// small (at most small_pairs contig pairs) and large.  Each lane is a worker
// thread with its own device context and stream.  Lane 0 takes large requests
// first and small ones when no large one waits; the other lanes take small
// requests only.  A lane that becomes free folds every queued request of its
// class, oldest first, that fits into the HBM budget left by the batches
// already running (admission against a global budget; a batch's reservation
// is released the moment it finishes, and the lanes waiting for memory are
// woken), up to max_batch requests and max_batch_pairs pairs, and runs them as
// one call: rbg_bin_graph for each large request, one rbg_bin_batch for the
// small ones.  So a request that arrives while others are on the
// GPU is admitted as soon as a lane of its class and the memory are free; a
// small request never waits behind a large batch, and the lanes' batches
// overlap on the device (their streams run concurrently).  Inside a batch the
// copies of later requests overlap the work of earlier ones.  A lane's device
// buffers grow to its largest batch and are kept for the next one.
//
// The plain mode runs one lane and one rbg_bin_graph call per request, in
// arrival order: the unbatched path, for comparisons on the same stream.
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
  int64_t reserved = 0;                 // device bytes of the batches running now
  Clock::time_point t_created;
  std::vector<rbg_ctx *> ctxs;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue[2];   // 0: large, 1: small
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
    int64_t bytes = 0;
    {
      std::unique_lock<std::mutex> lk(mu);
      for (;;) {
        // the queue this lane serves now: lane 0 large first, the others small only
        std::deque<std::shared_ptr<Request>> *q = nullptr;
        if (w == 0 && !queue[0].empty()) q = &queue[0];
        else if (!queue[1].empty() && (w > 0 || cfg.plain || queue[0].empty())) q = &queue[1];
        if (!q) {
          if (stop) return;                // stop requested and nothing left for this lane
          cv_work.wait(lk);
          continue;
        }
        int64_t pairs = 0;
        while (!q->empty() && take.size() < max_batch) {
          const std::shared_ptr<Request> &r = q->front();
          // admission against the budget the running batches leave; alone on an
          // idle device a request is always admitted (submit checked its size)
          const bool fits = reserved + bytes + r->est_bytes <= cfg.hbm_budget ||
                            (reserved == 0 && take.empty());
          if (!fits || (!take.empty() && pairs + r->pairs > cfg.max_batch_pairs)) break;
          bytes += r->est_bytes;
          pairs += r->pairs;
          take.push_back(r);
          q->pop_front();
        }
        if (!take.empty()) break;
        cv_work.wait(lk);                  // memory frees when a running batch finishes
      }
      reserved += bytes;
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
      reserved -= bytes;
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

// Large requests go through rbg_bin_graph one by one (its all-pairs pass over
// one assembly, behind that assembly's own input copy, is faster than the
// batch engine's shared kernel for one large assembly), the small ones of the
// batch through one rbg_bin_batch call.
void rbg_server::run_batch_of(int w, std::vector<std::shared_ptr<Request>> &take) {
  rbg_ctx *c = ctxs[w];
  const int nb = (int)take.size();
  std::vector<rbg_graph> outs(nb);
  std::vector<int> rcs(nb, RBG_OK);
  std::vector<std::string> errs(nb);
  std::vector<int> small;
  for (int i = 0; i < nb; ++i) {
    Request &r = *take[i];
    if (cfg.plain || r.pairs > cfg.small_pairs) {
      rcs[i] = rbg_bin_graph(c, &r.p, r.a.seqcat, r.a.offsets, r.a.n, r.a.depth, r.a.S, &outs[i]);
      if (rcs[i] != RBG_OK) errs[i] = rbg_last_error(c);
    } else {
      small.push_back(i);
    }
  }
  if (!small.empty()) {
    const int ns = (int)small.size();
    std::vector<rbg_assembly> asms(ns);
    std::vector<rbg_graph> so(ns);
    for (int t = 0; t < ns; ++t) {
      asms[t] = take[small[t]]->a;
      asms[t].params = &take[small[t]]->p;
    }
    const int rc = rbg_bin_batch(c, &defaults, asms.data(), ns, so.data(), nullptr);
    const std::string e = rc == RBG_OK ? std::string() : std::string(rbg_last_error(c));
    for (int t = 0; t < ns; ++t) {
      rcs[small[t]] = rc;
      errs[small[t]] = e;
      outs[small[t]] = so[t];
    }
  }
  std::lock_guard<std::mutex> lk(mu);
  for (int i = 0; i < nb; ++i) {
    take[i]->status = rcs[i];
    take[i]->err = errs[i];
    if (rcs[i] == RBG_OK) take[i]->g = outs[i];
    else err = errs[i];
  }
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
  if (s->cfg.workers <= 0) s->cfg.workers = 2;
  if (s->cfg.small_pairs <= 0) s->cfg.small_pairs = 200000000LL;
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
  if (r->est_bytes > s->cfg.hbm_budget) {
    s->err = "the request needs " + std::to_string(r->est_bytes) +
             " bytes of device memory, more than the HBM budget (" +
             std::to_string(s->cfg.hbm_budget) + ")";
    return RBG_ERR_NOMEM;
  }
  r->id = s->next_id++;
  r->t_submit = Clock::now();
  s->reqs[r->id] = r;
  // the plain mode keeps one arrival-order queue
  s->queue[!s->cfg.plain && r->pairs <= s->cfg.small_pairs ? 1 : 0].push_back(r);
  *request_id = r->id;
  s->cv_work.notify_all();
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
