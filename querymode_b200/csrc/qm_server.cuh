// Serving loop: continuous batching of single requests over resident tables
// with HBM budget admission (declared in include/qm_gpu.h, "serving loop").
// Included at the end of qm_api.cu: it drives the batched launch through
// that file's internal planning / layout / issue / collect steps.
//
// Several lanes run at once, each a worker thread with its own CUDA stream
// and batch buffers.  A lane that is free takes the requests queued at that
// moment (a heavy request alone, or up to max_batch light ones), plans and
// lays them out under the context lock, issues them on its stream and
// completes each request as soon as that request's result copy has landed.
// So a request that arrives while other batches are on the GPU starts on the
// next free lane at once and its work overlaps theirs; one lane only ever
// takes light requests, so a heavy request (e.g. a 16M-group aggregate)
// never holds back the small ones behind it.
#include <chrono>
#include <condition_variable>
#include <thread>
#include <unordered_map>

namespace {

using srv_clock = std::chrono::steady_clock;

enum ReqState { RQ_QUEUED, RQ_RUNNING, RQ_DONE };

struct Request {
  uint64_t ticket = 0;
  const qm_table *table = nullptr;
  OwnedQuery query;
  ReqState state = RQ_QUEUED;
  bool heavy = false;
  int code = QM_OK;
  std::string msg;
  qm_result *res = nullptr;
  srv_clock::time_point t_submit, t_take, t_launch, t_done;
  int batch_size = 0;
};

int64_t table_device_bytes(const qm_table *t) {
  int64_t b = 0;
  for (const DevCol &c : t->cols) {
    b += t->n_rows * (int64_t)dtype_size(c.dtype);
    if (c.nulls) b += (t->n_rows + 31) / 32 * 4;
  }
  return b;
}

int64_t us_between(srv_clock::time_point a, srv_clock::time_point b) {
  return std::chrono::duration_cast<std::chrono::microseconds>(b - a).count();
}

}  // namespace

struct qm_server;

namespace {

struct Lane {
  int id = 0;
  bool light_only = false;  // takes light requests only
  cudaStream_t stream = nullptr;
  qm_batch *batch = nullptr;
  std::thread th;
};

}  // namespace

struct qm_server {
  qm_ctx *ctx = nullptr;
  qm_server_config cfg{};
  std::mutex mu;  // queue, requests, budget, counters
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> reqs;
  std::unordered_map<const qm_table *, int64_t> tables;
  int64_t resident = 0;
  int64_t in_flight_bytes = 0;  // working memory of the batches on the GPU
  int64_t in_flight_reqs = 0;
  uint64_t budget_gen = 0;  // bumped whenever a batch gives its working memory back
  uint64_t next_ticket = 1;
  bool stop = false;
  qm_server_counters st{};
  std::mutex ctx_mu;  // planning, layout and single-query re-runs on the shared context
  std::vector<std::unique_ptr<Lane>> lanes;

  void complete(const std::shared_ptr<Request> &r, int code, const std::string &msg, qm_result *res) {
    std::lock_guard<std::mutex> lk(mu);
    r->code = code;
    r->msg = msg;
    r->res = res;
    r->t_done = srv_clock::now();
    r->state = RQ_DONE;
    if (code == QM_OK) st.completed++;
    else if (code == QM_ERR_CANCELLED) st.cancelled++;
    else st.failed++;
    if (code == QM_ERR_OOM) st.refused++;
    cv_done.notify_all();
  }

  bool eligible(const Lane &ln, const Request &r) const { return !(ln.light_only && r.heavy); }

  // Under mu: the requests this lane takes now (arrival order among the
  // ones it may take): a heavy request alone, else light requests up to
  // max_batch and max_batch_rows.
  std::vector<std::shared_ptr<Request>> take_for(const Lane &ln) {
    std::vector<std::shared_ptr<Request>> take;
    int64_t rows = 0;
    for (auto it = queue.begin(); it != queue.end();) {
      Request &r = **it;
      if (!eligible(ln, r) || (r.heavy && !take.empty())) {
        ++it;
        continue;
      }
      if (!take.empty() && cfg.max_batch_rows > 0 && rows + r.table->n_rows > cfg.max_batch_rows) {
        ++it;
        continue;
      }
      rows += r.table->n_rows;
      r.state = RQ_RUNNING;
      r.t_take = srv_clock::now();
      take.push_back(*it);
      it = queue.erase(it);
      if (take.back()->heavy || (int)take.size() >= cfg.max_batch) break;
    }
    return take;
  }

  bool has_work_for(const Lane &ln) const {
    for (auto &r : queue)
      if (eligible(ln, *r)) return true;
    return false;
  }

  void requeue_front(std::vector<std::shared_ptr<Request>> &rs) {
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = rs.rbegin(); it != rs.rend(); ++it) {
      (*it)->state = RQ_QUEUED;
      queue.push_front(*it);
    }
  }

  // Plan, admit, issue and collect one batch on lane `ln`.  Returns false
  // when nothing was admitted because the batches in flight hold the budget.
  bool run_batch(Lane &ln, std::vector<std::shared_ptr<Request>> &take) {
    qm_batch *b = ln.batch;
    std::vector<std::shared_ptr<Request>> admitted, deferred, heavy_back;
    int64_t working = 0;
    {
      std::unique_lock<std::mutex> cl(ctx_mu);
      batch_reset(b, (int)take.size());
      int64_t free_bytes;
      {
        std::lock_guard<std::mutex> lk(mu);
        free_bytes = cfg.hbm_budget_bytes - resident - in_flight_bytes;
      }
      const int64_t budget_alone = cfg.hbm_budget_bytes - resident;
      for (auto &r : take) {
        if (!deferred.empty()) {  // keep arrival order behind a deferred request
          deferred.push_back(r);
          continue;
        }
        const int k = (int)admitted.size();
        int rc = batch_plan_one(b, k, r->table, &r->query.q);
        if (rc) {
          complete(r, rc, ctx->err, nullptr);
          continue;
        }
        if (cfg.max_batch_groups > 0 && !r->heavy && b->est[k] > cfg.max_batch_groups &&
            (take.size() > 1 || ln.light_only)) {
          // planned heavy: back to the queue, where it runs alone on a lane that takes heavy requests
          r->heavy = true;
          heavy_back.push_back(r);
          continue;
        }
        const int64_t need = batch_query_bytes(b, k);
        if (need > budget_alone) {
          char m[200];
          snprintf(m, sizeof m, "request needs %lld device bytes; the HBM budget leaves %lld beside resident tables",
                   (long long)need, (long long)budget_alone);
          complete(r, QM_ERR_OOM, m, nullptr);
          continue;
        }
        if (working + need > free_bytes) {
          deferred.push_back(r);
          continue;
        }
        working += need;
        admitted.push_back(r);
      }
      if (!deferred.empty()) requeue_front(deferred);
      if (!heavy_back.empty()) {
        requeue_front(heavy_back);
        cv_work.notify_all();
      }
      const int n = (int)admitted.size();
      if (n == 0) return deferred.empty();
      // the planned queries are b's first n entries
      b->n = n;
      b->gts.resize(n);
      b->bq.resize(n);
      b->rows.resize(n);
      b->est.resize(n);
      b->tabs.resize(n);
      b->ex_plan.resize(n);
      b->queries.resize(n);
      b->total_rows = 0;
      b->bytes_scanned = 0;
      for (int i = 0; i < n; i++) {
        b->total_rows += b->rows[i];
        b->bytes_scanned += b->gts[i].pl.bytes_per_row * b->rows[i];
      }
      int rc = batch_layout(b);
      if (rc) {
        const std::string m = ctx->err;
        cl.unlock();
        for (auto &r : admitted) complete(r, rc, m, nullptr);
        return true;
      }
    }
    const int n = (int)admitted.size();
    const auto t_launch = srv_clock::now();
    {
      std::lock_guard<std::mutex> lk(mu);
      st.batches++;
      in_flight_bytes += working;
      in_flight_reqs += n;
      st.peak_working_bytes = std::max(st.peak_working_bytes, in_flight_bytes);
      st.peak_in_flight = std::max(st.peak_in_flight, in_flight_reqs);
      for (auto &r : admitted) {
        r->t_launch = t_launch;
        r->batch_size = n;
        if (r->heavy) st.heavy++;
      }
    }
    std::vector<int> codes(n, QM_OK);
    std::vector<qm_result *> results(n, nullptr);
    int rc = batch_issue(b, false);
    if (!rc)
      rc = batch_collect(b, results.data(), codes.data(), true, [&](int i, int code, qm_result *res) {
        if (code == QM_OK) complete(admitted[i], QM_OK, std::string(), res);
      });
    if (rc) {
      cudaStreamSynchronize(b->st());
      cudaStreamSynchronize(b->copy_stream);
      std::string m;
      {
        std::lock_guard<std::mutex> cl(ctx_mu);
        m = ctx->err;
      }
      for (int i = 0; i < n; i++)
        if (admitted[i]->state != RQ_DONE) {
          delete results[i];
          complete(admitted[i], rc, m, nullptr);
        }
    } else {
      for (int i = 0; i < n; i++) {
        if (codes[i] == QM_OK) continue;
        if (codes[i] == QM_ERR_CAPACITY) {
          // the group estimate was too small for the batched table: this
          // request alone, where its table regrows
          qm_result *res = nullptr;
          std::string m;
          int rc2;
          {
            std::lock_guard<std::mutex> cl(ctx_mu);
            rc2 = qm_query_run(ctx, admitted[i]->table, &admitted[i]->query.q, &res);
            if (rc2) m = ctx->err;
          }
          complete(admitted[i], rc2, m, res);
        } else {
          complete(admitted[i], codes[i], "device status error in the batched launch", nullptr);
        }
      }
    }
    std::lock_guard<std::mutex> lk(mu);
    in_flight_bytes -= working;
    in_flight_reqs -= n;
    budget_gen++;
    cv_work.notify_all();  // budget freed: other lanes may admit deferred requests
    return true;
  }

  void lane_loop(Lane &ln) {
    cudaSetDevice(ctx->device);
    for (;;) {
      std::vector<std::shared_ptr<Request>> take;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || has_work_for(ln); });
        if (stop) return;
        if (cfg.max_wait_us > 0 && (int)queue.size() < cfg.max_batch) {
          const auto deadline = queue.front()->t_submit + std::chrono::microseconds(cfg.max_wait_us);
          cv_work.wait_until(lk, deadline, [&] { return stop || (int)queue.size() >= cfg.max_batch; });
          if (stop) return;
        }
        take = take_for(ln);
      }
      if (take.empty()) continue;
      uint64_t gen;
      {
        std::lock_guard<std::mutex> lk(mu);
        gen = budget_gen;
      }
      if (!run_batch(ln, take)) {
        // the budget is held by batches in flight: wait for one to end
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || budget_gen != gen || in_flight_reqs == 0; });
      }
    }
  }
};

extern "C" {

int qm_server_create(qm_ctx *ctx, const qm_server_config *cfg, qm_server **out) {
  if (!ctx || !cfg || !out) return QM_ERR_INVALID;
  *out = nullptr;
  if (cfg->max_batch < 1 || cfg->max_batch > QM_BATCH_MAX || cfg->hbm_budget_bytes <= 0 || cfg->max_wait_us < 0 ||
      cfg->lanes < 0 || cfg->lanes > 64 || cfg->max_batch_groups < 0)
    return set_err(ctx, QM_ERR_INVALID,
                   "server config: max_batch 1..%d, a positive budget, max_wait_us >= 0, lanes 0..64, "
                   "max_batch_groups >= 0", QM_BATCH_MAX);
  cudaSetDevice(ctx->device);
  qm_server *s = new qm_server();
  s->ctx = ctx;
  s->cfg = *cfg;
  const int L = cfg->lanes > 0 ? cfg->lanes : 4;
  for (int i = 0; i < L; i++) {
    std::unique_ptr<Lane> ln(new Lane());
    ln->id = i;
    ln->light_only = L > 1 && i == L - 1;
    if (cudaStreamCreateWithFlags(&ln->stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      for (auto &l : s->lanes) {
        delete l->batch;
        cudaStreamDestroy(l->stream);
      }
      delete s;
      return set_err(ctx, QM_ERR_CUDA, "serving lane stream");
    }
    ln->batch = new qm_batch();
    ln->batch->ctx = ctx;
    ln->batch->stream = ln->stream;
    ln->batch->waves_req = 1;
    s->lanes.push_back(std::move(ln));
  }
  // Lanes grow their buffers with stream-ordered allocation from the
  // device's memory pool, which keeps what is freed.  Growing the pool itself
  // maps new memory (hundreds of milliseconds for a gigabyte, measured while
  // the other lanes ran); taking a block of it up front (2 GB per lane, at
  // most an eighth of the budget) and handing it back lets the lanes' large
  // batches reuse that memory instead.
  {
    const int64_t reserve = std::min<int64_t>((int64_t)L << 31, cfg->hbm_budget_bytes / 8);
    void *blk = nullptr;
    if (reserve > 0 && cudaMallocAsync(&blk, (size_t)reserve, ctx->stream) == cudaSuccess) {
      cudaFreeAsync(blk, ctx->stream);
      cudaStreamSynchronize(ctx->stream);
    } else {
      cudaGetLastError();
    }
  }
  // and page-lock 256 MB of result buffers per lane (carved by size class)
  // for the same reason: page-locking during serving holds up every lane's
  // CUDA calls for tens of milliseconds per buffer
  ctx->pool->reserve((size_t)L << 28);
  for (auto &ln : s->lanes) {
    Lane *p = ln.get();
    p->th = std::thread([s, p] { s->lane_loop(*p); });
  }
  *out = s;
  return QM_OK;
}

int qm_server_submit(qm_server *s, const qm_table *table, const qm_query *query, uint64_t *ticket) {
  if (!s || !table || !query || !ticket) return QM_ERR_INVALID;
  if (table->ctx != s->ctx) return QM_ERR_INVALID;
  auto r = std::make_shared<Request>();
  r->table = table;
  r->query.copy(*query);
  r->heavy = s->cfg.max_batch_rows > 0 && table->n_rows > s->cfg.max_batch_rows;
  r->t_submit = srv_clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return QM_ERR_CANCELLED;
    if (!s->tables.count(table)) {
      const int64_t b = table_device_bytes(table);
      s->tables[table] = b;
      s->resident += b;
    }
    r->ticket = s->next_ticket++;
    s->reqs[r->ticket] = r;
    s->queue.push_back(r);
    s->st.submitted++;
    *ticket = r->ticket;
  }
  s->cv_work.notify_all();
  return QM_OK;
}

int qm_server_cancel(qm_server *s, uint64_t ticket) {
  if (!s) return QM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end() || it->second->state != RQ_QUEUED) return QM_ERR_INVALID;
  auto r = it->second;
  for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
    if (*q == r) {
      s->queue.erase(q);
      break;
    }
  r->state = RQ_DONE;
  r->code = QM_ERR_CANCELLED;
  r->msg = "cancelled before launch";
  r->t_done = srv_clock::now();
  s->st.cancelled++;
  s->cv_done.notify_all();
  return QM_OK;
}

int qm_server_wait(qm_server *s, uint64_t ticket, int64_t timeout_us, qm_result **out, qm_server_timing *timing,
                   char *msg, size_t msg_len) {
  if (!s) return QM_ERR_INVALID;
  if (out) *out = nullptr;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return QM_ERR_INVALID;
  auto r = it->second;
  auto done = [&] { return r->state == RQ_DONE; };
  if (timeout_us < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), done)) {
    return QM_ERR_TIMEOUT;
  }
  s->reqs.erase(it);
  if (timing) {
    memset(timing, 0, sizeof *timing);
    const bool launched = r->batch_size > 0;
    timing->queued_us = us_between(r->t_submit, launched ? r->t_launch : r->t_done);
    timing->run_us = launched ? us_between(r->t_launch, r->t_done) : 0;
    timing->total_us = us_between(r->t_submit, r->t_done);
    timing->batch_size = r->batch_size;
    timing->plan_us = launched ? (int32_t)us_between(r->t_take, r->t_launch) : 0;
  }
  if (msg && msg_len) snprintf(msg, msg_len, "%s", r->msg.c_str());
  if (out) *out = r->res;
  else delete r->res;
  r->res = nullptr;
  return r->code;
}

int qm_server_stats(qm_server *s, qm_server_counters *out) {
  if (!s || !out) return QM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->resident_bytes = s->resident;
  out->queued = (int64_t)s->queue.size();
  out->lanes = (int64_t)s->lanes.size();
  return QM_OK;
}

int qm_server_destroy(qm_server *s) {
  if (!s) return QM_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto &ln : s->lanes)
    if (ln->th.joinable()) ln->th.join();
  for (auto &kv : s->reqs) {
    delete kv.second->res;
    kv.second->res = nullptr;
  }
  cudaSetDevice(s->ctx->device);
  for (auto &ln : s->lanes) {
    cudaStreamSynchronize(ln->stream);
    delete ln->batch;
    cudaStreamDestroy(ln->stream);
  }
  cudaStreamSynchronize(s->ctx->stream);
  delete s;
  return QM_OK;
}

}  // extern "C"
