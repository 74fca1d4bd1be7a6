// Serving loop: continuous batching of single requests over resident tables
// with HBM budget admission (declared in include/qm_gpu.h, "serving loop").
// Included at the end of qm_api.cu: it drives the batched launch through
// that file's internal planning / layout / execution steps.
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
  int code = QM_OK;
  std::string msg;
  qm_result *res = nullptr;
  srv_clock::time_point t_submit, t_launch, t_done;
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

struct qm_server {
  qm_ctx *ctx = nullptr;
  qm_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> reqs;
  std::unordered_map<const qm_table *, int64_t> tables;
  int64_t resident = 0;
  uint64_t next_ticket = 1;
  bool stop = false;
  qm_server_counters st{};
  qm_batch *batch = nullptr;
  std::thread worker;

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

  void run_batch(std::vector<std::shared_ptr<Request>> &take) {
    qm_batch *b = batch;
    int64_t free_bytes;
    {
      std::lock_guard<std::mutex> lk(mu);
      free_bytes = cfg.hbm_budget_bytes - resident;
    }
    batch_reset(b, (int)take.size());
    std::vector<std::shared_ptr<Request>> admitted, deferred;
    int64_t working = 0, rows = 0;
    for (auto &r : take) {
      if (!deferred.empty()) {  // keep arrival order behind a deferred request
        deferred.push_back(r);
        continue;
      }
      const int k = (int)admitted.size();
      if (k > 0 && cfg.max_batch_rows > 0 && rows + r->table->n_rows > cfg.max_batch_rows) {
        deferred.push_back(r);
        continue;
      }
      int rc = batch_plan_one(b, k, r->table, &r->query.q);
      if (rc) {
        complete(r, rc, ctx->err, nullptr);
        continue;
      }
      const int64_t need = batch_query_bytes(b, k);
      if (need > free_bytes) {
        char m[200];
        snprintf(m, sizeof m, "request needs %lld device bytes; the HBM budget leaves %lld beside resident tables",
                 (long long)need, (long long)free_bytes);
        complete(r, QM_ERR_OOM, m, nullptr);
        continue;
      }
      if (working + need > free_bytes) {
        deferred.push_back(r);
        continue;
      }
      working += need;
      rows += r->table->n_rows;
      admitted.push_back(r);
    }
    if (!deferred.empty()) {
      std::lock_guard<std::mutex> lk(mu);
      for (auto it = deferred.rbegin(); it != deferred.rend(); ++it) {
        (*it)->state = RQ_QUEUED;
        queue.push_front(*it);
      }
    }
    const int n = (int)admitted.size();
    if (n == 0) return;
    b->n = n;
    b->gts.resize(n);
    b->bq.resize(n);
    b->rows.resize(n);
    b->est.resize(n);
    b->total_rows = 0;
    b->bytes_scanned = 0;
    for (int i = 0; i < n; i++) {
      b->total_rows += b->rows[i];
      b->bytes_scanned += b->gts[i].pl.bytes_per_row * b->rows[i];
    }
    const auto t_launch = srv_clock::now();
    {
      std::lock_guard<std::mutex> lk(mu);
      st.batches++;
      st.peak_working_bytes = std::max(st.peak_working_bytes, working);
      for (auto &r : admitted) {
        r->t_launch = t_launch;
        r->batch_size = n;
      }
    }
    std::vector<qm_result *> results(n, nullptr);
    std::vector<int> codes(n, QM_OK);
    int rc = batch_layout(b);
    if (!rc) rc = batch_execute(b, results.data(), codes.data(), false);
    if (rc) {
      const std::string m = ctx->err;
      for (int i = 0; i < n; i++) {
        delete results[i];
        complete(admitted[i], rc, m, nullptr);
      }
      return;
    }
    for (int i = 0; i < n; i++) {
      if (codes[i] == QM_ERR_CAPACITY) {
        // the group estimate was too small for the batched table: run it
        // alone, where the table regrows
        qm_result *res = nullptr;
        int rc2 = qm_query_run(ctx, admitted[i]->table, &admitted[i]->query.q, &res);
        complete(admitted[i], rc2, rc2 ? ctx->err : std::string(), res);
      } else if (codes[i] != QM_OK) {
        complete(admitted[i], codes[i], "device status error in the batched launch", nullptr);
      } else {
        complete(admitted[i], QM_OK, std::string(), results[i]);
      }
    }
  }

  void loop() {
    cudaSetDevice(ctx->device);
    for (;;) {
      std::vector<std::shared_ptr<Request>> take;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || !queue.empty(); });
        if (stop) return;
        if (cfg.max_wait_us > 0 && (int)queue.size() < cfg.max_batch) {
          const auto deadline = queue.front()->t_submit + std::chrono::microseconds(cfg.max_wait_us);
          cv_work.wait_until(lk, deadline, [&] { return stop || (int)queue.size() >= cfg.max_batch; });
          if (stop) return;
        }
        while (!queue.empty() && (int)take.size() < cfg.max_batch) {
          take.push_back(queue.front());
          queue.pop_front();
          take.back()->state = RQ_RUNNING;
        }
      }
      if (!take.empty()) run_batch(take);
    }
  }
};

extern "C" {

int qm_server_create(qm_ctx *ctx, const qm_server_config *cfg, qm_server **out) {
  if (!ctx || !cfg || !out) return QM_ERR_INVALID;
  *out = nullptr;
  if (cfg->max_batch < 1 || cfg->max_batch > QM_BATCH_MAX || cfg->hbm_budget_bytes <= 0 || cfg->max_wait_us < 0)
    return set_err(ctx, QM_ERR_INVALID, "server config: max_batch 1..%d, a positive budget, max_wait_us >= 0",
                   QM_BATCH_MAX);
  qm_server *s = new qm_server();
  s->ctx = ctx;
  s->cfg = *cfg;
  s->batch = new qm_batch();
  s->batch->ctx = ctx;
  s->worker = std::thread([s] { s->loop(); });
  *out = s;
  return QM_OK;
}

int qm_server_submit(qm_server *s, const qm_table *table, const qm_query *query, uint64_t *ticket) {
  if (!s || !table || !query || !ticket) return QM_ERR_INVALID;
  if (table->ctx != s->ctx) return QM_ERR_INVALID;
  auto r = std::make_shared<Request>();
  r->table = table;
  r->query.copy(*query);
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
  s->cv_work.notify_one();
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
  return QM_OK;
}

int qm_server_destroy(qm_server *s) {
  if (!s) return QM_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (auto &kv : s->reqs) {
    delete kv.second->res;
    kv.second->res = nullptr;
  }
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  delete s->batch;
  delete s;
  return QM_OK;
}

}  // extern "C"
