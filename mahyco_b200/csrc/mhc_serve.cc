// mhc_serve.cc -- request loop over the batch engine: continuous batching
// of independent solves admitted by HBM budget.
//
// A request is one case (parameters) to be advanced a number of iterations.
// submit() queues it; every step() admits queued requests while their
// device footprint fits the budget (in arrival order, with bounded
// backfilling of smaller requests behind a blocked one), starts them, runs
// cycles of everything resident, then reads every case's status in one copy
// per batch and retires the cases that finished.  A retired case stays
// resident until the caller fetches its results and releases it, and its
// memory stays charged to the budget until then.
//
// Resident cases are split into size classes, each a batch on its own
// stream: all cases of a batch advance in lockstep (one launch per phase),
// so a small request sharing a batch with a large one would move at the
// large one's pace.  A request stops counting against its class's share
// once all its iterations are enqueued, so the next one is admitted behind
// it without a gap.  Each step gives every class the number of cycles that
// takes about as long as the slowest class's `cycles` (estimated from the
// launches and cells per cycle), and the classes' streams overlap on the
// GPU, the larger class at the higher stream priority.  A class advances a bounded number of cells at once (one large case,
// about two large cases' worth of medium ones, any number of small ones):
// cases that already fill the GPU gain nothing from sharing it.  Requests never change each other's arithmetic: each case's results
// are the same alone and in any mix.
//
// Host-only C++ over the public batch API; no counterpart in the reference,
// whose time loop runs one case per process.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <chrono>
#include <deque>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/mahyco_b200.h"

namespace {

constexpr int kClasses = 3;
// class of a request by its cells: [0, 3e4), [3e4, 1e6), [1e6, inf)
int size_class(long long cells) { return cells < 30000 ? 0 : (cells < 1000000 ? 1 : 2); }
// cells a class may advance at once: one large case already fills the GPU,
// so large cases run one after the other (sharing the GPU between them would
// only delay each), medium ones share up to about two large ones' worth;
// small cases are launch-bound and all run together
const long long kClassCells[kClasses] = {LLONG_MAX, 2000000, 1};

struct Request {
  long long ticket = 0;
  int cls = 0;
  long long cells = 0;
  mhc_case_params P;
  long long iterations = 0;
  long long enqueued = 0;     // iterations enqueued on the GPU so far
  double timeout_s = 0.;      // 0 = none
  long long bytes = 0;
  int state = MHC_REQ_QUEUED;
  int status = 0;
  int slot = -1;
  long long iteration = 0;
  double time = 0.;
  double t_submit = 0., t_admit = -1., t_done = -1.;
};

double now_s(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct mhc_server {
  mhc_batch* batch[kClasses] = {nullptr, nullptr, nullptr};
  cudaStream_t stream[kClasses] = {nullptr, nullptr, nullptr};
  long long budget = 0;
  long long in_use = 0;
  int max_bypass = 64;        // admissions allowed past a blocked queue head
  int bypassed = 0;
  long long next_ticket = 1;
  std::chrono::steady_clock::time_point t0;
  std::deque<long long> queue;                     // tickets, arrival order
  std::vector<long long> running;                  // tickets on the GPU
  std::unordered_map<long long, Request> reqs;

  int pending_poll[kClasses] = {-1, -1, -1};       // status read enqueued by the last step, per class
  std::vector<long long> completed_tickets;        // not yet handed out (mhc_server_take_completed)
  long long completed = 0;
};

int mhc_server_create(long long hbm_budget_bytes, mhc_server** out) {
  if (!out) return MHC_ERR_ARG;
  mhc_server* s = new mhc_server();
  // stream priorities: the large class first (its requests are the tail of
  // the latency distribution and already fill the GPU), the small class last
  // (its blocks fill whatever the others leave)
  int lo = 0, hi = 0;
  if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) { delete s; return MHC_ERR_CUDA; }
  for (int c = 0; c < kClasses; ++c) {
    const int prio = c == kClasses - 1 ? hi : (c == 0 ? lo : (lo + hi) / 2);
    if (cudaStreamCreateWithPriority(&s->stream[c], cudaStreamNonBlocking, prio) != cudaSuccess) {
      mhc_server_destroy(s);
      return MHC_ERR_CUDA;
    }
    int r = mhc_batch_create_on_stream(s->stream[c], &s->batch[c]);
    if (r) { mhc_server_destroy(s); return r; }
  }
  if (hbm_budget_bytes <= 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) { mhc_server_destroy(s); return MHC_ERR_CUDA; }
    hbm_budget_bytes = (long long)(0.9 * (double)fr);
  }
  s->budget = hbm_budget_bytes;
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return MHC_OK;
}

int mhc_server_destroy(mhc_server* s) {
  if (!s) return MHC_OK;
  for (int c = 0; c < kClasses; ++c) {
    mhc_batch_destroy(s->batch[c]);
    if (s->stream[c]) cudaStreamDestroy(s->stream[c]);
  }
  delete s;
  return MHC_OK;
}

void* mhc_server_stream(mhc_server* s, int cls) {
  return (s && cls >= 0 && cls < kClasses) ? mhc_batch_stream(s->batch[cls]) : nullptr;
}

long long mhc_server_launches(mhc_server* s) {
  if (!s) return MHC_ERR_ARG;
  long long n = 0;
  for (int c = 0; c < kClasses; ++c) n += mhc_batch_launches(s->batch[c]);
  return n;
}

int mhc_server_submit(mhc_server* s, const mhc_case_params* p, long long iterations, double timeout_s,
                      long long* ticket) {
  if (!s || !p || !ticket || iterations < 1) return MHC_ERR_ARG;
  Request q;
  q.ticket = s->next_ticket++;
  q.P = *p;
  q.iterations = iterations;
  q.timeout_s = timeout_s;
  q.bytes = mhc_case_device_bytes(p);
  if (q.bytes < 0) return MHC_ERR_ARG;
  q.cells = (long long)p->nx * p->ny * (p->dim == 3 ? p->nz : 1);
  q.cls = size_class(q.cells);
  q.t_submit = now_s(s->t0);
  if (q.bytes > s->budget) {
    // can never fit: refused at once
    q.state = MHC_REQ_FAILED;
    q.status = MHC_ST_OOM_ADMISSION;
    q.t_done = q.t_submit;
    s->reqs[q.ticket] = q;
    *ticket = q.ticket;
    return MHC_OK;
  }
  s->reqs[q.ticket] = q;
  s->queue.push_back(q.ticket);
  *ticket = q.ticket;
  return MHC_OK;
}

namespace {

void finish(mhc_server* s, Request& q, int state, int status, double t) {
  q.state = state;
  q.status = status;
  q.t_done = t;
  ++s->completed;
  s->completed_tickets.push_back(q.ticket);
}

int admit(mhc_server* s) {
  int added = 0;
  bool touched[kClasses] = {false, false, false};
  long long run_cells[kClasses] = {0, 0, 0};
  int run_cases[kClasses] = {0, 0, 0};
  // a request holds its class's share until all its iterations are
  // enqueued: its successor's cycles then queue right behind its last ones
  // instead of waiting for its completion to be read back
  for (long long tk : s->running) {
    const Request& q = s->reqs[tk];
    if (q.enqueued >= q.iterations) continue;
    run_cells[q.cls] += q.cells;
    run_cases[q.cls] += 1;
  }
  bool head_blocked = false;
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    Request& q = s->reqs[*it];
    const double t = now_s(s->t0);
    if (q.timeout_s > 0. && t - q.t_submit > q.timeout_s) {
      finish(s, q, MHC_REQ_FAILED, MHC_ST_TIMEOUT, t);
      it = s->queue.erase(it);
      continue;
    }
    if (run_cases[q.cls] > 0 && run_cells[q.cls] + q.cells > kClassCells[q.cls]) {
      ++it;  // its class is busy: wait, others may go ahead
      continue;
    }
    if (s->in_use + q.bytes > s->budget) {
      if (it == s->queue.begin()) head_blocked = true;
      ++it;
      continue;
    }
    if (head_blocked && it != s->queue.begin()) {
      if (s->bypassed >= s->max_bypass) break;  // let the head through first
      ++s->bypassed;
    }
    int slot = -1;
    int r = mhc_batch_add(s->batch[q.cls], &q.P, q.iterations, &slot);
    if (r == MHC_ERR_NOMEM || r == MHC_ERR_CUDA) {
      // the device refused the memory the budget allowed: wait for frees
      if (s->running.empty()) {
        finish(s, q, MHC_REQ_FAILED, MHC_ST_OOM_ADMISSION, t);
        it = s->queue.erase(it);
        continue;
      }
      break;
    }
    if (r) {
      finish(s, q, MHC_REQ_FAILED, MHC_ST_NAN, t);
      it = s->queue.erase(it);
      continue;
    }
    if (it == s->queue.begin()) s->bypassed = 0;
    q.slot = slot;
    q.state = MHC_REQ_RUNNING;
    q.t_admit = t;
    s->in_use += q.bytes;
    s->running.push_back(q.ticket);
    touched[q.cls] = true;
    run_cells[q.cls] += q.cells;
    run_cases[q.cls] += 1;
    it = s->queue.erase(it);
    ++added;
  }
  for (int c = 0; c < kClasses; ++c)
    if (touched[c]) {
      int r = mhc_batch_init(s->batch[c]);
      if (r) return r;
    }
  return added;
}

}  // namespace

int mhc_server_step(mhc_server* s, int cycles) {
  if (!s || cycles < 0) return MHC_ERR_ARG;
  const long long done0 = s->completed;
  int r = admit(s);
  if (r < 0) return r;
  // estimated seconds per cycle of each class: launches + streamed cells
  long long cells[kClasses] = {0, 0, 0}, remain[kClasses] = {0, 0, 0};
  int cases[kClasses] = {0, 0, 0}, nslot[kClasses] = {1, 1, 1};
  for (long long tk : s->running) {
    const Request& q = s->reqs[tk];
    cells[q.cls] += q.cells;
    cases[q.cls] += 1;
    nslot[q.cls] = std::max(nslot[q.cls], q.slot + 1);
    remain[q.cls] = std::max(remain[q.cls], q.iterations - q.enqueued);
  }
  double cost[kClasses], tmax = 0.;
  for (int c = 0; c < kClasses; ++c) {
    cost[c] = cases[c] ? 60e-6 + 1.0e-9 * (double)cells[c] : 0.;
    tmax = std::max(tmax, cost[c]);
  }
  // this step's cycles, then a status read of every class behind them
  int req[kClasses] = {-1, -1, -1};
  for (int c = 0; c < kClasses; ++c) {
    if (!cases[c]) continue;
    if (cycles > 0 && remain[c] > 0) {
      // no more cycles than the class's longest remaining request needs:
      // cycles past every member's limit would only launch empty kernels
      const double k = (double)cycles * tmax / cost[c];
      const int kc = (int)std::min((double)remain[c],
                                   std::min((double)(64 * cycles), std::max((double)cycles, k + 0.5)));
      if ((r = mhc_batch_cycle(s->batch[c], kc))) return r;
      for (long long tk : s->running) {
        Request& q = s->reqs[tk];
        if (q.cls == c) q.enqueued += kc;
      }
    }
    if ((req[c] = mhc_batch_poll_request(s->batch[c])) < 0) return req[c];
  }
  // while the GPU runs them, the previous step's status: retire what had
  // finished by then (a case past its iteration limit does not advance, so
  // its cycles of this step do nothing); with no previous read (first step
  // after an idle server) this step's own is waited for
  std::vector<long long> pit[kClasses];
  std::vector<int> pst[kClasses];
  std::vector<double> ptm[kClasses];
  bool have[kClasses] = {false, false, false};
  for (int c = 0; c < kClasses; ++c) {
    int rq = s->pending_poll[c] >= 0 ? s->pending_poll[c] : req[c];
    if (rq < 0) continue;
    const int n = nslot[c];  // the running requests' slots of the class
    pit[c].resize(n); pst[c].resize(n); ptm[c].resize(n);
    const int ns = mhc_batch_poll_wait(s->batch[c], rq, n, pit[c].data(), pst[c].data(), ptm[c].data());
    if (ns < 0) return ns;
    have[c] = true;
    if (rq == req[c]) req[c] = -1;  // already consumed
  }
  for (int c = 0; c < kClasses; ++c) s->pending_poll[c] = req[c];
  const double t = now_s(s->t0);
  std::vector<long long> still;
  for (long long tk : s->running) {
    Request& q = s->reqs[tk];
    if (!have[q.cls] || q.slot >= (int)pit[q.cls].size()) { still.push_back(tk); continue; }
    const long long it = pit[q.cls][q.slot];
    q.iteration = std::max(q.iteration, it);
    if (it > 0) q.time = ptm[q.cls][q.slot];
    const int st = pst[q.cls][q.slot];
    const int err = st & ~MHC_ST_STOP;
    bool end = false;
    if (err) { finish(s, q, MHC_REQ_FAILED, st, t); end = true; }
    else if ((st & MHC_ST_STOP) || q.iteration >= q.iterations) { finish(s, q, MHC_REQ_DONE, st, t); end = true; }
    else if (q.timeout_s > 0. && t - q.t_submit > q.timeout_s) {
      finish(s, q, MHC_REQ_FAILED, st | MHC_ST_TIMEOUT, t);
      end = true;
    }
    if (end) {
      if ((r = mhc_batch_detach(s->batch[q.cls], q.slot))) return r;
    } else {
      still.push_back(tk);
    }
  }
  s->running.swap(still);
  return (int)(s->completed - done0);
}

int mhc_server_take_completed(mhc_server* s, long long* tickets, int capacity) {
  if (!s || (capacity > 0 && !tickets)) return MHC_ERR_ARG;
  const int n = std::min(capacity, (int)s->completed_tickets.size());
  for (int i = 0; i < n; ++i) tickets[i] = s->completed_tickets[i];
  s->completed_tickets.erase(s->completed_tickets.begin(), s->completed_tickets.begin() + n);
  return n;
}

int mhc_server_poll(mhc_server* s, long long ticket, int* state, int* status, long long* iteration,
                    double* time) {
  if (!s) return MHC_ERR_ARG;
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return MHC_ERR_ARG;
  const Request& q = it->second;
  if (state) *state = q.state;
  if (status) *status = q.status;
  if (iteration) *iteration = q.iteration;
  if (time) *time = q.time;
  return MHC_OK;
}

int mhc_server_times(mhc_server* s, long long ticket, double* submit, double* admit_t, double* done) {
  if (!s) return MHC_ERR_ARG;
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return MHC_ERR_ARG;
  if (submit) *submit = it->second.t_submit;
  if (admit_t) *admit_t = it->second.t_admit;
  if (done) *done = it->second.t_done;
  return MHC_OK;
}

long long mhc_server_fetch(mhc_server* s, long long ticket, const char* name, int env, double* host,
                           long long capacity) {
  if (!s) return MHC_ERR_ARG;
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end() || it->second.slot < 0) return MHC_ERR_ARG;
  return mhc_batch_get_field(s->batch[it->second.cls], it->second.slot, name, env, host, capacity);
}

int mhc_server_release(mhc_server* s, long long ticket) {
  if (!s) return MHC_ERR_ARG;
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return MHC_ERR_ARG;
  Request& q = it->second;
  if (q.state == MHC_REQ_QUEUED || q.state == MHC_REQ_RUNNING) return MHC_ERR_ORDER;
  if (q.slot >= 0) {
    int r = mhc_batch_remove(s->batch[q.cls], q.slot);
    if (r) return r;
    s->in_use -= q.bytes;
  }
  s->reqs.erase(it);
  return MHC_OK;
}

int mhc_server_stats(mhc_server* s, long long* queued, long long* running, long long* bytes_in_use,
                     long long* budget) {
  if (!s) return MHC_ERR_ARG;
  if (queued) *queued = (long long)s->queue.size();
  if (running) *running = (long long)s->running.size();
  if (bytes_in_use) *bytes_in_use = s->in_use;
  if (budget) *budget = s->budget;
  return MHC_OK;
}
