// Serving loop: MD segment requests on one device, run as they arrive.
//
// ORAC has no counterpart (one system per process, src/mtsmd.f); this is
// the executor of a service that keeps many systems resident on one GPU.
// The caller (the host-side request loop) owns admission policy and the
// systems; the server owns
//   - the device-memory budget: reserve / unreserve of footprints
//     (orac_gpu_footprint gives a built context's exact bytes),
//   - the segment slots: at most max_active segments in flight, the rest
//     queued first come first served,
//   - a pump thread that launches every running segment's steps on its
//     own context stream, `chunk` captured step graphs at a time with at
//     most two chunks queued per stream, so a newly started segment gets
//     the device at once and the segments' kernels overlap,
//   - completion detection (one event per chunk) and time stamps on the
//     host's monotonic clock (arrival, start, end) for latency statistics.
// A context handed to orac_gpu_server_submit belongs to the pump thread
// until orac_gpu_server_poll reports its segment finished.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <deque>
#include <mutex>
#include <thread>

#include "common.cuh"

int md_step_graph(orac_gpu_ctx* ctx, int kind, cudaGraph_t* out);

namespace {

using Clock = std::chrono::steady_clock;

double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

struct Segment {
  int64_t ticket = 0, tag = 0;
  orac_gpu_ctx* ctx = nullptr;
  int nsteps = 0, launched = 0;
  std::deque<cudaEvent_t> inflight;  // one event per queued chunk
  double t_arrival = 0, t_start = 0, t_end = 0;
  int status = ORAC_OK;
};

}  // namespace

struct orac_gpu_server {
  int device = 0;
  int64_t budget = 0;
  int max_active = 1;
  int chunk = 1;
  std::mutex mu;  // guards everything below except the pump's private lists
  std::deque<Segment*> pending;
  std::vector<Segment*> running;
  std::vector<Segment*> finished;
  std::vector<cudaEvent_t> events;  // free events
  int64_t reserved = 0, peak = 0, next_ticket = 1;
  int64_t nsubmitted = 0, nfinished = 0, nlaunches = 0;
  std::atomic<bool> stop{false};
  std::thread pump;
  char err[512] = {0};
};

namespace {

int sfail(orac_gpu_server* s, int code, const char* what) {
  if (s) snprintf(s->err, sizeof(s->err), "%s", what);
  return code;
}

cudaEvent_t take_event(orac_gpu_server* s) {
  std::lock_guard<std::mutex> g(s->mu);
  if (!s->events.empty()) {
    cudaEvent_t e = s->events.back();
    s->events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  return e;
}

void give_event(orac_gpu_server* s, cudaEvent_t e) {
  std::lock_guard<std::mutex> g(s->mu);
  s->events.push_back(e);
}

// One pass over the running segments: retire finished chunks, queue new
// ones.  Returns true when it launched or retired anything.
bool pump_once(orac_gpu_server* s, std::vector<Segment*>& mine) {
  bool busy = false;
  {
    std::lock_guard<std::mutex> g(s->mu);
    while ((int)s->running.size() < s->max_active && !s->pending.empty()) {
      Segment* q = s->pending.front();
      s->pending.pop_front();
      q->t_start = now_s();
      s->running.push_back(q);
    }
    mine = s->running;
  }
  std::vector<Segment*> done;
  for (Segment* q : mine) {
    while (!q->inflight.empty()) {
      const cudaError_t r = cudaEventQuery(q->inflight.front());
      if (r == cudaErrorNotReady) break;
      if (r != cudaSuccess && q->status == ORAC_OK) q->status = ORAC_ERR_CUDA;
      give_event(s, q->inflight.front());
      q->inflight.pop_front();
      busy = true;
    }
    while (q->status == ORAC_OK && q->inflight.size() < 2 && q->launched < q->nsteps) {
      const int k = std::min(s->chunk, q->nsteps - q->launched);
      const int rc = orac_gpu_md_run_async(q->ctx, k);
      cudaEvent_t e = rc == ORAC_OK ? take_event(s) : nullptr;
      if (rc != ORAC_OK || !e || cudaEventRecord(e, q->ctx->stream) != cudaSuccess) {
        q->status = rc != ORAC_OK ? rc : ORAC_ERR_CUDA;
        if (e) give_event(s, e);
        break;
      }
      q->inflight.push_back(e);
      q->launched += k;
      busy = true;
      std::lock_guard<std::mutex> g(s->mu);
      s->nlaunches += k;
    }
    if (q->inflight.empty() && (q->launched >= q->nsteps || q->status != ORAC_OK)) {
      q->t_end = now_s();
      done.push_back(q);
    }
  }
  if (!done.empty()) {
    std::lock_guard<std::mutex> g(s->mu);
    for (Segment* q : done) {
      s->running.erase(std::find(s->running.begin(), s->running.end(), q));
      s->finished.push_back(q);
      s->nfinished++;
    }
    busy = true;
  }
  return busy;
}

void pump_main(orac_gpu_server* s) {
  cudaSetDevice(s->device);
  std::vector<Segment*> mine;
  while (!s->stop.load()) {
    if (!pump_once(s, mine)) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

}  // namespace

extern "C" {

double orac_gpu_server_now(void) { return now_s(); }

int orac_gpu_server_create(int device, int64_t budget_bytes, int max_active, int chunk, orac_gpu_server** out) {
  if (!out || budget_bytes <= 0 || max_active < 1 || chunk < 1) return ORAC_ERR_PARAM;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return ORAC_ERR_CUDA;
  orac_gpu_server* s = new orac_gpu_server();
  s->device = device;
  s->budget = budget_bytes;
  s->max_active = max_active;
  s->chunk = chunk;
  s->pump = std::thread(pump_main, s);
  *out = s;
  return ORAC_OK;
}

// Stops the pump after every submitted segment has finished (queued ones
// included) and frees the server; finished segments not yet polled are
// dropped.  The contexts stay with the caller.
int orac_gpu_server_destroy(orac_gpu_server* s) {
  if (!s) return ORAC_OK;
  for (;;) {
    {
      std::lock_guard<std::mutex> g(s->mu);
      if (s->pending.empty() && s->running.empty()) break;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
  s->stop.store(true);
  if (s->pump.joinable()) s->pump.join();
  for (Segment* q : s->finished) delete q;
  for (cudaEvent_t e : s->events) cudaEventDestroy(e);
  delete s;
  return ORAC_OK;
}

const char* orac_gpu_server_last_error(const orac_gpu_server* s) { return s ? s->err : "null server"; }

int orac_gpu_server_reserve(orac_gpu_server* s, int64_t bytes, int* granted) {
  if (!s || !granted || bytes < 0) return ORAC_ERR_PARAM;
  std::lock_guard<std::mutex> g(s->mu);
  *granted = s->reserved + bytes <= s->budget;
  if (*granted) {
    s->reserved += bytes;
    s->peak = std::max(s->peak, s->reserved);
  }
  return ORAC_OK;
}

int orac_gpu_server_unreserve(orac_gpu_server* s, int64_t bytes) {
  if (!s || bytes < 0) return ORAC_ERR_PARAM;
  std::lock_guard<std::mutex> g(s->mu);
  if (bytes > s->reserved) return sfail(s, ORAC_ERR_PARAM, "unreserve of more bytes than reserved");
  s->reserved -= bytes;
  return ORAC_OK;
}

int orac_gpu_server_submit(orac_gpu_server* s, orac_gpu_ctx* ctx, int nsteps, int64_t tag, double t_arrival,
                           int64_t* ticket) {
  if (!s || !ctx || nsteps < 1 || !ticket) return ORAC_ERR_PARAM;
  if (ctx->device != s->device) return sfail(s, ORAC_ERR_PARAM, "context on another device");
  // capture both step graphs here, in the caller's thread, so the pump only
  // launches; served contexts share the device with each other
  ctx->shared_device = true;
  for (int kind = 0; kind < 2; kind++) {
    cudaGraph_t g = nullptr;
    if (int rc = md_step_graph(ctx, kind, &g)) return sfail(s, rc, orac_gpu_last_error(ctx));
  }
  Segment* q = new Segment();
  q->ctx = ctx;
  q->nsteps = nsteps;
  q->tag = tag;
  q->t_arrival = t_arrival > 0 ? t_arrival : now_s();
  std::lock_guard<std::mutex> g(s->mu);
  q->ticket = s->next_ticket++;
  *ticket = q->ticket;
  s->pending.push_back(q);
  s->nsubmitted++;
  return ORAC_OK;
}

// Finished segments since the last call, at most `max`: ticket, tag,
// arrival / start / end times (seconds on orac_gpu_server_now's clock) and
// status (ORAC_OK, or the launch error; the run's own status flags are read
// with orac_gpu_md_collect on the context).
int orac_gpu_server_poll(orac_gpu_server* s, int max, int64_t* tickets, int64_t* tags, double* times3, int* status,
                         int* n) {
  if (!s || !n || max < 0) return ORAC_ERR_PARAM;
  std::lock_guard<std::mutex> g(s->mu);
  int k = 0;
  while (k < max && !s->finished.empty()) {
    Segment* q = s->finished.front();
    s->finished.erase(s->finished.begin());
    if (tickets) tickets[k] = q->ticket;
    if (tags) tags[k] = q->tag;
    if (times3) {
      times3[3 * k] = q->t_arrival;
      times3[3 * k + 1] = q->t_start;
      times3[3 * k + 2] = q->t_end;
    }
    if (status) status[k] = q->status;
    delete q;
    k++;
  }
  *n = k;
  return ORAC_OK;
}

// pending, running, finished (not polled), submitted, finished (all),
// reserved bytes, peak reserved bytes, step launches
int orac_gpu_server_stats(orac_gpu_server* s, int64_t* out8) {
  if (!s || !out8) return ORAC_ERR_PARAM;
  std::lock_guard<std::mutex> g(s->mu);
  out8[0] = (int64_t)s->pending.size();
  out8[1] = (int64_t)s->running.size();
  out8[2] = (int64_t)s->finished.size();
  out8[3] = s->nsubmitted;
  out8[4] = s->nfinished;
  out8[5] = s->reserved;
  out8[6] = s->peak;
  out8[7] = s->nlaunches;
  return ORAC_OK;
}

}  // extern "C"
