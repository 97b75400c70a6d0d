// Serving loop: compress and decompress requests admitted by a device-memory
// budget and coded in continuously formed batches.
//
// Requests wait in arrival order until their working set (field, stream and
// the batch scratch they need) fits in the budget; admitted requests that are
// not running yet are launched together, as one batch, as soon as one of the
// lanes (a CUDA stream with its own batch scratch) is free, so requests that
// arrive while others are on the GPU join the next batch and run beside the
// batches already in flight.  Each request's result is that of the
// single-array device call: a batch computes every array independently.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "zfpb_engine.h"
#include "zfpb_serve.h"

namespace zfpb {

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct ServeRequest {
  u64 tag;
  bool decompress;
  BatchJob job;
  u64 cost;
  u64 bytes;  // uncompressed bytes
  double t_submit, t_start;
};

struct ServeLane {
  cudaStream_t stream = nullptr;
  BatchRun* run = nullptr;
  std::vector<ServeRequest> reqs;
  std::vector<BatchJob> jobs;
  bool busy = false;
  bool finished = false;  // set by the stream callback
  bool launch_ok = false;
};

struct Server {
  u64 budget, in_use = 0;
  size_t max_batch;
  u64 batch_bytes;
  std::vector<ServeLane> lanes;
  std::deque<ServeRequest> waiting;   // submitted, not admitted
  std::deque<ServeRequest> admitted;  // admitted, not launched
  std::deque<ServeDone> done;
  size_t outstanding = 0;             // submitted, not yet polled
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::thread worker;
  bool stop = false;
  int device = 0;

  void loop();
  std::vector<ServeLane*> admit();
};

static void CUDART_CB lane_finished(void* p) {
  auto* pr = static_cast<std::pair<Server*, ServeLane*>*>(p);
  {
    std::lock_guard<std::mutex> l(pr->first->mu);
    pr->second->finished = true;
  }
  pr->first->cv.notify_one();
  delete pr;
}

// Under mu: admit waiting requests while they fit, then give every idle lane
// a batch of admitted requests of one kind (the oldest request's).  Returns
// the lanes to launch (outside the lock).
std::vector<ServeLane*> Server::admit() {
  std::vector<ServeLane*> go;
  while (!waiting.empty() && in_use + waiting.front().cost <= budget) {
    in_use += waiting.front().cost;
    admitted.push_back(waiting.front());
    waiting.pop_front();
  }
  for (ServeLane& L : lanes) {
    if (L.busy || admitted.empty()) continue;
    // The oldest request's kind; then, in arrival order, requests of that
    // kind while the batch stays under batch_bytes of data (a larger request
    // runs alone), so that small requests are not held behind large ones.
    const bool dec = admitted.front().decompress;
    L.reqs.clear();
    u64 bytes = 0;
    for (auto it = admitted.begin(); it != admitted.end() && L.reqs.size() < max_batch;) {
      if (it->decompress == dec && (L.reqs.empty() || bytes + it->bytes <= batch_bytes)) {
        bytes += it->bytes;
        L.reqs.push_back(*it);
        it = admitted.erase(it);
        if (bytes >= batch_bytes) break;
      } else {
        ++it;
      }
    }
    L.jobs.clear();
    const double t = now_s();
    for (ServeRequest& r : L.reqs) {
      r.t_start = t;
      L.jobs.push_back(r.job);
    }
    L.busy = true;
    L.finished = false;
    L.launch_ok = false;
    go.push_back(&L);
  }
  return go;
}

void Server::loop() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  while (true) {
    // Results of finished lanes.
    for (ServeLane& L : lanes) {
      if (!L.busy || !L.finished) continue;
      lk.unlock();
      Status st = L.launch_ok ? batch_collect(L.run, L.jobs.data()) : ERR_CUDA;
      const double t = now_s();
      lk.lock();
      for (size_t i = 0; i < L.reqs.size(); i++) {
        const ServeRequest& r = L.reqs[i];
        const BatchJob& J = L.jobs[i];
        ServeDone d;
        d.tag = r.tag;
        d.status = (!L.launch_ok || st == ERR_CUDA) ? (int)ERR_CUDA : (int)J.status;
        d.result = d.status == OK ? (J.end_bit + 63) / 64 * 8 : 0;
        d.queue_ms = (r.t_start - r.t_submit) * 1e3;
        d.latency_ms = (t - r.t_submit) * 1e3;
        done.push_back(d);
        in_use -= r.cost;
      }
      L.busy = false;
      done_cv.notify_all();
    }
    if (stop && waiting.empty() && admitted.empty() &&
        std::none_of(lanes.begin(), lanes.end(), [](const ServeLane& L) { return L.busy; }))
      break;
    std::vector<ServeLane*> go = admit();
    if (!go.empty()) {
      lk.unlock();
      for (ServeLane* L : go) {
        const bool dec = L->reqs.front().decompress;
        bool ok = batch_launch(L->run, L->jobs.data(), L->jobs.size(), !dec, L->stream) == OK;
        auto* pr = new std::pair<Server*, ServeLane*>(this, L);
        if (cudaLaunchHostFunc(L->stream, lane_finished, pr) != cudaSuccess) {
          delete pr;
          ok = false;
        }
        std::lock_guard<std::mutex> l(mu);
        L->launch_ok = ok;
        if (!ok) L->finished = true;
      }
      lk.lock();
      continue;
    }
    // Nothing to launch.  While batches are in flight, poll their events for
    // a short while (a stream callback also wakes the loop, later); when idle,
    // sleep until a submit or a callback.
    const bool inflight = std::any_of(lanes.begin(), lanes.end(), [](const ServeLane& L) { return L.busy; });
    if (inflight) {
      lk.unlock();
      const double until = now_s() + 200e-6;
      bool ready = false;
      while (!ready && now_s() < until) {
        for (ServeLane& L : lanes)
          if (L.busy && batch_ready(L.run)) ready = true;
        if (!ready) std::this_thread::yield();
      }
      lk.lock();
      if (ready) {
        for (ServeLane& L : lanes)
          if (L.busy && L.launch_ok && batch_ready(L.run)) L.finished = true;
        continue;
      }
    }
    if (!waiting.empty() || !admitted.empty()) {
      bool idle = std::any_of(lanes.begin(), lanes.end(), [](const ServeLane& L) { return !L.busy; });
      if (idle && !admitted.empty()) continue;
    }
    cv.wait_for(lk, std::chrono::milliseconds(1));
  }
}

Server* server_create(u64 budget, int nlanes, size_t max_batch, u64 batch_bytes) {
  Server* s = new Server();
  s->budget = budget;
  s->max_batch = max_batch ? max_batch : 4096;
  s->batch_bytes = batch_bytes ? batch_bytes : (64ull << 20);
  cudaGetDevice(&s->device);
  s->lanes.resize(nlanes > 0 ? nlanes : 4);
  for (ServeLane& L : s->lanes) {
    if (cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking) != cudaSuccess || !(L.run = batch_run_create())) {
      server_destroy(s);
      return nullptr;
    }
  }
  // Map scratch for the lanes up front (the pool keeps it once freed), so the
  // first large batches do not wait for memory to be mapped.
  if (!s->lanes.empty()) {
    const u64 reserve = std::min<u64>(budget / 4, 6ull << 30);
    cudaStream_t st = s->lanes[0].stream;
    if (reserve && batch_reserve(reserve, st)) cudaStreamSynchronize(st);
  }
  s->worker = std::thread([s] { s->loop(); });
  return s;
}

bool server_submit(Server* s, const BatchJob& job, bool decompress, u64 tag) {
  ServeRequest r;
  r.tag = tag;
  r.decompress = decompress;
  r.job = job;
  const u64 elem = (job.call.type == 1 || job.call.type == 3) ? 4 : 8;
  u64 values = 1;
  for (int d = 0; d < job.call.dims; d++) values *= job.call.f.n[d];
  r.bytes = values * elem;
  r.cost = r.bytes + job.stream_words * 8 + batch_scratch_bytes(job.call, !decompress);
  if (r.cost > s->budget) return false;
  r.t_submit = now_s();
  r.t_start = 0;
  {
    std::lock_guard<std::mutex> l(s->mu);
    s->waiting.push_back(r);
    s->outstanding++;
  }
  s->cv.notify_one();
  return true;
}

size_t server_poll(Server* s, ServeDone* out, size_t max, int wait_ms) {
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->done.empty() && wait_ms > 0)
    s->done_cv.wait_for(lk, std::chrono::milliseconds(wait_ms), [s] { return !s->done.empty(); });
  size_t n = 0;
  while (n < max && !s->done.empty()) {
    out[n++] = s->done.front();
    s->done.pop_front();
  }
  s->outstanding -= n;
  return n;
}

size_t server_outstanding(Server* s) {
  std::lock_guard<std::mutex> l(s->mu);
  return s->outstanding;
}

void server_destroy(Server* s) {
  if (!s) return;
  if (s->worker.joinable()) {
    {
      std::lock_guard<std::mutex> l(s->mu);
      s->stop = true;
    }
    s->cv.notify_one();
    s->worker.join();
  }
  for (ServeLane& L : s->lanes) {
    if (L.run) batch_run_destroy(L.run);
    if (L.stream) cudaStreamDestroy(L.stream);
  }
  delete s;
}

}  // namespace zfpb
