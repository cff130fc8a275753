// frsz2_serve.cu -- a compress / decompress request server with continuous
// batching over a device-memory budget.
//
// Requests (device input, output in caller memory or in the server's arena)
// become eligible at their arrival time.  A worker thread admits eligible
// requests in arrival order -- skipping, within a bounded window, requests
// whose output does not fit the arena right now -- into batches, and launches
// each batch on a free stream slot as soon as one exists, so batches that
// arrive while others run overlap on the device.  A batch's arrays are
// grouped by (direction, float type, width) and run through the batched
// kernels (frsz2_batch_kernels.cuh), one CTA per tile, from a device
// descriptor buffer and tile index of the slot; arrays those kernels do not
// take get their own launch.
// Completion is detected by polling the slot's event; outputs allocated in
// the arena stay there until released (or are released on completion when
// the request asks for it).
#include "frsz2_batch_kernels.cuh"
#include "frsz2_launch.hpp"

#include "../../include/frsz2_b200.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <time.h>

using namespace frsz2b;

namespace {

std::uint64_t now_ns()
{
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (std::uint64_t)ts.tv_sec * 1000000000ull + (std::uint64_t)ts.tv_nsec;
}

// First-fit arena over [0, cap) with coalescing free list; 256-byte granules.
class Arena
{
public:
  void init(std::uint64_t cap)
  {
    cap_ = cap;
    free_.clear();
    if (cap) free_[0] = cap;
    used_ = peak_ = 0;
  }
  bool alloc(std::uint64_t bytes, std::uint64_t* off)
  {
    bytes = round(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const std::uint64_t rest = it->second - bytes, start = it->first + bytes;
        free_.erase(it);
        if (rest) free_[start] = rest;
        used_ += bytes;
        peak_ = std::max(peak_, used_);
        return true;
      }
    }
    return false;
  }
  void release(std::uint64_t off, std::uint64_t bytes)
  {
    bytes = round(bytes);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  static std::uint64_t round(std::uint64_t b) { return ((b + 255) / 256) * 256; }
  std::uint64_t capacity() const { return cap_; }
  std::uint64_t used() const { return used_; }
  std::uint64_t peak() const { return peak_; }

private:
  std::map<std::uint64_t, std::uint64_t> free_; // offset -> length
  std::uint64_t cap_ = 0, used_ = 0, peak_ = 0;
};

struct Req
{
  frsz2_request r;
  std::uint64_t id = 0;
  std::uint64_t admit_ns = 0, done_ns = 0;
  std::uint64_t out_bytes = 0;
  std::uint64_t arena_off = 0;
  bool in_arena = false;
  int status = FRSZ2_OK;
};

constexpr int kSubStreams = 4; // a batch's class kernels are spread over these

struct Slot
{
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  cudaEvent_t fork = nullptr;
  cudaStream_t sub[kSubStreams] = {};
  cudaEvent_t join[kSubStreams] = {};
  BatchItem* d_desc = nullptr;
  BatchItem* h_desc = nullptr; // pinned
  // per tile of the batch's class kernels: the tile's descriptor within its
  // class (device, and its pinned staging), grown on demand
  std::uint32_t* d_tmap = nullptr;
  std::uint32_t* h_tmap = nullptr;
  std::uint64_t tmap_cap = 0;
  std::vector<Req*> reqs;
  bool busy = false;
};

constexpr int kBypassWindow = 64; // pending requests scanned past one that does not fit
constexpr int kKeys = 2 * 2 * 65; // (direction, float type, width)

} // namespace

struct frsz2_server
{
  Arena arena;
  std::uint8_t* d_arena = nullptr;
  int max_batch = 0;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Req*> pending;   // arrival order
  std::deque<Req*> completed; // not yet polled
  std::unordered_map<std::uint64_t, Req*> live; // admitted or completed, not released
  std::uint64_t next_id = 1;
  std::atomic<bool> stop{ false };
  std::thread worker;
  // statistics
  std::uint64_t n_completed = 0, n_failed = 0, n_batches = 0, bytes_done = 0, max_batch_seen = 0;
  std::uint64_t max_inflight_bytes = 0;
  int device = 0;
};

namespace {

std::uint64_t output_bytes(const frsz2_request& r)
{
  if (r.op == FRSZ2_OP_COMPRESS) return make_layout(r.n, r.bits, r.block_size).total_bytes;
  return r.n * (r.dtype == FRSZ2_DOUBLE ? 8 : 4);
}

int validate(const frsz2_request& r, std::uint64_t budget)
{
  if (r.op != FRSZ2_OP_COMPRESS && r.op != FRSZ2_OP_DECOMPRESS) return set_error(FRSZ2_EFAIL, "unknown request op");
  if (int rc = check_args(r.dtype, r.bits, r.block_size)) return rc;
  if (r.n > 0 && !r.input) return set_error(FRSZ2_EFAIL, "null request input");
  if (!r.output && Arena::round(output_bytes(r)) > budget)
    return set_error(FRSZ2_EFAIL, "request output larger than the server's memory budget");
  return FRSZ2_OK;
}

// Launch one admitted batch on slot s.
int launch_batch(frsz2_server* sv, Slot& s)
{
  NvtxRange nvtx("frsz2_server batch");
  std::uint64_t per_key[kKeys] = {};
  auto key = [](const Req* q) {
    return (q->r.op == FRSZ2_OP_COMPRESS ? 130 : 0) + (q->r.dtype == FRSZ2_DOUBLE ? 65 : 0) + q->r.bits;
  };
  auto job_of = [](const Req* q, void* out) {
    const frsz2_request& r = q->r;
    const Layout L = make_layout(r.n, r.bits, r.block_size);
    const bool comp = r.op == FRSZ2_OP_COMPRESS;
    return job_for_slice(L, r.dtype, 0, L.nb, comp ? r.input : nullptr, comp ? nullptr : out,
                         static_cast<std::uint8_t*>(comp ? out : const_cast<void*>(r.input)));
  };
  auto out_ptr = [sv](const Req* q) -> void* {
    return q->in_arena ? (void*)(sv->d_arena + q->arena_off) : q->r.output;
  };
  auto fast = [&](const Req* q) {
    if (q->r.n == 0) return false;
    const bool is64 = q->r.dtype == FRSZ2_DOUBLE;
    const batch_entry e = is64 ? batch_class_f64(q->r.bits, 0) : batch_class_f32(q->r.bits, 0);
    const int tv = fast_tile_values(is64 ? 8 : 4, kShapes[0].nt, kShapes[0].rpw);
    const Job j = job_of(q, out_ptr(q));
    const void* values = q->r.op == FRSZ2_OP_COMPRESS ? j.values_in : j.values_out;
    return e.launch_tiles != nullptr && q->r.block_size <= tv && fast_eligible(j, is64, values, j.words);
  };
  std::vector<char> is_fast(s.reqs.size());
  for (std::size_t i = 0; i < s.reqs.size(); ++i) {
    is_fast[i] = fast(s.reqs[i]);
    if (is_fast[i]) ++per_key[key(s.reqs[i])];
  }
  std::uint64_t start[kKeys], fill[kKeys], tiles[kKeys] = {}, used = 0;
  for (int k = 0; k < kKeys; ++k) {
    start[k] = fill[k] = used;
    used += per_key[k];
  }
  for (std::size_t i = 0; i < s.reqs.size(); ++i) {
    if (!is_fast[i]) continue;
    const Req* q = s.reqs[i];
    const int k = key(q);
    const int tv = fast_tile_values(q->r.dtype == FRSZ2_DOUBLE ? 8 : 4, kShapes[0].nt, kShapes[0].rpw);
    BatchItem& bi = s.h_desc[fill[k]++];
    bi.job = job_of(q, out_ptr(q));
    bi.job.tiles = (q->r.n + (std::uint64_t)tv - 1) / (std::uint64_t)tv;
    bi.job.tile_blocks = (std::uint32_t)(tv / q->r.block_size);
    bi.tile_begin = tiles[k];
    tiles[k] += bi.job.tiles;
  }
  if (used)
    if (int rc = cuda_status(
          cudaMemcpyAsync(s.d_desc, s.h_desc, used * sizeof(BatchItem), cudaMemcpyHostToDevice, s.stream),
          "descriptor upload"))
      return rc;
  // tile index of every class kernel: one CTA per tile reads its descriptor
  // from it (the slot is idle, so its buffers may be regrown)
  std::uint64_t tmap_start[kKeys], ntiles = 0;
  for (int k = 0; k < kKeys; ++k) {
    tmap_start[k] = ntiles;
    ntiles += tiles[k];
  }
  if (ntiles > s.tmap_cap) {
    const std::uint64_t cap = std::max<std::uint64_t>(ntiles, 2 * s.tmap_cap);
    if (s.d_tmap) cudaFree(s.d_tmap);
    if (s.h_tmap) cudaFreeHost(s.h_tmap);
    s.d_tmap = nullptr;
    s.h_tmap = nullptr;
    s.tmap_cap = 0;
    if (int rc = cuda_status(cudaMalloc(&s.d_tmap, cap * sizeof(std::uint32_t)), "tile index buffer")) return rc;
    if (int rc = cuda_status(cudaMallocHost(&s.h_tmap, cap * sizeof(std::uint32_t)), "tile index staging")) return rc;
    s.tmap_cap = cap;
  }
  for (int k = 0; k < kKeys; ++k) {
    std::uint32_t* m = s.h_tmap + tmap_start[k];
    for (std::uint64_t d = 0; d < per_key[k]; ++d) {
      const std::uint64_t t = s.h_desc[start[k] + d].job.tiles;
      std::fill(m, m + t, (std::uint32_t)d);
      m += t;
    }
  }
  if (ntiles)
    if (int rc = cuda_status(
          cudaMemcpyAsync(s.d_tmap, s.h_tmap, ntiles * sizeof(std::uint32_t), cudaMemcpyHostToDevice, s.stream),
          "tile index upload"))
      return rc;
  // class kernels side by side on the slot's sub-streams, one CTA per tile
  int nclass = 0;
  for (int k = 0; k < kKeys; ++k)
    if (per_key[k]) ++nclass;
  const bool fork = nclass > 1;
  if (fork) {
    if (int rc = cuda_status(cudaEventRecord(s.fork, s.stream), "fork")) return rc;
    for (int b = 0; b < kSubStreams; ++b)
      if (int rc = cuda_status(cudaStreamWaitEvent(s.sub[b], s.fork, 0), "fork wait")) return rc;
  }
  int ci = 0;
  for (int k = 0; k < kKeys; ++k) {
    if (!per_key[k]) continue;
    const bool comp = k >= 130;
    const int rest = k - (comp ? 130 : 0);
    const bool is64 = rest >= 65;
    const int bits = rest - (is64 ? 65 : 0);
    const batch_entry e = is64 ? batch_class_f64(bits, 0) : batch_class_f32(bits, 0);
    cudaStream_t st = fork ? s.sub[ci++ % kSubStreams] : s.stream;
    if (int rc = cuda_status(e.launch_tiles(comp, s.d_desc + start[k], s.d_tmap + tmap_start[k], tiles[k], st),
                             "batch launch"))
      return rc;
  }
  if (fork) {
    for (int b = 0; b < kSubStreams && b < nclass; ++b) {
      if (int rc = cuda_status(cudaEventRecord(s.join[b], s.sub[b]), "join")) return rc;
      if (int rc = cuda_status(cudaStreamWaitEvent(s.stream, s.join[b], 0), "join wait")) return rc;
    }
  }
  for (std::size_t i = 0; i < s.reqs.size(); ++i) {
    const Req* q = s.reqs[i];
    if (is_fast[i] || q->r.n == 0) continue;
    const Job j = job_of(q, out_ptr(q));
    const int rc = q->r.op == FRSZ2_OP_COMPRESS ? launch_compress(j, q->r.dtype, s.stream, nullptr)
                                                : launch_decompress(j, q->r.dtype, s.stream, nullptr);
    if (rc) return rc;
  }
  return cuda_status(cudaEventRecord(s.done, s.stream), "event record");
}

// Algorithmic bytes of a request: values + exponents + words.
std::uint64_t request_bytes(const frsz2_request& r)
{
  const Layout L = make_layout(r.n, r.bits, r.block_size);
  return r.n * (r.dtype == FRSZ2_DOUBLE ? 8 : 4) + L.nb * ((std::uint64_t)L.block_bytes + (std::uint64_t)(L.W / 8));
}

void finish(frsz2_server* sv, Req* q, int status, std::uint64_t t)
{
  q->status = status;
  q->done_ns = t;
  if (status == FRSZ2_OK) {
    ++sv->n_completed;
    sv->bytes_done += request_bytes(q->r);
  } else {
    ++sv->n_failed;
  }
  if (q->in_arena && (q->r.flags & FRSZ2_REQ_RELEASE_ON_COMPLETION)) {
    sv->arena.release(q->arena_off, q->out_bytes);
    q->in_arena = false;
  }
  sv->completed.push_back(q);
}

void worker_loop(frsz2_server* sv)
{
  cudaSetDevice(sv->device);
  std::unique_lock<std::mutex> lock(sv->mu);
  while (!sv->stop.load()) {
    const std::uint64_t t = now_ns();
    bool progressed = false;
    // completions
    for (auto& s : sv->slots) {
      if (!s.busy) continue;
      const cudaError_t e = cudaEventQuery(s.done);
      if (e == cudaErrorNotReady) continue;
      const int status = e == cudaSuccess ? FRSZ2_OK : FRSZ2_EFAIL;
      const std::uint64_t td = now_ns();
      for (Req* q : s.reqs) finish(sv, q, status, td);
      s.reqs.clear();
      s.busy = false;
      progressed = true;
    }
    // admission into free slots
    for (auto& s : sv->slots) {
      if (s.busy) continue;
      int skipped = 0;
      for (auto it = sv->pending.begin(); it != sv->pending.end() && (int)s.reqs.size() < sv->max_batch;) {
        Req* q = *it;
        if (q->r.arrival_ns > t) break; // arrival order: later ones are not eligible either
        if (!q->r.output) {
          std::uint64_t off = 0;
          if (!sv->arena.alloc(q->out_bytes, &off)) {
            if (++skipped > kBypassWindow) break;
            ++it;
            continue;
          }
          q->arena_off = off;
          q->in_arena = true;
        }
        q->admit_ns = t;
        s.reqs.push_back(q);
        it = sv->pending.erase(it);
      }
      if (s.reqs.empty()) break; // nothing admissible now; other free slots would find nothing either
      std::uint64_t inflight = 0;
      for (auto& o : sv->slots)
        for (Req* q : o.reqs) inflight += q->out_bytes;
      sv->max_inflight_bytes = std::max(sv->max_inflight_bytes, inflight);
      sv->max_batch_seen = std::max<std::uint64_t>(sv->max_batch_seen, s.reqs.size());
      ++sv->n_batches;
      const int rc = launch_batch(sv, s);
      if (rc) {
        const std::uint64_t td = now_ns();
        for (Req* q : s.reqs) finish(sv, q, rc, td);
        s.reqs.clear();
      } else {
        s.busy = true;
      }
      progressed = true;
    }
    if (progressed) {
      sv->cv.notify_all();
      continue;
    }
    bool any_busy = false;
    for (auto& s : sv->slots) any_busy |= s.busy;
    if (any_busy || (!sv->pending.empty() && sv->pending.front()->r.arrival_ns <= t + 20000)) {
      // work in flight or about to arrive: short pause without holding the lock
      lock.unlock();
      std::this_thread::yield();
      lock.lock();
    } else if (!sv->pending.empty()) {
      const std::uint64_t wait = std::min<std::uint64_t>(sv->pending.front()->r.arrival_ns - t, 1000000);
      sv->cv.wait_for(lock, std::chrono::nanoseconds(wait));
    } else {
      sv->cv.wait_for(lock, std::chrono::milliseconds(1));
    }
  }
}

} // namespace

extern "C" {

uint64_t frsz2_now_ns(void) { return now_ns(); }

int frsz2_server_create(uint64_t memory_budget, int max_batch, int streams, frsz2_server** out)
{
  if (!out) return set_error(FRSZ2_EFAIL, "null server pointer");
  *out = nullptr;
  if (max_batch < 1 || streams < 1 || streams > 64) return set_error(FRSZ2_EFAIL, "bad server shape");
  auto* sv = new frsz2_server();
  sv->max_batch = max_batch;
  cudaGetDevice(&sv->device);
  int rc = FRSZ2_OK;
  if (memory_budget) {
    rc = cuda_status(cudaMalloc(&sv->d_arena, memory_budget), "arena allocation");
    if (!rc) sv->arena.init(memory_budget);
  }
  sv->slots.resize(streams);
  for (auto& s : sv->slots) {
    if (rc) break;
    rc = cuda_status(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "stream create");
    if (!rc) rc = cuda_status(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming), "event create");
    if (!rc) rc = cuda_status(cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming), "event create");
    for (int b = 0; b < kSubStreams && !rc; ++b) {
      rc = cuda_status(cudaStreamCreateWithFlags(&s.sub[b], cudaStreamNonBlocking), "stream create");
      if (!rc) rc = cuda_status(cudaEventCreateWithFlags(&s.join[b], cudaEventDisableTiming), "event create");
    }
    if (!rc) rc = cuda_status(cudaMalloc(&s.d_desc, (std::size_t)max_batch * sizeof(BatchItem)), "descriptor buffer");
    if (!rc)
      rc = cuda_status(cudaMallocHost(&s.h_desc, (std::size_t)max_batch * sizeof(BatchItem)), "descriptor staging");
  }
  if (rc) {
    frsz2_server_destroy(sv);
    return rc;
  }
  sv->worker = std::thread(worker_loop, sv);
  *out = sv;
  return FRSZ2_OK;
}

int frsz2_server_submit(frsz2_server* sv, const frsz2_request* reqs, uint64_t count, uint64_t* first_id)
{
  if (!sv) return set_error(FRSZ2_EFAIL, "null server");
  if (count && !reqs) return set_error(FRSZ2_EFAIL, "null requests");
  std::lock_guard<std::mutex> lock(sv->mu);
  if (first_id) *first_id = sv->next_id;
  const std::uint64_t t = now_ns();
  for (std::uint64_t i = 0; i < count; ++i) {
    Req* q = new Req();
    q->r = reqs[i];
    if (q->r.flags & FRSZ2_REQ_ARRIVAL_RELATIVE)
      q->r.arrival_ns += t;
    else if (q->r.arrival_ns == 0)
      q->r.arrival_ns = t;
    q->id = sv->next_id++;
    sv->live[q->id] = q;
    const int rc = validate(q->r, sv->arena.capacity());
    if (rc) {
      q->admit_ns = t;
      finish(sv, q, rc, t);
      continue;
    }
    q->out_bytes = q->r.output ? 0 : output_bytes(q->r);
    // keep arrival order (submissions are usually already ordered)
    auto pos = sv->pending.end();
    while (pos != sv->pending.begin() && (*std::prev(pos))->r.arrival_ns > q->r.arrival_ns) --pos;
    sv->pending.insert(pos, q);
  }
  sv->cv.notify_all();
  return FRSZ2_OK;
}

int frsz2_server_cancel(frsz2_server* sv, uint64_t id)
{
  if (!sv) return set_error(FRSZ2_EFAIL, "null server");
  std::lock_guard<std::mutex> lock(sv->mu);
  for (auto it = sv->pending.begin(); it != sv->pending.end(); ++it) {
    if ((*it)->id == id) {
      Req* q = *it;
      sv->pending.erase(it);
      set_error(FRSZ2_EFAIL, "request cancelled");
      finish(sv, q, FRSZ2_ECANCELLED, now_ns());
      return FRSZ2_OK;
    }
  }
  return set_error(FRSZ2_EFAIL, "request is not pending (already admitted, finished or unknown)");
}

int frsz2_server_poll(frsz2_server* sv, frsz2_completion* out, uint64_t max, uint64_t* count, int wait_ms)
{
  if (!sv || !count) return set_error(FRSZ2_EFAIL, "null pointer");
  *count = 0;
  std::unique_lock<std::mutex> lock(sv->mu);
  if (sv->completed.empty() && wait_ms > 0)
    sv->cv.wait_for(lock, std::chrono::milliseconds(wait_ms), [sv] { return !sv->completed.empty(); });
  while (*count < max && !sv->completed.empty()) {
    Req* q = sv->completed.front();
    sv->completed.pop_front();
    frsz2_completion& c = out[(*count)++];
    c.id = q->id;
    c.status = q->status;
    c.op = q->r.op;
    c.output = q->in_arena ? (void*)(sv->d_arena + q->arena_off) : q->r.output;
    c.output_bytes = q->in_arena ? q->out_bytes : 0;
    c.bytes = q->status == FRSZ2_OK ? request_bytes(q->r) : 0;
    c.arrival_ns = q->r.arrival_ns;
    c.admit_ns = q->admit_ns;
    c.done_ns = q->done_ns;
    if (!q->in_arena) { // nothing left to release
      sv->live.erase(q->id);
      delete q;
    }
  }
  return FRSZ2_OK;
}

int frsz2_server_release(frsz2_server* sv, uint64_t id)
{
  if (!sv) return set_error(FRSZ2_EFAIL, "null server");
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->live.find(id);
  if (it == sv->live.end() || !it->second->in_arena || it->second->done_ns == 0)
    return set_error(FRSZ2_EFAIL, "no completed arena output for this request id");
  Req* q = it->second;
  sv->arena.release(q->arena_off, q->out_bytes);
  q->in_arena = false;
  sv->live.erase(it);
  // the completion may still be queued; it then frees the record when polled
  if (std::find(sv->completed.begin(), sv->completed.end(), q) == sv->completed.end()) delete q;
  sv->cv.notify_all();
  return FRSZ2_OK;
}

int frsz2_server_stats(frsz2_server* sv, frsz2_server_counters* st)
{
  if (!sv || !st) return set_error(FRSZ2_EFAIL, "null pointer");
  std::lock_guard<std::mutex> lock(sv->mu);
  std::memset(st, 0, sizeof(*st));
  st->completed = sv->n_completed;
  st->failed = sv->n_failed;
  st->batches = sv->n_batches;
  st->bytes = sv->bytes_done;
  st->pending = sv->pending.size();
  st->budget_bytes = sv->arena.capacity();
  st->arena_used_bytes = sv->arena.used();
  st->arena_peak_bytes = sv->arena.peak();
  st->max_batch = sv->max_batch_seen;
  st->max_inflight_output_bytes = sv->max_inflight_bytes;
  return FRSZ2_OK;
}

void frsz2_server_destroy(frsz2_server* sv)
{
  if (!sv) return;
  sv->stop.store(true);
  sv->cv.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  for (auto& s : sv->slots) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.stream) cudaStreamDestroy(s.stream);
    if (s.done) cudaEventDestroy(s.done);
    if (s.fork) cudaEventDestroy(s.fork);
    for (int b = 0; b < kSubStreams; ++b) {
      if (s.sub[b]) {
        cudaStreamSynchronize(s.sub[b]);
        cudaStreamDestroy(s.sub[b]);
      }
      if (s.join[b]) cudaEventDestroy(s.join[b]);
    }
    if (s.d_desc) cudaFree(s.d_desc);
    if (s.h_desc) cudaFreeHost(s.h_desc);
    if (s.d_tmap) cudaFree(s.d_tmap);
    if (s.h_tmap) cudaFreeHost(s.h_tmap);
  }
  if (sv->d_arena) cudaFree(sv->d_arena);
  std::vector<Req*> all;
  for (auto& kv : sv->live) all.push_back(kv.second);
  for (auto& s : sv->slots)
    for (Req* q : s.reqs) all.push_back(q);
  for (Req* q : sv->pending) all.push_back(q);
  for (Req* q : sv->completed) all.push_back(q);
  std::sort(all.begin(), all.end());
  all.erase(std::unique(all.begin(), all.end()), all.end());
  for (Req* q : all) delete q;
  delete sv;
}

} // extern "C"
