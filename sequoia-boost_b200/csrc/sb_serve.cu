// sb_serve.cu — the serving loop: a tree ensemble kept resident in HBM answers
// margin (BoostedModel::predict_margin, learner/model.rs:224-285) and TreeSHAP
// (predict_contribs, learner/shap.rs:321-367) requests with continuous
// batching.
//
//   submit  : any thread; the request joins one of three FIFO lanes: small
//             margin requests (at most SMALL_ROWS rows), larger margin
//             requests, TreeSHAP requests.
//   dispatcher thread : each lane has its own slots (a slot is a CUDA
//             stream; small margins get the highest stream priority, larger
//             margins the middle one, TreeSHAP the lowest). Whenever a slot
//             is free, the dispatcher takes the longest run at the head of
//             that lane's queue sharing a missing-value marker, up to the
//             lane's row cap, and admits it if its device buffers fit in the
//             free part of the loop's memory budget (first-fit arena);
//             otherwise that lane's head waits until a finishing batch frees
//             memory. The batch's rows are copied into one device buffer,
//             run as one set of kernel launches and copied back per request.
//             Several batches are in flight at once, so requests that arrive
//             while others are on the GPU are admitted as slots and memory
//             free up. A small request never queues behind a large batch, and
//             since every kernel is made of short blocks, the block scheduler
//             hands the SMs to the higher-priority stream as soon as its
//             kernel arrives.
//   completion : a host function queued behind each batch flags the slot; the
//             dispatcher then marks the requests done and frees their memory.
//
// The mutex is never held across a CUDA call (the completion host functions
// take it), so the loop cannot deadlock against the driver's callback thread.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "sb_internal.cuh"

namespace sb {

size_t margin_chunk_rows(const sb_model* m);
int margin_batch(sb_model* m, cudaStream_t st, const float* d_X, size_t n, size_t F, float missing,
                 float* d_buf, size_t buf_rows, float* d_out);
int contribs_bias(sb_model* m, std::vector<double>* bias);
int contribs_batch(sb_model* m, cudaStream_t st, const float* d_X, size_t n, size_t F, float missing,
                   double* d_acc, const double* d_bias, float* d_out);

struct Server;

namespace {

constexpr size_t ALIGN = 256;
constexpr size_t SMALL_ROWS = 4096;  // margin requests up to this size take the small lane
enum { LANE_SMALL = 0, LANE_MARGIN = 1, LANE_CONTRIBS = 2, N_LANES = 3 };
constexpr size_t LANE_BATCH_ROWS[N_LANES] = {16384, 65536, 65536};  // row cap of one batch

int lane_kind(int lane) { return lane == LANE_CONTRIBS ? SB_REQ_CONTRIBS : SB_REQ_MARGIN; }
int lane_of(int kind, size_t rows) {
  if (kind == SB_REQ_CONTRIBS) return LANE_CONTRIBS;
  return rows <= SMALL_ROWS ? LANE_SMALL : LANE_MARGIN;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t up(size_t x) { return (x + ALIGN - 1) / ALIGN * ALIGN; }

struct Request {
  uint64_t ticket = 0;
  int kind = 0;
  const float* X = nullptr;
  size_t n = 0;
  float missing = NAN;
  float* out = nullptr;
  int status = SB_OK;
  bool done = false;
  double t_submit = 0.0, t_done = 0.0;
};

// First-fit allocator over one device allocation (dispatcher thread only).
struct Arena {
  char* base = nullptr;
  size_t size = 0, used = 0, peak = 0;
  std::map<size_t, size_t> free_;  // offset -> length
  void init(char* b, size_t s) {
    base = b;
    size = s;
    free_.clear();
    if (s) free_[0] = s;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = up(std::max<size_t>(bytes, 1));
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      *off = it->first;
      const size_t rest = it->second - bytes;
      const size_t roff = it->first + bytes;
      free_.erase(it);
      if (rest) free_[roff] = rest;
      used += bytes;
      peak = std::max(peak, used);
      return true;
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = up(std::max<size_t>(bytes, 1));
    used -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct Slot {
  Server* srv = nullptr;
  cudaStream_t st = nullptr;
  int lane = 0;
  bool busy = false;
  bool finished = false;  // set by the completion host function (under the mutex)
  std::vector<std::shared_ptr<Request>> reqs;
  size_t mem_off = 0, mem_bytes = 0;
  int status = SB_OK;
};

}  // namespace

struct Server {
  sb_ctx* ctx = nullptr;
  sb_model* model = nullptr;
  int F = 0, K = 1, T = 0;
  size_t chunk_rows = 0;  // rows per margin leaf-buffer chunk
  char* d_mem = nullptr;
  double* d_bias = nullptr;
  Arena arena;
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv;       // dispatcher wake-ups
  std::condition_variable done_cv;  // request completions
  std::deque<std::shared_ptr<Request>> queue[N_LANES];
  std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
  uint64_t next_ticket = 1;
  bool stop = false;
  bool mem_blocked[N_LANES] = {};  // a lane's head waits for memory to be freed
  std::thread worker;
  sb_server_stats stats{};

  size_t out_floats(int kind, size_t n) const {
    return kind == SB_REQ_MARGIN ? n * K : n * K * (size_t)(F + 1);
  }
  // device bytes of a batch of `rows` rows
  size_t batch_bytes(int kind, size_t rows) const {
    size_t b = up(rows * F * 4) + up(out_floats(kind, rows) * 4);
    if (kind == SB_REQ_MARGIN) b += up(std::min(rows, chunk_rows) * (size_t)std::max(T, 1) * 4);  // leaf values
    else b += up(out_floats(kind, rows) * 8);  // f64 accumulator
    return b;
  }

  static void CUDART_CB on_done(void* p) {
    Slot* s = static_cast<Slot*>(p);
    {
      std::lock_guard<std::mutex> lk(s->srv->mu);
      s->finished = true;
    }
    s->srv->cv.notify_all();
  }

  int launch(Slot* s, int kind, float missing, size_t rows) {
    char* base = arena.base + s->mem_off;
    float* dX = reinterpret_cast<float*>(base);
    float* dOut = reinterpret_cast<float*>(base + up(rows * F * 4));
    char* scratch = base + up(rows * F * 4) + up(out_floats(kind, rows) * 4);
    cudaStream_t st = s->st;
    size_t r0 = 0;
    for (auto& r : s->reqs) {
      SB_CUDA(cudaMemcpyAsync(dX + r0 * F, r->X, r->n * F * 4, cudaMemcpyHostToDevice, st));
      r0 += r->n;
    }
    if (kind == SB_REQ_MARGIN)
      SB_TRY(margin_batch(model, st, dX, rows, F, missing, reinterpret_cast<float*>(scratch), chunk_rows, dOut));
    else
      SB_TRY(contribs_batch(model, st, dX, rows, F, missing, reinterpret_cast<double*>(scratch), d_bias, dOut));
    r0 = 0;
    for (auto& r : s->reqs) {
      const size_t w = out_floats(kind, 1);
      SB_CUDA(cudaMemcpyAsync(r->out, dOut + r0 * w, r->n * w * 4, cudaMemcpyDeviceToHost, st));
      r0 += r->n;
    }
    SB_CUDA(cudaLaunchHostFunc(st, on_done, s));
    return SB_OK;
  }

  // Marks a slot's requests done and frees its memory (mutex held; no CUDA call).
  void finish(Slot* s) {
    const double t = now_s();
    for (auto& r : s->reqs) {
      r->status = s->status;
      r->done = true;
      r->t_done = t;
      stats.completed++;
      if (s->status != SB_OK) stats.failed++;
    }
    s->reqs.clear();
    s->busy = false;
    s->finished = false;
    arena.release(s->mem_off, s->mem_bytes);
    for (bool& b : mem_blocked) b = false;
    done_cv.notify_all();
  }

  // Takes the longest admissible run at the head of a lane's queue into slot
  // s. Returns the run's rows, 0 when the head must wait for memory.
  size_t admit(Slot* s, int lane, float* miss_out) {
    std::deque<std::shared_ptr<Request>>& queue = this->queue[lane];
    const int kind = lane_kind(lane);
    const float miss = queue.front()->missing;
    const bool miss_nan = std::isnan(miss);
    const size_t cap = LANE_BATCH_ROWS[lane];
    size_t rows = 0, take = 0;
    for (auto& r : queue) {
      const bool same_miss = miss_nan ? std::isnan(r->missing) : r->missing == miss;
      if (!same_miss) break;
      if (take > 0 && rows + r->n > cap) break;
      rows += r->n;
      take++;
    }
    size_t off = 0, bytes = 0;
    for (;;) {  // admission by free memory: shorten the run until it fits
      bytes = batch_bytes(kind, rows);
      if (arena.alloc(bytes, &off)) break;
      if (take == 1) return 0;
      rows -= queue[take - 1]->n;
      take--;
    }
    s->reqs.assign(queue.begin(), queue.begin() + take);
    queue.erase(queue.begin(), queue.begin() + take);
    s->busy = true;
    s->finished = false;
    s->mem_off = off;
    s->mem_bytes = bytes;
    stats.batches++;
    stats.rows += rows;
    stats.max_batch_requests = std::max<uint64_t>(stats.max_batch_requests, take);
    stats.mem_peak = std::max<uint64_t>(stats.mem_peak, arena.used);
    *miss_out = miss;
    return rows;
  }

  Slot* free_slot(int lane) {
    for (auto& s : slots)
      if (s->lane == lane && !s->busy) return s.get();
    return nullptr;
  }

  bool can_admit(int lane) {
    return !queue[lane].empty() && !mem_blocked[lane] && free_slot(lane) != nullptr;
  }
  bool any_admissible() {
    for (int l = 0; l < N_LANES; ++l)
      if (can_admit(l)) return true;
    return false;
  }
  bool queues_empty() const {
    for (int l = 0; l < N_LANES; ++l)
      if (!queue[l].empty()) return false;
    return true;
  }

  void run() {
    cudaSetDevice(ctx->device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      for (auto& s : slots)
        if (s->busy && s->finished) finish(s.get());
      for (int lane = 0; lane < N_LANES; ++lane) {  // highest priority first
        std::deque<std::shared_ptr<Request>>& queue = this->queue[lane];
        const int kind = lane_kind(lane);
        while (can_admit(lane)) {
          Slot* slot = free_slot(lane);
          if (batch_bytes(kind, queue.front()->n) > arena.size) {  // can never fit
            auto r = queue.front();
            queue.pop_front();
            r->status = SB_ERR_OOM;
            r->done = true;
            r->t_done = now_s();
            stats.completed++;
            stats.failed++;
            done_cv.notify_all();
            continue;
          }
          float miss = NAN;
          const size_t rows = admit(slot, lane, &miss);
          if (rows == 0) {  // the head waits until a finishing batch frees memory
            mem_blocked[lane] = true;
            stats.memory_waits++;
            break;
          }
          lk.unlock();
          const int st = launch(slot, kind, miss, rows);
          if (st != SB_OK) cudaStreamSynchronize(slot->st);  // let anything already queued drain
          lk.lock();
          slot->status = st;
          if (st != SB_OK) finish(slot);
        }
      }
      bool any_busy = false;
      for (auto& s : slots) any_busy = any_busy || s->busy;
      if (stop && queues_empty() && !any_busy) break;
      // sleep (releasing the mutex, which the completion host functions
      // need) until a batch finishes, a queued request can be admitted, or
      // the loop may stop
      cv.wait(lk, [&] {
        bool busy = false;
        for (auto& s : slots) {
          if (s->busy && s->finished) return true;
          busy = busy || s->busy;
        }
        if (any_admissible()) return true;
        return stop && queues_empty() && !busy;
      });
    }
  }
};

}  // namespace sb

struct sb_server : sb::Server {};

extern "C" {

int sb_server_create(sb_ctx* ctx, sb_model* m, size_t mem_bytes, int n_slots, sb_server** out) {
  using namespace sb;
  SB_REQUIRE(ctx && m && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_slots >= 1 && n_slots <= 64, SB_ERR_INVALID_ARG, "n_slots must be in [1, 64]");
  *out = nullptr;
  SB_CUDA(cudaSetDevice(ctx->device));
  if (mem_bytes == 0) {  // half of the device memory free now
    size_t free_b = 0, total_b = 0;
    SB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    mem_bytes = free_b / 2;
  }
  SB_REQUIRE(mem_bytes >= (1u << 20), SB_ERR_INVALID_ARG, "mem_bytes must be at least 1 MiB");
  SB_TRY(model_upload(m));
  std::unique_ptr<sb_server> s(new sb_server);
  s->ctx = ctx;
  s->model = m;
  s->F = m->n_features;
  s->K = m->num_class >= 2 ? m->num_class : 1;
  s->T = m->dev.n_trees;
  s->chunk_rows = margin_chunk_rows(m);
  std::vector<double> bias;
  SB_TRY(contribs_bias(m, &bias));
  cudaError_t e = cudaMalloc(&s->d_bias, bias.size() * sizeof(double));
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("serving loop: allocation of the bias failed: %s", cudaGetErrorString(e));
    return SB_ERR_OOM;
  }
  SB_CUDA(cudaMemcpy(s->d_bias, bias.data(), bias.size() * sizeof(double), cudaMemcpyHostToDevice));
  e = cudaMalloc(&s->d_mem, mem_bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(s->d_bias);
    set_error("serving loop: allocation of %zu bytes failed: %s", mem_bytes, cudaGetErrorString(e));
    return SB_ERR_OOM;
  }
  s->arena.init(s->d_mem, mem_bytes);
  int lo_prio = 0, hi_prio = 0;  // numerically lower is higher priority
  SB_CUDA(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio));
  const int lane_slots[N_LANES] = {std::max(1, n_slots / 2), std::max(1, n_slots - n_slots / 2),
                                   std::max(1, n_slots / 2)};
  const int lane_prio[N_LANES] = {hi_prio, (lo_prio + hi_prio) / 2, lo_prio};
  for (int lane = 0; lane < N_LANES; ++lane)
    for (int i = 0; i < lane_slots[lane]; ++i) {
      std::unique_ptr<Slot> sl(new Slot);
      sl->srv = s.get();
      sl->lane = lane;
      SB_CUDA(cudaStreamCreateWithPriority(&sl->st, cudaStreamNonBlocking, lane_prio[lane]));
      s->slots.push_back(std::move(sl));
    }
  s->stats.mem_bytes = mem_bytes;
  s->worker = std::thread([p = s.get()] { p->run(); });
  *out = s.release();
  return SB_OK;
}

int sb_server_submit(sb_server* s, int kind, const float* X, size_t n_rows, size_t n_cols, float missing,
                     float* out, uint64_t* ticket) {
  using namespace sb;
  SB_REQUIRE(s && ticket && (X || n_rows == 0) && (out || n_rows == 0), SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(kind == SB_REQ_MARGIN || kind == SB_REQ_CONTRIBS, SB_ERR_INVALID_ARG, "unknown request kind %d", kind);
  SB_REQUIRE(n_cols == (size_t)s->F, SB_ERR_DIMENSION, "dimension mismatch: expected %d features, got %zu", s->F,
             n_cols);
  auto r = std::make_shared<Request>();
  r->kind = kind;
  r->X = X;
  r->n = n_rows;
  r->missing = missing;
  r->out = out;
  r->t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    SB_REQUIRE(!s->stop, SB_ERR_INVALID_ARG, "the serving loop is shutting down");
    r->ticket = s->next_ticket++;
    s->live[r->ticket] = r;
    s->stats.submitted++;
    if (n_rows == 0) {
      r->done = true;
      r->t_done = r->t_submit;
      s->stats.completed++;
    } else {
      s->queue[lane_of(kind, n_rows)].push_back(r);
    }
    *ticket = r->ticket;
  }
  s->cv.notify_all();
  return SB_OK;
}

int sb_server_wait(sb_server* s, uint64_t ticket, int timeout_ms, double* latency_ms) {
  using namespace sb;
  SB_REQUIRE(s, SB_ERR_INVALID_ARG, "NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->live.find(ticket);
  SB_REQUIRE(it != s->live.end(), SB_ERR_INVALID_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  std::shared_ptr<Request> r = it->second;
  auto pred = [&] { return r->done; };
  if (timeout_ms < 0) s->done_cv.wait(lk, pred);
  else if (!s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
    set_error("request %llu not finished after %d ms", (unsigned long long)ticket, timeout_ms);
    return SB_ERR_TIMEOUT;
  }
  s->live.erase(ticket);
  if (latency_ms) *latency_ms = (r->t_done - r->t_submit) * 1e3;
  if (r->status != SB_OK) set_error("request %llu failed with status %d", (unsigned long long)ticket, r->status);
  return r->status;
}

int sb_server_stats_get(sb_server* s, sb_server_stats* out) {
  using namespace sb;
  SB_REQUIRE(s && out, SB_ERR_INVALID_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  return SB_OK;
}

int sb_server_destroy(sb_server* s) {
  if (!s) return SB_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->ctx->device);
  for (auto& sl : s->slots)
    if (sl->st) cudaStreamSynchronize(sl->st), cudaStreamDestroy(sl->st);
  if (s->d_mem) cudaFree(s->d_mem);
  if (s->d_bias) cudaFree(s->d_bias);
  delete s;
  return SB_OK;
}

}  // extern "C"
