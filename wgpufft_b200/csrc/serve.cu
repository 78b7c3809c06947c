// Serving loop (b2f_server_*): requests of any configuration served with
// continuous batching; the crate has no counterpart (its plans only record
// into a caller's encoder).
//
// Clients submit transforms of any configuration with their data in host
// memory (copied in and out by the loop) or in device memory (transformed
// where it lies).  One scheduler thread owns the device side:
//   - two routes.  Line requests (1D complex f32 over axis 0, any length
//     and batch, no tuning) of one direction and normalization are
//     coalesced, whatever their lengths, into one batched launch of the
//     mixed-length line kernels (linebatch.h): every line of every request
//     of the group is a line of that launch.  Every other request runs on a
//     resident plan of its configuration; requests of the same
//     configuration are coalesced into one execution over their summed
//     batch (batches are contiguous blocks, so the requests' buffers sit
//     back to back in the staging buffers);
//   - resident plans are keyed by configuration without the batch and by a
//     power-of-two batch bucket: a group's batch B runs as the binary
//     decomposition of B over at most 13 cached plans, so no group size
//     builds a new plan once its buckets exist; a (configuration, batch)
//     seen a second time gets a plan of exactly that batch and runs as one
//     execution (recurring request shapes pay one plan build, not a
//     decomposition per request).  A group of one 1D complex f32 request
//     runs on a plan, not the line launch.  Plans count against the
//     HBM budget and the least recently used ones are evicted (after their
//     last execution has completed) when admission needs the room;
//   - admission: a group is admitted when its device bytes (staging, the
//     line launch's task lists and scratch, any new plan) fit the budget
//     next to everything in flight and resident; otherwise it waits for
//     in-flight groups to complete;
//   - continuous batching: arrivals join the next group while earlier
//     groups run; groups rotate over several streams so the copies of one
//     overlap the kernels of another.
// Completion is observed with events; waiting clients are woken, latency is
// recorded from submission to completion.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_map>
#include <vector>

#include "linebatch.h"
#include "plan.h"

namespace b2f {

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct SReq {
  uint64_t id = 0;
  Config cfg;
  int32_t kind = B2F_C2C;
  std::string key;   // group key: the line route's (direction, normalization) or the configuration
  bool line = false; // line route
  bool device = false;  // buffers in device memory
  const void* in = nullptr;
  void* out = nullptr;
  uint64_t in_bytes = 0, out_bytes = 0;  // the request's own sizes
  double t_submit = 0, t_done = 0;
  int state = 0;  // 0 queued, 1 in flight, 2 done, 3 failed
  b2f_status status = B2F_OK;
  std::string error;
};

struct SPlan {
  std::unique_ptr<Plan> plan;
  uint64_t bytes = 0;
  cudaEvent_t last = nullptr;  // completion of its last group
  bool used = false;
  std::list<std::string>::iterator lru;
};

struct SGroup {
  std::vector<SReq*> reqs;
  cudaEvent_t done = nullptr;
  uint64_t bytes = 0;  // device bytes held until completion
};

static std::string config_key(const Config& c, int32_t kind) {
  std::ostringstream os;
  os << kind << "|" << c.precision << "|" << c.direction << "|" << c.normalization << "|";
  for (auto s : c.shape) os << s << ",";
  os << "|";
  for (auto a : c.axes) os << a << ",";
  const Tuning& t = c.tuning;
  os << "|" << t.lines_per_block << "," << t.threads_per_block << "," << t.twiddle_table << ","
     << t.tensor_cores << "," << t.fuse_small_volumes << "," << t.rader_max_prime;
  for (auto a : t.force_rader_axes) os << ",r" << a;
  for (auto a : t.force_bluestein_axes) os << ",b" << a;
  return os.str();
}

// 1D complex f32 over axis 0 with default kernel tuning: the line route.
static bool line_config(const Config& c, int32_t kind) {
  const Tuning d;
  const Tuning& t = c.tuning;
  return kind == B2F_C2C && c.precision == B2F_F32 && c.shape.size() == 1 && c.axes.size() == 1 &&
         c.axes[0] == 0 && t.force_rader_axes.empty() && t.force_bluestein_axes.empty() &&
         t.lines_per_block == 0 && t.threads_per_block == 0 && t.tensor_cores == 0 &&
         t.rader_max_prime == d.rader_max_prime;
}

struct Server {
  int device = 0;
  uint64_t budget = 0;
  int nstreams = 4;
  uint32_t max_group = 64;
  uint64_t max_line_group_bytes = 512ull << 20;
  bool coalesce = true;
  std::vector<cudaStream_t> streams;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  bool held = false;  // b2f_server_hold: queue without dispatching
  std::deque<SReq*> queue;
  std::unordered_map<uint64_t, std::unique_ptr<SReq>> reqs;
  std::vector<SGroup> inflight;
  uint64_t used = 0;  // staging and launch bytes in flight
  uint64_t next_id = 1;
  int next_stream = 0;
  // resident plans: key -> plan, least recently used first in `lru`
  std::map<std::string, SPlan> plans;
  std::list<std::string> lru;
  uint64_t plan_bytes = 0;
  // line registries per (direction, normalization)
  LineRegistry* regs[2][4] = {};
  // statistics
  std::vector<double> lat;
  uint64_t completed = 0, failed = 0, groups = 0, line_groups = 0, coalesced = 0, transforms = 0;
  uint64_t evictions = 0;
  // executions seen per exact (configuration, batch): a batch seen before
  // runs on a plan of exactly that batch (one execution instead of the
  // power-of-two decomposition); the map is reset when it grows large
  std::unordered_map<std::string, uint32_t> seen_exact;
  double t_first = 0, t_last = 0;
  std::thread worker;

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv_work.notify_all();
    if (worker.joinable()) worker.join();
    cudaSetDevice(device);
    for (auto& g : inflight) {
      cudaEventSynchronize(g.done);
      cudaEventDestroy(g.done);
    }
    for (auto& kv : plans)
      if (kv.second.last) cudaEventDestroy(kv.second.last);
    plans.clear();
    for (auto& row : regs)
      for (auto* r : row) line_registry_free(r);
    for (auto s : streams) cudaStreamDestroy(s);
  }

  LineRegistry* registry(int32_t dir, int32_t norm) {
    LineRegistry*& r = regs[dir & 1][norm & 3];
    if (!r) r = line_registry_new(device, dir, norm);
    return r;
  }

  uint64_t registry_bytes() const {
    uint64_t b = 0;
    for (auto& row : regs)
      for (auto* r : row) b += line_registry_bytes(r);
    return b;
  }

  // Evicts least recently used plans that no group in flight uses until
  // `need` more bytes fit the budget (lock held).  Returns whether they fit.
  bool make_room(uint64_t need) {
    while (used + plan_bytes + registry_bytes() + need > budget && !lru.empty()) {
      bool evicted = false;
      for (auto it = lru.begin(); it != lru.end(); ++it) {
        SPlan& sp = plans[*it];
        if (sp.last && cudaEventQuery(sp.last) == cudaErrorNotReady) continue;
        cudaGetLastError();
        plan_bytes -= sp.bytes;
        if (sp.last) cudaEventDestroy(sp.last);
        const std::string k = *it;
        lru.erase(it);
        plans.erase(k);
        ++evictions;
        evicted = true;
        break;
      }
      if (!evicted) break;
    }
    return used + plan_bytes + registry_bytes() + need <= budget;
  }

  std::unique_lock<std::mutex>* run_lock = nullptr;  // the scheduler thread's hold on mu

  // The resident plan of cfg (a batch bucket or an exact batch), created when new.
  SPlan* get_plan(const Config& cfg, int32_t kind, b2f_status* st) {
    const std::string k = config_key(cfg, kind) + "|b" + std::to_string(cfg.batch);
    auto it = plans.find(k);
    if (it != plans.end()) {
      lru.erase(it->second.lru);
      lru.push_back(k);
      it->second.lru = std::prev(lru.end());
      return &it->second;
    }
    // built with the lock released (tables and workspace take allocations
    // and uploads): submitters and waiters are not held up meanwhile; only
    // this thread touches the plan map
    Plan* p = nullptr;
    if (run_lock) run_lock->unlock();
    *st = create_plan(cfg, kind, device, &p);
    if (run_lock) run_lock->lock();
    if (*st) return nullptr;
    SPlan& sp = plans[k];
    sp.plan.reset(p);
    sp.bytes = p->workspace_total() + p->table_bytes;
    cudaEventCreateWithFlags(&sp.last, cudaEventDisableTiming);
    lru.push_back(k);
    sp.lru = std::prev(lru.end());
    plan_bytes += sp.bytes;
    return &sp;
  }

  // Completes every group whose event has fired (lock held).
  void reap() {
    for (size_t i = 0; i < inflight.size();) {
      SGroup& g = inflight[i];
      cudaError_t q = cudaEventQuery(g.done);
      if (q == cudaErrorNotReady) {
        ++i;
        continue;
      }
      const double t = now_s();
      for (SReq* r : g.reqs) {
        if (q != cudaSuccess) {
          r->state = 3;
          r->status = B2F_ERR_DEVICE;
          r->error = cudaGetErrorString(q);
          ++failed;
        } else {
          r->state = 2;
          r->t_done = t;
          lat.push_back(t - r->t_submit);
          ++completed;
          transforms += r->cfg.batch;
        }
        t_last = t;
      }
      used -= g.bytes;
      cudaEventDestroy(g.done);
      inflight.erase(inflight.begin() + i);
    }
    cv_done.notify_all();
  }

  // Waits for the oldest group in flight with the lock released, so clients
  // keep submitting (and the queue keeps filling for coalescing) while the
  // scheduler is blocked on the device; then completes what has fired.
  // Only this thread changes `inflight`, so the event stays valid.
  void wait_oldest(std::unique_lock<std::mutex>& lk) {
    if (inflight.empty()) return;
    cudaEvent_t ev = inflight.front().done;
    lk.unlock();
    cudaEventSynchronize(ev);
    lk.lock();
    reap();
  }

  void fail_all(std::vector<SReq*>& members, b2f_status s, const std::string& msg) {
    for (SReq* r : members) {
      r->state = 3;
      r->status = s;
      r->error = msg;
      ++failed;
    }
    cv_done.notify_all();
  }

  // Copies the host requests' inputs into the staging buffer (device
  // requests are used where they lie).
  static cudaError_t copy_in(std::vector<SReq*>& members, char* din, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    uint64_t off = 0;
    for (SReq* r : members) {
      if (!r->device && e == cudaSuccess)
        e = cudaMemcpyAsync(din + off, r->in, r->in_bytes, cudaMemcpyHostToDevice, s);
      off += r->in_bytes;
    }
    return e;
  }
  static cudaError_t copy_out(std::vector<SReq*>& members, const char* dout, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    uint64_t off = 0;
    for (SReq* r : members) {
      if (!r->device && e == cudaSuccess)
        e = cudaMemcpyAsync(r->out, dout + off, r->out_bytes, cudaMemcpyDeviceToHost, s);
      off += r->out_bytes;
    }
    return e;
  }

  // A failed launch: nothing more is queued that touches the requests'
  // memory, the stream finishes the copies it already holds, then the
  // staging is freed and the requests are failed.
  void abort_group(std::vector<SReq*>& members, cudaStream_t s, void* din, void* dout,
                   b2f_status st, const std::string& msg) {
    if (din) cudaFreeAsync(din, s);
    if (dout) cudaFreeAsync(dout, s);
    cudaStreamSynchronize(s);
    cudaGetLastError();
    fail_all(members, st, msg);
  }

  // Runs one group on stream s (lock held; CUDA calls are asynchronous).
  // Returns false when admission must wait for memory.
  bool launch(std::vector<SReq*>& members) {
    const int si = next_stream;
    cudaStream_t s = streams[si];
    uint64_t in_total = 0, out_total = 0;
    bool all_device = true;
    for (SReq* r : members) {
      in_total += r->in_bytes;
      out_total += r->out_bytes;
      all_device = all_device && r->device;
    }
    // a line group of one request gains nothing from the batched line
    // launch: it runs on its resident plan (fewer launches, no task lists)
    const bool line = members[0]->line && members.size() > 1;
    // staging for host requests (a group is all host or all device requests)
    const bool stage = !all_device;
    const uint64_t stage_bytes = stage ? in_total + out_total : 0;
    if (line) {
      // line lists and scratch: bounded by about twice the group's points
      const uint64_t est = stage_bytes + 3 * in_total + (1u << 20);
      if (!make_room(est)) return false;
    } else if (!make_room(stage_bytes)) {
      return false;
    }
    next_stream = (next_stream + 1) % nstreams;
    char* din = nullptr;
    char* dout = nullptr;
    if (stage) {
      if (cudaMallocAsync((void**)&din, std::max<uint64_t>(in_total, 16), s) != cudaSuccess ||
          cudaMallocAsync((void**)&dout, std::max<uint64_t>(out_total, 16), s) != cudaSuccess) {
        cudaGetLastError();
        abort_group(members, s, din, nullptr, B2F_ERR_RESOURCE_ALLOCATION, "staging allocation failed");
        return true;
      }
    }
    cudaError_t e = stage ? copy_in(members, din, s) : cudaSuccess;
    if (e != cudaSuccess) {
      abort_group(members, s, din, dout, B2F_ERR_DEVICE, cudaGetErrorString(e));
      return true;
    }
    b2f_status st = B2F_OK;
    uint64_t extra = 0;
    if (line) {
      // every line of every request: (length, input offset, output offset)
      // relative to the staging buffers or to the lowest request address
      std::vector<uint64_t> lens, ioff, ooff;
      uintptr_t ibase = UINTPTR_MAX, obase = UINTPTR_MAX;
      if (!stage)
        for (SReq* r : members) {
          ibase = std::min(ibase, (uintptr_t)r->in);
          obase = std::min(obase, (uintptr_t)r->out);
        }
      uint64_t off = 0;
      for (SReq* r : members) {
        const uint64_t N = r->cfg.shape[0];
        const uint64_t i0 = stage ? off / 8 : ((uintptr_t)r->in - ibase) / 8;
        const uint64_t o0 = stage ? off / 8 : ((uintptr_t)r->out - obase) / 8;
        for (uint64_t b = 0; b < r->cfg.batch; ++b) {
          lens.push_back(N);
          ioff.push_back(i0 + b * N);
          ooff.push_back(o0 + b * N);
        }
        off += r->in_bytes;
      }
      LineRegistry* reg = registry(members[0]->cfg.direction, members[0]->cfg.normalization);
      st = reg ? line_batch_run(reg, s, lens.data(), ioff.data(), ooff.data(), lens.size(),
                                stage ? (const void*)din : (const void*)ibase,
                                stage ? (void*)dout : (void*)obase, &extra)
               : fail(B2F_ERR_RESOURCE_ALLOCATION, "line registry allocation failed");
      if (st == B2F_OK) ++line_groups;
    } else {
      // binary decomposition of the batch over bucketed resident plans
      uint64_t in_off = 0, out_off = 0;
      for (SReq* r : stage ? std::vector<SReq*>{members[0]} : members) {
        Config cfg = r->cfg;
        uint64_t left = 0;
        if (stage)
          for (SReq* q : members) left += q->cfg.batch;
        else
          left = cfg.batch;
        const uint64_t per_in = (stage ? in_total : r->in_bytes) / left;
        const uint64_t per_out = (stage ? out_total : r->out_bytes) / left;
        const char* src = stage ? din : (const char*)r->in;
        char* dst = stage ? dout : (char*)r->out;
        uint64_t done_b = 0;
        bool exact = false;
        {
          cfg.batch = left;
          const std::string ek = config_key(cfg, r->kind) + "|b" + std::to_string(left);
          if (seen_exact.size() > 65536) seen_exact.clear();
          exact = plans.count(ek) > 0 || seen_exact[ek]++ > 0;
        }
        while (left > 0 && st == B2F_OK) {
          uint64_t chunk = 1;
          while (chunk * 2 <= left && chunk * 2 <= 4096) chunk *= 2;
          if (exact) chunk = left;
          cfg.batch = chunk;
          SPlan* sp = get_plan(cfg, r->kind, &st);
          if (!sp) break;
          st = execute_plan(*sp->plan, s, src + done_b * per_in, chunk * per_in,
                            dst + done_b * per_out, chunk * per_out);
          cudaEventRecord(sp->last, s);
          done_b += chunk;
          left -= chunk;
        }
        in_off += r->in_bytes;
        out_off += r->out_bytes;
        if (st) break;
      }
    }
    if (st) {
      abort_group(members, s, din, dout, st, last_error());
      return true;
    }
    e = stage ? copy_out(members, dout, s) : cudaSuccess;
    if (stage) {
      cudaFreeAsync(din, s);
      cudaFreeAsync(dout, s);
    }
    SGroup g;
    g.reqs = members;
    g.bytes = stage_bytes + extra;
    cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(g.done, s);
    if (e != cudaSuccess) {
      cudaStreamSynchronize(s);
      cudaGetLastError();
      cudaEventDestroy(g.done);
      fail_all(members, B2F_ERR_DEVICE, cudaGetErrorString(e));
      return true;
    }
    for (SReq* r : members) r->state = 1;
    used += g.bytes;
    ++groups;
    if (members.size() > 1) coalesced += members.size();
    inflight.push_back(g);
    return true;
  }

  void run() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    run_lock = &lk;
    while (true) {
      // wake for new work at once; with groups in flight, poll their
      // completion every 20 us with the lock released (submitters and
      // waiters get the lock meanwhile)
      const auto poll = std::chrono::microseconds(inflight.empty() ? 2000 : 20);
      cv_work.wait_for(lk, poll, [&] { return stop || (!queue.empty() && !held); });
      if (stop && queue.empty() && inflight.empty()) break;
      reap();
      // admit and group: the queue head's key, then every other queued
      // request with the same key (continuous batching)
      while (!queue.empty() && (!held || stop)) {
        SReq* head = queue.front();
        std::vector<SReq*> members;
        uint64_t bytes = 0;
        for (auto it = queue.begin(); it != queue.end() && members.size() < max_group;) {
          SReq* r = *it;
          if (r->key != head->key || (!coalesce && !members.empty())) {
            ++it;
            continue;
          }
          const uint64_t b = r->in_bytes + r->out_bytes;
          if (!members.empty() && head->line && bytes + b > max_line_group_bytes) break;
          if (!members.empty() && used + bytes + b > budget) break;
          members.push_back(r);
          bytes += b;
          it = queue.erase(it);
        }
        if (bytes > budget) {
          fail_all(members, B2F_ERR_RESOURCE_ALLOCATION,
                   "request larger than the HBM admission budget");
          continue;
        }

        if (!launch(members)) {
          // wait for memory: put them back in front, in order
          for (auto it = members.rbegin(); it != members.rend(); ++it) queue.push_front(*it);
          if (inflight.empty()) {
            SReq* r = queue.front();
            queue.pop_front();
            std::vector<SReq*> one{r};
            fail_all(one, B2F_ERR_RESOURCE_ALLOCATION,
                     "request does not fit the HBM admission budget next to the resident plans");
            continue;
          }
          wait_oldest(lk);
          break;
        }
        // bound the work in flight: at most two groups per stream
        if ((int)inflight.size() >= 2 * nstreams) wait_oldest(lk);
      }
    }
  }
};

}  // namespace b2f

using namespace b2f;

struct b2f_server {
  Server* s;
};

static b2f_status submit_any(b2f_server* srv, const b2f_config* cfg, int32_t kind, bool device,
                             const void* in, uint64_t in_bytes, void* out, uint64_t out_bytes,
                             uint64_t* request_id) {
  if (!srv || !cfg || !in || !out || !request_id)
    return fail(B2F_ERR_INVALID_ARGUMENT, "null argument");
  b2f_status st = validate_config(cfg->cfg);
  if (st) return st;
  if (kind < B2F_C2C || kind > B2F_C2R) return fail(B2F_ERR_INVALID_ARGUMENT, "unknown kind");
  const Config& c = cfg->cfg;
  uint64_t total = c.batch, packed = c.batch;
  for (size_t d = 0; d < c.shape.size(); ++d) {
    total *= c.shape[d];
    packed *= d == 0 ? c.shape[0] / 2 + 1 : c.shape[d];
  }
  const uint64_t cb = c.precision == B2F_F32 ? 8 : 16, sb = cb / 2;
  uint64_t need_in = total * cb, need_out = total * cb;
  if (kind == B2F_R2C) {
    need_in = total * sb;
    need_out = packed * cb;
  } else if (kind == B2F_C2R) {
    need_in = packed * cb;
    need_out = total * sb;
  }
  if (in_bytes < need_in || out_bytes < need_out)
    return fail(B2F_ERR_BUFFER_TOO_SMALL, "BufferViewTooSmall: request buffers");
  Server* s = srv->s;
  std::unique_ptr<SReq> r(new SReq());
  r->cfg = c;
  r->kind = kind;
  r->device = device;
  r->line = line_config(c, kind) && (!device || ((uintptr_t)in % 8 == 0 && (uintptr_t)out % 8 == 0));
  if (r->line) {
    LineRegistry* reg;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      reg = s->registry(c.direction, c.normalization);
    }
    r->line = reg && line_registry_accepts(reg, c.shape[0]);
  }
  r->key = (r->line ? "lines|" + std::to_string(c.direction) + "|" + std::to_string(c.normalization)
                    : config_key(c, kind)) +
           (device ? "|dev" : "|host");
  r->in = in;
  r->out = out;
  r->in_bytes = need_in;
  r->out_bytes = need_out;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    r->t_submit = now_s();
    if (s->t_first == 0) s->t_first = r->t_submit;
    *request_id = r->id;
    s->queue.push_back(r.get());
    s->reqs[r->id] = std::move(r);
  }
  s->cv_work.notify_one();
  return B2F_OK;
}

extern "C" {

b2f_status b2f_server_new(b2f_server** out, int32_t device, uint64_t hbm_budget_bytes,
                          int32_t nstreams, int32_t coalesce) {
  if (!out) return fail(B2F_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  int dev = device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return fail(B2F_ERR_DEVICE, "no device");
  if (cudaSetDevice(dev) != cudaSuccess) return fail(B2F_ERR_DEVICE, "cudaSetDevice failed");
  std::unique_ptr<Server> s(new Server());
  s->device = dev;
  s->budget = hbm_budget_bytes ? hbm_budget_bytes : (120ull << 30);
  s->nstreams = std::max(1, std::min(16, (int)nstreams));
  s->coalesce = coalesce != 0;
  // the groups' stream-ordered allocations (staging, line task lists) come
  // from the device's default pool: keep up to the budget mapped across
  // synchronisations instead of returning it and mapping it anew per group
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (keep < s->budget) {
      keep = s->budget;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  cudaGetLastError();
  for (int i = 0; i < s->nstreams; ++i) {
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
      return fail(B2F_ERR_DEVICE, "stream creation failed");
    s->streams.push_back(st);
  }
  Server* raw = s.get();
  s->worker = std::thread([raw] { raw->run(); });
  *out = new b2f_server{s.release()};
  return B2F_OK;
}

void b2f_server_free(b2f_server* srv) {
  if (!srv) return;
  delete srv->s;
  delete srv;
}

b2f_status b2f_server_submit(b2f_server* srv, const b2f_config* cfg, int32_t kind,
                             const void* host_in, uint64_t in_bytes, void* host_out,
                             uint64_t out_bytes, uint64_t* request_id) {
  return submit_any(srv, cfg, kind, false, host_in, in_bytes, host_out, out_bytes, request_id);
}

b2f_status b2f_server_submit_device(b2f_server* srv, const b2f_config* cfg, int32_t kind,
                                    const void* dev_in, uint64_t in_bytes, void* dev_out,
                                    uint64_t out_bytes, uint64_t* request_id) {
  return submit_any(srv, cfg, kind, true, dev_in, in_bytes, dev_out, out_bytes, request_id);
}

b2f_status b2f_server_wait(b2f_server* srv, uint64_t request_id, double timeout_s) {
  if (!srv) return fail(B2F_ERR_INVALID_ARGUMENT, "null server");
  Server* s = srv->s;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return fail(B2F_ERR_INVALID_ARGUMENT, "unknown request id");
  SReq* r = it->second.get();
  const auto deadline = std::chrono::steady_clock::now() +
                        std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 3600.0);
  while (r->state < 2) {
    if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && r->state < 2)
      return fail(B2F_ERR_DEVICE, "timed out waiting for the request");
  }
  const b2f_status st = r->status;
  const std::string err = r->error;
  s->reqs.erase(it);
  if (st) return fail(st, err);
  return B2F_OK;
}

b2f_status b2f_server_drain(b2f_server* srv, double timeout_s) {
  if (!srv) return fail(B2F_ERR_INVALID_ARGUMENT, "null server");
  Server* s = srv->s;
  std::unique_lock<std::mutex> lk(s->mu);
  const auto deadline = std::chrono::steady_clock::now() +
                        std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 3600.0);
  while (!s->queue.empty() || !s->inflight.empty()) {
    s->cv_work.notify_all();
    if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
        (!s->queue.empty() || !s->inflight.empty()))
      return fail(B2F_ERR_DEVICE, "timed out draining the server");
  }
  return B2F_OK;
}

void b2f_server_hold(b2f_server* srv, int32_t hold) {
  if (!srv) return;
  {
    std::lock_guard<std::mutex> lk(srv->s->mu);
    srv->s->held = hold != 0;
  }
  srv->s->cv_work.notify_all();
}

b2f_status b2f_server_stats_json(b2f_server* srv, char* buf, uint64_t* len) {
  if (!srv || !len) return fail(B2F_ERR_INVALID_ARGUMENT, "null argument");
  Server* s = srv->s;
  std::string j;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> l = s->lat;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(p * l.size()))]; };
    const double span = s->t_last > s->t_first ? s->t_last - s->t_first : 0.0;
    std::ostringstream os;
    os << "{\"completed\":" << s->completed << ",\"failed\":" << s->failed
       << ",\"groups\":" << s->groups << ",\"line_groups\":" << s->line_groups
       << ",\"coalesced_requests\":" << s->coalesced
       << ",\"transforms\":" << s->transforms << ",\"p50_ms\":" << pct(0.50) * 1e3
       << ",\"p99_ms\":" << pct(0.99) * 1e3 << ",\"max_ms\":" << (l.empty() ? 0.0 : l.back() * 1e3)
       << ",\"span_s\":" << span << ",\"requests_per_s\":" << (span > 0 ? s->completed / span : 0.0)
       << ",\"ffts_per_s\":" << (span > 0 ? s->transforms / span : 0.0)
       << ",\"hbm_in_flight_bytes\":" << s->used << ",\"hbm_budget_bytes\":" << s->budget
       << ",\"resident_plans\":" << s->plans.size() << ",\"plan_bytes\":" << s->plan_bytes
       << ",\"plan_evictions\":" << s->evictions << ",\"line_registry_bytes\":" << s->registry_bytes()
       << ",\"streams\":" << s->nstreams << ",\"coalesce\":" << (s->coalesce ? "true" : "false")
       << "}";
    j = os.str();
  }
  const uint64_t cap = *len;
  *len = j.size();
  if (buf && cap > 0) {
    const uint64_t n = std::min<uint64_t>(cap - 1, j.size());
    std::memcpy(buf, j.data(), n);
    buf[n] = 0;
  }
  return B2F_OK;
}

void b2f_server_reset_stats(b2f_server* srv) {
  if (!srv) return;
  std::lock_guard<std::mutex> lk(srv->s->mu);
  Server* s = srv->s;
  s->lat.clear();
  s->completed = s->failed = s->groups = s->line_groups = s->coalesced = s->transforms = 0;
  s->evictions = 0;
  s->t_first = s->t_last = 0;
}

}  // extern "C"
