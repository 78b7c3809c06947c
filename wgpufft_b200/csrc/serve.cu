// Serving loop (b2f_server_*): requests of any configuration served with
// continuous batching; the crate has no counterpart (its plans only record
// into a caller's encoder).
//
// Clients submit transforms of any configuration with their data in host
// memory.  One scheduler thread owns the device side:
//   - admission: a request is admitted when the device bytes it needs (its
//     staging buffers, plus the workspace of the plan it runs on) fit the
//     HBM budget next to everything already in flight; otherwise it waits
//     until in-flight groups complete and release memory;
//   - continuous batching: admitted requests with the same configuration
//     are coalesced into one group and run as a single plan execution whose
//     batch is the sum of theirs (batches are contiguous blocks, so the
//     requests' buffers simply sit back to back); new arrivals join the next
//     group while earlier groups are still on the GPU;
//   - overlap: groups rotate over several streams, each group being
//     host->device copies, the transform, device->host copies, then a
//     stream-ordered free, so copies of one group overlap the kernels of
//     another;
//   - resident plans: plans (and their tables/workspaces) are cached by
//     configuration and reused.
// Completion is observed with events; waiting clients are woken, latency is
// recorded from submission to completion.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_map>
#include <vector>

#include "plan.h"

namespace b2f {

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct SReq {
  uint64_t id = 0;
  Config cfg;
  int32_t kind = B2F_C2C;
  std::string key;
  const void* host_in = nullptr;
  void* host_out = nullptr;
  uint64_t in_bytes = 0, out_bytes = 0;  // the request's own sizes
  double t_submit = 0, t_done = 0;
  int state = 0;  // 0 queued, 1 in flight, 2 done, 3 failed
  b2f_status status = B2F_OK;
  std::string error;
};

struct SGroup {
  std::vector<SReq*> reqs;
  int stream = 0;
  cudaEvent_t done = nullptr;
  uint64_t bytes = 0;  // device bytes held until completion
};

static std::string config_key(const Config& c, int32_t kind) {
  std::ostringstream os;
  os << kind << "|" << c.precision << "|" << c.direction << "|" << c.normalization << "|";
  for (auto s : c.shape) os << s << ",";
  os << "|";
  for (auto a : c.axes) os << a << ",";
  return os.str();
}

struct Server {
  int device = 0;
  uint64_t budget = 0;
  int nstreams = 4;
  uint32_t max_group = 64;
  bool coalesce = true;
  std::vector<cudaStream_t> streams;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::deque<SReq*> queue;
  std::unordered_map<uint64_t, std::unique_ptr<SReq>> reqs;
  std::vector<SGroup> inflight;
  uint64_t used = 0;
  uint64_t next_id = 1;
  int next_stream = 0;
  // plan cache: key (with the total batch) -> plan
  std::map<std::string, std::unique_ptr<Plan>> plans;
  // per cached plan, the end of its last execution: a plan's workspace is
  // shared by its executions, so one on another stream waits for it
  std::map<const Plan*, cudaEvent_t> plan_done;
  uint64_t plan_bytes = 0;
  // statistics
  std::vector<double> lat;
  uint64_t completed = 0, failed = 0, groups = 0, coalesced = 0, transforms = 0;
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
    for (auto& kv : plan_done) cudaEventDestroy(kv.second);
    for (auto s : streams) cudaStreamDestroy(s);
  }

  Plan* get_plan(const Config& cfg, int32_t kind, b2f_status* st) {
    const std::string k = config_key(cfg, kind) + "|b" + std::to_string(cfg.batch);
    auto it = plans.find(k);
    if (it != plans.end()) return it->second.get();
    Plan* p = nullptr;
    *st = create_plan(cfg, kind, device, &p);
    if (*st) return nullptr;
    plan_bytes += p->workspace_total() + p->table_bytes;
    plans[k].reset(p);
    return p;
  }

  // Completes every group whose event has fired (lock held).
  void reap(bool block_one) {
    for (size_t i = 0; i < inflight.size();) {
      SGroup& g = inflight[i];
      cudaError_t q = block_one && i == 0 ? cudaEventSynchronize(g.done) : cudaEventQuery(g.done);
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
      block_one = false;
    }
    cv_done.notify_all();
  }

  // Launches one group (lock held; the CUDA calls are asynchronous).
  void launch(std::vector<SReq*>& members) {
    SReq* r0 = members[0];
    Config cfg = r0->cfg;
    uint64_t total_batch = 0, in_total = 0, out_total = 0;
    for (SReq* r : members) {
      total_batch += r->cfg.batch;
      in_total += r->in_bytes;
      out_total += r->out_bytes;
    }
    cfg.batch = total_batch;
    b2f_status st = B2F_OK;
    Plan* plan = get_plan(cfg, r0->kind, &st);
    auto fail_all = [&](b2f_status s, const std::string& msg) {
      for (SReq* r : members) {
        r->state = 3;
        r->status = s;
        r->error = msg;
        ++failed;
      }
      cv_done.notify_all();
    };
    if (!plan) {
      fail_all(st, last_error());
      return;
    }
    const int si = next_stream;
    next_stream = (next_stream + 1) % nstreams;
    cudaStream_t s = streams[si];
    void* din = nullptr;
    void* dout = nullptr;
    if (cudaMallocAsync(&din, std::max<uint64_t>(in_total, 16), s) != cudaSuccess ||
        cudaMallocAsync(&dout, std::max<uint64_t>(out_total, 16), s) != cudaSuccess) {
      cudaGetLastError();
      if (din) cudaFreeAsync(din, s);
      fail_all(B2F_ERR_RESOURCE_ALLOCATION, "staging allocation failed");
      return;
    }
    uint64_t off = 0;
    for (SReq* r : members) {
      cudaMemcpyAsync((char*)din + off, r->host_in, r->in_bytes, cudaMemcpyHostToDevice, s);
      off += r->in_bytes;
    }
    cudaEvent_t& pd = plan_done[plan];
    if (!pd) cudaEventCreateWithFlags(&pd, cudaEventDisableTiming);
    else cudaStreamWaitEvent(s, pd, 0);  // after this group's copies in are queued
    st = execute_plan(*plan, s, din, in_total, dout, out_total);
    if (pd) cudaEventRecord(pd, s);
    off = 0;
    for (SReq* r : members) {
      cudaMemcpyAsync(r->host_out, (char*)dout + off, r->out_bytes, cudaMemcpyDeviceToHost, s);
      off += r->out_bytes;
    }
    cudaFreeAsync(din, s);
    cudaFreeAsync(dout, s);
    if (st) {
      fail_all(st, last_error());
      return;
    }
    SGroup g;
    g.reqs = members;
    g.stream = si;
    g.bytes = in_total + out_total;
    cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming);
    cudaEventRecord(g.done, s);
    for (SReq* r : members) r->state = 1;
    used += g.bytes;
    ++groups;
    if (members.size() > 1) coalesced += members.size();
    inflight.push_back(g);
  }

  void run() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
      cv_work.wait_for(lk, std::chrono::microseconds(200),
                       [&] { return stop || !queue.empty() || !inflight.empty(); });
      if (stop && queue.empty() && inflight.empty()) break;
      reap(false);
      // admit and group: take the queue head's configuration, then every
      // other queued request with the same configuration (continuous batching)
      while (!queue.empty()) {
        SReq* head = queue.front();
        std::vector<SReq*> members;
        uint64_t need = 0;
        for (auto it = queue.begin(); it != queue.end() && members.size() < max_group;) {
          SReq* r = *it;
          if (r->key != head->key || (!coalesce && !members.empty())) {
            ++it;
            continue;
          }
          const uint64_t b = r->in_bytes + r->out_bytes;
          if (!members.empty() && used + need + b > budget) break;
          members.push_back(r);
          need += b;
          it = queue.erase(it);
        }
        if (used + need > budget && !inflight.empty()) {
          // wait for memory: put them back in front, in order
          for (auto it = members.rbegin(); it != members.rend(); ++it) queue.push_front(*it);
          reap(true);
          break;
        }
        if (used + need > budget) {
          for (SReq* r : members) {
            r->state = 3;
            r->status = B2F_ERR_RESOURCE_ALLOCATION;
            r->error = "request larger than the HBM admission budget";
            ++failed;
          }
          cv_done.notify_all();
          continue;
        }
        launch(members);
        // bound the work in flight: at most two groups per stream
        if ((int)inflight.size() >= 2 * nstreams) reap(true);
      }
    }
  }
};

}  // namespace b2f

using namespace b2f;

struct b2f_server {
  Server* s;
};

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
  if (!srv || !cfg || !host_in || !host_out || !request_id)
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
  std::unique_ptr<SReq> r(new SReq());
  r->cfg = c;
  r->kind = kind;
  r->key = config_key(c, kind);
  r->host_in = host_in;
  r->host_out = host_out;
  r->in_bytes = need_in;
  r->out_bytes = need_out;
  Server* s = srv->s;
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
       << ",\"groups\":" << s->groups << ",\"coalesced_requests\":" << s->coalesced
       << ",\"transforms\":" << s->transforms << ",\"p50_ms\":" << pct(0.50) * 1e3
       << ",\"p99_ms\":" << pct(0.99) * 1e3 << ",\"max_ms\":" << (l.empty() ? 0.0 : l.back() * 1e3)
       << ",\"span_s\":" << span << ",\"requests_per_s\":" << (span > 0 ? s->completed / span : 0.0)
       << ",\"ffts_per_s\":" << (span > 0 ? s->transforms / span : 0.0)
       << ",\"hbm_in_use_bytes\":" << s->used << ",\"hbm_budget_bytes\":" << s->budget
       << ",\"resident_plans\":" << s->plans.size() << ",\"plan_bytes\":" << s->plan_bytes
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
  s->completed = s->failed = s->groups = s->coalesced = s->transforms = 0;
  s->t_first = s->t_last = 0;
}

}  // extern "C"
