// Frame server of libupbd.so (C ABI in include/upbd_server.h): continuous
// batching of scene requests over one scene batch.
//
// Threads: builder threads turn arrived requests into prepared scenes
// (host-only work: lattice lookup, fluid slots); the thread inside
// upbd_server_run owns the batch and the device: it admits prepared requests
// in arrival order while the HBM budget and the scene table allow, steps one
// batched frame of every live request, waits for it, stamps each live
// request's frame, and retires the finished ones (their memory returns to
// the batch's pool for the next admissions). One mutex guards the request
// table; the batch is touched by the serving thread only.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/upbd_server.h"
#include "upbd_batch_internal.h"
#include "upbd_scene.h"

using namespace upbd;

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  int64_t id = 0;
  upbd_request r{};
  std::vector<float> pos3, vel3;  // copies of the caller's arrays until prepared
  int state = UPBD_REQ_QUEUED;
  int status = UPBD_OK;
  PreparedScene ps;
  size_t bytes = 0;
  int32_t sid = -1;
  int frames_done = 0;
  int slots = 0;
  double admit = 0, done = 0, ready_t = 0, frame_ms_max = 0;
  std::vector<float> res_pos;
  std::vector<uint32_t> res_flags;
};

double pct(std::vector<float> v, double q) {
  if (v.empty()) return 0;
  const size_t k = (size_t)std::min<double>((double)v.size() - 1, std::floor(q * (double)(v.size() - 1) + 0.5));
  std::nth_element(v.begin(), v.begin() + k, v.end());
  return v[k];
}

thread_local std::string g_server_error;

}  // namespace

struct upbd_server {
  upbd_server_desc desc{};
  upbd_batch* batch = nullptr;
  std::mutex mu;
  std::condition_variable cv_build;  // builders wait for arrivals
  std::condition_variable cv_ready;  // the serving thread waits for prepared requests
  std::map<int64_t, Req> reqs;
  std::multimap<double, int64_t> by_arrival;  // requests not yet admitted or rejected
  int64_t next_id = 1;
  std::vector<std::thread> builders;
  bool stop = false;
  bool started = false;
  Clock::time_point t0;
  // statistics
  int64_t submitted = 0, admitted = 0, completed = 0, rejected = 0, scene_frames = 0, batch_frames = 0;
  double particle_substeps = 0, device_s = 0, wall_s = 0, scene_sum = 0;
  int32_t peak_scenes = 0;
  uint64_t peak_bytes = 0;
  std::vector<float> frame_ms, wait_ms, batch_ms;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

int sfail(upbd_server* s, int code, const std::string& msg) {
  if (s) s->err = msg;
  g_server_error = msg;
  return code;
}

// Builder thread: prepares the earliest-arriving queued request whose
// arrival time has come.
void builder_main(upbd_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    Req* pick = nullptr;
    double next_arrival = -1;
    if (s->started) {
      const double t = s->now();
      for (auto& kv : s->by_arrival) {  // arrival order; skips those being prepared or ready
        Req& r = s->reqs[kv.second];
        if (r.state != UPBD_REQ_QUEUED) continue;
        if (kv.first <= t) pick = &r;
        else next_arrival = kv.first;
        break;
      }
    }
    if (!pick) {
      if (next_arrival >= 0)
        s->cv_build.wait_for(lk, std::chrono::duration<double>(std::max(1e-4, next_arrival - s->now())));
      else
        s->cv_build.wait(lk);
      continue;
    }
    pick->state = UPBD_REQ_PREPARING;
    const int64_t id = pick->id;
    const upbd_request r = pick->r;
    std::vector<float> pos3 = std::move(pick->pos3), vel3 = std::move(pick->vel3);
    lk.unlock();
    PreparedScene ps;
    const char* why = prepare_scene(r.desc, r.params, r.n_fluid, pos3.empty() ? nullptr : pos3.data(),
                                    vel3.empty() ? nullptr : vel3.data(), r.fluid_mass, ps);
    size_t bytes = why ? 0 : prepared_bytes(ps);
    lk.lock();
    Req& q = s->reqs[id];
    if (why) {
      q.state = UPBD_REQ_REJECTED;
      q.status = UPBD_ERR_INVALID;
      s->rejected++;
      for (auto it = s->by_arrival.begin(); it != s->by_arrival.end(); ++it)
        if (it->second == id) {
          s->by_arrival.erase(it);
          break;
        }
    } else {
      q.ps = std::move(ps);
      q.bytes = bytes;
      q.slots = q.ps.lat->S + r.desc.max_fluid;
      q.state = UPBD_REQ_READY;
    }
    s->cv_ready.notify_all();
  }
}

// Admits prepared requests in arrival order while they fit; stops at the
// first arrived request that is not prepared yet or does not fit (arrival
// order is kept). Called with the lock held; releases it around uploads.
void admit(upbd_server* s, std::unique_lock<std::mutex>& lk) {
  const uint64_t budget = s->desc.batch.hbm_budget;
  while (true) {
    const double t = s->now();
    auto it = s->by_arrival.begin();
    if (it == s->by_arrival.end() || it->first > t) return;
    Req& r = s->reqs[it->second];
    if (r.state != UPBD_REQ_READY) return;
    if (budget && r.bytes > budget) {  // can never fit
      r.state = UPBD_REQ_REJECTED;
      r.status = UPBD_ERR_CAPACITY;
      s->rejected++;
      s->by_arrival.erase(it);
      continue;
    }
    upbd_batch_info bi;
    upbd_batch_get_info(s->batch, &bi);
    if (bi.scenes >= bi.max_scenes) return;
    if (budget && bi.bytes_in_use + r.bytes > budget) return;
    const int64_t id = r.id;
    const double arrival = it->first;
    s->by_arrival.erase(it);
    r.state = UPBD_REQ_RUNNING;  // no other thread touches a running request
    lk.unlock();
    int32_t sid = -1;
    const int rc = batch_add_prepared(s->batch, r.ps, &sid);  // map nodes are stable
    lk.lock();
    Req& q = s->reqs[id];
    if (rc == UPBD_ERR_CAPACITY || rc == UPBD_ERR_OOM) {
      if (bi.scenes > 0) {  // memory frees up when running requests finish: wait
        q.state = UPBD_REQ_READY;
        s->by_arrival.emplace(arrival, id);
        return;
      }
    }
    if (rc != UPBD_OK) {
      q.ps = PreparedScene();
      q.state = UPBD_REQ_REJECTED;
      q.status = rc;
      s->rejected++;
      continue;
    }
    q.ps = PreparedScene();  // the host copies are no longer needed
    q.sid = sid;
    q.admit = s->now();
    q.ready_t = q.r.arrival_s;
    s->admitted++;
    s->wait_ms.push_back((float)((q.admit - q.r.arrival_s) * 1e3));
  }
}

}  // namespace

extern "C" {

int upbd_server_default_desc(upbd_server_desc* d) {
  if (!d) return UPBD_ERR_INVALID;
  std::memset(d, 0, sizeof(*d));
  upbd_batch_default_desc(&d->batch);
  d->batch.max_scenes = 4096;
  d->dt = 1.0 / 60;
  d->substeps = 5;
  d->builders = 4;
  d->keep_results = 0;
  return UPBD_OK;
}

const char* upbd_server_last_error(upbd_server* s) { return s ? s->err.c_str() : g_server_error.c_str(); }

int upbd_server_create(const upbd_server_desc* d, upbd_server** out) {
  if (!d || !out) return sfail(nullptr, UPBD_ERR_INVALID, "null argument");
  *out = nullptr;
  if (!(d->dt > 0) || d->substeps < 1 || d->substeps > 1000)
    return sfail(nullptr, UPBD_ERR_INVALID, "dt must be > 0 and substeps in [1, 1000]");
  if (d->builders < 1 || d->builders > 64) return sfail(nullptr, UPBD_ERR_INVALID, "builders out of range [1, 64]");
  upbd_batch* b = nullptr;
  const int rc = upbd_batch_create(&d->batch, &b);
  if (rc != UPBD_OK) return sfail(nullptr, rc, upbd_batch_last_error(nullptr));
  upbd_server* s = new upbd_server();
  s->desc = *d;
  s->batch = b;
  if (cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) {
    upbd_server_destroy(s);
    return sfail(nullptr, UPBD_ERR_CUDA, "event creation failed");
  }
  for (int k = 0; k < d->builders; k++) s->builders.emplace_back(builder_main, s);
  *out = s;
  return UPBD_OK;
}

int upbd_server_destroy(upbd_server* s) {
  if (!s) return UPBD_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_build.notify_all();
  for (auto& t : s->builders) t.join();
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  upbd_batch_destroy(s->batch);
  delete s;
  return UPBD_OK;
}

int upbd_server_submit(upbd_server* s, const upbd_request* r, int64_t* id) {
  if (!s || !r || !id) return sfail(s, UPBD_ERR_INVALID, "null argument");
  if (r->frames < 1) return sfail(s, UPBD_ERR_INVALID, "frames must be >= 1");
  if (r->n_fluid < 0 || r->n_fluid > r->desc.max_fluid) return sfail(s, UPBD_ERR_INVALID, "n_fluid out of range");
  if (r->n_fluid > 0 && !r->fluid_pos3) return sfail(s, UPBD_ERR_INVALID, "fluid positions required");
  if (r->desc.solid_iters != s->desc.batch.solid_iters || r->desc.features != s->desc.batch.features)
    return sfail(s, UPBD_ERR_INVALID, "request solid_iters/features differ from the server's");
  if (const char* why = check_desc(&r->desc, &r->params)) return sfail(s, UPBD_ERR_INVALID, why);
  Req q;
  q.r = *r;
  q.r.fluid_pos3 = nullptr;
  q.r.fluid_vel3 = nullptr;
  if (r->n_fluid > 0) {
    q.pos3.assign(r->fluid_pos3, r->fluid_pos3 + 3 * (size_t)r->n_fluid);
    if (r->fluid_vel3) q.vel3.assign(r->fluid_vel3, r->fluid_vel3 + 3 * (size_t)r->n_fluid);
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    q.id = s->next_id++;
    *id = q.id;
    s->by_arrival.emplace(r->arrival_s, q.id);
    s->reqs.emplace(q.id, std::move(q));
    s->submitted++;
  }
  s->cv_build.notify_all();
  return UPBD_OK;
}

int upbd_server_run(upbd_server* s, double max_seconds) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->desc.batch.device);
  std::unique_lock<std::mutex> lk(s->mu);
  if (!s->started) {
    s->t0 = Clock::now();
    s->started = true;
  }
  s->cv_build.notify_all();
  const double deadline = s->now() + max_seconds;
  cudaStream_t st = batch_stream(s->batch);
  std::vector<int64_t> live;
  while (true) {
    admit(s, lk);
    live.clear();
    bool pending = !s->by_arrival.empty();
    for (auto& kv : s->reqs)
      if (kv.second.state == UPBD_REQ_RUNNING) live.push_back(kv.first);
    if (live.empty()) {
      if (!pending) break;  // everything submitted is finished
      if (s->now() >= deadline) {
        s->wall_s = s->now();
        return sfail(s, UPBD_ERR_TIMEOUT, "serving time limit reached");
      }
      // wait for the next arrival to be prepared (builders notify)
      s->cv_ready.wait_for(lk, std::chrono::milliseconds(1));
      continue;
    }
    lk.unlock();
    int rc = cudaEventRecord(s->ev0, st) == cudaSuccess ? UPBD_OK : UPBD_ERR_CUDA;
    if (rc == UPBD_OK) rc = upbd_batch_step(s->batch, s->desc.dt, s->desc.substeps);
    if (rc == UPBD_OK && cudaEventRecord(s->ev1, st) != cudaSuccess) rc = UPBD_ERR_CUDA;
    if (rc == UPBD_OK && cudaEventSynchronize(s->ev1) != cudaSuccess) rc = UPBD_ERR_CUDA;
    if (rc != UPBD_OK) {
      lk.lock();
      return sfail(s, rc, std::string("batched frame: ") + upbd_batch_last_error(s->batch));
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    lk.lock();
    const double t = s->now();
    s->batch_frames++;
    s->device_s += ms * 1e-3;
    s->batch_ms.push_back(ms);
    s->scene_sum += (double)live.size();
    s->peak_scenes = std::max<int32_t>(s->peak_scenes, (int32_t)live.size());
    {
      upbd_batch_info bi;
      upbd_batch_get_info(s->batch, &bi);
      s->peak_bytes = std::max<uint64_t>(s->peak_bytes, bi.bytes_in_use);
    }
    for (int64_t id : live) {
      Req& q = s->reqs[id];
      uint32_t active = 0, health = 0;
      int32_t solids = 0;
      batch_scene_counters(s->batch, q.sid, &active, &health, &solids);
      q.frames_done++;
      s->scene_frames++;
      const double fm = (t - q.ready_t) * 1e3;
      s->frame_ms.push_back((float)fm);
      q.frame_ms_max = std::max(q.frame_ms_max, fm);
      q.ready_t = t;
      s->particle_substeps += (double)(solids + (int64_t)active) * s->desc.substeps;
      const bool bad = (health & UPBD_HEALTH_NAN) != 0;
      if (q.frames_done >= q.r.frames || bad) {
        if (s->desc.keep_results) {
          q.res_pos.resize((size_t)q.slots * 4);
          q.res_flags.resize((size_t)q.slots);
          upbd_batch_read_state(s->batch, q.sid, q.res_pos.data(), nullptr, nullptr, nullptr, q.res_flags.data());
        }
        upbd_batch_remove_scene(s->batch, q.sid);
        q.sid = -1;
        q.state = UPBD_REQ_DONE;
        q.status = bad ? UPBD_ERR_NAN : UPBD_OK;
        q.done = t;
        s->completed++;
      }
    }
    s->wall_s = t;
    if (t >= deadline) {
      bool more = !s->by_arrival.empty();
      for (auto& kv : s->reqs) more = more || kv.second.state == UPBD_REQ_RUNNING;
      if (more) return sfail(s, UPBD_ERR_TIMEOUT, "serving time limit reached");
      break;
    }
  }
  s->wall_s = s->now();
  return UPBD_OK;
}

int upbd_server_get_stats(upbd_server* s, upbd_server_stats* o) {
  if (!s || !o) return UPBD_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(o, 0, sizeof(*o));
  o->submitted = s->submitted;
  o->admitted = s->admitted;
  o->completed = s->completed;
  o->rejected = s->rejected;
  o->scene_frames = s->scene_frames;
  o->batch_frames = s->batch_frames;
  o->particle_substeps = s->particle_substeps;
  o->wall_s = s->wall_s;
  o->device_s = s->device_s;
  o->frame_ms_p50 = pct(s->frame_ms, 0.50);
  o->frame_ms_p90 = pct(s->frame_ms, 0.90);
  o->frame_ms_p99 = pct(s->frame_ms, 0.99);
  o->frame_ms_max = s->frame_ms.empty() ? 0 : *std::max_element(s->frame_ms.begin(), s->frame_ms.end());
  double sum = 0;
  for (float x : s->frame_ms) sum += x;
  o->frame_ms_mean = s->frame_ms.empty() ? 0 : sum / (double)s->frame_ms.size();
  o->wait_ms_p50 = pct(s->wait_ms, 0.50);
  o->wait_ms_p99 = pct(s->wait_ms, 0.99);
  o->batch_ms_p50 = pct(s->batch_ms, 0.50);
  o->batch_ms_p99 = pct(s->batch_ms, 0.99);
  o->mean_scenes = s->batch_frames ? s->scene_sum / (double)s->batch_frames : 0;
  o->peak_scenes = s->peak_scenes;
  o->peak_bytes = s->peak_bytes;
  return UPBD_OK;
}

int upbd_server_result(upbd_server* s, int64_t id, upbd_request_result* res, float* pos4, uint32_t* flags) {
  if (!s || !res) return UPBD_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sfail(s, UPBD_ERR_INVALID, "no such request");
  const Req& q = it->second;
  std::memset(res, 0, sizeof(*res));
  res->state = q.state;
  res->status = q.status;
  res->frames_done = q.frames_done;
  res->slots = q.slots;
  res->arrival_s = q.r.arrival_s;
  res->admit_s = q.admit;
  res->done_s = q.done;
  res->frame_ms_max = q.frame_ms_max;
  if ((pos4 || flags) && q.state == UPBD_REQ_DONE) {
    if (q.res_pos.empty()) return sfail(s, UPBD_ERR_INVALID, "the server does not keep results");
    if (pos4) std::memcpy(pos4, q.res_pos.data(), q.res_pos.size() * 4);
    if (flags) std::memcpy(flags, q.res_flags.data(), q.res_flags.size() * 4);
  }
  return UPBD_OK;
}

}  // extern "C"
