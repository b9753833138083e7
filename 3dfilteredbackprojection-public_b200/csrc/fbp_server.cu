// Reconstruction server: continuous batching of independent FBP jobs on one
// GPU. No counterpart in the reference (one reconstruction per process on a
// GL context).
//
// A server owns `slots` worker threads, each with its own fbp_context (own
// CUDA stream and buffers). Jobs are queued in arrival order; a free worker
// takes the first queued job whose working-set estimate fits the HBM budget
// beside the jobs already running (looking at most kLookahead jobs past the
// head, so a large job is not starved), or the head job alone when nothing
// runs. A job's uploads, kernels and readback run on its worker's stream, so
// jobs admitted together overlap on the device (copies of one beside the
// kernels of another, small jobs beside large ones). Results are identical to
// the same job run alone: every job runs the same kernels with the same
// arguments on its own buffers.
//
// Worker buffers only grow (see alloc_stack), so after warm-up a slot stops
// allocating; the budget covers the working sets of running jobs, and each
// slot retains at most its largest job's buffers.
//
// Batching (on by default, for cone jobs of at most 1e10 voxel-view updates,
// fbp_server_set_batch_limit; larger ones run their own slab pipeline, whose
// volume readback overlaps its backprojection): a cone job's worker uploads, weights, filters and
// plans the backprojection (packing, footprint pass) on its own
// (high-priority) stream, then hands it to the server's engine thread, which
// feeds the tiles of all waiting jobs to the persistent multi-job
// backprojector (launch_bp_batch): each launch carries about kChunkUpdates
// voxel-view updates, taken from the jobs in arrival order, so a large job's
// tiles are spread over several launches and jobs that arrive meanwhile join
// the next one instead of waiting for the large job to finish. Launches
// alternate between two launcher streams, so one launch's CTAs take the SMs
// as the other's finish. A job's stream waits for every launch that computed
// some of its tiles, then its worker reads the volume back. Each tile is
// computed whole by one CTA in a fixed order, so a job's volume is the same
// bits alone and in any mix. Jobs whose geometry does not take the symmetric
// backprojector launch alone on their own stream.

#include "fbp_internal.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kLookahead = 8;    // queued jobs looked at past a head that does not fit
constexpr int kMaxBypass = 16;   // times a head may be passed over before it blocks the queue
constexpr double kChunkUpdates = 6e10;  // voxel-view updates per batched launch (about 20 ms)
// Larger cone jobs are not batched. A job of more than ~1e10 updates fills
// the GPU with its own grid, and jobs on the slots' own streams already share
// the SMs as their CTAs retire; through the engine, such jobs lost more to
// its chunked launches (at most two in flight) than they gained. On the
// serving mix (2000 jobs, 5 slots, one B200) the jobs other than the 768^3
// ones took 16.1 s with a 2.4e11 limit, 13.1 s with 1e10 and 12.8 s with no
// batching; the whole stream 106.0, 104.5 and 103.7 s (bound by the 768^3
// jobs' backprojections).
constexpr double kBatchMaxUpdates = 1e10;

// A cone job's backprojection handed from its worker to the engine.
struct BatchJob {
  fbp_context* ctx = nullptr;
  fbp_geometry geom{};
  int h = 0, v = 0;
  fbp::BPLaunchPlan* plan = nullptr;
  long long key = 0, tiles = 0, next = 0;
  double per_tile = 0;    // voxel-view updates of one tile
  bool planned = false;
  bool launched = false;  // every tile launched; the job's stream waits for them
  // set under the server's mutex when the engine hands the job back (all tiles
  // launched, or failed): the worker waits on this flag alone, so the engine's
  // earlier writes of status and error are visible to it and the engine no
  // longer touches the job (it lives on the worker's stack)
  bool returned = false;
  int status = FBP_OK;
  std::string error;
};

struct Job {
  fbp_request req;
  long long ticket = 0;
  size_t bytes = 0;
  int bypassed = 0;  // later jobs started while this one headed the queue
  int status = FBP_OK;
  bool done = false;
  bool claimed = false;  // a caller waits on this ticket (it is consumed by the wait)
  double queued = 0, started = 0, finished = 0;  // ms since the server started
  std::string error;
};

struct Worker {
  fbp_context* ctx = nullptr;
  float* d_in = nullptr;  // 2D jobs: sinogram and image on the device (grow only)
  float* d_out = nullptr;
  size_t in_cap = 0, out_cap = 0;
  std::thread thread;
};

size_t estimate_bytes(const fbp_request& r) {
  if (r.reserve_bytes > 0) return (size_t)r.reserve_bytes;
  const size_t cols4 = (size_t)(r.det_cols + 3) / 4 * 4;
  if (r.kind == FBP_JOB_CONE) {
    const size_t stack = cols4 * r.det_rows * r.views * 4;
    // packed views: FP16 quads 8 bytes per sample, 24-bit quads 12, FP32 pairs 8
    const size_t per = r.precision == FBP_PRECISION_MIXED24 ? 12 : 8;
    const size_t packed = r.precision != FBP_PRECISION_FP32
                              ? (size_t)r.views * (r.det_rows + 1) * (r.det_cols + 1) * per
                              : cols4 * (r.det_rows + 1) * r.views * 8;
    const size_t vol = (size_t)r.vol_h * r.vol_v * r.vol_h * 4;
    const size_t split = std::min<size_t>((size_t)r.det_rows * r.views, 65536) * (cols4 + 64) * 4;
    return stack + packed + vol + split + (64u << 20);
  }
  if (r.kind == FBP_JOB_FAN2D || r.kind == FBP_JOB_PARALLEL2D)
    return cols4 * r.views * 4 * 3 + (size_t)r.vol_h * r.vol_h * 4 + (16u << 20);
  return 0;
}

int device_buffer(float** p, size_t* cap, size_t bytes) {
  if (*p && *cap >= bytes) return FBP_OK;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return FBP_ERR_OUT_OF_MEMORY;
  }
  *cap = bytes;
  return FBP_OK;
}

}  // namespace

struct fbp_server {
  int device = -1;
  size_t budget = 0;
  bool batching = true;
  double chunk_updates = kChunkUpdates;  // voxel-view updates per batched launch
  double batch_max = kBatchMaxUpdates;    // larger cone jobs run their own slab pipelines
  // engine: the persistent multi-job backprojector's feeder
  std::thread engine;
  fbp_context* launcher[2] = {nullptr, nullptr};
  cudaEvent_t launched_ev[2] = {nullptr, nullptr};
  cudaEvent_t start_ev[2] = {nullptr, nullptr};  // timing of each launcher's launch in flight
  bool launcher_busy[2] = {false, false};
  // statistics (under mu): device time of the batched launches, host time in transfers
  double stat_batch_ms = 0, stat_upload_ms = 0, stat_readback_ms = 0;
  long long stat_launches = 0, stat_batched_jobs = 0;
  std::deque<BatchJob*> incoming;  // handed over, not yet planned (under mu)
  std::condition_variable engine_cv, batch_cv;
  bool engine_stop = false;
  std::vector<cudaStream_t> worker_streams;
  Clock::time_point t0;
  std::vector<Worker> workers;
  std::mutex mu;
  std::condition_variable work_cv, done_cv;
  std::deque<Job*> queue;
  std::unordered_map<long long, Job*> jobs;
  size_t reserved = 0;
  int running = 0;
  long long next_ticket = 1;
  bool stop = false;

  double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

  // first admissible queued job (caller holds mu)
  std::deque<Job*>::iterator pick() {
    int seen = 0;
    for (auto it = queue.begin(); it != queue.end() && seen <= kLookahead; ++it, ++seen) {
      if (running == 0 && it == queue.begin()) return it;  // nothing runs: the head goes, whatever its size
      if (reserved + (*it)->bytes <= budget) {
        if (it != queue.begin()) ++queue.front()->bypassed;
        return it;
      }
      if (queue.front()->bypassed >= kMaxBypass) break;  // the head waits for memory; nobody passes it
    }
    return queue.end();
  }

  int run(Worker& w, Job& j) {
    const fbp_request& r = j.req;
    if (r.kind == FBP_JOB_HOST_WAIT) {  // scheduler tests: holds the slot and the reservation for views us
      std::this_thread::sleep_for(std::chrono::microseconds(std::max(0, r.views)));
      return FBP_OK;
    }
    fbp_context* c = w.ctx;
    if (!c) {
      j.error = "server has no device";
      return FBP_ERR_STATE;
    }
    if (!r.input || !r.output) {
      j.error = "null input or output";
      return FBP_ERR_INVALID_ARGUMENT;
    }
    const fbp_geometry& g = r.geometry;
    int rc = fbp_set_precision(c, r.precision);
    // a cone job of more than batch_max updates runs its own slab
    // pipeline (readback of one slab under the next slab's backprojection);
    // batching pays for the jobs that a launch can mix
    const double updates = (double)r.vol_h * r.vol_h * r.vol_v * (double)r.views;
    bool batch;
    {
      std::lock_guard<std::mutex> lk(mu);
      batch = batching && updates <= batch_max;
    }
    if (r.kind == FBP_JOB_CONE && batch && launcher[0]) {
      // upload, weights and filter here; the engine backprojects; then readback
      if (!rc) rc = fbp_set_clip_after_backprojection(c, r.clip);
      const double tu = now_ms();
      if (!rc) rc = fbp_upload_projections(c, r.input, r.det_cols, r.det_rows, r.views, 0);
      {
        std::lock_guard<std::mutex> lk(mu);
        stat_upload_ms += now_ms() - tu;
      }
      if (!rc) rc = fbp_apply_fdk_weights_to_projections(c, g.source_distance, g.detector_distance, g.detector_width);
      if (!rc) rc = fbp_apply_filter_to_projections(c, r.filter_type);
      if (!rc) {
        BatchJob bj;
        bj.ctx = c;
        bj.geom = g;
        bj.geom.kind = FBP_GEOMETRY_CONE;
        bj.h = r.vol_h;
        bj.v = r.vol_v;
        // plan here, on this worker's stream (packing, footprint pass), so
        // that the engine thread only launches
        prepare(bj);
        if (bj.status == FBP_OK && bj.tiles > 0) {
          std::unique_lock<std::mutex> lk(mu);
          incoming.push_back(&bj);
          engine_cv.notify_all();
          batch_cv.wait(lk, [&] { return bj.returned; });
        }
        rc = bj.status;
        if (rc) j.error = bj.error;
        if (bj.plan) fbp::free_bp_plan(bj.plan);
      }
      const double tr = now_ms();
      if (!rc) rc = fbp_read_volume(c, r.output, 0);
      {
        std::lock_guard<std::mutex> lk(mu);
        stat_readback_ms += now_ms() - tr;
        ++stat_batched_jobs;
      }
    } else if (r.kind == FBP_JOB_CONE) {
      // one call: upload, weights, filter, slab-wise backprojection with the
      // volume readback overlapped (large volumes in 4 slabs)
      fbp_geometry gc = g;
      gc.kind = FBP_GEOMETRY_CONE;
      if (!rc) rc = fbp_set_clip_after_backprojection(c, r.clip);
      if (!rc)
        rc = fbp_reconstruct_fdk_to_host(c, r.input, r.det_cols, r.det_rows, r.views, &gc, r.filter_type, r.vol_h,
                                         r.vol_v, r.output, r.vol_v >= 256 ? 4 : 1);
    } else if (r.kind == FBP_JOB_FAN2D || r.kind == FBP_JOB_PARALLEL2D) {
      const size_t in = (size_t)r.det_cols * r.views * 4, out = (size_t)r.vol_h * r.vol_h * 4;
      rc = device_buffer(&w.d_in, &w.in_cap, in);
      if (!rc) rc = device_buffer(&w.d_out, &w.out_cap, out);
      cudaStream_t st = c->stream;
      if (!rc && cudaMemcpyAsync(w.d_in, r.input, in, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = FBP_ERR_CUDA;
      const bool fan = r.kind == FBP_JOB_FAN2D;
      const float sdd = fan ? g.source_distance + g.detector_distance : 0.f;
      if (!rc) rc = fbp2d_filter_sinogram(c, w.d_in, r.det_cols, r.views, r.filter_type, sdd, g.detector_width);
      fbp_geometry gg = g;
      gg.kind = fan ? FBP_GEOMETRY_CONE : FBP_GEOMETRY_PARALLEL;
      if (!rc) rc = fbp2d_project_backward(c, w.d_in, r.det_cols, r.views, &gg, w.d_out, r.vol_h, r.vol_h);
      if (!rc && cudaMemcpyAsync(r.output, w.d_out, out, cudaMemcpyDeviceToHost, st) != cudaSuccess) rc = FBP_ERR_CUDA;
      if (!rc) rc = fbp_synchronize(c);
    } else {
      j.error = "unknown job kind";
      return FBP_ERR_INVALID_ARGUMENT;
    }
    if (rc && j.error.empty()) j.error = fbp_last_error(c);
    return rc;
  }

  // The engine thread: plans handed-over jobs and launches their tiles in
  // chunks through the persistent multi-job backprojector.
  void engine_main() {
    if (device >= 0) cudaSetDevice(device);
    std::vector<BatchJob*> active;
    int turn = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        engine_cv.wait(lk, [&] { return !incoming.empty() || !active.empty() || engine_stop; });
        if (engine_stop && incoming.empty() && active.empty()) break;
        while (!incoming.empty()) {
          active.push_back(incoming.front());
          incoming.pop_front();
        }
      }
      finish(active);
      if (active.empty()) continue;
      // one launch: tiles of the waiting jobs in arrival order, about
      // kChunkUpdates updates, all of the first job's batch key
      fbp_context* L = launcher[turn];
      if (launcher_busy[turn]) {  // at most one launch per launcher in flight
        cudaEventSynchronize(launched_ev[turn]);
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, start_ev[turn], launched_ev[turn]) == cudaSuccess) {
          std::lock_guard<std::mutex> lk(mu);
          stat_batch_ms += ms;
        }
        launcher_busy[turn] = false;
      }
      const long long key = active.front()->key;
      std::vector<fbp::BPLaunchPlan*> plans;
      std::vector<long long> t0, t1;
      std::vector<BatchJob*> members;
      double budget;
      {
        std::lock_guard<std::mutex> lk(mu);
        budget = chunk_updates;
      }
      for (BatchJob* b : active) {
        if (b->key != key || budget <= 0) continue;
        const long long want = (long long)std::ceil(budget / std::max(1.0, b->per_tile));
        const long long take = std::max(1LL, std::min(b->tiles - b->next, want));
        plans.push_back(b->plan);
        t0.push_back(b->next);
        t1.push_back(b->next + take);
        members.push_back(b);
        budget -= take * b->per_tile;
      }
      int rc = FBP_OK;
      for (BatchJob* b : members)
        if (cudaStreamWaitEvent(L->stream, b->ctx->ev_sync, 0) != cudaSuccess) rc = FBP_ERR_CUDA;
      if (!rc && cudaEventRecord(start_ev[turn], L->stream) != cudaSuccess) rc = FBP_ERR_CUDA;
      if (!rc) rc = fbp::launch_bp_batch(L, plans.data(), (int)plans.size(), t0.data(), t1.data());
      if (!rc) {
        std::lock_guard<std::mutex> lk(mu);
        ++stat_launches;
      }
      if (!rc && cudaEventRecord(launched_ev[turn], L->stream) != cudaSuccess) rc = FBP_ERR_CUDA;
      launcher_busy[turn] = true;
      for (size_t i = 0; i < members.size(); ++i) {
        BatchJob* b = members[i];
        if (rc) {
          b->status = rc;
          b->error = fbp_last_error(L);
          continue;
        }
        if (cudaStreamWaitEvent(b->ctx->stream, launched_ev[turn], 0) != cudaSuccess) {
          b->status = FBP_ERR_CUDA;
          b->error = "stream wait on the batched backprojection failed";
          continue;
        }
        b->next = t1[i];
        b->ctx->last_bp[0] = FBP_BACKPROJECTOR_SYMMETRIC;
        b->ctx->minmax_valid = false;
      }
      turn ^= 1;
      finish(active);
    }
  }

  // Plan a handed-over job on its worker's stream; a job off the symmetric
  // path launches alone there (tiles stays 0).
  void prepare(BatchJob& b) {
    b.planned = true;
    b.plan = fbp::new_bp_plan();
    int rc = fbp::plan_cone_projections(b.ctx, b.geom, b.h, b.v, b.plan);
    if (!rc) {
      b.key = fbp::bp_plan_batch_key(*b.plan);
      if (b.key == 0) {
        rc = fbp::launch_bp_plan(b.ctx, *b.plan);
        b.next = b.tiles = 0;
      } else {
        b.tiles = fbp::bp_plan_tiles(*b.plan);
        const double all = (double)b.h * b.h * b.v * (double)b.ctx->proj.n;
        b.per_tile = all / (double)std::max(1LL, b.tiles);
        // the job's preparatory work (on its stream) precedes every launch of its tiles
        if (!b.ctx->ev_sync) cudaEventCreateWithFlags(&b.ctx->ev_sync, cudaEventDisableTiming);
        if (cudaEventRecord(b.ctx->ev_sync, b.ctx->stream) != cudaSuccess) rc = FBP_ERR_CUDA;
      }
    }
    if (rc) {
      b.status = rc;
      b.error = fbp_last_error(b.ctx);
    }
  }

  // hand back the jobs that failed or have all their tiles launched
  void finish(std::vector<BatchJob*>& active) {
    bool any = false;
    {
      std::lock_guard<std::mutex> lk(mu);
      for (auto it = active.begin(); it != active.end();) {
        BatchJob* b = *it;
        if (b->status != FBP_OK || (b->planned && b->next >= b->tiles)) {
          b->launched = b->status == FBP_OK;
          b->returned = true;
          it = active.erase(it);
          any = true;
        } else {
          ++it;
        }
      }
    }
    if (any) batch_cv.notify_all();
  }

  void worker_main(Worker& w) {
    if (device >= 0) cudaSetDevice(device);
    for (;;) {
      Job* j = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        std::deque<Job*>::iterator it = queue.end();
        // wake for an admissible job; leave once stopped with nothing queued
        work_cv.wait(lk, [&] { return (it = pick()) != queue.end() || (stop && queue.empty()); });
        if (it == queue.end()) return;
        j = *it;
        queue.erase(it);
        reserved += j->bytes;
        ++running;
        j->started = now_ms();
      }
      const int rc = run(w, *j);
      {
        std::lock_guard<std::mutex> lk(mu);
        j->status = rc;
        j->finished = now_ms();
        j->done = true;
        reserved -= j->bytes;
        --running;
      }
      done_cv.notify_all();
      work_cv.notify_all();  // memory and a slot freed up
    }
  }
};

extern "C" {

int fbp_server_create(fbp_server** out, int device, size_t hbm_budget_bytes, int slots) {
  if (!out || slots <= 0 || slots > 64) return FBP_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  fbp_server* s = new fbp_server();
  s->device = device;
  s->t0 = Clock::now();
  s->workers.resize(slots);
  if (device >= 0) {
    if (hbm_budget_bytes == 0) {
      size_t free_b = 0, total_b = 0;
      int prev = 0;
      cudaGetDevice(&prev);
      cudaSetDevice(device);
      cudaMemGetInfo(&free_b, &total_b);
      cudaSetDevice(prev);
      hbm_budget_bytes = free_b / 10 * 8;  // 80 % of what is free now
    }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);  // hi: the highest priority (numerically least)
    int rc = FBP_OK;
    for (auto& w : s->workers) {
      rc = fbp_create(&w.ctx, device);
      if (rc) break;
      // workers' uploads, filters and packing go ahead of queued backprojection launches
      cudaStream_t st = nullptr;
      if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, hi) != cudaSuccess) {
        rc = FBP_ERR_CUDA;
        break;
      }
      s->worker_streams.push_back(st);
      rc = fbp_set_stream(w.ctx, st);
      if (rc) break;
    }
    for (int i = 0; i < 2 && !rc; ++i) {
      rc = fbp_create(&s->launcher[i], device);
      if (!rc && (cudaEventCreate(&s->launched_ev[i]) != cudaSuccess || cudaEventCreate(&s->start_ev[i]) != cudaSuccess))
        rc = FBP_ERR_CUDA;
    }
    cudaSetDevice(prev);
    if (rc) {
      for (auto& v : s->workers) fbp_destroy(v.ctx);
      for (int i = 0; i < 2; ++i) {
        fbp_destroy(s->launcher[i]);
        if (s->launched_ev[i]) cudaEventDestroy(s->launched_ev[i]);
        if (s->start_ev[i]) cudaEventDestroy(s->start_ev[i]);
      }
      for (cudaStream_t st : s->worker_streams) cudaStreamDestroy(st);
      delete s;
      return rc;
    }
  }
  s->budget = hbm_budget_bytes;
  if (device >= 0) s->engine = std::thread([s] { s->engine_main(); });
  for (auto& w : s->workers) w.thread = std::thread([s, &w] { s->worker_main(w); });
  *out = s;
  return FBP_OK;
}

int fbp_server_set_batching(fbp_server* s, int enable, double chunk_updates) {
  if (!s) return FBP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  s->batching = enable != 0;
  s->chunk_updates = chunk_updates > 0 ? chunk_updates : kChunkUpdates;
  return FBP_OK;
}

int fbp_server_set_batch_limit(fbp_server* s, double max_updates) {
  if (!s) return FBP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  s->batch_max = max_updates > 0 ? max_updates : kBatchMaxUpdates;
  return FBP_OK;
}

int fbp_server_stats(fbp_server* s, double* batch_gpu_ms, double* upload_ms, double* readback_ms,
                     long long* batch_launches, long long* batched_jobs) {
  if (!s) return FBP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  if (batch_gpu_ms) *batch_gpu_ms = s->stat_batch_ms;
  if (upload_ms) *upload_ms = s->stat_upload_ms;
  if (readback_ms) *readback_ms = s->stat_readback_ms;
  if (batch_launches) *batch_launches = s->stat_launches;
  if (batched_jobs) *batched_jobs = s->stat_batched_jobs;
  return FBP_OK;
}

int fbp_server_submit(fbp_server* s, const fbp_request* req, long long* ticket) {
  if (!s || !req || !ticket) return FBP_ERR_INVALID_ARGUMENT;
  Job* j = new Job();
  j->req = *req;
  j->bytes = estimate_bytes(*req);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete j;
      return FBP_ERR_STATE;
    }
    j->ticket = s->next_ticket++;
    j->queued = s->now_ms();
    s->jobs[j->ticket] = j;
    s->queue.push_back(j);
    *ticket = j->ticket;
  }
  s->work_cv.notify_all();
  return FBP_OK;
}

int fbp_server_wait(fbp_server* s, long long ticket, fbp_job_result* result) {
  if (!s) return FBP_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return FBP_ERR_INVALID_ARGUMENT;
  Job* j = it->second;
  if (j->claimed) return FBP_ERR_STATE;  // another caller is waiting on this ticket
  j->claimed = true;
  s->done_cv.wait(lk, [&] { return j->done; });
  if (result) {
    result->status = j->status;
    result->queued_ms = j->queued;
    result->started_ms = j->started;
    result->finished_ms = j->finished;
    std::memset(result->error, 0, sizeof(result->error));
    std::strncpy(result->error, j->error.c_str(), sizeof(result->error) - 1);
  }
  s->jobs.erase(it);
  delete j;
  return FBP_OK;
}

int fbp_server_destroy(fbp_server* s) {
  if (!s) return FBP_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;  // queued jobs still run; then the workers leave
  }
  s->work_cv.notify_all();
  for (auto& w : s->workers)
    if (w.thread.joinable()) w.thread.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->engine_stop = true;
  }
  s->engine_cv.notify_all();
  if (s->engine.joinable()) s->engine.join();
  for (auto& w : s->workers) {
    cudaFree(w.d_in);
    cudaFree(w.d_out);
    fbp_destroy(w.ctx);
  }
  for (int i = 0; i < 2; ++i) {
    fbp_destroy(s->launcher[i]);
    if (s->launched_ev[i]) cudaEventDestroy(s->launched_ev[i]);
    if (s->start_ev[i]) cudaEventDestroy(s->start_ev[i]);
  }
  for (cudaStream_t st : s->worker_streams) cudaStreamDestroy(st);
  for (auto& kv : s->jobs) delete kv.second;
  delete s;
  return FBP_OK;
}

}  // extern "C"
