// serve.cu — continuous-batching commit engine.
//
// Jobs (a host trace to commit, optionally followed by the FRI commit phase on the
// alpha-reduced LDE) are submitted without blocking.  `slots` worker threads each
// own CUDA streams (one per job-size class, small jobs at the highest priority); a worker
// admits a queued job whose device-memory estimate fits what is left of the HBM budget
// (the oldest such job, or with ZKB_ADMIT_SMALLEST the one with the fewest cells, under a
// bound on how often a job is passed over), copies the trace
// in on its stream, keeps the LDE, the trees and the FRI layers device-resident until
// the job's answers are on the host, then releases the memory and wakes the queue.
// Jobs on different workers overlap on the GPU (one job's copy under another's
// kernels); each job's results depend only on its own inputs.
//
// The reference has a job-level concurrency scheduler for whole proofs
// (zkf-metal/src/batch_prover.rs:94-140) and a bounded in-flight command pipeline
// (zkf-metal/src/pipeline.rs:23-126); this engine is that role for commit jobs.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include "common.cuh"
#include "engine.cuh"

using namespace zkb;

namespace {

using Clock = std::chrono::steady_clock;

// ZKB_TRACE=1 prints the job lifecycle on stderr (admission, start, end, memory).
bool trace_on() {
  static const bool on = [] {
    const char *v = getenv("ZKB_TRACE");
    return v && *v && *v != '0';
  }();
  return on;
}
#define ENGINE_TRACE(...)                \
  do {                                   \
    if (trace_on()) {                    \
      fprintf(stderr, "[zkb engine] " __VA_ARGS__); \
      fflush(stderr);                    \
    }                                    \
  } while (0)

struct Job {
  uint64_t id = 0;
  zkb_job_desc desc{};
  HasherSpec spec;
  uint64_t mem_estimate = 0;
  Clock::time_point t_submit, t_start, t_done;
  JobStages stages;
  uint32_t bypassed = 0;  // times a younger job was admitted while this one waited
  int status = 1;  // 1 queued / running, 0 done, <0 error
  std::string error;
  uint32_t root[16] = {0};
  std::unique_ptr<zkb_fri_proof> fri;
};

// ZKB_JOB_LOG=<path>: one JSON line per finished job (shape, status, queue/run/latency ms,
// cells), appended, for per-job metrics next to the p50/p99 the caller computes.
Clock::time_point log_epoch() {
  static const Clock::time_point t0 = Clock::now();
  return t0;
}

void log_job(const Job &j, int rc, Clock::time_point done) {
  static const char *path = getenv("ZKB_JOB_LOG");
  if (!path || !*path) return;
  static std::mutex mu;
  using ms = std::chrono::duration<double, std::milli>;
  std::lock_guard<std::mutex> lk(mu);
  FILE *f = fopen(path, "a");
  if (!f) return;
  fprintf(f,
          "{\"job\": %llu, \"field\": %d, \"log_h\": %u, \"width\": %u, \"log_blowup\": %u, \"fri\": %d, "
          "\"status\": %d, \"cells\": %llu, \"queue_ms\": %.3f, \"run_ms\": %.3f, \"latency_ms\": %.3f, "
          "\"uploaded_ms\": %.3f, \"lock_ms\": %.3f, \"tree_ms\": %.3f, \"fri_alloc_ms\": %.3f, "
          "\"fri_enqueued_ms\": %.3f, \"fri_answers_ms\": %.3f, \"released_ms\": %.3f, \"start_ms\": %.3f}\n",
          (unsigned long long)j.id, j.desc.hasher.field, j.desc.log_h, j.desc.width, j.desc.log_blowup,
          j.desc.with_fri, rc, (unsigned long long)((1ull << j.desc.log_h) * j.desc.width),
          ms(j.t_start - j.t_submit).count(), ms(done - j.t_start).count(), ms(done - j.t_submit).count(),
          // stage ends, from the job's start
          ms(j.stages.uploaded - j.t_start).count(), ms(j.stages.lock_taken - j.t_start).count(),
          ms(j.stages.tree_built - j.t_start).count(), ms(j.stages.fri_alloc - j.t_start).count(),
          ms(j.stages.fri_enqueued - j.t_start).count(), ms(j.stages.fri_answers - j.t_start).count(),
          ms(j.stages.released - j.t_start).count(),
          // the job's start on the engine's clock (its first job's submission)
          ms(j.t_start - log_epoch()).count());
  fclose(f);
}

uint64_t job_bytes(const zkb_job_desc &d) {
  const uint64_t es = d.hasher.field == ZKB_FIELD_BABYBEAR ? 4 : 8;
  const uint64_t n = 1ull << d.log_h, N = n << d.log_blowup;
  uint64_t b = n * d.width * es        // staged trace (the inverse passes run in place on it)
               + N * d.width * es      // LDE
               + 2 * N * 64;           // digest layers (upper bound)
  // a trace uploaded in column slabs carries its rows' sponge states between slabs
  if (d.hasher.field == ZKB_FIELD_BABYBEAR && d.hasher.width == 16 && d.width >= 128 && d.log_h >= 1) b += N * 64;
  if (d.with_fri) b += N * 16 + N * 64;  // codeword + FRI layers and trees
  return b + (64ull << 20);
}

}  // namespace

struct zkb_engine {
  int device = 0;
  uint64_t budget = 0, in_use = 0;
  uint32_t policy = ZKB_ADMIT_FIFO;
  std::mutex mu;
  // one trace piece crosses PCIe at a time, the fewest bytes left first; an upload that 64
  // pieces of later (smaller) uploads have passed over (16 GiB) goes next
  UploadGate upload_mu{64};
  // One job of each size class runs its LDE and tree at a time: equal jobs pipeline one's
  // upload under another's kernels instead of interleaving their kernels block by block;
  // jobs of different classes still overlap, the smaller at the higher stream priority.
  std::mutex compute_mu[3];
  std::condition_variable cv_queue, cv_done;
  std::deque<std::shared_ptr<Job>> queue;
  std::map<uint64_t, std::shared_ptr<Job>> jobs;
  std::vector<std::thread> workers;
  uint64_t next_id = 1;
  bool stopping = false;
  uint64_t completed = 0, peak_in_use = 0;

  static uint64_t cells(const Job &j) { return ((uint64_t)j.desc.width) << j.desc.log_h; }

  // The queued job to admit now (queue.end(): none).  Called with mu held.
  std::deque<std::shared_ptr<Job>>::iterator pick() {
    auto fits = [&](const std::shared_ptr<Job> &j) { return in_use + j->mem_estimate <= budget; };
    if (policy != ZKB_ADMIT_SMALLEST) {
      // the oldest fitting job; a job that younger ones have passed ZKB_ADMIT_MAX_BYPASS
      // times is admitted next, and nothing passes it while it waits for memory
      for (auto it = queue.begin(); it != queue.end(); ++it) {
        if (fits(*it)) return it;
        if ((*it)->bypassed >= ZKB_ADMIT_MAX_BYPASS) return queue.end();
      }
      return queue.end();
    }
    auto best = queue.end();
    for (auto it = queue.begin(); it != queue.end(); ++it) {
      if ((*it)->bypassed >= ZKB_ADMIT_MAX_BYPASS) return fits(*it) ? it : queue.end();  // it goes next
      if (fits(*it) && (best == queue.end() || cells(**it) < cells(**best))) best = it;
    }
    return best;
  }

  // Stream priority by job size: small jobs' kernels are scheduled ahead of large jobs'
  // as blocks retire, so a small job does not wait behind a large job's whole kernel.
  static int size_class(const Job &j) {
    const uint64_t c = cells(j);
    return c < (1ull << 26) ? 0 : c < (1ull << 30) ? 1 : 2;
  }

  void worker_loop() {
    cudaSetDevice(device);
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    const int prio[3] = {greatest, (least + greatest) / 2, least};
    cudaStream_t streams[3] = {nullptr, nullptr, nullptr};
    for (int k = 0; k < 3; k++)
      if (cudaStreamCreateWithPriority(&streams[k], cudaStreamNonBlocking, prio[k]) != cudaSuccess) {
        for (int q = 0; q < k; q++) cudaStreamDestroy(streams[q]);
        return;
      }
    for (;;) {
      std::shared_ptr<Job> job;
      {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
          if (stopping && queue.empty()) break;
          auto it = pick();
          if (it != queue.end()) {
            job = *it;
            // every older job still queued was passed over once more
            for (auto o = queue.begin(); o != it; ++o) (*o)->bypassed++;
            queue.erase(it);
            in_use += job->mem_estimate;
            peak_in_use = in_use > peak_in_use ? in_use : peak_in_use;
            break;
          }
          cv_queue.wait(lk);
        }
      }
      if (!job) break;
      ENGINE_TRACE("start job %llu log_h=%u width=%u fri=%d est=%llu in_use=%llu\n",
                   (unsigned long long)job->id, job->desc.log_h, job->desc.width, job->desc.with_fri,
                   (unsigned long long)job->mem_estimate, (unsigned long long)in_use);
      job->t_start = Clock::now();
      std::unique_ptr<zkb_fri_proof> fri;
      if (job->desc.with_fri) fri = std::make_unique<zkb_fri_proof>();
      zkb_fri_params prm = job->desc.fri;
      cudaStream_t s = streams[size_class(*job)];
      int rc = pcs_job_run(job->spec, job->desc.trace, job->desc.log_h, job->desc.width,
                           job->desc.log_blowup, job->desc.alpha, job->desc.with_fri ? &prm : nullptr,
                           job->root, fri ? &fri->f : nullptr, s, &upload_mu,
                           &compute_mu[size_class(*job)], &job->stages, streams[0]);
      std::string err = rc == ZKB_OK ? "" : zkb_last_error_message();
      ENGINE_TRACE("end job %llu rc=%d %s\n", (unsigned long long)job->id, rc, err.c_str());
      log_job(*job, rc, Clock::now());
      {
        std::lock_guard<std::mutex> lk(mu);
        job->t_done = Clock::now();
        job->status = rc == ZKB_OK ? 0 : rc;
        job->error = err;
        job->fri = std::move(fri);
        in_use -= job->mem_estimate;
        completed++;
      }
      cv_queue.notify_all();
      cv_done.notify_all();
    }
    for (cudaStream_t q : streams) cudaStreamDestroy(q);
  }
};

extern "C" {

int zkb_engine_create(const zkb_engine_config *cfg, zkb_engine **out) {
  clear_error();
  ZKB_REQUIRE(cfg != nullptr && out != nullptr, "null arguments");
  ZKB_REQUIRE(cfg->slots >= 1 && cfg->slots <= 64, "slots must be in [1, 64]");
  ZKB_TRY(library_gate());
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    set_error("no CUDA device available");
    return ZKB_DECLINED;
  }
  auto e = std::make_unique<zkb_engine>();
  ZKB_CHECK_CUDA(cudaGetDevice(&e->device));
  size_t free_b = 0, total_b = 0;
  ZKB_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
  // memory this process's pool keeps after earlier jobs is free for the engine's jobs too
  uint64_t pool_idle = 0;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, e->device) == cudaSuccess) {
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
      pool_idle = reserved - used;
  }
  const uint64_t reserve = 2ull << 30;
  const uint64_t avail = free_b + pool_idle > reserve ? free_b + pool_idle - reserve : 0;
  e->budget = cfg->hbm_budget ? (cfg->hbm_budget < avail ? cfg->hbm_budget : avail) : avail;
  ZKB_REQUIRE(cfg->policy == ZKB_ADMIT_FIFO || cfg->policy == ZKB_ADMIT_SMALLEST, "unknown admission policy %u",
              cfg->policy);
  e->policy = cfg->policy;
  zkb_engine *raw = e.get();
  for (uint32_t i = 0; i < cfg->slots; i++) e->workers.emplace_back([raw] { raw->worker_loop(); });
  *out = e.release();
  return ZKB_OK;
}

int zkb_engine_submit(zkb_engine *e, const zkb_job_desc *desc, uint64_t *job_id) {
  clear_error();
  ZKB_REQUIRE(e != nullptr && desc != nullptr && job_id != nullptr, "null arguments");
  ZKB_TRY(library_gate());
  ZKB_REQUIRE(desc->trace != nullptr && desc->width > 0 && desc->log_h + desc->log_blowup < 31,
              "bad job shape");
  auto job = std::make_shared<Job>();
  job->desc = *desc;
  if (!make_hasher_spec(desc->hasher.field, (int)desc->hasher.width, desc->hasher.seed, &job->spec)) {
    set_error("unsupported hasher");
    return ZKB_ERR_UNSUPPORTED;
  }
  ZKB_REQUIRE(!desc->with_fri || desc->hasher.field == ZKB_FIELD_BABYBEAR,
              "the FRI job runs over the BabyBear quartic extension");
  job->mem_estimate = job_bytes(*desc);
  {
    std::lock_guard<std::mutex> lk(e->mu);
    ZKB_REQUIRE(job->mem_estimate <= e->budget,
                "job needs ~%llu bytes of device memory, more than the engine budget %llu",
                (unsigned long long)job->mem_estimate, (unsigned long long)e->budget);
    job->id = e->next_id++;
    job->t_submit = Clock::now();
    (void)log_epoch();  // the job log's clock starts at the first submission
    e->jobs[job->id] = job;
    e->queue.push_back(job);
  }
  e->cv_queue.notify_all();
  *job_id = job->id;
  return ZKB_OK;
}

int zkb_engine_wait(zkb_engine *e, uint64_t job_id, zkb_job_result *res, zkb_fri_proof **fri_out) {
  clear_error();
  ZKB_REQUIRE(e != nullptr && res != nullptr, "null arguments");
  std::shared_ptr<Job> job;
  {
    std::unique_lock<std::mutex> lk(e->mu);
    auto it = e->jobs.find(job_id);
    ZKB_REQUIRE(it != e->jobs.end(), "unknown job %llu", (unsigned long long)job_id);
    job = it->second;
    e->cv_done.wait(lk, [&] { return job->status != 1; });
    e->jobs.erase(job_id);
  }
  std::memset(res, 0, sizeof *res);
  res->status = job->status;
  std::memcpy(res->root, job->root, sizeof res->root);
  using ms = std::chrono::duration<double, std::milli>;
  res->queue_ms = ms(job->t_start - job->t_submit).count();
  res->run_ms = ms(job->t_done - job->t_start).count();
  res->latency_ms = ms(job->t_done - job->t_submit).count();
  if (fri_out) *fri_out = job->fri.release();
  if (job->status != 0) set_error("%s", job->error.c_str());
  return job->status == 0 ? ZKB_OK : job->status;
}

int zkb_engine_cancel(zkb_engine *e, uint64_t job_id) {
  clear_error();
  ZKB_REQUIRE(e != nullptr, "null engine");
  {
    std::lock_guard<std::mutex> lk(e->mu);
    auto it = e->jobs.find(job_id);
    ZKB_REQUIRE(it != e->jobs.end(), "unknown job %llu", (unsigned long long)job_id);
    std::shared_ptr<Job> job = it->second;
    auto q = std::find(e->queue.begin(), e->queue.end(), job);
    if (q == e->queue.end()) {
      set_error("job %llu has already started or finished", (unsigned long long)job_id);
      return ZKB_DECLINED;
    }
    e->queue.erase(q);
    job->t_start = job->t_done = Clock::now();
    job->status = ZKB_ERR_CANCELLED;
    job->error = "cancelled before it started";
  }
  e->cv_done.notify_all();
  e->cv_queue.notify_all();
  return ZKB_OK;
}

int zkb_engine_stats(zkb_engine *e, zkb_engine_stats_t *st) {
  clear_error();
  ZKB_REQUIRE(e != nullptr && st != nullptr, "null arguments");
  std::lock_guard<std::mutex> lk(e->mu);
  st->queued = e->queue.size();
  st->completed = e->completed;
  st->hbm_budget = e->budget;
  st->hbm_in_use = e->in_use;
  st->hbm_peak = e->peak_in_use;
  return ZKB_OK;
}

void zkb_engine_destroy(zkb_engine *e) {
  if (!e) return;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    e->stopping = true;
  }
  e->cv_queue.notify_all();
  for (auto &t : e->workers) t.join();
  delete e;
}

}  // extern "C"
