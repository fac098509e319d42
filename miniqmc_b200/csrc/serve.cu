// serve.cu -- several walker batches advanced by shared launches (qmc_group),
// the launch-configuration autotuner (qmc_autotune) and the request loop
// that admits VMC jobs as they arrive (qmc_server).
//
// The fused sweep runs over a list of SweepTasks, each with its own system
// (spline table, lattice, Jastrows), electron count and walker state: in
// the work-queue form (the default) every resident CTA slot takes units of
// any task's walkers, in the static form one CTA per walker.  A group fills
// that list once with its batches, so one launch per MC step moves every
// walker of every system; the launch can be captured once as a CUDA graph
// (with the zeroing of its schedule words) and replayed per step.
// The server keeps a group of the running jobs and rebuilds the list only
// when a job starts or ends.
#include "host_api.hpp"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>

using namespace qmc;

namespace
{
// launch block size for a set of batches: the largest any of them asked for
int group_threads(const std::vector<qmc_walkers*>& b)
{
  int t = 64;
  for (auto* w : b)
    t = std::max(t, w->threads);
  return t;
}

struct TaskList
{
  SweepTask* d = nullptr;
  int cap = 0, n = 0, blocks = 0, threads = 64, max_npad = 0, max_k = 0;
  bool fp32 = true, tc = false, j3 = false, epoch = false;
  // the work-queue form (QMC_SCHED_AUTO / QUEUE; STATIC launches one CTA
  // per walker): per task its walkers, electrons and up electrons, the CTAs
  // of a launch, and the schedule words prepared for n_substeps
  int sched_mode = QMC_SCHED_AUTO, sched_unit = QMC_SCHED_UNIT_DEFAULT, sched_ctas = 0;
  std::vector<int> task_W, task_N, task_nup;
  int queue_ctas = 0, prepared_substeps = -1;
  size_t total_units = 0, n_words = 0, cap_sched = 0;
  int* sched = nullptr;

  ~TaskList()
  {
    cudaFree(d);
    cudaFree(sched);
  }

  // fill the device task list for `batches` (stream-ordered copy)
  int build(const std::vector<qmc_walkers*>& batches, int launch_threads, cudaStream_t st)
  {
    n = (int)batches.size();
    if (n > cap)
    {
      cudaStreamSynchronize(st);
      cudaFree(d);
      d = nullptr;
      CK(cudaMalloc(&d, (size_t)n * sizeof(SweepTask)));
      cap = n;
    }
    std::vector<SweepTask> h;
    blocks = 0, max_npad = 0, max_k = 0, tc = false, j3 = false, epoch = false;
    threads = launch_threads;
    task_W.clear();
    task_N.clear();
    task_nup.clear();
    double inflight = 0;
    for (auto* w : batches)
    {
      task_W.push_back(w->dw.W);
      task_N.push_back(w->dw.N);
      task_nup.push_back(w->sys->h.n_up);
      SweepTask t = sweep_task(w, blocks);
      t.tc        = (w->use_tc && threads >= 128) ? 1 : 0;
      tc          = tc || t.tc;
      blocks += w->dw.W;
      max_npad = std::max(max_npad, w->dw.npad);
      max_k    = std::max(max_k, w->dw.k);
      inflight += (double)w->dw.W * 16 * 4 * w->dw.npad * (w->fp32 ? 4 : 8);
      fp32 = w->fp32;
      j3   = j3 || (w->sys->h.comp & QMC_WF_J3) != 0;
      epoch = epoch || w->max_moves > 1;
      h.push_back(t);
    }
    // the next-move L2 prefetch only while all walkers' stencils fit well
    for (size_t i = 0; i < h.size(); ++i)
    {
      const int mode = batches[i]->prefetch_mode;
      h[i].prefetch  = mode == QMC_PREFETCH_ON || (mode == QMC_PREFETCH_AUTO && inflight <= 32.0e6);
    }
    if (n)
      CK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(SweepTask), cudaMemcpyHostToDevice, st));
    queue_ctas        = 0;
    prepared_substeps = -1;
    if (n && sched_mode != QMC_SCHED_STATIC)
    {
      int dev = 0, sms = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      const int per_sm = sweep_occupancy(fp32, threads, max_k, tc, j3, epoch, true);
      if (per_sm < 1)
        return fail(QMC_ERR_CUDA, "occupancy query failed");
      queue_ctas = sched_ctas > 0 ? sched_ctas : per_sm * sms;
    }
    return QMC_OK;
  }

  // the schedule words of a work-queue launch of n_substeps, allocated here
  // (outside any stream capture); *moved: the buffer changed, so a graph
  // that captured the old one must go
  int prepare(int n_substeps, cudaStream_t st, bool* moved)
  {
    *moved = false;
    if (!queue_ctas || prepared_substeps == n_substeps)
      return QMC_OK;
    size_t units = 0;
    for (size_t i = 0; i < task_W.size(); ++i)
      units += (size_t)task_W[i] * sweep_queue_units(task_N[i], task_nup[i], n_substeps, sched_unit);
    const size_t words = sweep_queue_words(blocks, queue_ctas, units);
    if (words > (size_t)INT32_MAX)
      return fail(QMC_ERR_ARG, "too many work-queue units in one launch: take longer units");
    if (cap_sched < words)
    {
      CK(cudaStreamSynchronize(st));
      cudaFree(sched);
      sched = nullptr;
      CK(cudaMalloc(&sched, words * sizeof(int)));
      cap_sched = words;
      *moved    = true;
    }
    total_units       = units;
    n_words           = words;
    prepared_substeps = n_substeps;
    return QMC_OK;
  }

  cudaError_t launch(int n_substeps, double accept, cudaStream_t st) const
  {
    if (!queue_ctas)
      return launch_sweep(fp32, d, n, blocks, n_substeps, accept, threads, max_npad, max_k, st, tc, j3, epoch);
    if (prepared_substeps != n_substeps)
      return cudaErrorInvalidValue; // prepare() first
    cudaError_t e = cudaMemsetAsync(sched, 0, n_words * sizeof(int), st);
    if (e != cudaSuccess)
      return e;
    const QueueLaunch q{d,          n,       blocks, (int)total_units, n_substeps, sched_unit,
                        queue_ctas, threads, accept, tc,               sched};
    return launch_sweep_queue(fp32, q, max_k, j3, epoch, st);
  }
};

// one MC step's bookkeeping of a batch swept by a shared launch: the
// periodic FP64 refresh of its inverses
int after_step(qmc_walkers* w, int recompute_every)
{
  ++w->steps_done;
  if (recompute_every > 0 && w->steps_done % recompute_every == 0 && (w->sys->h.comp & QMC_WF_DET))
  {
    int st = recompute_dets(w);
    if (st)
      return st;
    CK(launch_gl(w->fp32, w->sys->d, w->dw, w->threads, w->stream));
    w->launches++;
  }
  return QMC_OK;
}

double now_s()
{
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
} // namespace

// --------------------------------------------------------------- groups --
struct qmc_group_s
{
  std::vector<qmc_walkers*> batches;
  std::vector<cudaStream_t> saved;
  std::vector<bool> saved_own;
  cudaStream_t stream = nullptr;
  TaskList tasks;
  int threads      = 64;
  bool use_graph   = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_substeps   = -1;
  double graph_accept  = 0;
  bool launched        = false;
  int64_t launches     = 0;
  int64_t graph_launches = 0;

  void drop_graph()
  {
    if (exec)
      cudaGraphExecDestroy(exec);
    if (graph)
      cudaGraphDestroy(graph);
    exec  = nullptr;
    graph = nullptr;
  }
};

extern "C" {

int qmc_group_create(qmc_walkers* const* batches, int n_batches, qmc_group** out)
{
  if (!batches || !out || n_batches < 1)
    return fail(QMC_ERR_ARG, "a group needs at least one batch");
  for (int i = 0; i < n_batches; ++i)
  {
    if (!batches[i])
      return fail(QMC_ERR_ARG, "null batch");
    if (batches[i]->fp32 != batches[0]->fp32)
      return fail(QMC_ERR_ARG, "all batches of a group must have the same precision");
    for (int j = 0; j < i; ++j)
      if (batches[j] == batches[i])
        return fail(QMC_ERR_ARG, "a batch appears twice in the group");
  }
  auto* g = new qmc_group_s;
  g->batches.assign(batches, batches + n_batches);
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess)
  {
    delete g;
    return fail(QMC_ERR_CUDA, cudaGetErrorString(e));
  }
  // every batch works on the group's stream while the group exists
  for (auto* w : g->batches)
  {
    cudaStreamSynchronize(w->stream);
    g->saved.push_back(w->stream);
    g->saved_own.push_back(w->own_stream);
    w->stream     = g->stream;
    w->own_stream = false;
  }
  g->threads = group_threads(g->batches);
  int st     = g->tasks.build(g->batches, g->threads, g->stream);
  if (st)
  {
    qmc_group_destroy(g);
    return st;
  }
  *out = g;
  return QMC_OK;
}

int qmc_group_destroy(qmc_group* g)
{
  if (!g)
    return QMC_OK;
  cudaStreamSynchronize(g->stream);
  g->drop_graph();
  for (size_t i = 0; i < g->batches.size(); ++i)
  {
    g->batches[i]->stream     = g->saved[i];
    g->batches[i]->own_stream = g->saved_own[i];
  }
  cudaStreamDestroy(g->stream);
  delete g;
  return QMC_OK;
}

int qmc_group_set_threads(qmc_group* g, int threads)
{
  if (!g)
    return fail(QMC_ERR_ARG, "null handle");
  int kmax = 1;
  for (auto* w : g->batches)
    kmax = std::max(kmax, w->dw.k);
  if (threads % 32 || threads < std::max(std::max(64, 2 * kmax), group_threads(g->batches)) || threads > 256)
    return fail(QMC_ERR_ARG, "group threads must be a multiple of 32, at least every batch's own, at most 256");
  g->threads = threads;
  g->drop_graph();
  return g->tasks.build(g->batches, g->threads, g->stream);
}

int qmc_group_set_schedule(qmc_group* g, int mode, int unit_moves, int ctas)
{
  if (!g || mode < QMC_SCHED_AUTO || mode > QMC_SCHED_QUEUE || unit_moves < 0 || ctas < 0)
    return fail(QMC_ERR_ARG, "bad schedule");
  CK(cudaStreamSynchronize(g->stream));
  g->drop_graph();
  g->tasks.sched_mode = mode;
  g->tasks.sched_unit = unit_moves ? unit_moves : QMC_SCHED_UNIT_DEFAULT;
  g->tasks.sched_ctas = ctas;
  return g->tasks.build(g->batches, g->threads, g->stream);
}

int qmc_group_use_graph(qmc_group* g, int enable)
{
  if (!g)
    return fail(QMC_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(g->stream));
  g->use_graph = enable != 0;
  if (!g->use_graph)
    g->drop_graph();
  return QMC_OK;
}

int qmc_group_sweep(qmc_group* g, int n_steps, int n_substeps, double accept, int recompute_every)
{
  if (!g || n_steps < 0 || n_substeps < 1)
    return fail(QMC_ERR_ARG, "bad sweep options");
  for (int step = 0; step < n_steps; ++step)
  {
    bool moved = false;
    if (int st = g->tasks.prepare(n_substeps, g->stream, &moved))
      return st;
    if (moved)
      g->drop_graph();
    if (g->use_graph && g->launched)
    {
      if (!g->exec || g->graph_substeps != n_substeps || g->graph_accept != accept)
      {
        g->drop_graph();
        CK(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t le = g->tasks.launch(n_substeps, accept, g->stream);
        cudaError_t ce = cudaStreamEndCapture(g->stream, &g->graph);
        CK(le);
        CK(ce);
        CK(cudaGraphInstantiate(&g->exec, g->graph, 0));
        g->graph_substeps = n_substeps;
        g->graph_accept   = accept;
      }
      CK(cudaGraphLaunch(g->exec, g->stream));
      g->graph_launches++;
    }
    else
      CK(g->tasks.launch(n_substeps, accept, g->stream)); // first launch eager: sets the kernel attributes
    g->launched = true;
    g->launches++;
    for (auto* w : g->batches)
    {
      w->launches++;
      int st = after_step(w, recompute_every);
      if (st)
        return st;
    }
  }
  return QMC_OK;
}

int qmc_group_sync(qmc_group* g)
{
  if (!g)
    return fail(QMC_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(g->stream));
  for (auto* w : g->batches)
    if (int st = device_status(w))
      return st;
  return QMC_OK;
}

int qmc_group_stream(const qmc_group* g, void** stream)
{
  if (!g || !stream)
    return fail(QMC_ERR_ARG, "null pointer");
  *stream = g->stream;
  return QMC_OK;
}

int qmc_group_stats(const qmc_group* g, int* threads, int64_t* launches, int64_t* graph_launches)
{
  if (!g)
    return fail(QMC_ERR_ARG, "null handle");
  if (threads)
    *threads = g->threads;
  if (launches)
    *launches = g->launches;
  if (graph_launches)
    *graph_launches = g->graph_launches;
  return QMC_OK;
}

// ------------------------------------------------------------ autotuner --
int qmc_autotune(qmc_system* sys, int n_walkers, const int* delays, int n_delays, int n_steps,
                 qmc_tune_result* results, int max_results, int* n_results, qmc_tune_result* best)
{
  if (!sys || n_walkers < 1 || !delays || n_delays < 1 || n_steps < 1 || !best)
    return fail(QMC_ERR_ARG, "bad autotune arguments");
  std::vector<qmc_tune_result> all;
  std::vector<uint32_t> seeds(n_walkers);
  for (int i = 0; i < n_walkers; ++i)
    seeds[i] = 1009u + 7919u * (uint32_t)i;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int status = QMC_OK;
  for (int di = 0; di < n_delays && status == QMC_OK; ++di)
  {
    const int k = delays[di];
    qmc_walkers* w = nullptr;
    if (qmc_walkers_create(sys, n_walkers, k, &w) != QMC_OK)
      continue; // delay rank not valid for this system
    int def_threads = w->threads;
    std::vector<int> thread_opts = {def_threads};
    for (int t : {128, 192, 256})
      if (t > def_threads)
        thread_opts.push_back(t);
    if ((status = qmc_walkers_init_random(w, seeds.data())) || (status = qmc_wf_evaluate_log(w, nullptr)))
    {
      qmc_walkers_destroy(w);
      break;
    }
    for (int threads : thread_opts)
      for (int tc = 0; tc <= 1 && status == QMC_OK; ++tc)
        for (int moves : {1, EPOCH_MAX})
        {
          if (tc && !(w->tc_capable && threads >= 128))
            continue;
          w->use_tc = false;
          if (qmc_walkers_set_threads(w, threads) != QMC_OK)
            continue;
          w->use_tc    = tc != 0;
          w->max_moves = moves;
          if ((status = qmc_sweep_async(w, 1, 1, 0.5, 0)))
            break;
          CK(cudaEventRecord(e0, w->stream));
          if ((status = qmc_sweep_async(w, n_steps, 1, 0.5, 0)))
            break;
          CK(cudaEventRecord(e1, w->stream));
          CK(cudaEventSynchronize(e1));
          if ((status = device_status(w)))
            break;
          float ms = 0;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          all.push_back({k, threads, tc, moves, (double)ms / n_steps});
        }
    qmc_walkers_destroy(w);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status)
    return status;
  if (all.empty())
    return fail(QMC_ERR_ARG, "no candidate configuration was valid for this system");
  *best = *std::min_element(all.begin(), all.end(),
                            [](const qmc_tune_result& a, const qmc_tune_result& b) { return a.ms_per_step < b.ms_per_step; });
  if (n_results)
    *n_results = (int)all.size();
  if (results)
    for (int i = 0; i < (int)all.size() && i < max_results; ++i)
      results[i] = all[i];
  return QMC_OK;
}

} // extern "C"

// --------------------------------------------------------------- server --
namespace
{
// pinned host space a retiring job's results land in
struct ResultSlot
{
  int cap            = 0;
  long long* acc     = nullptr; // [cap]
  double* lp         = nullptr; // [cap]
  unsigned* status   = nullptr; // [1]
  cudaEvent_t done   = nullptr; // recorded after the copies
};

struct Job
{
  int64_t id;
  qmc_system* sys;
  int W, steps, delay;
  uint32_t seed;
  size_t bytes = 0;
  qmc_walkers* w = nullptr;
  int state      = QMC_JOB_WAITING;
  int steps_done = 0;
  double t_submit = 0, t_start = 0, t_done = 0;
  int64_t accepted = 0;
  double logpsi_mean = 0;
  int status = QMC_OK;
  ResultSlot slot;
};
} // namespace

struct qmc_server_s
{
  size_t budget = 0, used = 0;
  int threads = 128, recompute_every = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool  = nullptr; // every job's device memory, stream-ordered on `stream`
  double t0 = 0;
  int64_t next_id = 1;
  std::map<int64_t, Job> jobs;
  std::deque<int64_t> waiting;
  std::vector<int64_t> running;
  std::deque<int64_t> retiring; // swept to the end; results in flight to the host
  std::vector<ResultSlot> free_slots;
  TaskList tasks;
  bool dirty = true;
  int64_t launches = 0, moves = 0;
};

namespace
{
// admission: the batch's memory from the server's pool, its electrons and
// evaluateLog enqueued on the server stream; nothing waits for the device
// (an error of evaluateLog, e.g. a singular Slater matrix, lands in the
// job's own status word and fails the job when it retires)
int start_job(qmc_server_s* s, Job& j)
{
  int st = walkers_create_pooled(j.sys, j.W, j.delay, s->stream, s->pool, &j.w);
  if (st)
    return st;
  std::vector<uint32_t> seeds(j.W);
  for (int i = 0; i < j.W; ++i)
    seeds[i] = j.seed + 7919u * (uint32_t)i;
  if ((st = walkers_init_random(j.w, seeds.data(), false)))
    return st;
  if ((st = evaluate_log_launch(j.w)))
    return st;
  CK(cudaMemsetAsync(j.w->dw.accepted, 0, j.W * sizeof(long long), s->stream));
  return QMC_OK;
}

int get_slot(qmc_server_s* s, int W, ResultSlot& out)
{
  for (size_t i = 0; i < s->free_slots.size(); ++i)
    if (s->free_slots[i].cap >= W)
    {
      out = s->free_slots[i];
      s->free_slots.erase(s->free_slots.begin() + (long)i);
      return QMC_OK;
    }
  ResultSlot r;
  r.cap = std::max(W, 256);
  CK(cudaMallocHost(&r.acc, r.cap * sizeof(long long)));
  CK(cudaMallocHost(&r.lp, r.cap * sizeof(double)));
  CK(cudaMallocHost(&r.status, sizeof(unsigned)));
  CK(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming));
  out = r;
  return QMC_OK;
}

// the job has made its steps: its results and status word start towards
// pinned host memory behind its last launch; the job retires when they land
int begin_retire(qmc_server_s* s, Job& j)
{
  int st = get_slot(s, j.W, j.slot);
  if (st)
    return st;
  CK(cudaMemcpyAsync(j.slot.acc, j.w->dw.accepted, j.W * sizeof(long long), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(j.slot.lp, j.w->dw.logpsi, j.W * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(j.slot.status, j.w->dw.status, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaEventRecord(j.slot.done, s->stream));
  s->retiring.push_back(j.id);
  return QMC_OK;
}

// the job's walkers are gone (stream-ordered) and its memory is free for
// admission; status QMC_OK with a clean status word means done
void finish_job(qmc_server_s* s, Job& j, int status)
{
  if (j.w)
  {
    qmc_walkers_destroy(j.w); // pooled: cudaFreeAsync on the server stream
    j.w = nullptr;
  }
  s->used -= j.bytes;
  j.status = status;
  j.state  = status == QMC_OK ? QMC_JOB_DONE : QMC_JOB_FAILED;
  j.t_done = now_s() - s->t0;
  if (j.slot.done)
  {
    s->free_slots.push_back(j.slot);
    j.slot = ResultSlot();
  }
}

// retire every job whose results have landed (wait for the oldest if
// `block`); returns how many retired
int poll_retiring(qmc_server_s* s, bool block)
{
  int n = 0;
  while (!s->retiring.empty())
  {
    Job& j = s->jobs[s->retiring.front()];
    cudaError_t q = block && n == 0 ? cudaEventSynchronize(j.slot.done) : cudaEventQuery(j.slot.done);
    if (q == cudaErrorNotReady)
      break;
    s->retiring.pop_front();
    int status = q == cudaSuccess ? status_from_bits(*j.slot.status) : QMC_ERR_CUDA;
    if (status == QMC_OK)
    {
      j.accepted    = 0;
      j.logpsi_mean = 0;
      for (int i = 0; i < j.W; ++i)
      {
        j.accepted += j.slot.acc[i];
        j.logpsi_mean += j.slot.lp[i] / j.W;
      }
    }
    finish_job(s, j, status);
    ++n;
  }
  return n;
}
} // namespace

extern "C" {

int qmc_server_create(size_t memory_budget, int threads, int recompute_every, qmc_server** out)
{
  if (!out || memory_budget == 0 || threads % 32 || threads < 64 || threads > 256 || recompute_every < 0)
    return fail(QMC_ERR_ARG, "bad server arguments");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  auto* s            = new qmc_server_s;
  s->budget          = memory_budget;
  s->threads         = threads;
  s->recompute_every = recompute_every;
  s->t0              = now_s();
  cudaError_t e      = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  cudaMemPoolProps props{};
  props.allocType     = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id   = dev;
  if (e == cudaSuccess)
    e = cudaMemPoolCreate(&s->pool, &props);
  if (e == cudaSuccess)
  {
    // keep freed job memory in the pool for the next admissions
    uint64_t keep = ~0ull;
    e             = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (e != cudaSuccess)
  {
    if (s->stream)
      cudaStreamDestroy(s->stream);
    if (s->pool)
      cudaMemPoolDestroy(s->pool);
    delete s;
    return fail(QMC_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = s;
  return QMC_OK;
}

int qmc_server_destroy(qmc_server* s)
{
  if (!s)
    return QMC_OK;
  cudaStreamSynchronize(s->stream);
  for (auto& kv : s->jobs)
  {
    if (kv.second.w)
      qmc_walkers_destroy(kv.second.w);
    if (kv.second.slot.done)
      s->free_slots.push_back(kv.second.slot);
  }
  cudaStreamSynchronize(s->stream);
  for (auto& r : s->free_slots)
  {
    cudaFreeHost(r.acc);
    cudaFreeHost(r.lp);
    cudaFreeHost(r.status);
    cudaEventDestroy(r.done);
  }
  cudaMemPoolDestroy(s->pool);
  cudaStreamDestroy(s->stream);
  delete s;
  return QMC_OK;
}

int qmc_server_submit(qmc_server* s, qmc_system* sys, int n_walkers, int n_steps, int delay, uint32_t seed,
                      int64_t* job)
{
  if (!s || !sys || !job || n_walkers < 1 || n_steps < 1 || delay < 1 || delay > 64 || delay > sys->h.norb)
    return fail(QMC_ERR_ARG, "bad job");
  const int nvec = sys->h.npad / (sys->fp32 ? 4 : 2);
  const int need = std::min(256, std::max(std::max(64, 2 * delay), round_up(nvec, 32)));
  if (need > s->threads)
    return fail(QMC_ERR_ARG, "the job needs more threads per walker than the server launches with");
  Job j;
  j.id = s->next_id++, j.sys = sys, j.W = n_walkers, j.steps = n_steps, j.delay = delay, j.seed = seed;
  j.bytes = walkers_footprint(sys, n_walkers, delay);
  if (j.bytes > s->budget)
    return fail(QMC_ERR_ADMISSION, "the job's walker state is larger than the server's memory budget");
  j.t_submit = now_s() - s->t0;
  s->jobs[j.id] = j;
  s->waiting.push_back(j.id);
  *job = j.id;
  return QMC_OK;
}

int qmc_server_tick(qmc_server* s, int* n_running, int* n_waiting)
{
  if (!s)
    return fail(QMC_ERR_ARG, "null handle");
  // jobs whose results have landed free their memory first; with nothing
  // left to launch, wait for the oldest instead of spinning
  poll_retiring(s, s->running.empty() && !s->retiring.empty());
  // admit, in arrival order, every waiting job that fits the budget now
  for (auto it = s->waiting.begin(); it != s->waiting.end();)
  {
    Job& j = s->jobs[*it];
    if (s->used + j.bytes > s->budget)
    {
      ++it;
      continue;
    }
    s->used += j.bytes;
    j.state   = QMC_JOB_RUNNING;
    j.t_start = now_s() - s->t0;
    int st    = start_job(s, j);
    if (st)
      finish_job(s, j, st);
    else
    {
      s->running.push_back(j.id);
      s->dirty = true;
    }
    it = s->waiting.erase(it);
  }
  if (!s->running.empty())
  {
    if (s->dirty)
    {
      std::vector<qmc_walkers*> b;
      for (int64_t id : s->running)
        b.push_back(s->jobs[id].w);
      if (int st = s->tasks.build(b, s->threads, s->stream))
        return st;
      s->dirty = false;
    }
    // one shared launch moves every walker of every running job by one step
    bool moved = false;
    if (int st = s->tasks.prepare(1, s->stream, &moved))
      return st;
    CK(s->tasks.launch(1, 0.5, s->stream));
    s->launches++;
    std::vector<int64_t> still;
    for (int64_t id : s->running)
    {
      Job& j = s->jobs[id];
      j.w->launches++;
      s->moves += (int64_t)j.W * j.w->dw.N;
      int st = after_step(j.w, s->recompute_every);
      if (st)
      {
        finish_job(s, j, st);
        s->dirty = true;
        continue;
      }
      if (++j.steps_done == j.steps)
      {
        if ((st = begin_retire(s, j)))
          finish_job(s, j, st);
        s->dirty = true;
      }
      else
        still.push_back(id);
    }
    s->running.swap(still);
  }
  if (n_running)
    *n_running = (int)(s->running.size() + s->retiring.size());
  if (n_waiting)
    *n_waiting = (int)s->waiting.size();
  return QMC_OK;
}

int qmc_server_job(qmc_server* s, int64_t job, qmc_job_info* info)
{
  if (!s || !info)
    return fail(QMC_ERR_ARG, "null pointer");
  auto it = s->jobs.find(job);
  if (it == s->jobs.end())
    return fail(QMC_ERR_ARG, "unknown job");
  const Job& j     = it->second;
  info->state      = j.state;
  info->status     = j.status;
  info->steps_done = j.steps_done;
  info->n_accepted = j.accepted;
  info->logpsi_mean = j.logpsi_mean;
  info->t_submit   = j.t_submit;
  info->t_start    = j.t_start;
  info->t_done     = j.t_done;
  return QMC_OK;
}

int qmc_server_stats(const qmc_server* s, size_t* bytes_in_use, int64_t* launches, int64_t* electron_moves)
{
  if (!s)
    return fail(QMC_ERR_ARG, "null handle");
  if (bytes_in_use)
    *bytes_in_use = s->used;
  if (launches)
    *launches = s->launches;
  if (electron_moves)
    *electron_moves = s->moves;
  return QMC_OK;
}

} // extern "C"
