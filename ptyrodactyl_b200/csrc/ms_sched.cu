// Multi-job scheduler: continuous batching of multislice forward and gradient jobs.
//
// Jobs (simulations or gradient solves of any grid edge, slice count and scan
// size) are submitted at any time. A job is admitted when its scratch fits in the
// scheduler's arena (caller-provided device memory; nothing is allocated per job)
// and its probes-in-flight fit in the slot budget. Every tick advances each running
// job by one pass: the passes of all running jobs with the same grid edge go out
// as ONE multi-job launch per (forward/adjoint, axis), each CTA row reading its own
// job's arguments, so jobs that arrive while others run share the same kernels and
// fill the GPU together. Grid edges have their own streams and overlap. A job
// leaves when its last pass has completed; its memory returns to the arena.
//
// Gradient jobs: per probe batch, the forward with checkpoint residuals, a fused
// amplitude-loss kernel (L = sum (sqrt(I + eps) - sqrt(target))^2, dL/dI), then the
// adjoint passes with deterministic dV reductions; finally the probe gradient.
#include <algorithm>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "engine.cuh"

namespace ptyro {

constexpr float kLossEps = 1e-12f;

// amplitude loss of one pattern per CTA (256 threads), fixed-order tree reduction
static __global__ void __launch_bounds__(256) k_amp_loss(const float* __restrict__ I, const float* __restrict__ target,
                                                         int nn, float eps, float* __restrict__ g,
                                                         float* __restrict__ partial) {
  const size_t base = (size_t)blockIdx.x * nn;
  float acc = 0.f;
  for (int i = threadIdx.x; i < nn; i += blockDim.x) {
    const float a = sqrtf(I[base + i] + eps);
    const float d = a - sqrtf(fmaxf(target[base + i], 0.f));
    acc = fmaf(d, d, acc);
    g[base + i] = d / a;
  }
  __shared__ float red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

static __global__ void __launch_bounds__(256) k_sum_partials(const float* __restrict__ partial, int count, float* out) {
  float acc = 0.f;
  for (int i = threadIdx.x; i < count; i += blockDim.x) acc += partial[i];
  __shared__ float red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

static int launch_pass_multi(int n, int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st, int var) {
  if (nr <= 0) return PTYRO_OK;
  int rc;
  switch (n) {
    case 16: rc = launch_pass_multi_16(axis, d, r, nr, st, var); break;
    case 32: rc = launch_pass_multi_32(axis, d, r, nr, st, var); break;
    case 64: rc = launch_pass_multi_64(axis, d, r, nr, st, var); break;
    case 128: rc = launch_pass_multi_128(axis, d, r, nr, st, var); break;
    case 256: rc = launch_pass_multi_256(axis, d, r, nr, st, var); break;
    case 512: rc = launch_pass_multi_512(axis, d, r, nr, st, var); break;
    case 1024: rc = launch_pass_multi_1024(axis, d, r, nr, st, var); break;
    default: return fail(PTYRO_ERR_UNSUPPORTED, "grid edge not compiled");
  }
  return rc ? fail(PTYRO_ERR_CUDA, std::string("ms_pass_multi_kernel: ") + cudaGetErrorString((cudaError_t)rc)) : 0;
}

// paired steady passes of several jobs (grid edges up to 512)
static int launch_pass_pair_multi(int n, int axis, const PassArgs* d, const int2* r, int nr, cudaStream_t st) {
  if (nr <= 0) return PTYRO_OK;
  int rc;
  switch (n) {
    case 16: rc = launch_pass_pair_multi_16(axis, d, r, nr, st); break;
    case 32: rc = launch_pass_pair_multi_32(axis, d, r, nr, st); break;
    case 64: rc = launch_pass_pair_multi_64(axis, d, r, nr, st); break;
    case 128: rc = launch_pass_pair_multi_128(axis, d, r, nr, st); break;
    case 256: rc = launch_pass_pair_multi_256(axis, d, r, nr, st); break;
    case 512: rc = launch_pass_pair_multi_512(axis, d, r, nr, st); break;
    default: return fail(PTYRO_ERR_UNSUPPORTED, "paired multi-job pass: grid edge not served");
  }
  if (rc != 0) return fail(PTYRO_ERR_CUDA, std::string("ms_pass_pair_multi_kernel: ") + cudaGetErrorString((cudaError_t)rc));
  return PTYRO_OK;
}

static int launch_bwd_multi(int n, int axis, const BwdArgs* d, const int2* r, int nr, cudaStream_t st) {
  if (nr <= 0) return PTYRO_OK;
  int rc;
  switch (n) {
    case 16: rc = launch_bwd_multi_16(axis, d, r, nr, st); break;
    case 32: rc = launch_bwd_multi_32(axis, d, r, nr, st); break;
    case 64: rc = launch_bwd_multi_64(axis, d, r, nr, st); break;
    case 128: rc = launch_bwd_multi_128(axis, d, r, nr, st); break;
    case 256: rc = launch_bwd_multi_256(axis, d, r, nr, st); break;
    case 512: rc = launch_bwd_multi_512(axis, d, r, nr, st); break;
    case 1024: rc = launch_bwd_multi_1024(axis, d, r, nr, st); break;
    default: return fail(PTYRO_ERR_UNSUPPORTED, "grid edge not compiled");
  }
  return rc ? fail(PTYRO_ERR_CUDA, std::string("ms_bwd_multi_kernel: ") + cudaGetErrorString((cudaError_t)rc)) : 0;
}

// ---------------------------------------------------------------- arena
class Arena {
 public:
  void init(char* base, size_t bytes) {
    base_ = base;
    free_.clear();
    if (bytes) free_[0] = bytes;
  }
  // first fit, 256-byte granules; returns false when nothing fits
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 255) & ~(size_t)255;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes, start = it->first + bytes;
        free_.erase(it);
        if (rest) free_[start] = rest;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
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
  size_t free_bytes() const {
    size_t s = 0;
    for (auto& kv : free_) s += kv.second;
    return s;
  }
  char* base() const { return base_; }

 private:
  char* base_ = nullptr;
  std::map<size_t, size_t> free_;  // offset -> size
};

// ---------------------------------------------------------------- jobs
struct JobPlan {
  ptyro_ms_params p;  // batch resolved
  int grad = 0, K = 1, C = 0;
  Layout L;
  size_t off_fwd = 0, off_res = 0, off_g = 0, off_lam = 0, off_contrib = 0, off_beam = 0, off_lossp = 0;
  size_t bytes = 0;
};

static int plan_job(const ptyro_job_desc* d, JobPlan* jp) {
  if (!d) return fail(PTYRO_ERR_INVALID, "job descriptor is NULL");
  int rc = validate(&d->p);
  if (rc) return rc;
  if (d->kind != PTYRO_JOB_FORWARD && d->kind != PTYRO_JOB_GRADIENT)
    return fail(PTYRO_ERR_INVALID, "job kind must be PTYRO_JOB_FORWARD or PTYRO_JOB_GRADIENT");
  if (!d->potential || !d->modes || !d->weights || !d->positions || !d->patterns)
    return fail(PTYRO_ERR_INVALID, "NULL array argument");
  if (d->kind == PTYRO_JOB_GRADIENT && (!d->targets || !d->grad_potential || !d->grad_modes || !d->loss))
    return fail(PTYRO_ERR_INVALID, "gradient jobs need targets, grad_potential, grad_modes and loss");
  JobPlan& j = *jp;
  j.p = d->p;
  if (j.p.batch <= 0) {
    // probes in flight: a 32 MiB batch of wave slots, so several jobs share the GPU
    const double slot = 8.0 * j.p.n * (double)j.p.n * j.p.num_modes;
    j.p.batch = (int)std::max(1.0, std::min((double)std::max(j.p.num_probes, 1), 32.0 * 1024 * 1024 / slot));
  }
  j.grad = d->kind == PTYRO_JOB_GRADIENT;
  j.L = layout_for(&j.p);
  const size_t nn = (size_t)j.p.n * j.p.n;
  const size_t slots = (size_t)j.L.batch * j.p.num_modes;
  size_t o = 0;
  j.off_fwd = o; o = align_up(o + j.L.total);
  if (j.grad) {
    j.K = d->ckpt_every > 0 ? d->ckpt_every : std::max(1, (int)ceil(sqrt((double)j.p.num_slices)));
    j.C = (j.p.num_slices + j.K - 1) / j.K;
    j.off_res = o; o = align_up(o + 8 * nn * (size_t)(j.C + 1) * slots);
    j.off_g = o; o = align_up(o + 4 * nn * (size_t)j.L.batch);
    j.off_lam = o; o = align_up(o + 8 * nn * slots);
    j.off_contrib = o; o = align_up(o + 4 * nn * slots);
    j.off_beam = o; o = align_up(o + 8 * nn * j.p.num_modes);
    j.off_lossp = o; o = align_up(o + 4 * (size_t)std::max(j.p.num_probes, 1));
  }
  j.bytes = o;
  return PTYRO_OK;
}

struct Job {
  int64_t id = 0;
  ptyro_job_desc d;
  JobPlan plan;
  size_t arena_off = 0;
  char* base = nullptr;
  int state = PTYRO_JOB_QUEUED;
  int phase = 0;  // 0: forward passes of the batch, 1: adjoint passes of the batch
  int b0 = 0, nb = 0, k = 0;
  bool issued_all = false;
  cudaEvent_t done = nullptr;
  int rows_reserved = 0;
};

struct GridClass {
  int n = 0;
  cudaStream_t stream = nullptr;
  // staging ring for the per-tick descriptors and row tables
  static constexpr int kRing = 4;
  char* dev[kRing] = {};
  char* host[kRing] = {};
  cudaEvent_t used[kRing] = {};
  int next = 0;
};

}  // namespace ptyro

using namespace ptyro;

struct ptyro_sched {
  int device = 0;
  Arena arena;
  size_t arena_bytes = 0;
  int max_slots = 0;
  int active_slots = 0;
  size_t stage_bytes = 0;
  std::mutex mu;                 // guards jobs and queue
  int64_t next_id = 1;
  std::map<int64_t, std::unique_ptr<Job>> jobs;
  std::deque<int64_t> queue;     // submitted, not admitted, in arrival order
  std::vector<int64_t> running;  // admitted, not yet released
  std::map<int, GridClass> classes;
};

namespace ptyro {

static int class_for(ptyro_sched* s, int n, GridClass** out) {
  auto it = s->classes.find(n);
  if (it == s->classes.end()) {
    GridClass c;
    c.n = n;
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail(PTYRO_ERR_CUDA, "cudaStreamCreateWithFlags failed");
    for (int i = 0; i < GridClass::kRing; ++i) {
      size_t off;
      if (!s->arena.alloc(s->stage_bytes, &off))
        return fail(PTYRO_ERR_WORKSPACE, "arena too small for the scheduler's staging buffers");
      c.dev[i] = s->arena.base() + off;
      if (cudaHostAlloc((void**)&c.host[i], s->stage_bytes, cudaHostAllocDefault) != cudaSuccess)
        return fail(PTYRO_ERR_CUDA, "cudaHostAlloc failed");
      cudaEventCreateWithFlags(&c.used[i], cudaEventDisableTiming);
    }
    it = s->classes.emplace(n, c).first;
  }
  *out = &it->second;
  return PTYRO_OK;
}

static FwdBuffers job_fwd_buffers(Job& j) { return fwd_buffers(j.plan.L, j.base + j.plan.off_fwd); }

static BwdBuffers job_bwd_buffers(Job& j) {
  const FwdBuffers f = job_fwd_buffers(j);
  BwdBuffers b;
  b.psi = f.waves;  // the forward wave slots are free while the batch runs backwards
  b.lam = (float2*)(j.base + j.plan.off_lam);
  b.contrib = (float*)(j.base + j.plan.off_contrib);
  b.trans = f.trans;
  b.trans_t = f.trans_t;
  b.pf = f.pf;
  b.tw = f.tw;
  b.ramp_y = f.ramp_y;
  b.ramp_x = f.ramp_x;
  return b;
}

// the job's status word cleared, its tables and probe spectra built, gradient sums zeroed
static int job_setup(Job& j, cudaStream_t st) {
  const ptyro_ms_params* p = &j.plan.p;
  int rc;
  if ((rc = clear_status(j.base + j.plan.off_fwd + j.plan.L.status, st))) return rc;
  if ((rc = forward_setup(p, j.plan.L, j.base + j.plan.off_fwd, j.d.potential, j.d.modes, st))) return rc;
  if (j.plan.grad) {
    const int F = field_of(p);
    const size_t nn = (size_t)p->n * p->n;
    k_zero_pot<<<blocks_for((size_t)F * F * p->num_slices, 256), 256, 0, st>>>(
        j.d.grad_potential, p->pot_stride_y, p->pot_stride_x, p->pot_stride_s, F, p->num_slices);
    k_zero2<<<blocks_for(nn * p->num_modes, 256), 256, 0, st>>>((float2*)(j.base + j.plan.off_beam),
                                                                 nn * p->num_modes);
    if ((rc = check_launch("gradient job setup", 2))) return rc;
  }
  return PTYRO_OK;
}

// the pass counters of a job that starts
static void job_start(Job& j) {
  j.state = PTYRO_JOB_RUNNING;
  j.phase = 0;
  j.b0 = 0;
  j.nb = std::min(j.plan.L.batch, j.plan.p.num_probes);
  j.k = 0;
  if (j.plan.p.num_probes == 0) j.issued_all = true;
}

static int admit(ptyro_sched* s, Job& j, GridClass& c) {
  (void)s;
  int rc;
  if (j.d.ready_event && cudaStreamWaitEvent(c.stream, (cudaEvent_t)j.d.ready_event, 0) != cudaSuccess)
    return fail(PTYRO_ERR_CUDA, "cudaStreamWaitEvent on the job's ready event failed");
  if ((rc = job_setup(j, c.stream))) return rc;
  job_start(j);
  return PTYRO_OK;
}

// the last kernels of a job (gradient jobs: the probe gradient and the loss)
static int job_epilogue(Job& j, cudaStream_t st) {
  const ptyro_ms_params* p = &j.plan.p;
  int rc = PTYRO_OK;
  if (j.plan.grad && p->num_probes > 0) {
    const FwdBuffers f = job_fwd_buffers(j);
    const int n = p->n, M = p->num_modes;
    const size_t nn = (size_t)n * n;
    float2* beam = (float2*)(j.base + j.plan.off_beam);
    if ((rc = fft2_planes(n, M, true, beam, f.tw, st))) return rc;
    k_write_grad_modes<<<(unsigned)((nn * M + 255) / 256), 256, 0, st>>>(
        beam, n, M, (float2*)j.d.grad_modes, p->mode_stride_y, p->mode_stride_x, p->mode_stride_m);
    k_sum_partials<<<1, 256, 0, st>>>((const float*)(j.base + j.plan.off_lossp), p->num_probes, j.d.loss);
    if ((rc = check_launch("gradient job epilogue", 2))) return rc;
  }
  return PTYRO_OK;
}

// the epilogue, then the job's completion event
static int finish_job(Job& j, GridClass& c) {
  int rc = job_epilogue(j, c.stream);
  if (rc) return rc;
  if (cudaEventCreateWithFlags(&j.done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventRecord(j.done, c.stream) != cudaSuccess)
    return fail(PTYRO_ERR_CUDA, "cudaEventRecord failed");
  j.issued_all = true;
  return PTYRO_OK;
}

struct TickRows {
  std::vector<PassArgs> fdesc;
  std::vector<BwdArgs> bdesc;
  // forward axis 0, forward axis 1, adjoint axis 0, adjoint axis 1, paired steady
  // forward axis 0, paired steady forward axis 1
  std::vector<int2> rows[6];
};

// the per-job kernels that follow a tick's multi-job launches
struct Follow {
  Job* j;
  int b0, nb, slice;
  bool loss, beam;
};

struct RampReq {
  Job* j;
  int b0, nb;
};

// One pass of every job in `jobs`: the descriptors and CTA rows of the multi-job
// launches, the probe batches whose shift ramps must be built first, and the
// follow-up kernels.
static void build_tick(std::vector<Job*>& jobs, TickRows& t, std::vector<RampReq>& ramps,
                       std::vector<Follow>& follow) {
  for (Job* j : jobs) {
    const ptyro_ms_params* p = &j->plan.p;
    const int S = p->num_slices;
    if (j->k == 0 && j->phase == 0) ramps.push_back({j, j->b0, j->nb});
    Follow fl{j, j->b0, j->nb, -1, false, false};
    if (j->phase == 0) {
      float2* res = j->plan.grad ? (float2*)(j->base + j->plan.off_res) : nullptr;
      const FwdPlan f = fwd_pass_plan(p, job_fwd_buffers(*j), j->d.weights, j->d.patterns, res, j->plan.K,
                                      j->plan.grad ? j->plan.C : 0, j->b0, j->nb, j->k);
      const int di = (int)t.fdesc.size();
      t.fdesc.push_back(f.a);
      // steady passes of grids up to 512 run in paired arithmetic (two lines per thread
      // up to 256, the two halves of each line at 512)
      const int table = (p->n <= 512 && is_steady_pass(f.a)) ? 4 + f.axis : f.axis;
      for (int r = 0; r < f.rows; ++r) t.rows[table].push_back(make_int2(di, r));
      if (j->plan.grad && j->k == S + 1) fl.loss = true;
    } else {
      const BwdBuffers b = job_bwd_buffers(*j);
      const BwdPlan pl = bwd_pass_plan(p, b, j->d.weights, (const float2*)(j->base + j->plan.off_res),
                                       (const float*)(j->base + j->plan.off_g), j->plan.K, j->plan.C, j->b0, j->nb,
                                       j->k);
      const int di = (int)t.bdesc.size();
      t.bdesc.push_back(pl.a);
      for (int r = 0; r < pl.rows; ++r) t.rows[2 + pl.axis].push_back(make_int2(di, r));
      fl.slice = pl.slice;
      fl.beam = j->k == S + 1;
    }
    follow.push_back(fl);
  }
}

static int launch_ramps(const RampReq& r, cudaStream_t st) {
  const ptyro_ms_params* p = &r.j->plan.p;
  const FwdBuffers f = job_fwd_buffers(*r.j);
  k_ramps<<<(r.nb * p->n + 255) / 256, 256, 0, st>>>(r.j->d.positions + 2 * (size_t)r.b0, r.nb, p->n,
                                                      p->shift_calib_ang, (float2*)f.ramp_y, (float2*)f.ramp_x);
  return check_launch("k_ramps");
}

// bytes of one tick's descriptors and row tables as laid out by pack_tick
static size_t tick_bytes(const TickRows& t) {
  size_t bytes = align_up(t.fdesc.size() * sizeof(PassArgs)) + align_up(t.bdesc.size() * sizeof(BwdArgs));
  for (int i = 0; i < 6; ++i) bytes += align_up(t.rows[i].size() * sizeof(int2));
  return bytes;
}

// the device addresses a tick's launches read, for a packed copy at `dptr`
struct TickPtrs {
  const PassArgs* fd;
  const BwdArgs* bd;
  const int2* rows[6];
  int nrows[6];
};

static TickPtrs pack_tick(const TickRows& t, char* h, char* dptr) {
  TickPtrs q;
  size_t o = 0;
  q.fd = (const PassArgs*)(dptr + o);
  if (h) memcpy(h + o, t.fdesc.data(), t.fdesc.size() * sizeof(PassArgs));
  o += align_up(t.fdesc.size() * sizeof(PassArgs));
  q.bd = (const BwdArgs*)(dptr + o);
  if (h) memcpy(h + o, t.bdesc.data(), t.bdesc.size() * sizeof(BwdArgs));
  o += align_up(t.bdesc.size() * sizeof(BwdArgs));
  for (int i = 0; i < 6; ++i) {
    q.rows[i] = (const int2*)(dptr + o);
    q.nrows[i] = (int)t.rows[i].size();
    if (h) memcpy(h + o, t.rows[i].data(), t.rows[i].size() * sizeof(int2));
    o += align_up(t.rows[i].size() * sizeof(int2));
  }
  return q;
}

static int launch_tick(int n, const TickPtrs& q, cudaStream_t st) {
  const int tune = 3;
  int rc;
  if ((rc = launch_pass_multi(n, 0, q.fd, q.rows[0], q.nrows[0], st, tune))) return rc;
  if ((rc = launch_pass_multi(n, 1, q.fd, q.rows[1], q.nrows[1], st, tune))) return rc;
  if ((rc = launch_pass_pair_multi(n, 0, q.fd, q.rows[4], q.nrows[4], st))) return rc;
  if ((rc = launch_pass_pair_multi(n, 1, q.fd, q.rows[5], q.nrows[5], st))) return rc;
  if ((rc = launch_bwd_multi(n, 0, q.bd, q.rows[2], q.nrows[2], st))) return rc;
  return launch_bwd_multi(n, 1, q.bd, q.rows[3], q.nrows[3], st);
}

static int launch_follow(const Follow& fl, cudaStream_t st) {
  Job& j = *fl.j;
  const ptyro_ms_params* p = &j.plan.p;
  const int n = p->n, M = p->num_modes;
  const size_t nn = (size_t)n * n;
  int rc;
  if (fl.loss) {
    k_amp_loss<<<fl.nb, 256, 0, st>>>(j.d.patterns + (size_t)fl.b0 * nn, j.d.targets + (size_t)fl.b0 * nn, (int)nn,
                                       kLossEps, (float*)(j.base + j.plan.off_g),
                                       (float*)(j.base + j.plan.off_lossp) + fl.b0);
    if ((rc = check_launch("k_amp_loss"))) return rc;
  }
  if (fl.slice >= 0 &&
      (rc = launch_reduce_dv_any(p, (const float*)(j.base + j.plan.off_contrib), fl.nb, fl.b0, j.d.grad_potential,
                                 fl.slice, st)))
    return rc;
  if (fl.beam) {
    k_reduce_beam<<<(unsigned)((nn * M + 255) / 256), 256, 0, st>>>((const float2*)(j.base + j.plan.off_lam), fl.nb,
                                                                     M, n, (float2*)(j.base + j.plan.off_beam));
    if ((rc = check_launch("k_reduce_beam"))) return rc;
  }
  return PTYRO_OK;
}

// past one pass: returns true when the job has issued its last pass
static bool job_advance(Job& j) {
  const ptyro_ms_params* p = &j.plan.p;
  if (++j.k <= p->num_slices + 1) return false;
  j.k = 0;
  if (j.phase == 0 && j.plan.grad) {
    j.phase = 1;
    return false;
  }
  j.phase = 0;
  j.b0 += j.nb;
  if (j.b0 >= p->num_probes) return true;
  j.nb = std::min(j.plan.L.batch, p->num_probes - j.b0);
  return false;
}

// one pass of every running job of grid class c
static int tick_class(ptyro_sched* s, GridClass& c, std::vector<Job*>& jobs) {
  TickRows t;
  std::vector<RampReq> ramps;
  std::vector<Follow> follow;
  int rc;
  build_tick(jobs, t, ramps, follow);
  for (const RampReq& r : ramps)
    if ((rc = launch_ramps(r, c.stream))) return rc;
  // upload descriptors and rows through the staging ring
  const size_t bytes = tick_bytes(t);
  if (bytes > s->stage_bytes) return fail(PTYRO_ERR_INVALID, "tick descriptors exceed the staging buffer");
  const int slot = c.next;
  c.next = (c.next + 1) % GridClass::kRing;
  cudaEventSynchronize(c.used[slot]);  // the copy that last used this slot has finished
  const TickPtrs q = pack_tick(t, c.host[slot], c.dev[slot]);
  if (cudaMemcpyAsync(c.dev[slot], c.host[slot], bytes, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
    return fail(PTYRO_ERR_CUDA, "descriptor upload failed");
  cudaEventRecord(c.used[slot], c.stream);
  if ((rc = launch_tick(c.n, q, c.stream))) return rc;
  for (const Follow& fl : follow) {
    if ((rc = launch_follow(fl, c.stream))) return rc;
    if (job_advance(*fl.j) && (rc = finish_job(*fl.j, c))) return rc;
  }
  return PTYRO_OK;
}

// ---------------------------------------------------------------- recorded batch plans
// A fixed set of jobs (any mix of grid edges, slice counts, scan sizes, forward and
// gradient) as one recorded sequence of launches: the scheduler's lockstep ticks are
// simulated once on the host and every tick's descriptors and row tables are copied
// once into the plan's arena, so launching the plan only enqueues kernels and memsets
// on the caller's stream (no host synchronisation, copies or events) and can be
// captured in a CUDA graph and replayed.
struct PlanOp {
  enum Kind { SETUP, RAMPS, TICK, FOLLOW, EPILOGUE } kind;
  int cls = 0;   // grid class: the op goes on that class's stream
  int job = -1;  // SETUP, EPILOGUE
  RampReq ramp{};
  Follow follow{};
  int n = 0;  // TICK: grid edge
  TickPtrs q{};
};

struct PlanJobs {
  std::vector<Job> jobs;  // reserved up front: ops hold pointers into it
  std::vector<PlanOp> ops;
  std::vector<char> blob;  // the packed ticks
  std::vector<int> class_edges;  // grid edge of each class, ascending
  size_t job_bytes = 0;
};

static int plan_record(const ptyro_job_desc* descs, int num_jobs, char* arena, PlanJobs& pj) {
  if (num_jobs < 1 || !descs) return fail(PTYRO_ERR_INVALID, "a plan needs at least one job");
  pj.jobs.clear();
  pj.jobs.reserve((size_t)num_jobs);
  pj.ops.clear();
  pj.blob.clear();
  size_t o = 0;
  for (int i = 0; i < num_jobs; ++i) {
    pj.jobs.emplace_back();
    Job& j = pj.jobs.back();
    int rc = plan_job(&descs[i], &j.plan);
    if (rc) return rc;
    if (descs[i].ready_event)
      return fail(PTYRO_ERR_INVALID, "plan jobs take no ready events: order their inputs on the launch stream");
    j.d = descs[i];
    j.id = i;
    j.arena_off = o;
    j.base = arena ? arena + o : nullptr;
    o = align_up(o + j.plan.bytes);
  }
  pj.job_bytes = o;
  char* desc_base = arena ? arena + o : nullptr;
  std::map<int, int> cls_of;  // grid edge -> class index
  for (Job& j : pj.jobs) cls_of.emplace(j.plan.p.n, 0);
  for (auto& kv : cls_of) {
    kv.second = (int)pj.class_edges.size();
    pj.class_edges.push_back(kv.first);
  }
  std::map<int, std::vector<Job*>> classes;
  for (Job& j : pj.jobs) {
    PlanOp op;
    op.kind = PlanOp::SETUP;
    op.cls = cls_of[j.plan.p.n];
    op.job = (int)j.id;
    pj.ops.push_back(op);
    job_start(j);
    if (!j.issued_all) classes[j.plan.p.n].push_back(&j);
  }
  for (auto& kv : classes) {
    const int cls = cls_of[kv.first];
    for (;;) {
      std::vector<Job*> running;
      for (Job* j : kv.second)
        if (!j->issued_all) running.push_back(j);
      if (running.empty()) break;
      TickRows t;
      std::vector<RampReq> ramps;
      std::vector<Follow> follow;
      build_tick(running, t, ramps, follow);
      for (const RampReq& r : ramps) {
        PlanOp op;
        op.kind = PlanOp::RAMPS;
        op.cls = cls;
        op.ramp = r;
        pj.ops.push_back(op);
      }
      const size_t off = pj.blob.size();  // a multiple of 256: every packed piece is
      pj.blob.resize(off + tick_bytes(t));
      PlanOp tick;
      tick.kind = PlanOp::TICK;
      tick.cls = cls;
      tick.n = kv.first;
      tick.q = pack_tick(t, pj.blob.data() + off, desc_base + off);
      pj.ops.push_back(tick);
      for (const Follow& fl : follow) {
        PlanOp op;
        op.kind = PlanOp::FOLLOW;
        op.cls = cls;
        op.follow = fl;
        pj.ops.push_back(op);
        if (job_advance(*fl.j)) {
          fl.j->issued_all = true;
          PlanOp ep;
          ep.kind = PlanOp::EPILOGUE;
          ep.cls = cls;
          ep.job = (int)fl.j->id;
          pj.ops.push_back(ep);
        }
      }
    }
  }
  return PTYRO_OK;
}

}  // namespace ptyro

// Grid classes run on their own streams, forked from and joined back to the launch
// stream with events (under stream capture the graph gets one branch per class).
struct ptyro_plan {
  int device = 0;
  ptyro::PlanJobs pj;
  std::vector<cudaStream_t> streams;  // one per grid class
  std::vector<cudaEvent_t> joins;     // one per grid class
  cudaEvent_t fork = nullptr;
  ~ptyro_plan() {
    for (cudaStream_t s : streams)
      if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : joins)
      if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
  }
};

extern "C" {

size_t ptyro_plan_bytes(const ptyro_job_desc* jobs, int32_t num_jobs) {
  ptyro::PlanJobs pj;
  if (ptyro::plan_record(jobs, num_jobs, nullptr, pj)) return 0;
  return pj.job_bytes + ptyro::align_up(pj.blob.size());
}

int ptyro_plan_create(int32_t device, const ptyro_job_desc* jobs, int32_t num_jobs, void* arena, size_t arena_bytes,
                      ptyro_plan** out) {
  using namespace ptyro;
  if (!out) return fail(PTYRO_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (!arena || ((uintptr_t)arena & 255)) return fail(PTYRO_ERR_WORKSPACE, "arena must be 256-byte aligned");
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != device) return fail(PTYRO_ERR_INVALID, "create the plan with its device current");
  auto plan = std::make_unique<ptyro_plan>();
  plan->device = device;
  int rc = plan_record(jobs, num_jobs, (char*)arena, plan->pj);
  if (rc) return rc;
  const size_t need = plan->pj.job_bytes + align_up(plan->pj.blob.size());
  if (arena_bytes < need)
    return fail(PTYRO_ERR_WORKSPACE, "plan needs " + std::to_string(need) + " arena bytes; got " +
                                         std::to_string(arena_bytes));
  if (!plan->pj.blob.empty() &&
      cudaMemcpy((char*)arena + plan->pj.job_bytes, plan->pj.blob.data(), plan->pj.blob.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(PTYRO_ERR_CUDA, "plan descriptor upload failed");
  if (cudaEventCreateWithFlags(&plan->fork, cudaEventDisableTiming) != cudaSuccess)
    return fail(PTYRO_ERR_CUDA, "cudaEventCreateWithFlags failed");
  for (size_t c = 0; c < plan->pj.class_edges.size(); ++c) {
    cudaStream_t cs = nullptr;
    cudaEvent_t ev = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess)
      return fail(PTYRO_ERR_CUDA, "cudaStreamCreateWithFlags failed");
    plan->streams.push_back(cs);
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
      return fail(PTYRO_ERR_CUDA, "cudaEventCreateWithFlags failed");
    plan->joins.push_back(ev);
  }
  *out = plan.release();
  return PTYRO_OK;
}

int ptyro_plan_launch(ptyro_plan* plan, void* stream) {
  using namespace ptyro;
  if (!plan) return fail(PTYRO_ERR_INVALID, "plan is NULL");
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != plan->device) return fail(PTYRO_ERR_INVALID, "launch the plan with its device current");
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaEventRecord(plan->fork, st) != cudaSuccess) return fail(PTYRO_ERR_CUDA, "plan fork: cudaEventRecord failed");
  for (cudaStream_t cs : plan->streams)
    if (cudaStreamWaitEvent(cs, plan->fork, 0) != cudaSuccess)
      return fail(PTYRO_ERR_CUDA, "plan fork: cudaStreamWaitEvent failed");
  int rc = PTYRO_OK;
  for (const PlanOp& op : plan->pj.ops) {
    cudaStream_t cs = plan->streams[op.cls];
    switch (op.kind) {
      case PlanOp::SETUP: rc = job_setup(plan->pj.jobs[op.job], cs); break;
      case PlanOp::RAMPS: rc = launch_ramps(op.ramp, cs); break;
      case PlanOp::TICK: rc = launch_tick(op.n, op.q, cs); break;
      case PlanOp::FOLLOW: rc = launch_follow(op.follow, cs); break;
      case PlanOp::EPILOGUE: rc = job_epilogue(plan->pj.jobs[op.job], cs); break;
    }
    if (rc) break;
  }
  // join every class stream back to the launch stream, also after a failed launch
  for (size_t c = 0; c < plan->streams.size(); ++c) {
    if (cudaEventRecord(plan->joins[c], plan->streams[c]) != cudaSuccess ||
        cudaStreamWaitEvent(st, plan->joins[c], 0) != cudaSuccess)
      return rc ? rc : fail(PTYRO_ERR_CUDA, "plan join failed");
  }
  return rc;
}

int ptyro_plan_job_status(const ptyro_plan* plan, int32_t job, void** status_word) {
  if (!plan || !status_word) return ptyro::fail(PTYRO_ERR_INVALID, "plan or status_word is NULL");
  if (job < 0 || job >= (int)plan->pj.jobs.size()) return ptyro::fail(PTYRO_ERR_INVALID, "job index out of range");
  const ptyro::Job& j = plan->pj.jobs[job];
  *status_word = j.base + j.plan.off_fwd + j.plan.L.status;
  return PTYRO_OK;
}

int ptyro_plan_destroy(ptyro_plan* plan) {
  delete plan;
  return PTYRO_OK;
}

size_t ptyro_sched_job_bytes(const ptyro_job_desc* d) {
  JobPlan jp;
  if (plan_job(d, &jp)) return 0;
  return jp.bytes;
}

int ptyro_sched_create(int32_t device, void* arena, size_t arena_bytes, int32_t max_slots, ptyro_sched** out) {
  if (!out) return fail(PTYRO_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (!arena || ((uintptr_t)arena & 255)) return fail(PTYRO_ERR_WORKSPACE, "arena must be 256-byte aligned");
  if (max_slots < 1) return fail(PTYRO_ERR_INVALID, "max_slots must be >= 1");
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != device) return fail(PTYRO_ERR_INVALID, "create the scheduler with its device current");
  auto* s = new ptyro_sched();
  s->device = device;
  s->max_slots = max_slots;
  s->arena.init((char*)arena, arena_bytes);
  s->arena_bytes = arena_bytes;
  // per tick: up to max_slots rows in each of 6 tables plus one descriptor per job
  s->stage_bytes = align_up((size_t)6 * max_slots * sizeof(int2) + (size_t)max_slots * (sizeof(PassArgs) +
                                                                                        sizeof(BwdArgs)) + 4096);
  *out = s;
  return PTYRO_OK;
}

int ptyro_sched_destroy(ptyro_sched* s) {
  if (!s) return PTYRO_OK;
  for (auto& kv : s->classes) {
    cudaStreamSynchronize(kv.second.stream);
    for (int i = 0; i < GridClass::kRing; ++i) {
      cudaFreeHost(kv.second.host[i]);
      cudaEventDestroy(kv.second.used[i]);
    }
    cudaStreamDestroy(kv.second.stream);
  }
  for (auto& kv : s->jobs)
    if (kv.second->done) cudaEventDestroy(kv.second->done);
  delete s;
  return PTYRO_OK;
}

int ptyro_sched_submit(ptyro_sched* s, const ptyro_job_desc* d, int64_t* id) {
  if (!s || !id) return fail(PTYRO_ERR_INVALID, "scheduler or id is NULL");
  auto j = std::make_unique<Job>();
  int rc = plan_job(d, &j->plan);
  if (rc) return rc;
  // a job that could not fit even in an empty arena is rejected now; others wait for memory
  if (j->plan.bytes + (size_t)GridClass::kRing * s->stage_bytes > s->arena_bytes)
    return fail(PTYRO_ERR_WORKSPACE, "job needs " + std::to_string(j->plan.bytes) + " bytes of scratch; the arena holds " +
                                         std::to_string(s->arena_bytes));
  if (j->plan.L.batch * j->plan.p.num_modes > s->max_slots)
    return fail(PTYRO_ERR_INVALID, "job's probes in flight exceed the scheduler's slot budget (lower p.batch)");
  j->d = *d;
  std::lock_guard<std::mutex> lock(s->mu);
  j->id = s->next_id++;
  *id = j->id;
  s->queue.push_back(j->id);
  s->jobs.emplace(j->id, std::move(j));
  return PTYRO_OK;
}

int ptyro_sched_cancel(ptyro_sched* s, int64_t id) {
  if (!s) return fail(PTYRO_ERR_INVALID, "scheduler is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return fail(PTYRO_ERR_INVALID, "unknown job id");
  Job& j = *it->second;
  if (j.state == PTYRO_JOB_QUEUED) {
    s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), id), s->queue.end());
    j.state = PTYRO_JOB_CANCELLED;
    return PTYRO_OK;
  }
  if (j.state == PTYRO_JOB_RUNNING && !j.issued_all) {
    // stop issuing passes; memory returns once the passes already issued complete
    GridClass* c = nullptr;
    int rc = class_for(s, j.plan.p.n, &c);
    if (rc) return rc;
    if (cudaEventCreateWithFlags(&j.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(j.done, c->stream) != cudaSuccess)
      return fail(PTYRO_ERR_CUDA, "cudaEventRecord failed");
    j.issued_all = true;
    j.state = PTYRO_JOB_CANCELLED;
  }
  return PTYRO_OK;
}

int ptyro_sched_step(ptyro_sched* s, int32_t* running, int32_t* queued) {
  if (!s) return fail(PTYRO_ERR_INVALID, "scheduler is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  int rc = PTYRO_OK;
  // 1. retire jobs whose last work has completed
  for (size_t i = 0; i < s->running.size();) {
    Job& j = *s->jobs[s->running[i]];
    if (j.issued_all && j.done && cudaEventQuery(j.done) == cudaSuccess) {
      s->arena.release(j.arena_off, j.plan.bytes);
      s->active_slots -= j.rows_reserved;
      if (j.state == PTYRO_JOB_RUNNING) j.state = PTYRO_JOB_DONE;
      s->running.erase(s->running.begin() + i);
    } else {
      ++i;
    }
  }
  // 2. admit queued jobs in arrival order while memory and slots allow
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    Job& j = *s->jobs[*it];
    const int rows = j.plan.L.batch * j.plan.p.num_modes;
    size_t off;
    if (s->active_slots + rows > s->max_slots) break;
    GridClass* c = nullptr;
    if ((rc = class_for(s, j.plan.p.n, &c))) return rc;
    if (!s->arena.alloc(j.plan.bytes, &off)) {
      ++it;  // a smaller job behind it may still fit
      continue;
    }
    j.arena_off = off;
    j.base = s->arena.base() + off;
    j.rows_reserved = rows;
    s->active_slots += rows;
    if ((rc = admit(s, j, *c))) {
      j.state = PTYRO_JOB_FAILED;
      j.issued_all = true;
      cudaEventCreateWithFlags(&j.done, cudaEventDisableTiming);
      cudaEventRecord(j.done, c->stream);
      s->running.push_back(j.id);
      it = s->queue.erase(it);
      continue;
    }
    if (j.issued_all && !j.done) finish_job(j, *c);
    s->running.push_back(j.id);
    it = s->queue.erase(it);
  }
  // 3. one pass of every running job, grouped by grid edge
  std::map<int, std::vector<Job*>> by_class;
  for (int64_t id : s->running) {
    Job* j = s->jobs[id].get();
    if (!j->issued_all) by_class[j->plan.p.n].push_back(j);
  }
  for (auto& kv : by_class) {
    GridClass* c = nullptr;
    if ((rc = class_for(s, kv.first, &c))) return rc;
    if ((rc = tick_class(s, *c, kv.second))) {
      for (Job* j : kv.second) {
        j->state = PTYRO_JOB_FAILED;
        if (!j->done) {
          cudaEventCreateWithFlags(&j->done, cudaEventDisableTiming);
          cudaEventRecord(j->done, c->stream);
        }
        j->issued_all = true;
      }
      return rc;
    }
  }
  if (running) *running = (int32_t)s->running.size();
  if (queued) *queued = (int32_t)s->queue.size();
  return PTYRO_OK;
}

int ptyro_sched_job_state(ptyro_sched* s, int64_t id, int32_t* state) {
  if (!s || !state) return fail(PTYRO_ERR_INVALID, "scheduler or state is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return fail(PTYRO_ERR_INVALID, "unknown job id");
  *state = it->second->state;
  return PTYRO_OK;
}

int ptyro_sched_release(ptyro_sched* s, int64_t id) {
  if (!s) return fail(PTYRO_ERR_INVALID, "scheduler is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return fail(PTYRO_ERR_INVALID, "unknown job id");
  const int st = it->second->state;
  if (st == PTYRO_JOB_QUEUED || (st == PTYRO_JOB_RUNNING) ||
      (std::find(s->running.begin(), s->running.end(), id) != s->running.end()))
    return fail(PTYRO_ERR_INVALID, "job has not finished");
  if (it->second->done) cudaEventDestroy(it->second->done);
  s->jobs.erase(it);
  return PTYRO_OK;
}

int ptyro_sched_memory(ptyro_sched* s, size_t* free_bytes, int32_t* free_slots) {
  if (!s) return fail(PTYRO_ERR_INVALID, "scheduler is NULL");
  std::lock_guard<std::mutex> lock(s->mu);
  if (free_bytes) *free_bytes = s->arena.free_bytes();
  if (free_slots) *free_slots = s->max_slots - s->active_slots;
  return PTYRO_OK;
}

}  // extern "C"
