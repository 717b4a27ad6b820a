// Ensemble of independent 2D pseudospectral DP45 problems stepped together.
//
// No counterpart in the reference, which integrates one problem per process.  Every
// member keeps its own state, step size and controller (the DP45Ctl of the single-problem
// engine, one per member in device memory); one attempt of the ensemble is the six
// batched stage launches 2..7 of SpectralBatch plus one controller launch with a block
// per member, captured once as a CUDA graph (stage 1, k1 = f(y), runs at the start of
// every solve, as in the single-problem solver).  Members
// that reached their end time stop being stepped (their work items return at once),
// so each member takes exactly the accepted/rejected sequence the single-problem
// solver takes, with bitwise identical states.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

#include "dp45_ctl.cuh"
#include "ensemble.h"

namespace rdcu {
namespace {

__global__ void k_ens_arm(DP45Ctl* ctl, int m, double t1, double hmin, double hmax) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) dp45_arm(ctl + i, 1, t1, hmin, hmax, 0, 0, INT_MAX);
}

__global__ void __launch_bounds__(kCtlThreads) k_ens_ctl(DP45Ctl* ctl, const double* const* parts, const double* nN) {
  const int i = blockIdx.x;
  dp45_control(ctl + i, parts[i], nullptr, nullptr, nullptr, nN[i], nullptr);
}

__global__ void k_ens_running(const DP45Ctl* ctl, int m, int* out) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int c = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) c += ctl[i].running;
  atomicAdd(&cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) *out = cnt;
}

}  // namespace

#define RDCU_TRY(x)                   \
  do {                                \
    cudaError_t _e = (x);             \
    if (_e != cudaSuccess) return _e; \
  } while (0)

bool EnsembleEngine::init(const std::vector<EnsembleProblem>& probs, double rtol, double atol, cudaStream_t st,
                          std::string* msg) {
  release();
  probs_ = probs;
  st_ = st;
  rtol_ = rtol;
  atol_ = atol;
  const int m = (int)probs.size();
  if (m < 1) {
    *msg = "empty ensemble";
    return false;
  }
  size_t total = 0;
  std::vector<size_t> off(m);
  for (int i = 0; i < m; ++i) {
    const auto& p = probs[i];
    std::unique_ptr<SpectralPlan> sp(new SpectralPlan);
    if (!sp->init(p.n, 2, p.Ns, p.Ls, p.terms, msg)) {
      *msg = "ensemble member " + std::to_string(i) + ": " + *msg;
      return false;
    }
    device_bytes += sp->device_bytes;
    nN_.push_back((long long)p.n * sp->N);
    off[i] = total;
    total += (size_t)nN_[i] * 10 + (size_t)std::max(1, sp->nparts_max);
    total = (total + 31) / 32 * 32;  // 256-byte alignment of every member's block
    plans_.push_back(std::move(sp));
  }
  if (cudaMalloc((void**)&state_mem_, total * sizeof(double)) != cudaSuccess) {
    *msg = "out of device memory (ensemble states)";
    return false;
  }
  device_bytes += total * sizeof(double);
  if (cudaMalloc((void**)&d_ctl_, m * sizeof(DP45Ctl)) != cudaSuccess ||
      cudaMallocHost((void**)&h_ctl_, m * sizeof(DP45Ctl)) != cudaSuccess ||
      cudaMalloc((void**)&d_parts_, m * sizeof(double*)) != cudaSuccess ||
      cudaMalloc((void**)&d_nN_, m * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&d_running_, sizeof(int)) != cudaSuccess ||
      cudaMallocHost((void**)&h_running_, sizeof(int)) != cudaSuccess) {
    *msg = "out of device memory (ensemble controllers)";
    return false;
  }
  std::vector<double*> parts(m);
  std::vector<double> nNd(m);
  members_.resize(m);
  for (int i = 0; i < m; ++i) {
    double* base = state_mem_ + off[i];
    BatchMember& b = members_[i];
    b.plan = plans_[i].get();
    for (int k = 0; k < 3; ++k) b.bufs.ybuf[k] = base + (size_t)k * nN_[i];
    for (int k = 0; k < 7; ++k) b.bufs.kbuf[k] = base + (size_t)(3 + k) * nN_[i];
    b.err_part = base + (size_t)10 * nN_[i];
    b.ctl = d_ctl_ + i;
    parts[i] = b.err_part;
    nNd[i] = (double)nN_[i];
    DP45Ctl c{};
    c.atol = atol;
    c.rtol = rtol;
    c.fixed = 0;
    c.y_slot = 0;
    c.yn_slot = 1;
    c.yl_slot = 2;
    c.k1_buf = 0;
    c.k7_buf = 6;
    c.last_k1_buf = 0;
    c.last_k7_buf = 6;
    c.log_cap = 0;  // no attempt log: the ensemble reports counters only
    c.nparts = plans_[i]->nparts_max;
    c.hmax = INFINITY;
    h_ctl_[i] = c;
  }
  if (cudaMemcpy(d_ctl_, h_ctl_, m * sizeof(DP45Ctl), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(d_parts_, parts.data(), m * sizeof(double*), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(d_nN_, nNd.data(), m * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(state_mem_, 0, total * sizeof(double)) != cudaSuccess) {
    *msg = "ensemble set-up copy failed";
    return false;
  }
  if (build_batch(tile_elems) != cudaSuccess) {
    *msg = "ensemble batch set-up failed";
    return false;
  }
  return true;
}

cudaError_t EnsembleEngine::build_batch(int elems) {
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  std::string msg;
  if (!batch_.init(members_, elems, &msg)) return cudaErrorInvalidValue;
  tile_elems = batch_.elems;
  return cudaSuccess;
}

void EnsembleEngine::release() {
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  batch_.release();
  plans_.clear();
  members_.clear();
  nN_.clear();
  if (state_mem_) cudaFree(state_mem_);
  if (d_ctl_) cudaFree(d_ctl_);
  if (h_ctl_) cudaFreeHost(h_ctl_);
  if (d_parts_) cudaFree(d_parts_);
  if (d_nN_) cudaFree(d_nN_);
  if (d_running_) cudaFree(d_running_);
  if (h_running_) cudaFreeHost(h_running_);
  state_mem_ = nullptr;
  d_ctl_ = nullptr;
  h_ctl_ = nullptr;
  d_parts_ = nullptr;
  d_nN_ = nullptr;
  d_running_ = nullptr;
  h_running_ = nullptr;
  device_bytes = 0;
}

cudaError_t EnsembleEngine::sync_ctl() {
  RDCU_TRY(cudaMemcpyAsync(h_ctl_, d_ctl_, probs_.size() * sizeof(DP45Ctl), cudaMemcpyDeviceToHost, st_));
  return cudaStreamSynchronize(st_);
}

cudaError_t EnsembleEngine::set_state(int i, double t, double h, const double* y) {
  if (i < 0 || i >= size()) return cudaErrorInvalidValue;
  RDCU_TRY(sync_ctl());
  DP45Ctl c = h_ctl_[i];
  c.t = t;
  c.h = h;
  c.t_last = t;
  c.y_slot = 0;
  c.yn_slot = 1;
  c.yl_slot = 2;
  c.k1_buf = 0;
  c.k7_buf = 6;
  c.last_k1_buf = 0;
  c.last_k7_buf = 6;
  c.running = 0;
  c.accepted = 0;
  c.n_attempts = 0;
  c.n_accepted = 0;
  h_ctl_[i] = c;
  RDCU_TRY(cudaMemcpyAsync(d_ctl_ + i, &h_ctl_[i], sizeof(DP45Ctl), cudaMemcpyHostToDevice, st_));
  if (y)
    RDCU_TRY(cudaMemcpyAsync(members_[i].bufs.ybuf[0], y, (size_t)nN_[i] * sizeof(double), cudaMemcpyDefault, st_));
  return cudaStreamSynchronize(st_);
}

cudaError_t EnsembleEngine::get_state(int i, double* t, double* h, double* y) {
  if (i < 0 || i >= size()) return cudaErrorInvalidValue;
  RDCU_TRY(sync_ctl());
  if (t) *t = h_ctl_[i].t;
  if (h) *h = h_ctl_[i].h;
  if (y)
    RDCU_TRY(cudaMemcpyAsync(y, members_[i].bufs.ybuf[h_ctl_[i].y_slot], (size_t)nN_[i] * sizeof(double),
                             cudaMemcpyDefault, st_));
  return cudaStreamSynchronize(st_);
}

cudaError_t EnsembleEngine::counters(int i, long long* accepted, long long* attempts) {
  if (i < 0 || i >= size()) return cudaErrorInvalidValue;
  RDCU_TRY(sync_ctl());
  if (accepted) *accepted = h_ctl_[i].n_accepted;
  if (attempts) *attempts = h_ctl_[i].n_attempts;
  return cudaSuccess;
}

cudaError_t EnsembleEngine::set_tolerances(int i, double rtol, double atol) {
  if (i < 0 || i >= size()) return cudaErrorInvalidValue;
  RDCU_TRY(sync_ctl());
  h_ctl_[i].rtol = rtol;
  h_ctl_[i].atol = atol;
  RDCU_TRY(cudaMemcpyAsync(d_ctl_ + i, &h_ctl_[i], sizeof(DP45Ctl), cudaMemcpyHostToDevice, st_));
  return cudaStreamSynchronize(st_);
}

cudaError_t EnsembleEngine::launch_attempt() {
  for (int s = 2; s <= 7; ++s) RDCU_TRY(batch_.launch_stage(s, st_));
  k_ens_ctl<<<size(), kCtlThreads, 0, st_>>>(d_ctl_, d_parts_, d_nN_);
  return cudaGetLastError();
}

cudaError_t EnsembleEngine::ensure_graph() {
  if (graph_) return cudaSuccess;
  RDCU_TRY(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = launch_attempt();
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(st_, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&graph_, g, 0);
  if (g) cudaGraphDestroy(g);
  return e;
}

cudaError_t EnsembleEngine::solve(double t1, double hmin, double hmax) {
  const int m = size();
  attempt_launches = 0;
  k_ens_arm<<<(m + 127) / 128, 128, 0, st_>>>(d_ctl_, m, t1, hmin, hmax);
  RDCU_TRY(cudaGetLastError());
  // FSAL start (dp45.cu:157): k1 = f(y) of every running member, as the single-problem
  // solve does at its start
  RDCU_TRY(batch_.launch_stage(1, st_));
  RDCU_TRY(ensure_graph());
  // attempts in chunks; the host checks between chunks whether any member still runs
  int chunk = 16;
  for (long long guard = 0; guard < 100000000LL; guard += chunk) {
    for (int k = 0; k < chunk; ++k) RDCU_TRY(cudaGraphLaunch(graph_, st_));
    attempt_launches += chunk;
    k_ens_running<<<1, 256, 0, st_>>>(d_ctl_, m, d_running_);
    RDCU_TRY(cudaGetLastError());
    RDCU_TRY(cudaMemcpyAsync(h_running_, d_running_, sizeof(int), cudaMemcpyDeviceToHost, st_));
    RDCU_TRY(cudaStreamSynchronize(st_));
    if (*h_running_ == 0) return sync_ctl();
    chunk = std::min(chunk * 2, 256);
  }
  return cudaErrorUnknown;
}

cudaError_t EnsembleEngine::tune(std::vector<std::pair<int, double>>* trials) {
  // A trial runs stage 4 of every member: it writes only the stage-4 state slot and slope
  // k4, which the next solve recomputes (solve starts from y and a fresh k1), so the
  // members' states need no saving.
  const int m = size();
  RDCU_TRY(sync_ctl());
  std::vector<DP45Ctl> saved(h_ctl_, h_ctl_ + m);
  const int cand[] = {512, 1024, 2048, 4096};
  int best = tile_elems;
  double best_ms = 1e300;
  cudaEvent_t e0, e1;
  RDCU_TRY(cudaEventCreate(&e0));
  RDCU_TRY(cudaEventCreate(&e1));
  for (int c : cand) {
    if (build_batch(c) != cudaSuccess) continue;
    k_ens_arm<<<(m + 127) / 128, 128, 0, st_>>>(d_ctl_, m, INFINITY, 0.0, INFINITY);
    RDCU_TRY(cudaGetLastError());
    RDCU_TRY(batch_.launch_stage(4, st_));
    RDCU_TRY(cudaEventRecord(e0, st_));
    for (int r = 0; r < 5; ++r) RDCU_TRY(batch_.launch_stage(4, st_));
    RDCU_TRY(cudaEventRecord(e1, st_));
    RDCU_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    RDCU_TRY(cudaEventElapsedTime(&ms, e0, e1));
    if (trials) trials->push_back({batch_.elems, ms / 5});
    if (ms < best_ms) {
      best_ms = ms;
      best = batch_.elems;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  RDCU_TRY(build_batch(best));
  // controllers as before the trials (not running)
  std::copy(saved.begin(), saved.end(), h_ctl_);
  RDCU_TRY(cudaMemcpyAsync(d_ctl_, h_ctl_, m * sizeof(DP45Ctl), cudaMemcpyHostToDevice, st_));
  return cudaStreamSynchronize(st_);
}

}  // namespace rdcu
