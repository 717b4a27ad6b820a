// Ensemble of independent 2D pseudospectral DP45 problems stepped together.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "internal.h"
#include "spectral.h"

namespace rdcu {

struct EnsembleProblem {
  int n = 0;
  int Ns[2] = {0, 0};
  double Ls[2] = {0, 0};
  std::vector<HostTerm> terms;
};

class EnsembleEngine {
 public:
  bool init(const std::vector<EnsembleProblem>& probs, double rtol, double atol, cudaStream_t st, std::string* msg);
  void release();
  ~EnsembleEngine() { release(); }

  // state of member i (y host or device, n*N doubles)
  cudaError_t set_state(int i, double t, double h, const double* y);
  cudaError_t get_state(int i, double* t, double* h, double* y);
  // every member from its own (t, h) until its first accepted step reaching t1 (or h <= hmin)
  cudaError_t solve(double t1, double hmin, double hmax);
  // accepted steps and attempts of member i since its last set_state
  cudaError_t counters(int i, long long* accepted, long long* attempts);
  cudaError_t set_tolerances(int i, double rtol, double atol);
  // Autotuner: times one batched RHS stage for each candidate tile size (complex values
  // per CTA) on the current states and keeps the fastest; the states are kept.
  cudaError_t tune(std::vector<std::pair<int, double>>* trials);

  int size() const { return (int)probs_.size(); }
  long long state_len(int i) const { return nN_[i]; }
  size_t device_bytes = 0;
  int tile_elems = 1024;
  long long attempt_launches = 0;  // batched attempts launched by the last solve

 private:
  std::vector<EnsembleProblem> probs_;
  std::vector<std::unique_ptr<SpectralPlan>> plans_;
  std::vector<long long> nN_;
  std::vector<BatchMember> members_;
  SpectralBatch batch_;
  cudaStream_t st_ = nullptr;
  double rtol_ = 0, atol_ = 0;
  double* state_mem_ = nullptr;  // every member's 3 state + 7 slope buffers and error partials
  DP45Ctl* d_ctl_ = nullptr;
  DP45Ctl* h_ctl_ = nullptr;  // pinned mirror
  double** d_parts_ = nullptr;
  double* d_nN_ = nullptr;
  int* d_running_ = nullptr;
  int* h_running_ = nullptr;
  cudaGraphExec_t graph_ = nullptr;
  cudaError_t build_batch(int elems);
  cudaError_t ensure_graph();
  cudaError_t launch_attempt();
  cudaError_t sync_ctl();
};

}  // namespace rdcu
