// Device-controlled Dormand-Prince 4(5) integrator over the fused spectral RHS.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "internal.h"
#include "spectral.h"

namespace rdcu {

struct AttemptRecord {
  double h;
  int accepted;
};

class DP45Engine {
 public:
  bool init(SpectralPlan* sp, double atol, double rtol, int fixed, cudaStream_t st, std::string* msg);
  void release();
  ~DP45Engine() { release(); }

  // State (t, h, y); y is a host or device pointer of n*N doubles.
  cudaError_t set_state(double t, double h, const double* y);
  cudaError_t get_state(double* t, double* h, double* y_dst, cudaMemcpyKind kind);
  // One attempt (dp45_step); synchronous.
  cudaError_t step(double* t, double* h, double hmin, double hmax, int* accepted);
  // Dense output of the last accepted step (dp45_eval); y_eval device pointer.
  cudaError_t eval(double t_eval, double* y_eval);
  // Whole integration with device-side control; on_attempt/on_output are called in
  // reference order.  on_output(eval index) is called once per due output time after
  // an accepted step, then on_checkpoint().
  cudaError_t solve(double t1, double hmin, double hmax, const std::vector<double>& t_eval,
                    const std::function<int(double t, double h, int acc, long long steps)>& on_attempt,
                    const std::function<int(int idx, const double* y_eval)>& on_eval,
                    const std::function<int(double t, double h, long long steps)>& on_checkpoint,
                    int* cb_status);

  // per-pass timing of stage 4 (see rdcu_profile_passes)
  cudaError_t profile(int reps, std::vector<SpectralPlan::PassTime>* out);
  // n attempts on the device (graph launches), one sync at the end
  cudaError_t advance(int n, double hmin, double hmax, long long* accepted);
  // Launches one attempt (stages 2..7 and the controller) on the stream; no sync.
  cudaError_t launch_attempt();
  // launch_attempt with the stage states of stages 2..6 written to ytemp_out[2..6]
  // (entries may be null) instead of the scratch state slot
  cudaError_t launch_attempt_capture(double* const* ytemp_out);
  cudaError_t launch_k1();
  // the RhsIO of DP45 stage s (2..7) of this engine's attempt
  RhsIO stage_io(int s) const;
  // device copy of the current state y (slot chosen on the device); no sync
  cudaError_t copy_current_y(double* dst);
  // sets the step size of the next attempt on the device; no sync
  cudaError_t set_h_async(double h);
  // (t, h) and the slot assignment of set_state, queued on the stream (no sync, no
  // copy: the caller fills bufs.ybuf[0]); stream-capturable
  cudaError_t reset_async(double t, double h);
  int log_cap() const { return log_cap_; }
  cudaError_t arm(int check, double t1, double hmin, double hmax, int eval_i, int n_eval,
                  int max_attempts);
  // the cached slope k1 = f(y) is stale (new coefficients): recompute it before the next attempt
  void invalidate_k1() {
    k1_valid_ = false;
    have_step_ = false;
  }
  cudaError_t sync_ctl();  // copies the controller state to host_ctl (synchronises)

  DP45Ctl host_ctl{};
  long long solve_attempts = 0, solve_accepted = 0;
  double* y_eval = nullptr;
  DP45Bufs bufs{};
  size_t device_bytes = 0;
  bool use_graph = true;

 private:
  SpectralPlan* sp_ = nullptr;
  cudaStream_t st_ = nullptr;
  long long nN_ = 0;
  DP45Ctl* d_ctl_ = nullptr;
  DP45Ctl* h_ctl_pinned_ = nullptr;
  double* err_part_ = nullptr;
  double* log_h_ = nullptr;
  int* log_acc_ = nullptr;
  double* log_t_ = nullptr;
  double* h_log_t_ = nullptr;
  double* h_log_h_ = nullptr;
  int* h_log_acc_ = nullptr;
  double* d_teval_ = nullptr;
  int teval_cap_ = 0;
  int log_cap_ = 4096;
  bool k1_valid_ = false;
  bool have_step_ = false;
  int fixed_ = 0;
  double atol_ = 0, rtol_ = 0;
  cudaGraphExec_t graph_exec_ = nullptr;
  cudaGraph_t graph_ = nullptr;
  int graph_gen_ = -1;  // the plan's buffers_gen when the attempt graph was captured
  double* err_aux_ = nullptr;  // stage-7 slope sums (nN doubles) when the plan wants them
  cudaError_t ensure_graph();
};

}  // namespace rdcu
