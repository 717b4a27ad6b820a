// Variable-order NDF/BDF integrator (ode15s style) on the finite-difference RHS.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "fd.h"
#include "internal.h"

namespace rdcu {

class BDFEngine {
 public:
  bool init(FDProblem* fd, double atol, double rtol, int fixed, cudaStream_t st, std::string* msg);
  void release();
  ~BDFEngine() { release(); }

  cudaError_t set_state(double t, double h, const double* y, int order, const double* D);
  cudaError_t get_state(double* t, double* h, int* order, double* y, double* D);
  // one attempt (bdf_step); *status receives an RDCU_ERR_* code for solver failures
  cudaError_t step(double* t, double* h, double hmin, double hmax, int* accepted, int* status);
  cudaError_t eval(double t_eval, double* y_eval);
  cudaError_t solve(double t1, double hmin, double hmax, const std::vector<double>& t_eval,
                    const std::function<int(double, double, int, long long)>& on_attempt,
                    const std::function<int(int, const double*)>& on_eval,
                    const std::function<int(double, double, long long)>& on_checkpoint, int* cb_status,
                    int* status);

  int order() const { return order_; }
  double t() const { return t_; }
  double h() const { return h_; }
  const double* D_ptr() const { return D_; }

  long long solve_attempts = 0, solve_accepted = 0;
  size_t device_bytes = 0;
  std::string last_msg;
  // linear-solver statistics
  long long lin_iters = 0, lin_solves = 0, lin_cycles = 0;

  struct Impl;

 private:
  Impl* impl_ = nullptr;
  FDProblem* fd_ = nullptr;
  cudaStream_t st_ = nullptr;
  double* D_ = nullptr;  // 8 blocks of n*N (bdf.cu:416)
  int order_ = 0;
  double t_ = 0, h_ = 0;
};

}  // namespace rdcu
