// Discrete adjoint of fixed-step DP45 on the pseudospectral dictionary RHS.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "dp45.h"
#include "internal.h"
#include "spectral.h"

namespace rdcu {

class AdjointEngine {
 public:
  bool init(SpectralPlan* fwd, DP45Engine* dp, const std::vector<HostTerm>& terms, int n, int ndim, const int* Ns,
            const double* Ls, cudaStream_t st, std::string* msg);
  void release();
  ~AdjointEngine() { release(); }

  // Forward run from y0 (host or device) over the step sizes hs[0..nsteps) (host; a
  // fixed step or a recorded accepted sequence), keeping the state every K steps; yT
  // (host or device, may be null) receives the final state.
  cudaError_t forward(const double* y0, const double* hs, int nsteps, int K, double* yT);
  // Reverse sweep from lambdaT = dL/dy(T): grad_y0 (host or device, n*N) and grad_C
  // (host, one entry per coupling term) of the last forward run.
  cudaError_t backward(const double* lambdaT, double* grad_y0, double* grad_C);
  cudaError_t set_coefficients(const std::vector<double>& C);
  bool recorded() const { return !ckpt_.empty(); }

  size_t device_bytes = 0;
  int nterms = 0;
  bool use_graphs = true;  // replay full segments as CUDA graphs (uniform step size)

 private:
  SpectralPlan* fwd_ = nullptr;
  DP45Engine* dp_ = nullptr;
  cudaStream_t st_ = nullptr;
  int n_ = 0;
  long long N_ = 0, nN_ = 0;
  // forward record
  std::vector<double> hs_;
  bool uniform_h_ = true;
  int nsteps_ = 0, K_ = 0;
  std::vector<double*> ckpt_;       // state at steps 0, K, 2K, ... of the last forward run
  std::vector<double*> ckpt_pool_;  // every checkpoint buffer allocated so far
  // segment store: stage states Y_1..Y_6 of up to K steps
  double* store_ = nullptr;
  int store_steps_ = 0;
  // reverse sweep buffers
  double* lam_ = nullptr;           // adjoint state
  double* Yb_ = nullptr;            // stage adjoints (6 blocks)
  double* tin_ = nullptr;           // transposed-operator input: [kbar (n), Qbar (nq)]
  double* tout_ = nullptr;          // transposed-operator output (ng channels)
  double* qv_ = nullptr;            // derivative quantities of the stage state (nq)
  double* ubar_ = nullptr;          // pointwise field adjoint (n)
  double* part_ = nullptr;          // per-term partial sums [nterms][kBlocks]
  double* gC_ = nullptr;            // coefficient gradient accumulator [nterms]
  // plans
  SpectralPlan planQ_, planT_;
  bool have_q_ = false;
  int nq_ = 0, ng_ = 0, nfold_pairs_ = 0;
  size_t pw_smem_ = 0;  // dynamic shared memory of the pointwise kernel
  // tables (device)
  struct Tables;
  Tables* tab_ = nullptr;
  std::vector<HostTerm> terms_;
  struct SegGraphs {
    int steps;
    double h;
    cudaGraphExec_t rec, rev;
  };
  std::vector<SegGraphs> graphs_;
  cudaError_t stage_kernels(const double* Y, int stage, double h, const double* Yprev, int sprev);
  cudaError_t ensure_store(int steps);
  void drop_graphs();
  cudaError_t launch_recompute(int j0, int steps);
  cudaError_t launch_reverse(int j0, int steps);
};

}  // namespace rdcu
