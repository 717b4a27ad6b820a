// Variable-order NDF/BDF integrator on the finite-difference RHS (in progress).
#include <cmath>
#include <cstring>

#include "bdf.h"

namespace rdcu {

struct BDFEngine::Impl {};

bool BDFEngine::init(FDProblem* fd, double, double, int, cudaStream_t st, std::string* msg) {
  fd_ = fd;
  st_ = st;
  const size_t b = (size_t)fd->nN * 8 * sizeof(double);
  if (cudaMalloc((void**)&D_, b) != cudaSuccess) {
    *msg = "out of device memory (BDF differences)";
    return false;
  }
  device_bytes = b;
  return true;
}

void BDFEngine::release() {
  if (D_) cudaFree(D_);
  D_ = nullptr;
}

cudaError_t BDFEngine::set_state(double t, double h, const double* y, int order, const double* D) {
  t_ = t;
  h_ = h;
  order_ = order;
  const size_t sb = (size_t)fd_->nN * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(D_, y, sb, cudaMemcpyDefault, st_);
  if (e == cudaSuccess && order > 0 && D) e = cudaMemcpyAsync(D_ + fd_->nN, D, sb * order, cudaMemcpyDefault, st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  return e;
}

cudaError_t BDFEngine::get_state(double* t, double* h, int* order, double* y, double* D) {
  if (t) *t = t_;
  if (h) *h = h_;
  if (order) *order = order_;
  const size_t sb = (size_t)fd_->nN * sizeof(double);
  cudaError_t e = cudaSuccess;
  if (y) e = cudaMemcpyAsync(y, D_, sb, cudaMemcpyDefault, st_);
  if (e == cudaSuccess && D && order_ > 0) e = cudaMemcpyAsync(D, D_ + fd_->nN, sb * order_, cudaMemcpyDefault, st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  return e;
}

cudaError_t BDFEngine::step(double*, double*, double, double, int*, int* status) {
  *status = RDCU_ERR_UNSUPPORTED;
  last_msg = "BDF stepping not built";
  return cudaSuccess;
}

cudaError_t BDFEngine::eval(double, double*) { return cudaErrorNotSupported; }

cudaError_t BDFEngine::solve(double t1, double hmin, double, const std::vector<double>&,
                             const std::function<int(double, double, int, long long)>&,
                             const std::function<int(int, const double*)>&,
                             const std::function<int(double, double, long long)>&, int*, int* status) {
  *status = RDCU_OK;
  if (!(t_ < t1 && h_ > hmin)) return cudaSuccess;
  *status = RDCU_ERR_UNSUPPORTED;
  last_msg = "BDF stepping not built";
  return cudaSuccess;
}

}  // namespace rdcu
