// Finite-difference RHS and analytic CSR Jacobian of the dictionary (BDF path).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "internal.h"
#include "spectral.h"

namespace rdcu {

// One Jacobian contribution: term t, factor jf (reference jac loop, rdcu.cu:202-245).
struct JacContrib {
  int term;     // index into the term table
  int jf;       // factor position within the term
  int yind;     // Y block of the factor (stencil)
  int src;      // field of the factor (column block)
};

// Device term table of the FD path: all factors kept (zero powers included, as the
// reference's Jacobian loops over them).
struct FDTerm {
  int field, nf, off, pad;
  double C;
};
struct FDFactor {
  int k, eta;   // Y index, power
};

struct FDTables {
  int n, ndim, nY, nterms, ncontrib;
  int Ns[3];
  double inv_dx[3];      // 1/dx per axis (first derivative scale uses 0.5/dx exactly as below)
  double s1[3];          // 0.5/dx_a  (rdcu.cu:442-446)
  double s2[3][3];       // 1/(dx_a dx_b) (rdcu.cu:496,502-504,561-564)
  const FDTerm* terms;
  const FDFactor* fac;
  const int* field_begin;      // terms grouped by field [n+1]
  const JacContrib* contrib;   // grouped by row field, term order kept
  const int* contrib_begin;    // [n+1]
  long long N;
};

class FDProblem {
 public:
  bool init(int n, int ndim, const int* Ns, const double* Ls, const std::vector<HostTerm>& terms,
            cudaStream_t st, std::string* msg);
  void release();
  ~FDProblem() { release(); }

  // f = dydt(y); if Y != nullptr all real FD blocks in Y.dat layout (imaginary parts 0)
  cudaError_t rhs(const double* y, double* f, double* Y);
  // Jacobian values at y into the handle's CSR (vals_); optional copy to caller arrays
  cudaError_t jac_values(const double* y);
  cudaError_t jac_csr(const double* y, int* rows, int* cols, double* vals);

  int n = 0, ndim = 0, Ns[3] = {1, 1, 1};
  double Ls[3] = {1, 1, 1};
  long long N = 0, nN = 0;
  long long nnz = 0;
  int* rows_ = nullptr;   // CSR pattern of J (device)
  int* cols_ = nullptr;
  double* vals_ = nullptr;
  int* diag_ = nullptr;   // position of the diagonal entry in each row, -1 if none
  size_t device_bytes = 0;
  FDTables tab{};
  cudaStream_t st = nullptr;
  std::vector<HostTerm> terms;

 private:
  FDTerm* d_terms_ = nullptr;
  FDFactor* d_fac_ = nullptr;
  int* d_field_begin_ = nullptr;
  JacContrib* d_contrib_ = nullptr;
  int* d_contrib_begin_ = nullptr;
};

}  // namespace rdcu
