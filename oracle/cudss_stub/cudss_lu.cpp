/* A solving stand-in for the cuDSS calls of the reference's BDF path (reference
 * bdf.cu:26-29, 154-159, 341-368, 450-452, 487-489), for an image without cuDSS.
 *
 * The reference factorises A = I + alpha J with cuDSS's sparse LU and solves A dd = b
 * once per Newton iteration.  This stand-in does the same with cuSOLVER's host sparse
 * LU (partial pivoting) after a nested-dissection reordering of A's pattern:
 *   ANALYSIS         -> pattern to the host, reordering p, permuted pattern, symbolic LU
 *   (RE)FACTORIZATION-> values to the host, numeric LU of A(p, p)
 *   SOLVE            -> b to the host, x = solve, x to the device
 * so the reference's unmodified rdcu.cu/bdf.cu can run its BDF path on a GPU machine and
 * produce fixtures.  Test infrastructure only (oracle/build_ref.sh links it into
 * oracle/_ref/rdcu_ref_lu); librdcu never uses it.  The declarations are those of
 * cudss.h beside it (names and signatures from the reference's call sites). */
#include <cuda_runtime.h>
#include <cusolverSp.h>
#include <cusolverSp_LOWLEVEL_PREVIEW.h>
#include <cusparse.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <utility>
#include <vector>

#include "cudss.h"

struct cudss_stub_handle {
  cusolverSpHandle_t sp = nullptr;
};
struct cudss_stub_config {
  int unused = 0;
};
struct cudss_stub_matrix {
  bool csr = false;
  int n = 0, nnz = 0;
  int* rows = nullptr;  // device CSR (the reference's buffers)
  int* cols = nullptr;
  double* vals = nullptr;
  double* dn = nullptr;  // device dense vector
};
struct cudss_stub_data {
  int n = 0, nnz = 0;
  std::vector<int> p;          // reordering: row/column i of A(p,p) is p[i] of A
  std::vector<int> brow, bcol;  // pattern of A(p,p)
  std::vector<int> map;        // valB = valA[map]
  std::vector<double> aval, bval, rhs, xp, x, bsave;
  std::vector<int> arow, acol;  // A's own pattern (residual check)
  cusparseMatDescr_t descr = nullptr;
  csrluInfoHost_t info = nullptr;
  std::vector<char> buffer;
  bool factored = false;
  int info_code = 0;
};

static cudssStatus_t fail(cudss_stub_data* d, const char* what, int code) {
  std::fprintf(stderr, "cudss stand-in: %s failed (%d)\n", what, code);
  if (d) d->info_code = code ? code : -1;
  return CUDSS_STATUS_NOT_SUPPORTED;
}

extern "C" {

cudssStatus_t cudssCreate(cudssHandle_t* h) {
  *h = new cudss_stub_handle();
  if (cusolverSpCreate(&(*h)->sp) != CUSOLVER_STATUS_SUCCESS) return CUDSS_STATUS_NOT_SUPPORTED;
  return CUDSS_STATUS_SUCCESS;
}
cudssStatus_t cudssDestroy(cudssHandle_t h) {
  if (h) {
    if (h->sp) cusolverSpDestroy(h->sp);
    delete h;
  }
  return CUDSS_STATUS_SUCCESS;
}
cudssStatus_t cudssConfigCreate(cudssConfig_t* c) {
  *c = new cudss_stub_config();
  return CUDSS_STATUS_SUCCESS;
}
cudssStatus_t cudssConfigDestroy(cudssConfig_t c) {
  delete c;
  return CUDSS_STATUS_SUCCESS;
}
cudssStatus_t cudssDataCreate(cudssHandle_t, cudssData_t* d) {
  *d = new cudss_stub_data();
  return CUDSS_STATUS_SUCCESS;
}
cudssStatus_t cudssDataDestroy(cudssHandle_t, cudssData_t d) {
  if (d) {
    if (d->info) cusolverSpDestroyCsrluInfoHost(d->info);
    if (d->descr) cusparseDestroyMatDescr(d->descr);
    delete d;
  }
  return CUDSS_STATUS_SUCCESS;
}
cudssStatus_t cudssDataGet(cudssHandle_t, cudssData_t d, cudssDataParam_t, void* v, size_t sz, size_t* written) {
  if (v && sz >= sizeof(int)) *(int*)v = d ? d->info_code : -1;
  if (written) *written = sizeof(int);
  return CUDSS_STATUS_SUCCESS;
}
cudssStatus_t cudssMatrixCreateCsr(cudssMatrix_t* m, int64_t nrows, int64_t, int64_t nnz, void* rowStart, void*,
                                   void* colIndices, void* values, cudssStubType_t, cudssStubType_t, cudssStubType_t,
                                   cudssMatrixType_t, cudssMatrixViewType_t, cudssIndexBase_t) {
  cudss_stub_matrix* a = new cudss_stub_matrix();
  a->csr = true;
  a->n = (int)nrows;
  a->nnz = (int)nnz;
  a->rows = (int*)rowStart;
  a->cols = (int*)colIndices;
  a->vals = (double*)values;
  *m = a;
  return CUDSS_STATUS_SUCCESS;
}
cudssStatus_t cudssMatrixCreateDn(cudssMatrix_t* m, int64_t nrows, int64_t, int64_t, void* values, cudssStubType_t,
                                  cudssLayout_t) {
  cudss_stub_matrix* a = new cudss_stub_matrix();
  a->n = (int)nrows;
  a->dn = (double*)values;
  *m = a;
  return CUDSS_STATUS_SUCCESS;
}
cudssStatus_t cudssMatrixDestroy(cudssMatrix_t m) {
  delete m;
  return CUDSS_STATUS_SUCCESS;
}

cudssStatus_t cudssExecute(cudssHandle_t h, cudssPhase_t phase, cudssConfig_t, cudssData_t d, cudssMatrix_t A,
                           cudssMatrix_t x, cudssMatrix_t b) {
  if (!h || !d || !A || !A->csr) return fail(d, "arguments", -1);
  const int n = A->n;
  if (phase == CUDSS_PHASE_ANALYSIS) {
    cudaDeviceSynchronize();
    d->n = n;
    d->nnz = A->nnz;
    std::vector<int> row(n + 1), col(A->nnz);
    if (cudaMemcpy(row.data(), A->rows, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(col.data(), A->cols, sizeof(int) * A->nnz, cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(d, "pattern copy", -2);
    if (!d->descr) {
      cusparseCreateMatDescr(&d->descr);
      cusparseSetMatType(d->descr, CUSPARSE_MATRIX_TYPE_GENERAL);
      cusparseSetMatIndexBase(d->descr, CUSPARSE_INDEX_BASE_ZERO);
    }
    d->arow = row;
    d->acol = col;
    d->p.assign(n, 0);
    cusolverStatus_t s = cusolverSpXcsrmetisndHost(h->sp, n, A->nnz, d->descr, row.data(), col.data(), nullptr,
                                                   d->p.data());
    if (s != CUSOLVER_STATUS_SUCCESS) {
      std::fprintf(stderr, "cudss stand-in: nested dissection failed (%d), trying AMD\n", (int)s);
      s = cusolverSpXcsrsymamdHost(h->sp, n, A->nnz, d->descr, row.data(), col.data(), d->p.data());
    }
    if (s != CUSOLVER_STATUS_SUCCESS) {
      std::fprintf(stderr, "cudss stand-in: AMD failed (%d), natural order\n", (int)s);
      for (int i = 0; i < n; ++i) d->p[i] = i;
    }
    {
      std::vector<char> seen(n, 0);
      for (int i = 0; i < n; ++i) {
        if (d->p[i] < 0 || d->p[i] >= n || seen[d->p[i]]) return fail(d, "reordering (not a permutation)", -6);
        seen[d->p[i]] = 1;
      }
    }
    // B = A(p, p) built explicitly (row i of B is row p[i] of A, columns renumbered by
    // the inverse permutation and sorted), with valB = valA[map]
    std::vector<int> pinv(n);
    for (int i = 0; i < n; ++i) pinv[d->p[i]] = i;
    d->brow.assign(n + 1, 0);
    d->bcol.clear();
    d->map.clear();
    std::vector<std::pair<int, int>> ent;
    for (int i = 0; i < n; ++i) {
      const int r = d->p[i];
      ent.clear();
      for (int q = row[r]; q < row[r + 1]; ++q) ent.push_back({pinv[col[q]], q});
      std::sort(ent.begin(), ent.end());
      for (const auto& e : ent) {
        d->bcol.push_back(e.first);
        d->map.push_back(e.second);
      }
      d->brow[i + 1] = (int)d->bcol.size();
    }
    if (d->info) cusolverSpDestroyCsrluInfoHost(d->info);
    cusolverSpCreateCsrluInfoHost(&d->info);
    cusolverStatus_t s2 = cusolverSpXcsrluAnalysisHost(h->sp, n, A->nnz, d->descr, d->brow.data(), d->bcol.data(), d->info);
    s = s2;
    if (s != CUSOLVER_STATUS_SUCCESS) return fail(d, "symbolic LU", (int)s);
    d->aval.resize(A->nnz);
    d->bval.assign(A->nnz, 0.0);
    size_t internal = 0, work = 0;
    s = cusolverSpDcsrluBufferInfoHost(h->sp, n, A->nnz, d->descr, d->bval.data(), d->brow.data(), d->bcol.data(),
                                       d->info, &internal, &work);
    if (s != CUSOLVER_STATUS_SUCCESS) return fail(d, "LU workspace", (int)s);
    d->buffer.assign(work + 16, 0);
    d->factored = false;
    return CUDSS_STATUS_SUCCESS;
  }
  if (phase == CUDSS_PHASE_FACTORIZATION || phase == CUDSS_PHASE_REFACTORIZATION) {
    if (d->n != n || d->nnz != A->nnz) return fail(d, "factorization before analysis", -3);
    cudaDeviceSynchronize();
    if (cudaMemcpy(d->aval.data(), A->vals, sizeof(double) * A->nnz, cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(d, "value copy", -2);
    for (int i = 0; i < A->nnz; ++i) d->bval[i] = d->aval[d->map[i]];
    // the reference's first factorization (bdf_run, before any step) is of A with
    // alpha = -h / 0 (order 0): non-finite values; its first step refactorises with the
    // step's alpha before solving.  Like the library call, accept it and factor nothing.
    for (int i = 0; i < A->nnz; ++i)
      if (!std::isfinite(d->bval[i])) {
        d->factored = false;
        return CUDSS_STATUS_SUCCESS;
      }
    cusolverStatus_t s = cusolverSpDcsrluFactorHost(h->sp, n, A->nnz, d->descr, d->bval.data(), d->brow.data(),
                                                    d->bcol.data(), d->info, 1.0, d->buffer.data());
    if (s != CUSOLVER_STATUS_SUCCESS) return fail(d, "numeric LU", (int)s);
    int pos = -1;
    cusolverSpDcsrluZeroPivotHost(h->sp, d->info, 0.0, &pos);
    if (pos >= 0) std::fprintf(stderr, "cudss stand-in: zero pivot at %d\n", pos);
    d->factored = true;
    return CUDSS_STATUS_SUCCESS;
  }
  if (phase == CUDSS_PHASE_SOLVE) {
    if (!d->factored || !x || !b) return fail(d, "solve before factorization", -4);
    cudaDeviceSynchronize();
    d->rhs.resize(n);
    d->xp.resize(n);
    d->x.resize(n);
    if (cudaMemcpy(d->x.data(), b->dn, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(d, "right-hand side copy", -2);
    for (int i = 0; i < n; ++i) d->rhs[i] = d->x[d->p[i]];
    cusolverStatus_t s = cusolverSpDcsrluSolveHost(h->sp, n, d->rhs.data(), d->xp.data(), d->info, d->buffer.data());
    if (s != CUSOLVER_STATUS_SUCCESS) return fail(d, "LU solve", (int)s);
    d->bsave = d->x;
    for (int i = 0; i < n; ++i) d->x[d->p[i]] = d->xp[i];
    // max-norm residual of A x = b (a wrong solve would otherwise only show as failed
    // Newton iterations)
    double rn = 0.0, bn = 0.0;
    for (int i = 0; i < n; ++i) {
      double acc = -d->bsave[i];
      for (int q = d->arow[i]; q < d->arow[i + 1]; ++q) acc += d->aval[q] * d->x[d->acol[q]];
      rn = std::fmax(rn, std::fabs(acc));
      bn = std::fmax(bn, std::fabs(d->bsave[i]));
    }
    if (rn > 1e-8 * (bn > 0 ? bn : 1.0)) {
      std::fprintf(stderr, "cudss stand-in: solve residual %.3e (max |b| %.3e)\n", rn, bn);
      return fail(d, "LU solve (residual)", -5);
    }
    if (cudaMemcpy(x->dn, d->x.data(), sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(d, "solution copy", -2);
    return CUDSS_STATUS_SUCCESS;
  }
  return fail(d, "phase", (int)phase);
}

}  // extern "C"
