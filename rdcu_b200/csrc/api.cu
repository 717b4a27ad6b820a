// C ABI of librdcu (include/rdcu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/rdcu.h"
#include "adjoint.h"
#include "bdf.h"
#include "dp45.h"
#include "ensemble.h"
#include "fd.h"
#include "spectral.h"

using namespace rdcu;

struct rdcu_handle {
  rdcu_spec spec{};
  std::vector<HostTerm> terms;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  long long N = 0, nN = 0;
  int nY = 0;
  // DP45 (pseudospectral)
  std::unique_ptr<SpectralPlan> sp;
  std::unique_ptr<DP45Engine> dp;
  std::unique_ptr<AdjointEngine> adj;  // created by the first rdcu_adjoint_forward
  // BDF (finite differences)
  std::unique_ptr<FDProblem> fd;
  std::unique_ptr<BDFEngine> bdf;
  long long last_accepted = 0, last_attempts = 0;
  // device staging for host pointers passed to rdcu_rhs / rdcu_jac / rdcu_eval
  double* scr_y = nullptr;
  double* scr_f = nullptr;
  double* scr_Y = nullptr;
  int* scr_rows = nullptr;
  int* scr_cols = nullptr;
  double* scr_vals = nullptr;
  ~rdcu_handle() {
    void* p[] = {scr_y, scr_f, scr_Y, scr_rows, scr_cols, scr_vals};
    for (void* q : p)
      if (q) cudaFree(q);
  }
};

static bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <typename T>
static cudaError_t ensure_scratch(T** p, size_t count) {
  if (*p) return cudaSuccess;
  return cudaMalloc((void**)p, std::max<size_t>(1, count) * sizeof(T));
}

static thread_local std::string g_create_error;

static int set_err(rdcu_t* h, int code, const std::string& msg) {
  if (h)
    h->err = msg;
  else
    g_create_error = msg;
  return code;
}

namespace rdcu {
void set_thread_error(const std::string& msg) { g_create_error = msg; }
}  // namespace rdcu

static int cuda_err(rdcu_t* h, cudaError_t e, const char* where) {
  return set_err(h, RDCU_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CHECK_CUDA(h, x, where)                          \
  do {                                                   \
    cudaError_t _e = (x);                                \
    if (_e != cudaSuccess) return cuda_err(h, _e, where); \
  } while (0)

static int activate(rdcu_t* h) {
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_err(h, e, "cudaSetDevice");
  return RDCU_OK;
}

extern "C" {

const char* rdcu_error_string(int code) {
  switch (code) {
    case RDCU_OK: return "ok";
    case RDCU_ERR_INVALID: return "invalid argument";
    case RDCU_ERR_CUDA: return "CUDA error";
    case RDCU_ERR_UNSUPPORTED: return "unsupported";
    case RDCU_ERR_TIMEOUT: return "timeout";
    case RDCU_ERR_NOMEM: return "out of memory";
    case RDCU_ERR_NUMERIC: return "numerical failure";
    case RDCU_ERR_STATE: return "call out of order";
    case RDCU_ERR_CALLBACK: return "callback aborted";
    default: return "unknown error";
  }
}

const char* rdcu_last_error(rdcu_t* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int rdcu_create(rdcu_t** out, const rdcu_spec* spec) {
  if (!out || !spec) return set_err(nullptr, RDCU_ERR_INVALID, "null argument");
  *out = nullptr;
  if (spec->n < 1) return set_err(nullptr, RDCU_ERR_INVALID, "n must be >= 1");
  if (spec->ndim < 1 || spec->ndim > 3) return set_err(nullptr, RDCU_ERR_INVALID, "ndim must be 1, 2 or 3");
  for (int a = 0; a < spec->ndim; ++a) {
    if (spec->Ns[a] < 1) return set_err(nullptr, RDCU_ERR_INVALID, "grid sizes must be >= 1");
    if (!(spec->Ls[a] > 0) && !(spec->Ls[a] < 0))
      return set_err(nullptr, RDCU_ERR_INVALID, "domain lengths must be nonzero");
  }
  if (spec->nterms < 0 || (spec->nterms > 0 && (!spec->C || !spec->nprods || !spec->c)))
    return set_err(nullptr, RDCU_ERR_INVALID, "bad coupling-term arrays");
  if (spec->method != RDCU_METHOD_DP45 && spec->method != RDCU_METHOD_BDF)
    return set_err(nullptr, RDCU_ERR_INVALID, "unknown method");
  std::unique_ptr<rdcu_handle> h(new rdcu_handle);
  h->spec = *spec;
  h->spec.C = nullptr;
  h->spec.nprods = nullptr;
  h->spec.c = nullptr;
  h->device = spec->device;
  h->N = 1;
  for (int a = 0; a < spec->ndim; ++a) h->N *= spec->Ns[a];
  h->nN = h->N * spec->n;
  h->nY = 1 + spec->ndim + spec->ndim * spec->ndim;
  for (int i = 0; i < spec->nterms; ++i) {
    HostTerm t;
    t.C = spec->C[i];
    const int np = spec->nprods[i];
    if (np < 0 || (np > 0 && !spec->c[i])) return set_err(nullptr, RDCU_ERR_INVALID, "bad coupling term list");
    t.ints.assign(spec->c[i], spec->c[i] + np);
    const int field = np > 0 ? t.ints[0] : 0;
    if (field < 0 || field >= spec->n)
      return set_err(nullptr, RDCU_ERR_INVALID, "coupling term " + std::to_string(i) + ": field out of range");
    for (int j = 1; j < np; j += 2)
      if (t.ints[j] < 0 || t.ints[j] >= h->nY * spec->n)
        return set_err(nullptr, RDCU_ERR_INVALID,
                       "coupling term " + std::to_string(i) + ": Y index " + std::to_string(t.ints[j]) +
                           " out of range");
    h->terms.push_back(std::move(t));
  }
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return set_err(nullptr, RDCU_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return set_err(nullptr, RDCU_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
  std::string msg;
  if (spec->method == RDCU_METHOD_DP45) {
    h->sp.reset(new SpectralPlan);
    if (!h->sp->init(spec->n, spec->ndim, spec->Ns, spec->Ls, h->terms, &msg)) {
      const int code = msg.find("memory") != std::string::npos ? RDCU_ERR_NOMEM : RDCU_ERR_UNSUPPORTED;
      cudaStreamDestroy(h->stream);
      return set_err(nullptr, code, msg);
    }
    h->dp.reset(new DP45Engine);
    if (!h->dp->init(h->sp.get(), spec->atol, spec->rtol, spec->fixed, h->stream, &msg)) {
      cudaStreamDestroy(h->stream);
      return set_err(nullptr, RDCU_ERR_NOMEM, msg);
    }
  } else {
    h->fd.reset(new FDProblem);
    if (!h->fd->init(spec->n, spec->ndim, spec->Ns, spec->Ls, h->terms, h->stream, &msg)) {
      cudaStreamDestroy(h->stream);
      return set_err(nullptr, msg.find("memory") != std::string::npos ? RDCU_ERR_NOMEM : RDCU_ERR_UNSUPPORTED, msg);
    }
    h->bdf.reset(new BDFEngine);
    if (!h->bdf->init(h->fd.get(), spec->atol, spec->rtol, spec->fixed, h->stream, &msg)) {
      cudaStreamDestroy(h->stream);
      return set_err(nullptr, msg.find("memory") != std::string::npos ? RDCU_ERR_NOMEM : RDCU_ERR_UNSUPPORTED, msg);
    }
  }
  // The set-up uploads its tables with cudaMemcpy from pageable host memory, which can
  // return before the copy has landed; the handle's stream is non-blocking, so nothing
  // orders its first launches after those copies.  Wait for the device here.
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaStreamDestroy(h->stream);
    return set_err(nullptr, RDCU_ERR_CUDA, std::string("set-up: ") + cudaGetErrorString(e));
  }
  *out = h.release();
  return RDCU_OK;
}

int rdcu_destroy(rdcu_t* h) {
  if (!h) return RDCU_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  h->adj.reset();
  h->dp.reset();
  h->sp.reset();
  h->bdf.reset();
  h->fd.reset();
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return RDCU_OK;
}

int rdcu_get_info(rdcu_t* h, rdcu_info* info) {
  if (!h || !info) return set_err(h, RDCU_ERR_INVALID, "null argument");
  std::memset(info, 0, sizeof(*info));
  info->state_len = h->nN;
  info->Y_len = h->nN * h->nY;
  info->stream = (void*)h->stream;
  if (h->sp) {
    info->n_channels = h->sp->nch;
    info->device_bytes = (long long)(h->sp->device_bytes + h->dp->device_bytes);
    info->nnz_max = 0;
  } else {
    info->nnz_max = h->fd->nnz;
    info->order = h->bdf->order();
    info->device_bytes = (long long)(h->fd->device_bytes + h->bdf->device_bytes);
  }
  return RDCU_OK;
}

int rdcu_set_state(rdcu_t* h, double t, double hstep, const double* y, int order, const double* D) {
  if (!h || !y) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (int rc = activate(h)) return rc;
  if (h->dp) {
    CHECK_CUDA(h, h->dp->set_state(t, hstep, y), "rdcu_set_state");
    return RDCU_OK;
  }
  if (order < 0 || order > 5 || (order > 0 && !D)) return set_err(h, RDCU_ERR_INVALID, "bad BDF order or D");
  CHECK_CUDA(h, h->bdf->set_state(t, hstep, y, order, D), "rdcu_set_state");
  return RDCU_OK;
}

int rdcu_get_state(rdcu_t* h, double* t, double* hstep, int* order, double* y, double* D) {
  if (!h) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (int rc = activate(h)) return rc;
  if (h->dp) {
    CHECK_CUDA(h, h->dp->get_state(t, hstep, y, cudaMemcpyDefault), "rdcu_get_state");
    if (order) *order = 0;
    return RDCU_OK;
  }
  CHECK_CUDA(h, h->bdf->get_state(t, hstep, order, y, D), "rdcu_get_state");
  return RDCU_OK;
}

int rdcu_rhs(rdcu_t* h, double t, const double* y, double* f, double* Y) {
  (void)t;  // the dictionary is autonomous (dydt ignores t, rdcu.cu:167-184)
  if (!h || !y || !f) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (int rc = activate(h)) return rc;
  const size_t sb = (size_t)h->nN * sizeof(double);
  const size_t Yb = (size_t)h->nN * h->nY * 2 * sizeof(double);
  const double* yd = y;
  double* fd = f;
  double* Yd = Y;
  if (!is_device_ptr(y)) {
    CHECK_CUDA(h, ensure_scratch(&h->scr_y, (size_t)h->nN), "rdcu_rhs staging");
    CHECK_CUDA(h, cudaMemcpyAsync(h->scr_y, y, sb, cudaMemcpyHostToDevice, h->stream), "rdcu_rhs");
    yd = h->scr_y;
  }
  const bool f_host = !is_device_ptr(f);
  if (f_host) {
    CHECK_CUDA(h, ensure_scratch(&h->scr_f, (size_t)h->nN), "rdcu_rhs staging");
    fd = h->scr_f;
  }
  const bool Y_host = Y && !is_device_ptr(Y);
  if (Y_host) {
    CHECK_CUDA(h, ensure_scratch(&h->scr_Y, (size_t)h->nN * h->nY * 2), "rdcu_rhs staging");
    Yd = h->scr_Y;
  }
  if (h->sp) {
    RhsIO io{};
    io.mode = 0;
    io.y = yd;
    io.f = fd;
    CHECK_CUDA(h, h->sp->run(io, h->stream), "rdcu_rhs");
    if (Yd) CHECK_CUDA(h, h->sp->run_Y(yd, Yd, h->stream), "rdcu_rhs (Y)");
  } else {
    CHECK_CUDA(h, h->fd->rhs(yd, fd, Yd), "rdcu_rhs");
  }
  if (f_host) CHECK_CUDA(h, cudaMemcpyAsync(f, fd, sb, cudaMemcpyDeviceToHost, h->stream), "rdcu_rhs");
  if (Y_host) CHECK_CUDA(h, cudaMemcpyAsync(Y, Yd, Yb, cudaMemcpyDeviceToHost, h->stream), "rdcu_rhs");
  CHECK_CUDA(h, cudaStreamSynchronize(h->stream), "rdcu_rhs");
  if (h->sp && h->sp->take_pipe_error())
    return set_err(h, RDCU_ERR_CUDA, "rdcu_rhs: a tile pass gave up waiting for its copies");
  return RDCU_OK;
}

int rdcu_jac(rdcu_t* h, double t, const double* y, int* nnz, int* rows, int* cols, double* vals) {
  (void)t;
  if (!h || !y || !nnz || !rows) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (int rc = activate(h)) return rc;
  const size_t rb = (size_t)(h->nN + 1) * sizeof(int);
  if (h->sp) {
    // no stencils without -S: the reference's jac then assembles nothing
    if (is_device_ptr(rows))
      CHECK_CUDA(h, cudaMemsetAsync(rows, 0, rb, h->stream), "rdcu_jac");
    else
      std::memset(rows, 0, rb);
    CHECK_CUDA(h, cudaStreamSynchronize(h->stream), "rdcu_jac");
    *nnz = 0;
    return RDCU_OK;
  }
  if (!cols || !vals) return set_err(h, RDCU_ERR_INVALID, "null argument");
  const double* yd = y;
  if (!is_device_ptr(y)) {
    CHECK_CUDA(h, ensure_scratch(&h->scr_y, (size_t)h->nN), "rdcu_jac staging");
    CHECK_CUDA(h, cudaMemcpyAsync(h->scr_y, y, (size_t)h->nN * sizeof(double), cudaMemcpyHostToDevice, h->stream),
               "rdcu_jac");
    yd = h->scr_y;
  }
  CHECK_CUDA(h, h->fd->jac_values(yd), "rdcu_jac");
  const size_t nz = (size_t)h->fd->nnz;
  CHECK_CUDA(h, cudaMemcpyAsync(rows, h->fd->rows_, rb, cudaMemcpyDefault, h->stream), "rdcu_jac");
  if (nz) {
    CHECK_CUDA(h, cudaMemcpyAsync(cols, h->fd->cols_, nz * sizeof(int), cudaMemcpyDefault, h->stream), "rdcu_jac");
    CHECK_CUDA(h, cudaMemcpyAsync(vals, h->fd->vals_, nz * sizeof(double), cudaMemcpyDefault, h->stream), "rdcu_jac");
  }
  CHECK_CUDA(h, cudaStreamSynchronize(h->stream), "rdcu_jac");
  *nnz = (int)nz;
  return RDCU_OK;
}

int rdcu_step(rdcu_t* h, double* t, double* hstep, double hmin, double hmax, int* accepted) {
  if (!h || !t || !hstep || !accepted) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (int rc = activate(h)) return rc;
  if (h->dp) {
    CHECK_CUDA(h, h->dp->step(t, hstep, hmin, hmax, accepted), "rdcu_step");
    return RDCU_OK;
  }
  int st = 0;
  CHECK_CUDA(h, h->bdf->step(t, hstep, hmin, hmax, accepted, &st), "rdcu_step");
  if (st) return set_err(h, st, h->bdf->last_msg);
  return RDCU_OK;
}

int rdcu_eval(rdcu_t* h, double t_eval, double* y_eval) {
  if (!h || !y_eval) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (int rc = activate(h)) return rc;
  const bool host = !is_device_ptr(y_eval);
  double* out = y_eval;
  if (host) {
    CHECK_CUDA(h, ensure_scratch(&h->scr_f, (size_t)h->nN), "rdcu_eval staging");
    out = h->scr_f;
  }
  if (h->dp) {
    if (h->dp->host_ctl.n_accepted == 0) return set_err(h, RDCU_ERR_STATE, "rdcu_eval needs an accepted step");
    if (!h->dp->host_ctl.accepted)
      return set_err(h, RDCU_ERR_STATE, "rdcu_eval after a rejected attempt: the stage slopes are overwritten");
    CHECK_CUDA(h, h->dp->eval(t_eval, out), "rdcu_eval");
  } else {
    CHECK_CUDA(h, h->bdf->eval(t_eval, out), "rdcu_eval");
  }
  if (host)
    CHECK_CUDA(h, cudaMemcpy(y_eval, out, (size_t)h->nN * sizeof(double), cudaMemcpyDeviceToHost), "rdcu_eval");
  return RDCU_OK;
}

int rdcu_memcpy(rdcu_t* h, void* dst, const void* src, unsigned long long bytes) {
  if (!h || (!dst && bytes) || (!src && bytes)) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (int rc = activate(h)) return rc;
  if (bytes) {
    CHECK_CUDA(h, cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDefault, h->stream), "rdcu_memcpy");
    CHECK_CUDA(h, cudaStreamSynchronize(h->stream), "rdcu_memcpy");
  }
  return RDCU_OK;
}

int rdcu_solve(rdcu_t* h, double t1, double hmin, double hmax, const double* t_eval, int n_eval,
               rdcu_out_cb cb, void* user) {
  if (!h || n_eval < 0 || (n_eval > 0 && !t_eval)) return set_err(h, RDCU_ERR_INVALID, "bad argument");
  if (int rc = activate(h)) return rc;
  std::vector<double> te(t_eval, t_eval + n_eval);
  int order_now = 0;
  auto on_attempt = [&](double t, double hh, int acc, long long steps) -> int {
    if (!cb) return 0;
    rdcu_event ev{};
    ev.kind = RDCU_EV_ATTEMPT;
    ev.accepted = acc;
    ev.steps = (int)steps;
    ev.t = t;
    ev.h = hh;
    ev.order = h->bdf ? h->bdf->order() : 0;
    return cb(user, &ev);
  };
  double ev_t = 0, ev_h = 0;
  long long ev_steps = 0;
  auto on_eval = [&](int idx, const double* ye) -> int {
    if (!cb) return 0;
    rdcu_event ev{};
    ev.kind = RDCU_EV_EVAL;
    ev.eval_index = idx;
    ev.t_eval = te[idx];
    ev.y = ye;
    if (h->dp) {
      ev.t = h->dp->host_ctl.t;
      ev.h = h->dp->host_ctl.h;
    } else {
      ev.t = h->bdf->t();
      ev.h = h->bdf->h();
      ev.order = h->bdf->order();
    }
    return cb(user, &ev);
  };
  auto on_ckpt = [&](double t, double hh, long long steps) -> int {
    if (!cb) return 0;
    rdcu_event ev{};
    ev.kind = RDCU_EV_CHECKPOINT;
    ev.t = t;
    ev.h = hh;
    ev.steps = (int)steps;
    if (h->dp) {
      ev.y = h->dp->bufs.ybuf[h->dp->host_ctl.y_slot];
    } else {
      ev.y = h->bdf->D_ptr();
      ev.order = h->bdf->order();
    }
    return cb(user, &ev);
  };
  (void)order_now;
  (void)ev_t;
  (void)ev_h;
  (void)ev_steps;
  int cbst = 0;
  if (h->dp) {
    CHECK_CUDA(h, h->dp->solve(t1, hmin, hmax, te, on_attempt, on_eval, on_ckpt, &cbst), "rdcu_solve");
    h->last_accepted = h->dp->solve_accepted;
    h->last_attempts = h->dp->solve_attempts;
  } else {
    int st = 0;
    CHECK_CUDA(h, h->bdf->solve(t1, hmin, hmax, te, on_attempt, on_eval, on_ckpt, &cbst, &st), "rdcu_solve");
    h->last_accepted = h->bdf->solve_accepted;
    h->last_attempts = h->bdf->solve_attempts;
    if (st) return set_err(h, st, h->bdf->last_msg);
  }
  if (cbst) return set_err(h, RDCU_ERR_CALLBACK, "output callback returned " + std::to_string(cbst));
  return RDCU_OK;
}

int rdcu_advance(rdcu_t* h, int n_attempts, double hmin, double hmax, long long* accepted) {
  if (!h || n_attempts < 0) return set_err(h, RDCU_ERR_INVALID, "bad argument");
  if (!h->dp) return set_err(h, RDCU_ERR_UNSUPPORTED, "rdcu_advance is implemented for DP45 handles");
  if (int rc = activate(h)) return rc;
  long long acc = 0;
  CHECK_CUDA(h, h->dp->advance(n_attempts, hmin, hmax, &acc), "rdcu_advance");
  if (accepted) *accepted = acc;
  return RDCU_OK;
}

int rdcu_random_ic(double* y, int n, long long N, double A, double A0, int seed) {
  if (!y || n < 1 || N < 1) return set_err(nullptr, RDCU_ERR_INVALID, "bad argument");
  srand(seed);
  for (int i = 0; i < n; i++)
    for (long long j = 0; j < N; j++) y[N * i + j] = A0 + A / 2 * (2.0 / RAND_MAX * rand() - 1);
  return RDCU_OK;
}

int rdcu_profile_passes(rdcu_t* h, int reps, rdcu_pass_timing* out, int max_passes, int* npass) {
  if (!h || !out || !npass || reps < 1) return set_err(h, RDCU_ERR_INVALID, "bad argument");
  if (!h->dp) return set_err(h, RDCU_ERR_UNSUPPORTED, "pass profiling is implemented for DP45 handles");
  if (int rc = activate(h)) return rc;
  std::vector<SpectralPlan::PassTime> pt;
  CHECK_CUDA(h, h->dp->profile(reps, &pt), "rdcu_profile_passes");
  const int m = std::min((int)pt.size(), max_passes);
  for (int i = 0; i < m; ++i) {
    out[i].name = pt[i].name;
    out[i].ms = pt[i].ms;
    out[i].bytes = pt[i].bytes;
  }
  *npass = m;
  return RDCU_OK;
}

int rdcu_get_counters(rdcu_t* h, long long* accepted, long long* attempts) {
  if (!h) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (accepted) *accepted = h->last_accepted;
  if (attempts) *attempts = h->last_attempts;
  return RDCU_OK;
}

int rdcu_get_linear_stats(rdcu_t* h, long long* iterations, long long* solves, long long* cycles) {
  if (!h) return set_err(h, RDCU_ERR_INVALID, "null argument");
  const BDFEngine* b = h->bdf.get();
  if (iterations) *iterations = b ? b->lin_iters : 0;
  if (solves) *solves = b ? b->lin_solves : 0;
  if (cycles) *cycles = b ? b->lin_cycles : 0;
  return RDCU_OK;
}

int rdcu_set_coefficients(rdcu_t* h, const double* C) {
  if (!h || (!C && !h->terms.empty())) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (!h->sp) return set_err(h, RDCU_ERR_UNSUPPORTED, "coefficients can be replaced on pseudospectral handles");
  if (int rc = activate(h)) return rc;
  std::vector<double> c(C, C + h->terms.size());
  for (size_t i = 0; i < c.size(); ++i) {
    if (!std::isfinite(c[i])) return set_err(h, RDCU_ERR_INVALID, "coefficients must be finite");
    h->terms[i].C = c[i];
  }
  CHECK_CUDA(h, cudaStreamSynchronize(h->stream), "rdcu_set_coefficients");
  CHECK_CUDA(h, h->sp->set_coefficients(c), "rdcu_set_coefficients");
  if (h->adj) CHECK_CUDA(h, h->adj->set_coefficients(c), "rdcu_set_coefficients");
  // the new tables went up with cudaMemcpy (see rdcu_create)
  CHECK_CUDA(h, cudaDeviceSynchronize(), "rdcu_set_coefficients");
  h->dp->invalidate_k1();
  return RDCU_OK;
}

int rdcu_adjoint_forward(rdcu_t* h, const double* y0, const double* hs, int nsteps, int K, double* yT) {
  if (!h || !y0 || (!hs && nsteps > 0) || nsteps < 0 || K < 1) return set_err(h, RDCU_ERR_INVALID, "bad argument");
  if (!h->sp) return set_err(h, RDCU_ERR_UNSUPPORTED, "the adjoint is implemented for pseudospectral DP45 handles");
  if (!h->spec.fixed) return set_err(h, RDCU_ERR_STATE, "the adjoint needs a handle created with fixed = 1");
  for (int j = 0; j < nsteps; ++j)
    if (!(hs[j] > 0) || !std::isfinite(hs[j])) return set_err(h, RDCU_ERR_INVALID, "step sizes must be positive and finite");
  if (int rc = activate(h)) return rc;
  if (!h->adj) {
    std::string msg;
    std::unique_ptr<AdjointEngine> a(new AdjointEngine);
    if (!a->init(h->sp.get(), h->dp.get(), h->terms, h->spec.n, h->spec.ndim, h->spec.Ns, h->spec.Ls, h->stream,
                 &msg))
      return set_err(h, msg.find("memory") != std::string::npos ? RDCU_ERR_NOMEM : RDCU_ERR_UNSUPPORTED, msg);
    h->adj = std::move(a);
    // its tables were uploaded with cudaMemcpy (see rdcu_create)
    CHECK_CUDA(h, cudaDeviceSynchronize(), "rdcu_adjoint_forward set-up");
  }
  CHECK_CUDA(h, h->adj->forward(y0, hs, nsteps, K, yT), "rdcu_adjoint_forward");
  return RDCU_OK;
}

int rdcu_adjoint_backward(rdcu_t* h, const double* lambdaT, double* grad_y0, double* grad_C) {
  if (!h || !lambdaT) return set_err(h, RDCU_ERR_INVALID, "null argument");
  if (!h->adj || !h->adj->recorded()) return set_err(h, RDCU_ERR_STATE, "rdcu_adjoint_forward has not run");
  if (int rc = activate(h)) return rc;
  CHECK_CUDA(h, h->adj->backward(lambdaT, grad_y0, grad_C), "rdcu_adjoint_backward");
  return RDCU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------- ensembles
struct rdcu_ensemble {
  EnsembleEngine eng;
  cudaStream_t stream = nullptr;
  int device = 0;
  std::string err;
};

static thread_local std::string g_ens_create_error;

static int ens_err(rdcu_ensemble_t* e, int code, const std::string& msg) {
  if (e)
    e->err = msg;
  else
    g_ens_create_error = msg;
  return code;
}

#define ENS_CUDA(e, x, where)                                                                            \
  do {                                                                                                   \
    cudaError_t _c = (x);                                                                                \
    if (_c != cudaSuccess) return ens_err(e, RDCU_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(_c)); \
  } while (0)

extern "C" {

int rdcu_ensemble_create(rdcu_ensemble_t** out, const rdcu_spec* specs, int count) {
  if (!out || !specs || count < 1) return ens_err(nullptr, RDCU_ERR_INVALID, "bad argument");
  *out = nullptr;
  std::vector<EnsembleProblem> probs(count);
  const int dev = specs[0].device;
  for (int i = 0; i < count; ++i) {
    const rdcu_spec& s = specs[i];
    const std::string who = "member " + std::to_string(i) + ": ";
    if (s.method != RDCU_METHOD_DP45 || s.ndim != 2 || s.fixed)
      return ens_err(nullptr, RDCU_ERR_UNSUPPORTED, who + "ensembles take adaptive 2D DP45 problems");
    if (s.device != dev) return ens_err(nullptr, RDCU_ERR_INVALID, who + "all members must use one device");
    if (s.n < 1 || s.Ns[0] < 1 || s.Ns[1] < 1 || !(s.Ls[0] != 0) || !(s.Ls[1] != 0))
      return ens_err(nullptr, RDCU_ERR_INVALID, who + "bad n, grid or lengths");
    if (s.nterms < 0 || (s.nterms > 0 && (!s.C || !s.nprods || !s.c)))
      return ens_err(nullptr, RDCU_ERR_INVALID, who + "bad coupling-term arrays");
    EnsembleProblem& p = probs[i];
    p.n = s.n;
    p.Ns[0] = s.Ns[0];
    p.Ns[1] = s.Ns[1];
    p.Ls[0] = s.Ls[0];
    p.Ls[1] = s.Ls[1];
    const int nY = 1 + 2 + 4;
    for (int k = 0; k < s.nterms; ++k) {
      HostTerm t;
      t.C = s.C[k];
      const int np = s.nprods[k];
      if (np < 0 || (np > 0 && !s.c[k])) return ens_err(nullptr, RDCU_ERR_INVALID, who + "bad coupling term list");
      t.ints.assign(s.c[k], s.c[k] + np);
      const int field = np > 0 ? t.ints[0] : 0;
      if (field < 0 || field >= s.n) return ens_err(nullptr, RDCU_ERR_INVALID, who + "field out of range");
      for (int j = 1; j < np; j += 2)
        if (t.ints[j] < 0 || t.ints[j] >= nY * s.n) return ens_err(nullptr, RDCU_ERR_INVALID, who + "Y index out of range");
      p.terms.push_back(std::move(t));
    }
  }
  std::unique_ptr<rdcu_ensemble> e(new rdcu_ensemble);
  e->device = dev;
  cudaError_t c = cudaSetDevice(dev);
  if (c != cudaSuccess) return ens_err(nullptr, RDCU_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(c));
  c = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (c != cudaSuccess) return ens_err(nullptr, RDCU_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(c));
  std::string msg;
  // per-member tolerances: the controllers hold them; the engine takes the first pair
  // and the loop below overrides each member's
  if (!e->eng.init(probs, specs[0].rtol, specs[0].atol, e->stream, &msg)) {
    e->eng.release();
    cudaStreamDestroy(e->stream);
    return ens_err(nullptr, msg.find("memory") != std::string::npos ? RDCU_ERR_NOMEM : RDCU_ERR_UNSUPPORTED, msg);
  }
  for (int i = 0; i < count; ++i) {
    c = e->eng.set_tolerances(i, specs[i].rtol, specs[i].atol);
    if (c != cudaSuccess) {
      e->eng.release();
      cudaStreamDestroy(e->stream);
      return ens_err(nullptr, RDCU_ERR_CUDA, std::string("ensemble tolerances: ") + cudaGetErrorString(c));
    }
  }
  // set-up copies made with cudaMemcpy may still be in flight (see rdcu_create)
  c = cudaDeviceSynchronize();
  if (c != cudaSuccess) {
    e->eng.release();
    cudaStreamDestroy(e->stream);
    return ens_err(nullptr, RDCU_ERR_CUDA, std::string("ensemble set-up: ") + cudaGetErrorString(c));
  }
  *out = e.release();
  return RDCU_OK;
}

int rdcu_ensemble_destroy(rdcu_ensemble_t* e) {
  if (!e) return RDCU_OK;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  e->eng.release();
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return RDCU_OK;
}

int rdcu_ensemble_set_state(rdcu_ensemble_t* e, int i, double t, double hstep, const double* y) {
  if (!e || !y) return ens_err(e, RDCU_ERR_INVALID, "null argument");
  if (i < 0 || i >= e->eng.size()) return ens_err(e, RDCU_ERR_INVALID, "member index out of range");
  ENS_CUDA(e, cudaSetDevice(e->device), "cudaSetDevice");
  ENS_CUDA(e, e->eng.set_state(i, t, hstep, y), "rdcu_ensemble_set_state");
  return RDCU_OK;
}

int rdcu_ensemble_get_state(rdcu_ensemble_t* e, int i, double* t, double* hstep, double* y) {
  if (!e) return ens_err(e, RDCU_ERR_INVALID, "null argument");
  if (i < 0 || i >= e->eng.size()) return ens_err(e, RDCU_ERR_INVALID, "member index out of range");
  ENS_CUDA(e, cudaSetDevice(e->device), "cudaSetDevice");
  ENS_CUDA(e, e->eng.get_state(i, t, hstep, y), "rdcu_ensemble_get_state");
  return RDCU_OK;
}

int rdcu_ensemble_solve(rdcu_ensemble_t* e, double t1, double hmin, double hmax) {
  if (!e) return ens_err(e, RDCU_ERR_INVALID, "null argument");
  ENS_CUDA(e, cudaSetDevice(e->device), "cudaSetDevice");
  ENS_CUDA(e, e->eng.solve(t1, hmin, hmax), "rdcu_ensemble_solve");
  return RDCU_OK;
}

int rdcu_ensemble_counters(rdcu_ensemble_t* e, int i, long long* accepted, long long* attempts) {
  if (!e) return ens_err(e, RDCU_ERR_INVALID, "null argument");
  if (i < 0 || i >= e->eng.size()) return ens_err(e, RDCU_ERR_INVALID, "member index out of range");
  ENS_CUDA(e, cudaSetDevice(e->device), "cudaSetDevice");
  ENS_CUDA(e, e->eng.counters(i, accepted, attempts), "rdcu_ensemble_counters");
  return RDCU_OK;
}

int rdcu_ensemble_tune(rdcu_ensemble_t* e, int* tile_elems) {
  if (!e) return ens_err(e, RDCU_ERR_INVALID, "null argument");
  ENS_CUDA(e, cudaSetDevice(e->device), "cudaSetDevice");
  ENS_CUDA(e, e->eng.tune(nullptr), "rdcu_ensemble_tune");
  if (tile_elems) *tile_elems = e->eng.tile_elems;
  return RDCU_OK;
}

int rdcu_ensemble_info(rdcu_ensemble_t* e, int* count, void** stream, long long* device_bytes) {
  if (!e) return ens_err(e, RDCU_ERR_INVALID, "null argument");
  if (count) *count = e->eng.size();
  if (stream) *stream = (void*)e->stream;
  if (device_bytes) *device_bytes = (long long)e->eng.device_bytes;
  return RDCU_OK;
}

const char* rdcu_ensemble_last_error(rdcu_ensemble_t* e) { return e ? e->err.c_str() : g_ens_create_error.c_str(); }

}  // extern "C"
