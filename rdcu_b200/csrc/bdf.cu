// Variable-order NDF/BDF integrator (ode15s style) on the finite-difference RHS.
//
// The step logic restates bdf_step (reference bdf.cu:135-323) on the host, with every
// vector operation a kernel here: predictor and error scale (step0/errscale,
// bdf.cu:85-101), Newton right-hand side (rhs, bdf.cu:104-113), scaled RMS norms
// (scale_err + cublasDnrm2, bdf.cu:127-132,166,238), the difference updates after an
// accepted step (bdf.cu:262-271), the step-size rescaling of the differences (updateD,
// bdf.cu:72-83, with makeRU bdf.cu:35-69) and dense output (interpolate,
// bdf.cu:115-125).
//
// Linear solves.  The reference factorises A = I + alpha*J with cuDSS (LU, refactorised
// whenever h or the order changes) and solves once per Newton iteration.  cuDSS is not
// available here; A dd = b is solved by restarted GMRES with right preconditioning,
// A applied as dd + alpha*(J dd) on the CSR Jacobian the FD kernels assemble.  The
// preconditioner is the exact inverse of I + alpha*J_lin, J_lin the constant-
// coefficient linear part of the dictionary (diffusion and linear reaction terms):
// the reference's stencils are circulant, so the FFT diagonalises J_lin and each
// Fourier mode is an n x n solve (spectral.cu k_mid_solve).  GMRES runs to a relative
// residual of 1e-12, far below the Newton tolerance, so Newton and step decisions are
// those of an exact solve.  The Newton loop of an attempt, with its linear solves (GMRES
// restarts of up to 40 Arnoldi iterations), is one CUDA graph of nested WHILE nodes
// whose tests run on the device: the host reads back one small record per attempt.  If
// that graph cannot be built, each restart cycle alone is a graph and the host runs
// the Newton and restart loops.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

#include "bdf.h"
#include "spectral.h"

namespace rdcu {
namespace {

// bdf.cu:8-9
const double kKappa[6] = {0.0, -0.1850, -1.0 / 9, -0.0823, -0.0415, 0.0};
const double kGamma[6] = {0.0, 1.0, 1.0 + 1.0 / 2, 1.0 + 1.0 / 2 + 1.0 / 3, 1.0 + 1.0 / 2 + 1.0 / 3 + 1.0 / 4,
                          1.0 + 1.0 / 2 + 1.0 / 3 + 1.0 / 4 + 1.0 / 5};
constexpr int kNwit = 4;  // bdf.cu:23

struct Small {
  double v[36];
};

constexpr int kRedBlocks = 296;
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_reduce(double v) {
  __shared__ double red[kRedThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kRedThreads / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

// step0 + errscale (bdf.cu:93-101, 85-90)
__global__ void k_predict(const double* D, long long nN, int order, double atl, double rtl, double* ytemp,
                          double* yscale) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  double y = D[i];
  for (int j = 1; j <= order; ++j) y += D[nN * j + i];
  ytemp[i] = y;
  if (yscale) yscale[i] = atl + rtl * fabs(y);
}

__global__ void k_errscale(const double* y, long long nN, double atl, double rtl, double* yscale) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nN) yscale[i] = atl + rtl * fabs(y[i]);
}

// rhs kernel (bdf.cu:104-113): b = h/alpha f - sum_j D_j gamma_j/alpha - d
__global__ void k_newton_rhs(double* b, const double* f, const double* d, const double* D, long long nN, int order,
                             double h, double alpha, Small gam) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  double v = h / alpha * f[i];
  for (int j = 1; j <= order; ++j) v -= D[nN * j + i] * gam.v[j] / alpha;
  v -= d[i];
  b[i] = v;
}

// partial sums of (x/yscale)^2 (scale_err + Dnrm2)
__global__ void k_wsq(const double* x, const double* yscale, long long nN, double* part) {
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nN; i += (long long)gridDim.x * blockDim.x) {
    const double v = x[i] / yscale[i];
    s += v * v;
  }
  s = block_reduce(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// dots of w with V[0..nvec) (row blockIdx.y) and, in row nvec, w . w
__global__ void k_dots(const double* V, int nvec, const double* w, long long nN, double* part) {
  const int row = blockIdx.y;
  const double* a = row < nvec ? V + (long long)row * nN : w;
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nN; i += (long long)gridDim.x * blockDim.x)
    s += a[i] * w[i];
  s = block_reduce(s);
  if (threadIdx.x == 0) part[(long long)row * gridDim.x + blockIdx.x] = s;
}

__global__ void k_sum_rows(const double* part, int nrow, int ncol, double* out) {
  const int r = blockIdx.x;
  if (r >= nrow) return;
  double s = 0.0;
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) s += part[(long long)r * ncol + c];
  s = block_reduce(s);
  if (threadIdx.x == 0) out[r] = s;
}

__global__ void k_scale(const double* x, double s, double* y, long long nN) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nN) y[i] = s * x[i];
}

__global__ void k_axpy(double a, const double* x, double* y, long long nN) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nN) y[i] += a * x[i];
}

// r = b - A x
__global__ void k_residual(const int* rows, const int* cols, const double* vals, double alpha, const double* x,
                           const double* b, double* r, long long nN) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  double acc = 0.0;
  for (int p = rows[i]; p < rows[i + 1]; ++p) acc += vals[p] * x[cols[p]];
  r[i] = b[i] - (x[i] + alpha * acc);
}

// ---------------------------------------------------------------- device-resident GMRES
// One restart cycle of GMRES(m) runs as a CUDA graph with a WHILE node (see
// build_cycle_graph).  What changes between iterations and calls lives here, on the
// device: the column j, alpha, the Givens factors, g and the Hessenberg matrix.  The
// scalar update uses round-to-nearest intrinsics without contraction, so every value
// is the one the same recurrence gives on the host.
constexpr int kGmresM = 40;  // restart length m

struct GmresState {
  double alpha;   // A = I + alpha J
  double tol;     // absolute residual target
  double inv_hn;  // 1 / ||w|| of the last column: scale of the next basis vector
  int j;          // column being built
  int jdone;      // columns done
  int total;      // iterations over all cycles of this solve
  int max_total;
  int cont;       // the loop goes on (the next basis vector was formed)
  int conv;
  int guard;      // iterations of this cycle: bounds the loop whatever j does
  int pad;
  double cs[kGmresM], sn[kGmresM], g[kGmresM + 1];
  double H[kGmresM * kGmresM];  // H[k * m + j], k <= j
  double y[kGmresM];            // least-squares solution (back-substitution)
};

__global__ void k_gm_init(GmresState* s, double alpha, double tol, double beta, int total, int max_total) {
  for (int k = threadIdx.x; k <= kGmresM; k += blockDim.x) s->g[k] = k == 0 ? beta : 0.0;
  if (threadIdx.x == 0) {
    s->alpha = alpha;
    s->tol = tol;
    s->inv_hn = 0.0;
    s->j = 0;
    s->jdone = 0;
    s->total = total;
    s->max_total = max_total;
    s->cont = 0;
    s->conv = 0;
    s->guard = 0;
  }
}

// Start of iteration j: for j > 0, V_j = w / ||w|| from the previous iteration (the
// scaling k_scale did); out = V_j, the preconditioner's input.
__global__ void k_gm_take(double* V, const GmresState* s, const double* w, double* out, long long nN) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  const int j = s->j;
  double v;
  if (j > 0) {
    v = s->inv_hn * w[i];
    V[(long long)j * nN + i] = v;
  } else {
    v = V[i];
  }
  out[i] = v;
}

// y = x + alpha * (J x), alpha read on the device: the action of A = I + alpha J
// (csrgeam2 of bdf.cu:153)
__global__ void k_apply_A_dev(const int* rows, const int* cols, const double* vals, const double* alpha,
                              const double* x, double* y, long long nN) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nN) return;
  const double al = *alpha;
  double acc = 0.0;
  for (int p = rows[r]; p < rows[r + 1]; ++p) acc += vals[p] * x[cols[p]];
  y[r] = x[r] + al * acc;
}

// k_dots then k_sum_rows over the j + 1 basis vectors (nvec < 0: j + 1 read on the
// device; rows past it return) in one launch: the last block of each row to finish
// sums that row's partials with the threads and order of k_sum_rows (bitwise the
// same), then clears the row's arrival count.
__global__ void k_dots_sum(const double* V, const GmresState* s, int nvec, const double* w, long long nN,
                           double* part, unsigned int* count, double* out) {
  if (nvec < 0) nvec = s->j + 1;
  const int row = blockIdx.y;
  if (row > nvec) return;
  const double* a = row < nvec ? V + (long long)row * nN : w;
  double sum = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nN; i += (long long)gridDim.x * blockDim.x)
    sum += a[i] * w[i];
  sum = block_reduce(sum);
  __shared__ int last;
  if (threadIdx.x == 0) {
    part[(long long)row * gridDim.x + blockIdx.x] = sum;
    __threadfence();
    last = atomicAdd(&count[row], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (int c = threadIdx.x; c < (int)gridDim.x; c += blockDim.x) t += __ldcg(&part[(long long)row * gridDim.x + c]);
  t = block_reduce(t);
  if (threadIdx.x == 0) {
    out[row] = t;
    count[row] = 0u;
  }
}

__global__ void k_vsub_j(const double* V, const GmresState* s, const double* h, double* w, long long nN) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  const int nvec = s->j + 1;
  double acc = w[i];
  for (int k = 0; k < nvec; ++k) acc -= h[k] * V[(long long)k * nN + i];
  w[i] = acc;
}

// Column j of the Hessenberg matrix from the two Gram-Schmidt passes (dots rows 0 and
// 1, stride `row`) and the norm of w (row 2); Givens rotations; stop test; the loop
// condition.  One thread.
__global__ void k_gm_update(GmresState* s, const double* dots, int row, cudaGraphConditionalHandle cond) {
  if (threadIdx.x != 0) return;
  const int j = s->j;
  double hcol[kGmresM + 1];
  for (int k = 0; k <= j; ++k) hcol[k] = __dadd_rn(__dadd_rn(0.0, dots[k]), dots[row + k]);
  const double hn = sqrt(dots[2 * row]);
  const int total = s->total + 1;
  s->total = total;
  for (int k = 0; k < j; ++k) {
    const double a = __dadd_rn(__dmul_rn(s->cs[k], hcol[k]), __dmul_rn(s->sn[k], hcol[k + 1]));
    hcol[k + 1] = __dadd_rn(__dmul_rn(-s->sn[k], hcol[k]), __dmul_rn(s->cs[k], hcol[k + 1]));
    hcol[k] = a;
  }
  const double den = sqrt(__dadd_rn(__dmul_rn(hcol[j], hcol[j]), __dmul_rn(hn, hn)));
  const double c = den > 0 ? hcol[j] / den : 1.0;
  const double sj = den > 0 ? hn / den : 0.0;
  s->cs[j] = c;
  s->sn[j] = sj;
  hcol[j] = den;
  const double gj = s->g[j];
  s->g[j + 1] = __dmul_rn(-sj, gj);
  s->g[j] = __dmul_rn(c, gj);
  for (int k = 0; k <= j; ++k) s->H[k * kGmresM + j] = hcol[k];
  s->jdone = j + 1;
  const bool met = fabs(s->g[j + 1]) <= s->tol || !(hn > 0);
  const bool stop = met || total >= s->max_total;
  s->conv = met ? 1 : 0;
  const int guard = s->guard + 1;
  s->guard = guard;
  const int cont = (!stop && j + 1 < kGmresM && guard < kGmresM) ? 1 : 0;
  s->cont = cont;
  if (cont) {
    s->inv_hn = 1.0 / hn;
    s->j = j + 1;
  }
  cudaGraphSetConditional(cond, (unsigned int)cont);
}

// back-substitution H y = g over the columns done (one thread)
__global__ void k_gm_backsub(GmresState* s) {
  if (threadIdx.x != 0) return;
  const int jd = s->jdone;
  for (int k = jd - 1; k >= 0; --k) {
    double acc = s->g[k];
    for (int q = k + 1; q < jd; ++q) acc = __dsub_rn(acc, __dmul_rn(s->H[k * kGmresM + q], s->y[q]));
    const double d = s->H[k * kGmresM + k];
    s->y[k] = d != 0 ? acc / d : 0.0;
  }
}

// u = sum_{k < jdone} y_k V_k
__global__ void k_vcomb_j(const double* V, const GmresState* s, double* u, long long nN) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  const int nvec = s->jdone;
  double acc = 0.0;
  for (int k = 0; k < nvec; ++k) acc += s->y[k] * V[(long long)k * nN + i];
  u[i] = acc;
}

// ytemp += dd; d += dd (the two Daxpy of bdf.cu:187-188)
__global__ void k_newton_update(const double* dd, double* ytemp, double* d, long long nN) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  ytemp[i] += dd[i];
  d[i] += dd[i];
}

// updateD (bdf.cu:72-83) in place: Dnew[k] = sum_j RU[(order+1)*j+k] D[j]
__global__ void k_updateD(double* D, long long nN, int order, Small RU) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  double dj[6];
  for (int j = 0; j <= order; ++j) dj[j] = D[nN * j + i];
  for (int k = 0; k <= order; ++k) {
    double val = 0;
    for (int j = 0; j <= order; ++j) val += RU.v[(order + 1) * j + k] * dj[j];
    D[nN * k + i] = val;
  }
}

// accepted step (bdf.cu:262-271): D0 = ytemp; D[k+2] = d - D[k+1]; D[k+1] = d;
// D[i] += D[i+1] for i = k..1
__global__ void k_accept(double* D, const double* d, const double* ytemp, long long nN, int order) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  double Dv[8];
  for (int j = 0; j <= order + 1; ++j) Dv[j] = D[nN * j + i];
  const double di = d[i];
  Dv[0] = ytemp[i];
  Dv[order + 2] = di - Dv[order + 1];
  Dv[order + 1] = di;
  for (int j = order; j >= 1; --j) Dv[j] = Dv[j] + Dv[j + 1];
  for (int j = 0; j <= order + 2; ++j) D[nN * j + i] = Dv[j];
}

// interpolate (bdf.cu:115-125) with the factors computed on the host in the same order
__global__ void k_interp(const double* D, long long nN, int order, Small fac, double* y) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  double v = D[i];
  for (int j = 1; j <= order; ++j) v += D[nN * j + i] * fac.v[j];
  y[i] = v;
}

// ---------------------------------------------------------------- device-resident Newton loop
// The Newton iteration of one attempt (bdf.cu:147-190) runs as one CUDA graph (see
// build_newton_graph): WHILE nodes for the Newton iterations, for the GMRES restarts of
// each linear solve and for the Arnoldi iterations of each restart, with the scalar
// logic -- norms, the rate tests, the restart tests -- in one-thread kernels on this
// record.  After the loop the graph forms the squared error norm of the correction d
// (bdf.cu:231-239).  The host writes the attempt's inputs with k_newton_arm and reads
// the record back once per attempt.
struct NewtonCtl {
  // inputs of the attempt
  double hh;         // step size
  double coef;       // (1 - kappa_k) gamma_k of the order
  double alpha_new;  // -hh / coef: alpha after a refactorisation
  double gam[6];     // gamma_j
  int order;
  int refactor;      // a refactorisation is due (cleared when done)
  // persistent
  double alpha;      // alpha of the current "factorisation"
  // loop state
  double dnorm, dnormold, rate, beta, tol;
  int it, converged, update, restart, proceed, total;
  // results
  double errsq;  // sum of (d / yscale)^2 after the loop
  long long lin_iters, lin_cycles, lin_solves;
};

__global__ void k_newton_arm(NewtonCtl* c, double hh, double coef, double alpha_new, int order, int refactor,
                             Small gam) {
  c->hh = hh;
  c->coef = coef;
  c->alpha_new = alpha_new;
  for (int j = 0; j < 6; ++j) c->gam[j] = gam.v[j];
  c->order = order;
  if (refactor) c->refactor = 1;
  c->lin_iters = 0;
  c->lin_cycles = 0;
  c->lin_solves = 0;
}

// start of the Newton loop (the loop variables of bdf.cu:147-150)
__global__ void k_newton_start(NewtonCtl* c, cudaGraphConditionalHandle cond) {
  c->it = 0;
  c->dnorm = 0.0;
  c->dnormold = 0.0;
  c->rate = 0.0;
  c->converged = 0;
  c->update = 0;
  cudaGraphSetConditional(cond, 1u);
}

// start of an iteration: the refactorisation's alpha (bdf.cu:152-156)
__global__ void k_newton_begin(NewtonCtl* c) {
  if (c->refactor) {
    c->alpha = c->alpha_new;
    c->refactor = 0;
  }
}

// k_newton_rhs with the order, h and coefficients of the record
__global__ void k_newton_rhs_dev(double* b, const double* f, const double* d, const double* D, long long nN,
                                 const NewtonCtl* c) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  const int order = c->order;
  const double h = c->hh, alpha = c->coef;
  double v = h / alpha * f[i];
  for (int j = 1; j <= order; ++j) v -= D[nN * j + i] * c->gam[j] / alpha;
  v -= d[i];
  b[i] = v;
}

// k_wsq then k_sum_rows in one launch (k_dots_sum's last-block pattern, bitwise the
// same sums): out[0] = sum of (x / yscale)^2
__global__ void k_wsq_sum(const double* x, const double* yscale, long long nN, double* part, unsigned int* count,
                          double* out) {
  double sum = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nN; i += (long long)gridDim.x * blockDim.x) {
    const double v = x[i] / yscale[i];
    sum += v * v;
  }
  sum = block_reduce(sum);
  __shared__ int last;
  if (threadIdx.x == 0) {
    part[blockIdx.x] = sum;
    __threadfence();
    last = atomicAdd(count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) t += __ldcg(&part[q]);
  t = block_reduce(t);
  if (threadIdx.x == 0) {
    out[0] = t;
    *count = 0u;
  }
}

// start of a linear solve (gmres): beta0 = ||b||, the tolerance, the restart loop's
// condition (no restart when b = 0: x stays 0)
__global__ void k_solve_begin(NewtonCtl* c, const double* bb, double lin_tol, cudaGraphConditionalHandle cond) {
  const double beta0 = sqrt(bb[0]);
  c->beta = beta0;
  c->tol = lin_tol * beta0;
  c->total = 0;
  c->restart = 0;
  c->proceed = 0;
  c->lin_solves += 1;
  cudaGraphSetConditional(cond, beta0 > 0 ? 1u : 0u);
}

// r = b - A x from the second restart on
__global__ void k_residual_dev(const int* rows, const int* cols, const double* vals, const NewtonCtl* c,
                               const double* x, const double* b, double* r, long long nN) {
  if (c->restart == 0) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  const double alpha = c->alpha;
  double acc = 0.0;
  for (int p = rows[i]; p < rows[i + 1]; ++p) acc += vals[p] * x[cols[p]];
  r[i] = b[i] - (x[i] + alpha * acc);
}

// restart test (beta = ||r|| > tol from the second restart on), V_0 = r / beta and the
// cycle's GMRES state (k_gm_init); the Arnoldi loop runs only when the cycle goes on
__global__ void k_restart_begin(NewtonCtl* c, GmresState* s, const double* rr, int max_total,
                                cudaGraphConditionalHandle cond) {
  if (c->restart > 0) c->beta = sqrt(rr[0]);
  const int proceed = (c->restart == 0 || c->beta > c->tol) ? 1 : 0;
  c->proceed = proceed;
  for (int k = 0; k <= kGmresM; ++k) s->g[k] = k == 0 ? c->beta : 0.0;
  s->alpha = c->alpha;
  s->tol = c->tol;
  s->inv_hn = 0.0;
  s->j = 0;
  s->jdone = 0;
  s->total = c->total;
  s->max_total = max_total;
  s->cont = 0;
  s->conv = 0;
  s->guard = 0;
  if (proceed) c->lin_cycles += 1;
  cudaGraphSetConditional(cond, (unsigned)proceed);
}

// V_0 = (1 / beta) * (b on the first restart, else r)
__global__ void k_scale_dev(const NewtonCtl* c, const double* b, const double* r, double* V, long long nN) {
  if (!c->proceed) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  const double s = 1.0 / c->beta;
  V[i] = s * (c->restart == 0 ? b[i] : r[i]);
}

// end of a restart: iterations so far, convergence, the restart loop's condition
__global__ void k_restart_end(NewtonCtl* c, const GmresState* s, int max_total, cudaGraphConditionalHandle cond) {
  int cont = 0;
  if (c->proceed) {
    c->total = s->total;
    c->restart += 1;
    cont = (!s->conv && c->restart < 50 && c->total < max_total) ? 1 : 0;
  }
  cudaGraphSetConditional(cond, (unsigned)cont);
}

__global__ void k_solve_end(NewtonCtl* c) { c->lin_iters += c->total; }

// Newton convergence tests (bdf.cu:168-183) on ||dd|| (weighted RMS): stop, converge,
// or apply the correction and go on
__global__ void k_newton_ctl(NewtonCtl* c, const double* ss, double sqN, double ntol, int nwit,
                             cudaGraphConditionalHandle cond) {
  const double dnorm = sqrt(ss[0]) / sqN;
  c->dnorm = dnorm;
  const double dnormold = c->dnormold;
  double rate = c->rate;
  if (dnormold > 0) rate = dnorm / dnormold;
  c->rate = rate;
  const int it = c->it;
  bool stop = false;
  if (rate >= 1)
    stop = true;
  else if (pow(rate, (double)(nwit - it)) / (1 - rate) * dnorm > ntol)
    stop = true;
  else if (dnormold > 0 && rate / (1 - rate) * dnorm < ntol) {
    c->converged = 1;
    stop = true;
  }
  int cont = 0;
  c->update = stop ? 0 : 1;
  if (!stop) {
    c->dnormold = dnorm;
    c->it = it + 1;
    cont = it + 1 < nwit ? 1 : 0;
  }
  cudaGraphSetConditional(cond, (unsigned)cont);
}

// ytemp += dd; d += dd when the iteration goes on
__global__ void k_newton_update_dev(const NewtonCtl* c, const double* dd, double* ytemp, double* d, long long nN) {
  if (!c->update) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nN) return;
  ytemp[i] += dd[i];
  d[i] += dd[i];
}

__global__ void k_zero(double* x, long long nN) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nN) x[i] = 0.0;
}

// makeRU (bdf.cu:35-69)
void make_RU(int order, double factor, double* RU) {
  double R[36], U[36];
  double prod;
  for (int i = 0; i <= order; i++)
    for (int j = 0; j <= order; j++) {
      prod = 1.0 / std::max(i, 1);
      for (int k = 0; k < i; k++) prod *= (k - factor * j) / std::max(k, 1);
      R[(order + 1) * i + j] = prod;
    }
  for (int i = 0; i <= order; i++)
    for (int j = 0; j <= order; j++) {
      prod = 1.0 / std::max(i, 1);
      for (int k = 0; k < i; k++) prod *= (k - j) * 1.0 / std::max(k, 1);
      U[(order + 1) * i + j] = prod;
    }
  for (int i = 0; i <= order; i++)
    for (int j = 0; j <= order; j++) {
      RU[(order + 1) * i + j] = 0;
      for (int k = 0; k <= order; k++) RU[(order + 1) * i + j] += R[(order + 1) * i + k] * U[(order + 1) * k + j];
    }
}

}  // namespace

#define RDCU_TRY(x)                   \
  do {                                \
    cudaError_t _e = (x);             \
    if (_e != cudaSuccess) return _e; \
  } while (0)

struct BDFEngine::Impl {
  SpectralPlan prec;
  bool have_prec = false;
  long long nN = 0;
  int blocks = 0;
  double *ytemp = nullptr, *yscale = nullptr, *f = nullptr, *d = nullptr, *dd = nullptr, *b = nullptr;
  double *y_eval = nullptr, *w = nullptr, *z = nullptr, *vj = nullptr, *r = nullptr;
  double* V = nullptr;
  int m = kGmresM;
  double* part = nullptr;   // [(m+2)][kRedBlocks]
  double* dots = nullptr;   // 3 rows of [m+2] (device)
  double* hdots = nullptr;  // pinned
  // the restart cycle as a graph (build_cycle_graph), its device state and a pinned
  // copy of the state's header
  GmresState* gm = nullptr;
  GmresState* gm_host = nullptr;
  unsigned int* arrivals = nullptr;  // per-row block counts of k_dots_sum (zero between launches)
  cudaGraph_t cycle_graph = nullptr;
  cudaGraphExec_t cycle_exec = nullptr;
  double* cycle_x = nullptr;  // the solution vector the graph updates
  // the Newton loop of an attempt as a graph (build_newton_graph), its record and a
  // pinned copy; newton_failed: the graph could not be built (host loop instead)
  NewtonCtl* nctl = nullptr;
  NewtonCtl* nctl_host = nullptr;
  double* ndots = nullptr;  // ||b||^2, ||r||^2, ||dd||^2 (weighted) of the graph
  cudaGraph_t newton_graph = nullptr;
  cudaGraphExec_t newton_exec = nullptr;
  bool newton_failed = false;
  int refactor = 1, rejac = 1;
  double nconststeps = 0;
  double ntol = 0;
  double alpha = 0;  // alpha of the current "factorisation" (bdf.cu:152)
  double atl = 0, rtl = 0;
  int fixed = 0;
  bool jac_ready = false;
  bool started = false;  // bdf_run set-up done for the current state
  double lin_tol = 1e-12;
  int lin_max_iters = 400;
};

static std::vector<LinEntry> linear_part(const FDProblem& fd) {
  std::vector<LinEntry> out;
  const int n = fd.n, ndim = fd.ndim;
  for (const auto& t : fd.terms) {
    const int field = t.ints.empty() ? 0 : t.ints[0];
    int cnt = 0, k = -1, p = 0;
    const int np = (int)t.ints.size();
    for (int j = 1; j < np; j += 2) {
      const int pw = j + 1 < np ? t.ints[j + 1] : 0;
      if (pw != 0) {
        ++cnt;
        k = t.ints[j];
        p = pw;
      }
    }
    if (cnt != 1 || p != 1) continue;
    LinEntry e{};
    e.row = field;
    e.src = k % n;
    const int yind = k / n;
    if (yind == 0) {
      e.nax = 0;
    } else if (yind <= ndim) {
      e.nax = 1;
      e.ax0 = yind - 1;
    } else {
      const int q = yind - ndim - 1;
      e.nax = 2;
      e.ax0 = q / ndim;
      e.ax1 = q % ndim;
    }
    e.coef = t.C;
    out.push_back(e);
  }
  return out;
}

bool BDFEngine::init(FDProblem* fd, double atol, double rtol, int fixed, cudaStream_t st, std::string* msg) {
  release();
  fd_ = fd;
  st_ = st;
  impl_ = new Impl;
  Impl& I = *impl_;
  I.nN = fd->nN;
  I.atl = atol;
  I.rtl = rtol;
  I.fixed = fixed;
  // ntol (bdf.cu:395-401)
  I.ntol = 0.03;
  if (std::pow(rtol, 0.5) < 0.03) I.ntol = std::pow(rtol, 0.5);
  if (10 * std::pow(2, -52) / rtol > I.ntol) I.ntol = 10 * std::pow(2, -52) / (rtol + std::pow(2, -52));
  I.blocks = (int)((I.nN + 255) / 256);
  const size_t sb = (size_t)I.nN * sizeof(double);
  auto fail = [&](const char* what) {
    *msg = std::string("out of device memory (") + what + ")";
    return false;
  };
  if (cudaMalloc((void**)&D_, sb * 8) != cudaSuccess) return fail("BDF differences");
  double** vecs[] = {&I.ytemp, &I.yscale, &I.f, &I.d, &I.dd, &I.b, &I.y_eval, &I.w, &I.z, &I.vj, &I.r};
  for (double** p : vecs)
    if (cudaMalloc((void**)p, sb) != cudaSuccess) return fail("BDF vectors");
  if (cudaMalloc((void**)&I.V, sb * (I.m + 1)) != cudaSuccess) return fail("GMRES basis");
  if (cudaMalloc((void**)&I.part, sizeof(double) * (I.m + 2) * kRedBlocks) != cudaSuccess) return fail("reductions");
  // three rows of m+2: the two Gram-Schmidt passes and the new vector's norm
  if (cudaMalloc((void**)&I.dots, sizeof(double) * 3 * (I.m + 2)) != cudaSuccess) return fail("reductions");
  if (cudaMalloc((void**)&I.gm, sizeof(GmresState)) != cudaSuccess) return fail("GMRES state");
  if (cudaMalloc((void**)&I.arrivals, sizeof(unsigned int) * (I.m + 2)) != cudaSuccess ||
      cudaMemset(I.arrivals, 0, sizeof(unsigned int) * (I.m + 2)) != cudaSuccess)
    return fail("GMRES state");
  if (cudaMallocHost((void**)&I.hdots, sizeof(double) * 3 * (I.m + 2)) != cudaSuccess) return fail("pinned");
  if (cudaMallocHost((void**)&I.gm_host, sizeof(GmresState)) != cudaSuccess) return fail("pinned");
  if (cudaMalloc((void**)&I.nctl, sizeof(NewtonCtl)) != cudaSuccess ||
      cudaMemset(I.nctl, 0, sizeof(NewtonCtl)) != cudaSuccess ||
      cudaMalloc((void**)&I.ndots, sizeof(double) * 4) != cudaSuccess)
    return fail("Newton state");
  if (cudaMallocHost((void**)&I.nctl_host, sizeof(NewtonCtl)) != cudaSuccess) return fail("pinned");
  device_bytes = sb * (8 + 11 + I.m + 1) + fd->device_bytes;
  std::vector<LinEntry> lin = linear_part(*fd);
  if (!lin.empty() && fd->n <= kMaxPrecFields) {
    std::string pm;
    if (I.prec.init_precond(fd->n, fd->ndim, fd->Ns, fd->Ls, lin, &pm)) {
      I.have_prec = true;
      device_bytes += I.prec.device_bytes;
    }
  }
  return true;
}

void BDFEngine::release() {
  if (impl_) {
    Impl& I = *impl_;
    if (I.cycle_exec) cudaGraphExecDestroy(I.cycle_exec);
    if (I.cycle_graph) cudaGraphDestroy(I.cycle_graph);
    if (I.newton_exec) cudaGraphExecDestroy(I.newton_exec);
    if (I.newton_graph) cudaGraphDestroy(I.newton_graph);
    if (I.nctl) cudaFree(I.nctl);
    if (I.ndots) cudaFree(I.ndots);
    if (I.nctl_host) cudaFreeHost(I.nctl_host);
    double* vecs[] = {I.ytemp, I.yscale, I.f, I.d, I.dd, I.b, I.y_eval, I.w, I.z, I.vj, I.r, I.V, I.part, I.dots};
    for (double* p : vecs)
      if (p) cudaFree(p);
    if (I.gm) cudaFree(I.gm);
    if (I.arrivals) cudaFree(I.arrivals);
    if (I.hdots) cudaFreeHost(I.hdots);
    if (I.gm_host) cudaFreeHost(I.gm_host);
    delete impl_;
    impl_ = nullptr;
  }
  if (D_) cudaFree(D_);
  D_ = nullptr;
}

cudaError_t BDFEngine::set_state(double t, double h, const double* y, int order, const double* D) {
  t_ = t;
  h_ = h;
  order_ = order;
  const size_t sb = (size_t)fd_->nN * sizeof(double);
  RDCU_TRY(cudaMemcpyAsync(D_, y, sb, cudaMemcpyDefault, st_));
  if (order > 0 && D) RDCU_TRY(cudaMemcpyAsync(D_ + fd_->nN, D, sb * order, cudaMemcpyDefault, st_));
  RDCU_TRY(cudaStreamSynchronize(st_));
  impl_->refactor = 1;
  impl_->rejac = 1;
  impl_->nconststeps = 0;
  impl_->started = false;
  impl_->jac_ready = false;
  return cudaSuccess;
}

cudaError_t BDFEngine::get_state(double* t, double* h, int* order, double* y, double* D) {
  if (t) *t = t_;
  if (h) *h = h_;
  if (order) *order = order_;
  const size_t sb = (size_t)fd_->nN * sizeof(double);
  if (y) RDCU_TRY(cudaMemcpyAsync(y, D_, sb, cudaMemcpyDefault, st_));
  if (D && order_ > 0) RDCU_TRY(cudaMemcpyAsync(D, D_ + fd_->nN, sb * order_, cudaMemcpyDefault, st_));
  return cudaStreamSynchronize(st_);
}

// ---------------------------------------------------------------- helpers (host)
namespace {

cudaError_t wnorm(BDFEngine::Impl& I, const double* x, cudaStream_t st, double* out) {
  k_wsq<<<kRedBlocks, kRedThreads, 0, st>>>(x, I.yscale, I.nN, I.part);
  k_sum_rows<<<1, kRedThreads, 0, st>>>(I.part, 1, kRedBlocks, I.dots);
  RDCU_TRY(cudaMemcpyAsync(I.hdots, I.dots, sizeof(double), cudaMemcpyDeviceToHost, st));
  RDCU_TRY(cudaStreamSynchronize(st));
  *out = std::sqrt(I.hdots[0]);
  return cudaGetLastError();
}

// dots[0..nvec) = V^T w, dots[nvec] = w.w  (host copy in I.hdots)
cudaError_t vdots(BDFEngine::Impl& I, int nvec, const double* w, cudaStream_t st) {
  dim3 grid(kRedBlocks, nvec + 1);
  k_dots<<<grid, kRedThreads, 0, st>>>(I.V, nvec, w, I.nN, I.part);
  k_sum_rows<<<nvec + 1, kRedThreads, 0, st>>>(I.part, nvec + 1, kRedBlocks, I.dots);
  RDCU_TRY(cudaMemcpyAsync(I.hdots, I.dots, sizeof(double) * (nvec + 1), cudaMemcpyDeviceToHost, st));
  RDCU_TRY(cudaStreamSynchronize(st));
  return cudaGetLastError();
}

}  // namespace

// The GMRES(m) restart cycle as one CUDA graph: a WHILE node whose body is one Arnoldi
// iteration -- V_j = w/||w|| of the previous iteration, z = P^-1 V_j, w = A z, two
// classical Gram-Schmidt passes, ||w||, the Givens update (which clears the loop
// condition on convergence, after m columns or on the iteration limit) -- then the
// back-substitution and x += P^-1 (V y).  No host round trip per iteration: the host
// launches the graph once per cycle and reads back the state's header.
static cudaError_t build_cycle_graph(BDFEngine::Impl& I, const FDProblem& fd, double* x, cudaStream_t st) {
  if (I.cycle_exec) cudaGraphExecDestroy(I.cycle_exec);
  if (I.cycle_graph) cudaGraphDestroy(I.cycle_graph);
  I.cycle_exec = nullptr;
  I.cycle_graph = nullptr;
  const long long nN = I.nN;
  const int nb = I.blocks;
  const int m = I.m;
  const int row = m + 2;
  const double* alpha_dev = &I.gm->alpha;
  cudaGraph_t graph = nullptr;
  RDCU_TRY(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle cond;
  cudaError_t e = cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault);
  cudaGraphNode_t loop = nullptr;
  cudaGraph_t body = nullptr;
  if (e == cudaSuccess) {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&loop, graph, nullptr, 0, &cp);
    if (e == cudaSuccess) body = cp.conditional.phGraph_out[0];
  }
  // one Arnoldi iteration
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t el = cudaSuccess;
    const double* zin = I.have_prec ? I.z : I.vj;
    k_gm_take<<<nb, 256, 0, st>>>(I.V, I.gm, I.w, I.vj, nN);
    if (I.have_prec) el = I.prec.precond(I.vj, I.z, 0.0, alpha_dev, st);
    k_apply_A_dev<<<nb, 256, 0, st>>>(fd.rows_, fd.cols_, fd.vals_, alpha_dev, zin, I.w, nN);
    for (int pass = 0; pass < 2; ++pass) {
      k_dots_sum<<<dim3(kRedBlocks, m + 1), kRedThreads, 0, st>>>(I.V, I.gm, -1, I.w, nN, I.part, I.arrivals,
                                                                  I.dots + pass * row);
      k_vsub_j<<<nb, 256, 0, st>>>(I.V, I.gm, I.dots + pass * row, I.w, nN);
    }
    k_dots_sum<<<dim3(kRedBlocks, 1), kRedThreads, 0, st>>>(I.V, I.gm, 0, I.w, nN, I.part, I.arrivals,
                                                            I.dots + 2 * row);
    k_gm_update<<<1, 32, 0, st>>>(I.gm, I.dots, row, cond);
    if (el == cudaSuccess) el = cudaGetLastError();
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(st, &captured);
    if (e == cudaSuccess) e = el;
  }
  // after the loop: x += P^-1 (V y)
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(st, graph, &loop, nullptr, 1, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t el = cudaSuccess;
    k_gm_backsub<<<1, 32, 0, st>>>(I.gm);
    k_vcomb_j<<<nb, 256, 0, st>>>(I.V, I.gm, I.w, nN);
    if (I.have_prec) {
      el = I.prec.precond(I.w, I.z, 0.0, alpha_dev, st);
      k_axpy<<<nb, 256, 0, st>>>(1.0, I.z, x, nN);
    } else {
      k_axpy<<<nb, 256, 0, st>>>(1.0, I.w, x, nN);
    }
    if (el == cudaSuccess) el = cudaGetLastError();
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(st, &captured);
    if (e == cudaSuccess) e = el;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&I.cycle_exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    I.cycle_exec = nullptr;
    return e;
  }
  I.cycle_graph = graph;
  I.cycle_x = x;
  return cudaSuccess;
}

// Solves (I + alpha J) x = b.  Returns the number of GMRES iterations and restart
// cycles.  The residual norm of each restart is taken on the host; each restart cycle
// is one launch of the cycle graph and one read of its state.
static cudaError_t gmres(BDFEngine::Impl& I, const FDProblem& fd, double alpha, const double* b, double* x,
                         cudaStream_t st, int* iters, int* cycles) {
  const long long nN = I.nN;
  const int nb = I.blocks;
  *iters = 0;
  *cycles = 0;
  RDCU_TRY(vdots(I, 0, b, st));
  const double beta0 = std::sqrt(I.hdots[0]);
  RDCU_TRY(cudaMemsetAsync(x, 0, sizeof(double) * nN, st));
  if (!(beta0 > 0)) return cudaStreamSynchronize(st);
  if (!I.cycle_exec || I.cycle_x != x) RDCU_TRY(build_cycle_graph(I, fd, x, st));
  const double tol = I.lin_tol * beta0;
  const double* r = b;
  double beta = beta0;
  int total = 0;
  for (int restart = 0; restart < 50 && total < I.lin_max_iters; ++restart) {
    if (restart > 0) {
      k_residual<<<nb, 256, 0, st>>>(fd.rows_, fd.cols_, fd.vals_, alpha, x, b, I.r, nN);
      RDCU_TRY(vdots(I, 0, I.r, st));
      beta = std::sqrt(I.hdots[0]);
      if (!(beta > tol)) break;
      r = I.r;
    }
    k_scale<<<nb, 256, 0, st>>>(r, 1.0 / beta, I.V, nN);
    k_gm_init<<<1, 64, 0, st>>>(I.gm, alpha, tol, beta, total, I.lin_max_iters);
    RDCU_TRY(cudaGetLastError());
    RDCU_TRY(cudaGraphLaunch(I.cycle_exec, st));
    ++*cycles;
    RDCU_TRY(cudaMemcpyAsync(I.gm_host, I.gm, offsetof(GmresState, cs), cudaMemcpyDeviceToHost, st));
    RDCU_TRY(cudaStreamSynchronize(st));
    total = I.gm_host->total;
    if (I.gm_host->conv) break;
  }
  *iters = total;
  return cudaGetLastError();
}

// A WHILE node on handle h after the capture's current frontier in graph g (being
// captured on st); the capture continues after it.  *body receives its body graph.
static cudaError_t add_while_node(cudaGraph_t g, cudaStream_t st, cudaGraphConditionalHandle h, cudaGraph_t* body) {
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  RDCU_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &nd));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  RDCU_TRY(cudaGraphAddNode(&node, g, deps, nd, &cp));
  *body = cp.conditional.phGraph_out[0];
  return cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
}

// Captures `fill` into graph g on st.
template <typename F>
static cudaError_t capture_into(cudaGraph_t g, cudaStream_t st, F&& fill) {
  RDCU_TRY(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = fill();
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaGraph_t captured = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(st, &captured);
  return e != cudaSuccess ? e : e2;
}

// The Newton loop of one attempt (bdf.cu:147-190) with its linear solves (gmres above)
// as one graph: Newton WHILE { f = F(ytemp); alpha on refactorisation; b; ||b||; x = 0;
// restart WHILE { r = b - A x and ||r|| (from the second restart); test; V_0; Arnoldi
// WHILE { one iteration, as in build_cycle_graph }; x += P^-1 V y }; ||dd||; tests;
// update }, then yscale at ytemp and ||d||^2 for the error test (bdf.cu:231-239).
static cudaError_t build_newton_graph(BDFEngine::Impl& I, FDProblem& fd, const double* D, cudaStream_t st) {
  const long long nN = I.nN;
  const int nb = I.blocks, m = I.m, row = m + 2;
  const double* alpha_dev = &I.gm->alpha;
  const double sqN = std::pow((double)nN, 0.5);
  double* x = I.dd;
  cudaGraph_t G = nullptr;
  RDCU_TRY(cudaGraphCreate(&G, 0));
  cudaGraphConditionalHandle hn, hr, ha;
  cudaGraph_t Bn = nullptr, Br = nullptr, Ba = nullptr;
  cudaError_t e = cudaGraphConditionalHandleCreate(&hn, G, 0, cudaGraphCondAssignDefault);
  if (e == cudaSuccess)
    e = capture_into(G, st, [&]() -> cudaError_t {
      k_newton_start<<<1, 1, 0, st>>>(I.nctl, hn);
      RDCU_TRY(add_while_node(G, st, hn, &Bn));
      k_errscale<<<nb, 256, 0, st>>>(I.ytemp, nN, I.atl, I.rtl, I.yscale);
      k_wsq_sum<<<kRedBlocks, kRedThreads, 0, st>>>(I.d, I.yscale, nN, I.part, I.arrivals, &I.nctl->errsq);
      return cudaSuccess;
    });
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hr, Bn, 0, cudaGraphCondAssignDefault);
  if (e == cudaSuccess)
    e = capture_into(Bn, st, [&]() -> cudaError_t {
      RDCU_TRY(fd.rhs(I.ytemp, I.f, nullptr));
      k_newton_begin<<<1, 1, 0, st>>>(I.nctl);
      k_newton_rhs_dev<<<nb, 256, 0, st>>>(I.b, I.f, I.d, D, nN, I.nctl);
      k_dots_sum<<<dim3(kRedBlocks, 1), kRedThreads, 0, st>>>(I.V, I.gm, 0, I.b, nN, I.part, I.arrivals, I.ndots);
      k_solve_begin<<<1, 1, 0, st>>>(I.nctl, I.ndots, I.lin_tol, hr);
      k_zero<<<nb, 256, 0, st>>>(x, nN);
      RDCU_TRY(add_while_node(Bn, st, hr, &Br));
      k_solve_end<<<1, 1, 0, st>>>(I.nctl);
      k_wsq_sum<<<kRedBlocks, kRedThreads, 0, st>>>(x, I.yscale, nN, I.part, I.arrivals, I.ndots + 2);
      k_newton_ctl<<<1, 1, 0, st>>>(I.nctl, I.ndots + 2, sqN, I.ntol, kNwit, hn);
      k_newton_update_dev<<<nb, 256, 0, st>>>(I.nctl, x, I.ytemp, I.d, nN);
      return cudaSuccess;
    });
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&ha, Br, 0, cudaGraphCondAssignDefault);
  if (e == cudaSuccess)
    e = capture_into(Br, st, [&]() -> cudaError_t {
      k_residual_dev<<<nb, 256, 0, st>>>(fd.rows_, fd.cols_, fd.vals_, I.nctl, x, I.b, I.r, nN);
      k_dots_sum<<<dim3(kRedBlocks, 1), kRedThreads, 0, st>>>(I.V, I.gm, 0, I.r, nN, I.part, I.arrivals,
                                                              I.ndots + 1);
      k_restart_begin<<<1, 1, 0, st>>>(I.nctl, I.gm, I.ndots + 1, I.lin_max_iters, ha);
      k_scale_dev<<<nb, 256, 0, st>>>(I.nctl, I.b, I.r, I.V, nN);
      RDCU_TRY(add_while_node(Br, st, ha, &Ba));
      k_gm_backsub<<<1, 32, 0, st>>>(I.gm);
      k_vcomb_j<<<nb, 256, 0, st>>>(I.V, I.gm, I.w, nN);
      if (I.have_prec) {
        RDCU_TRY(I.prec.precond(I.w, I.z, 0.0, alpha_dev, st));
        k_axpy<<<nb, 256, 0, st>>>(1.0, I.z, x, nN);
      } else {
        k_axpy<<<nb, 256, 0, st>>>(1.0, I.w, x, nN);
      }
      k_restart_end<<<1, 1, 0, st>>>(I.nctl, I.gm, I.lin_max_iters, hr);
      return cudaSuccess;
    });
  if (e == cudaSuccess)
    e = capture_into(Ba, st, [&]() -> cudaError_t {
      const double* zin = I.have_prec ? I.z : I.vj;
      k_gm_take<<<nb, 256, 0, st>>>(I.V, I.gm, I.w, I.vj, nN);
      if (I.have_prec) RDCU_TRY(I.prec.precond(I.vj, I.z, 0.0, alpha_dev, st));
      k_apply_A_dev<<<nb, 256, 0, st>>>(fd.rows_, fd.cols_, fd.vals_, alpha_dev, zin, I.w, nN);
      for (int pass = 0; pass < 2; ++pass) {
        k_dots_sum<<<dim3(kRedBlocks, m + 1), kRedThreads, 0, st>>>(I.V, I.gm, -1, I.w, nN, I.part, I.arrivals,
                                                                    I.dots + pass * row);
        k_vsub_j<<<nb, 256, 0, st>>>(I.V, I.gm, I.dots + pass * row, I.w, nN);
      }
      k_dots_sum<<<dim3(kRedBlocks, 1), kRedThreads, 0, st>>>(I.V, I.gm, 0, I.w, nN, I.part, I.arrivals,
                                                              I.dots + 2 * row);
      k_gm_update<<<1, 32, 0, st>>>(I.gm, I.dots, row, ha);
      return cudaSuccess;
    });
  if (e == cudaSuccess) e = cudaGraphInstantiate(&I.newton_exec, G, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(G);
    I.newton_exec = nullptr;
    cudaGetLastError();
    return e;
  }
  I.newton_graph = G;
  return cudaSuccess;
}

// bdf_run set-up (bdf.cu:333-374): f and J at D_0; order 0 -> D_1 = h f
static cudaError_t bdf_setup(BDFEngine::Impl& I, FDProblem& fd, double* D, int* order, double h,
                             cudaStream_t st) {
  RDCU_TRY(fd.rhs(D, I.f, nullptr));
  RDCU_TRY(fd.jac_values(D));
  I.jac_ready = true;
  if (*order == 0) {
    k_scale<<<I.blocks, 256, 0, st>>>(I.f, h, D + I.nN, I.nN);
    RDCU_TRY(cudaGetLastError());
    *order = 1;
  }
  I.started = true;
  return cudaSuccess;
}

cudaError_t BDFEngine::step(double* t, double* h, double hmin, double hmax, int* accepted, int* status) {
  *status = RDCU_OK;
  Impl& I = *impl_;
  if (!I.started) {
    RDCU_TRY(bdf_setup(I, *fd_, D_, &order_, *h, st_));
  }
  t_ = *t;
  h_ = *h;
  const long long nN = I.nN;
  const int nb = I.blocks;
  const double sqN = std::pow((double)nN, 0.5);
  int order = order_;
  int converged = 0, it = 0;
  double dnorm = 0, dnormold = 0, rate = 0, factor = 1.0;
  const double h0 = h_;
  double hh = h_, tt = t_;
  k_predict<<<nb, 256, 0, st_>>>(D_, nN, order, I.atl, I.rtl, I.ytemp, I.yscale);
  RDCU_TRY(cudaMemsetAsync(I.d, 0, sizeof(double) * nN, st_));
  Small gam{};
  for (int j = 0; j < 6; ++j) gam.v[j] = kGamma[j];
  if (!I.newton_exec && !I.newton_failed && build_newton_graph(I, *fd_, D_, st_) != cudaSuccess)
    I.newton_failed = true;
  // the graph also leaves yscale at ytemp and ||d||^2 for the error test
  bool errsq_ready = false;
  double errsq = 0.0;
  if (I.newton_exec) {
    // the Newton loop on the device: one launch, one record read back
    const double coef = (1 - kKappa[order]) * kGamma[order];
    k_newton_arm<<<1, 1, 0, st_>>>(I.nctl, hh, coef, -hh / coef, order, I.refactor, gam);
    RDCU_TRY(cudaGetLastError());
    RDCU_TRY(cudaGraphLaunch(I.newton_exec, st_));
    RDCU_TRY(cudaMemcpyAsync(I.nctl_host, I.nctl, sizeof(NewtonCtl), cudaMemcpyDeviceToHost, st_));
    RDCU_TRY(cudaStreamSynchronize(st_));
    const NewtonCtl& c = *I.nctl_host;
    converged = c.converged;
    it = c.it;
    I.alpha = c.alpha;
    I.refactor = c.refactor;
    lin_iters += c.lin_iters;
    lin_cycles += c.lin_cycles;
    lin_solves += c.lin_solves;
    errsq = c.errsq;
    errsq_ready = true;
  }
  for (it = I.newton_exec ? it : 0; !I.newton_exec && it < kNwit; it++) {
    RDCU_TRY(fd_->rhs(I.ytemp, I.f, nullptr));
    if (I.refactor) {
      I.alpha = -hh / ((1 - kKappa[order]) * kGamma[order]);
      I.refactor = 0;
    }
    k_newton_rhs<<<nb, 256, 0, st_>>>(I.b, I.f, I.d, D_, nN, order, hh, (1 - kKappa[order]) * kGamma[order], gam);
    int iters = 0, cycles = 0;
    RDCU_TRY(gmres(I, *fd_, I.alpha, I.b, I.dd, st_, &iters, &cycles));
    lin_iters += iters;
    lin_cycles += cycles;
    ++lin_solves;
    RDCU_TRY(wnorm(I, I.dd, st_, &dnorm));
    dnorm /= sqN;
    if (dnormold > 0) rate = dnorm / dnormold;
    if (rate >= 1) break;
    if (std::pow(rate, kNwit - it) / (1 - rate) * dnorm > I.ntol) break;
    if (dnormold > 0 && rate / (1 - rate) * dnorm < I.ntol) {
      converged = 1;
      break;
    }
    k_newton_update<<<nb, 256, 0, st_>>>(I.dd, I.ytemp, I.d, nN);
    dnormold = dnorm;
  }
  *accepted = 0;
  if (!converged) {
    if (I.rejac) {
      k_predict<<<nb, 256, 0, st_>>>(D_, nN, order, I.atl, I.rtl, I.ytemp, nullptr);
      RDCU_TRY(fd_->jac_values(I.ytemp));
      I.refactor = 1;
      I.rejac = 0;
      RDCU_TRY(cudaStreamSynchronize(st_));
      *t = tt;
      *h = hh;
      return cudaSuccess;
    } else if (!I.fixed) {
      factor = 0.5;
      hh *= factor;
      h_ = hh;
      *h = hh;
      *t = tt;
      if (hh < hmin) return cudaStreamSynchronize(st_);
      Small RU{};
      make_RU(order, factor, RU.v);
      k_updateD<<<nb, 256, 0, st_>>>(D_, nN, order, RU);
      I.refactor = 1;
      I.nconststeps = 0;
      return cudaStreamSynchronize(st_);
    }
  }
  if (I.fixed) {
    RDCU_TRY(cudaMemcpyAsync(D_, I.ytemp, sizeof(double) * nN, cudaMemcpyDeviceToDevice, st_));
    hh = h0;
    tt = tt + hh;
    t_ = tt;
    h_ = hh;
    *t = tt;
    *h = hh;
    *accepted = 1;
    return cudaStreamSynchronize(st_);
  }
  // error test (bdf.cu:231-259)
  const double safety = (2 * kNwit + 1) * 0.9 / (2 * kNwit + it + 1);
  double errnorm;
  if (errsq_ready) {
    errnorm = std::sqrt(errsq);
  } else {
    k_errscale<<<nb, 256, 0, st_>>>(I.ytemp, nN, I.atl, I.rtl, I.yscale);
    RDCU_TRY(wnorm(I, I.d, st_, &errnorm));
  }
  errnorm *= (kKappa[order] * kGamma[order] + 1.0 / (order + 1)) / sqN;
  factor = safety * std::pow(errnorm, (-1.0 / (order + 1)));
  if (errnorm > 1) {
    if (factor < 0.2) factor = 0.2;
    hh = hh * factor;
    h_ = hh;
    *h = hh;
    *t = tt;
    if (hh < hmin) return cudaStreamSynchronize(st_);
    Small RU{};
    make_RU(order, factor, RU.v);
    k_updateD<<<nb, 256, 0, st_>>>(D_, nN, order, RU);
    I.refactor = 1;
    I.nconststeps = 0;
    return cudaStreamSynchronize(st_);
  }
  // accept (bdf.cu:262-271)
  tt = tt + hh;
  k_accept<<<nb, 256, 0, st_>>>(D_, I.d, I.ytemp, nN, order);
  I.rejac = 1;
  I.nconststeps++;
  if (I.nconststeps > order) {
    double errm = INFINITY, errp = INFINITY, fm = 0.0, fp = 0.0;
    if (order > 1) {
      RDCU_TRY(wnorm(I, D_ + nN * order, st_, &errm));
      errm *= (kKappa[order - 1] * kGamma[order - 1] + 1.0 / (order)) / sqN;
      fm = safety * std::pow(errm, (-1.0 / (order)));
    }
    if (order < 5) {
      RDCU_TRY(wnorm(I, D_ + nN * (order + 2), st_, &errp));
      errp *= (kKappa[order + 1] * kGamma[order + 1] + 1.0 / (order + 2)) / sqN;
      fp = safety * std::pow(errp, (-1.0 / (order + 2)));
    }
    int dorder = 0;
    if (order > 1 && fm > factor && fm > fp) {
      factor = fm;
      dorder = -1;
    } else if (order < 5 && fp > factor) {
      factor = fp;
      dorder = 1;
    }
    if (factor > 10) factor = 10;
    if (hh * factor > hmax) {
      factor = hmax / hh;
      hh = hmax;
    } else {
      hh = hh * factor;
    }
    order += dorder;
    Small RU{};
    make_RU(order, factor, RU.v);
    k_updateD<<<nb, 256, 0, st_>>>(D_, nN, order, RU);
    I.nconststeps = 0;
    I.refactor = 1;
  }
  order_ = order;
  t_ = tt;
  h_ = hh;
  *t = tt;
  *h = hh;
  *accepted = 1;
  return cudaStreamSynchronize(st_);
}

cudaError_t BDFEngine::eval(double t_eval, double* y_eval) {
  Small fac{};
  double factor = 1.0;
  for (int j = 1; j <= order_; j++) {
    factor *= (t_eval - t_ + j * h_) / (j * h_);
    fac.v[j] = factor;
  }
  k_interp<<<impl_->blocks, 256, 0, st_>>>(D_, impl_->nN, order_, fac, y_eval);
  RDCU_TRY(cudaGetLastError());
  return cudaStreamSynchronize(st_);
}

cudaError_t BDFEngine::solve(double t1, double hmin, double hmax, const std::vector<double>& t_eval,
                             const std::function<int(double, double, int, long long)>& on_attempt,
                             const std::function<int(int, const double*)>& on_eval,
                             const std::function<int(double, double, long long)>& on_checkpoint, int* cb_status,
                             int* status) {
  *cb_status = 0;
  *status = RDCU_OK;
  Impl& I = *impl_;
  // bdf_run (bdf.cu:330-383): set-up, then attempt while t < t1 and h > hmin
  RDCU_TRY(bdf_setup(I, *fd_, D_, &order_, h_, st_));
  RDCU_TRY(cudaStreamSynchronize(st_));
  solve_attempts = 0;
  solve_accepted = 0;
  long long steps = 0;
  int eval_i = 0;
  const int n_eval = (int)t_eval.size();
  while (t_ < t1 && h_ > hmin) {
    double t = t_, h = h_;
    int acc = 0, st = 0;
    RDCU_TRY(step(&t, &h, hmin, hmax, &acc, &st));
    if (st) {
      *status = st;
      return cudaSuccess;
    }
    ++solve_attempts;
    if (acc) ++steps;
    solve_accepted = steps;
    if (on_attempt) {
      const int rc = on_attempt(t_, h_, acc, steps);
      if (rc) {
        *cb_status = rc;
        return cudaSuccess;
      }
    }
    if (!acc) continue;
    bool any = false;
    while (eval_i < n_eval && t_ >= t_eval[eval_i]) {
      RDCU_TRY(eval(t_eval[eval_i], I.y_eval));
      if (on_eval) {
        const int rc = on_eval(eval_i, I.y_eval);
        if (rc) {
          *cb_status = rc;
          return cudaSuccess;
        }
      }
      ++eval_i;
      any = true;
    }
    if (any && on_checkpoint) {
      const int rc = on_checkpoint(t_, h_, steps);
      if (rc) {
        *cb_status = rc;
        return cudaSuccess;
      }
    }
  }
  return cudaSuccess;
}

}  // namespace rdcu
