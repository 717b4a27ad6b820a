// Internal types of librdcu (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/rdcu.h"

namespace rdcu {

// ----------------------------------------------------------------------------- FFT plans
constexpr int kMaxStages = 16;
constexpr int kMaxLine = 4096;  // longest complex line one CTA transforms in shared memory

// Division of 0 <= n < 2^31 by an invariant d >= 1 with a multiply and a shift
// (Granlund & Montgomery, "Division by invariant integers using multiplication",
// PLDI 1994): s = ceil(log2 d), m = ceil(2^(31+s) / d) < 2^32, q = (n*m) >> (31+s).
// Exact because the rounding error of m is below d and n*error < 2^(31+s).
struct FastDiv {
  unsigned m;
  int s;
};
inline FastDiv make_fastdiv(unsigned d) {
  int s = 0;
  while ((1ull << s) < d) ++s;
  const unsigned long long num = 1ull << (31 + s);
  FastDiv f;
  f.m = (unsigned)((num + d - 1) / d);
  f.s = s;
  return f;
}
// make_fastdiv for a divisor known at compile time
__host__ __device__ constexpr FastDiv make_fastdiv_c(unsigned d) {
  int s = 0;
  while ((1ull << s) < d) ++s;
  const unsigned long long num = 1ull << (31 + s);
  return FastDiv{(unsigned)((num + d - 1) / d), s};
}
#ifdef __CUDACC__
__device__ __forceinline__ int fdiv(int n, FastDiv f) {
  return (int)(((unsigned long long)(unsigned)n * f.m) >> (31 + f.s));
}
#endif

// Mixed-radix Stockham plan for one complex line length.
struct LinePlan {
  int L;
  int nstages;
  int radix[kMaxStages];
  FastDiv div_m[kMaxStages];   // L / radix[s] (butterflies per line at stage s)
  FastDiv div_ns[kMaxStages];  // span Ns before stage s
};

bool make_line_plan(int L, LinePlan* p);
// exp(-2 pi i t / L) for t < L, rounded from long double.
void make_twiddles(int L, std::vector<double2>& tw);

// ----------------------------------------------------------------------------- spectra
// One entry of an inverse-transform channel: coef * Mpart(k) * U_src(k), where
// Mpart is the real-part (part 0) or imaginary-part (part 1) multiplier of the
// derivative operator on axes ax0 (and ax1) -- see spectral.cu.
struct ChanEntry {
  int src;   // source field
  int nax;   // 0: identity, 1: d_ax0, 2: d_ax0 d_ax1
  int ax0, ax1;
  int part;  // 0: Re of the reference's complex Y block, 1: Im
  int pad;
  double coef;
};

struct ChanTable {
  int nch;
  const int* off;         // [nch+1] entry ranges
  const ChanEntry* ent;
  const double* kv;       // wavenumbers, axis a at kv + kv_off[a]
  int kv_off[3];
  int Ns[3];
  int ndim;
  int kv_total;  // sum of Ns over the axes (length of kv)
};

// Dictionary terms left after folding the linear derivative terms into channels.
struct DictTerm {
  int field;
  int nf;   // factors
  int off;  // first factor
  int pad;
  double C;
};
struct DictFactor {
  int q;    // quantity: < n physical field, else channel q-n
  int eta;  // integer power (never 0: zero powers are dropped, pow(x,0) == 1)
};
struct DictTable {
  int n;
  int nterms;
  const DictTerm* terms;      // grouped by field, reference order kept within a field
  const DictFactor* fac;
  const int* field_begin;     // [n+1]
  const int* fold;            // [n] channel holding the folded linear part, -1 if none
  int nfac;                   // number of factors (fac length)
  // Dense form when every term is a product of fields of total degree <= 3 in poly_nf
  // (= n <= 3) fields: f_i = fold_i + sum_m poly[i * poly_count + m] * monomial_m (Mono
  // order); poly_nf = 0 otherwise.
  const double* poly;
  int poly_nf, poly_count;
};

// Monomials of total degree <= 3 in NF variables, in a fixed order: monomial 0 is 1 and
// monomial m > 0 is monomial parent(m) times variable var(m).
template <int NF>
struct Mono;
template <>
struct Mono<1> {
  static constexpr int count = 4;
  __host__ __device__ static constexpr int parent(int m) { return m - 1; }
  __host__ __device__ static constexpr int var(int) { return 0; }
};
template <>
struct Mono<2> {
  static constexpr int count = 10;  // 1 u v uu uv vv uuu uuv uvv vvv
  __host__ __device__ static constexpr int parent(int m) {
    return m == 1 || m == 2 ? 0 : m == 3 || m == 4 ? 1 : m == 5 ? 2 : m == 6 || m == 7 ? 3 : m == 8 ? 4 : 5;
  }
  __host__ __device__ static constexpr int var(int m) { return m == 1 || m == 3 || m == 6 ? 0 : 1; }
};
template <>
struct Mono<3> {
  static constexpr int count = 20;
  __host__ __device__ static constexpr int parent(int m) {
    constexpr int p[20] = {-1, 0, 0, 0, 1, 1, 1, 2, 2, 3, 4, 4, 4, 5, 5, 6, 7, 7, 8, 9};
    return p[m];
  }
  __host__ __device__ static constexpr int var(int m) {
    constexpr int v[20] = {-1, 0, 1, 2, 0, 1, 2, 1, 2, 2, 0, 1, 2, 1, 2, 2, 1, 2, 2, 2};
    return v[m];
  }
};

// Constant-coefficient linear part of the finite-difference Jacobian, one entry per
// linear term: row field, source field, FD operator, coefficient.  Its symbol at
// wavenumber theta_a = 2 pi m_a / N_a is exact for the reference's stencils:
// identity 1; d_a -> i sin(theta_a)/dx_a; d_a d_a -> (2 cos(theta_a) - 2)/dx_a^2;
// d_a d_b -> -2 sin(theta_a) sin(theta_b)/(dx_a dx_b) (the reference's 0.5 factor).
struct LinEntry {
  int row, src, nax, ax0, ax1, pad;
  double coef;
};
constexpr int kMaxPrecFields = 4;  // per-mode dense solve size of the preconditioner

struct LinTable {
  int n, nent, ndim;
  const LinEntry* ent;
  const double* sinv;  // sin(2 pi m / N_a) at sinv + off[a]
  const double* cosv;
  int off[3];
  int Ns[3];
  double dx[3];
  double alpha;        // preconditioner of I + alpha * J_lin
  const double* alpha_dev;  // when set, alpha is read from here (device-resident solves)
};

// ----------------------------------------------------------------------------- DP45
enum StopReason { kStopNone = 0, kStopDone = 1, kStopOutput = 2, kStopLog = 3, kStopChunk = 4 };

// Device-resident DP45 controller state.  Kernels of one attempt read the buffer
// slots from here, so a step sequence can run (and be captured in a CUDA graph)
// without host round trips.
struct DP45Ctl {
  double t, h, hmin, hmax, t1;
  double t_last;        // start of the last accepted step
  double err_norm;      // last RMS error norm
  double atol, rtol;
  long long n_attempts, n_accepted;
  int running;          // kernels of an attempt return at once when 0
  int stop_reason;
  int accepted;         // last attempt accepted
  int fixed;
  int check_t1;         // solve mode: stop at t >= t1 or h <= hmin
  int y_slot, yn_slot, yl_slot;    // which ybuf is y, the stage state / y_new, y_last
  int k1_buf, k7_buf;              // kbuf index of logical k1 and k7 (FSAL swap)
  int last_k1_buf, last_k7_buf;    // mapping of the last accepted step (dense output)
  int log_count, log_cap;
  int eval_i, n_eval;
  int max_attempts;     // per launch sequence
  int attempts_this_launch;
  int nparts;           // error partial sums written by the stage-7 epilogue
  int pipe_err;         // nonzero: a pass on TMA tiles gave up waiting for its copies
};

struct DP45Bufs {
  double* ybuf[3];
  double* kbuf[7];
};

// Sets the message rdcu_last_error(NULL) returns on this thread (api.cu).
void set_thread_error(const std::string& msg);

}  // namespace rdcu
