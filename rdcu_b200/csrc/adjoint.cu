// Discrete adjoint of fixed-step DP45 on the pseudospectral dictionary RHS.
//
// Step map (fixed h, dp45.cu:34-69 with the b row of dp45.cu:11):
//   Y_i = y_n + h sum_{j<i} a_ij k_j,  k_i = f(Y_i; C),  y_{n+1} = y_n + h sum_i b_i k_i.
// Reverse sweep for lambda = dL/dy_{n+1}, stages i = 6..1 (stage 7 only feeds the error
// estimate and FSAL, so it is absent from the fixed-step map):
//   kbar_i = h b_i lambda + h sum_{l>i} a_li Ybar_l,   Ybar_i = J_f(Y_i)^T kbar_i,
//   Cbar  += (df/dC)(Y_i)^T kbar_i,                    dL/dy_n = lambda + sum_i Ybar_i.
// The VJP of f = sum_t C_t prod_q Q_q^eta (Q: fields and spectral derivative blocks)
// splits into
//   * a pointwise kernel over the monomials: d/dQ_q of every term (product rule over its
//     factors) times the cotangent, and the C-gradients <w_field, term> (reductions);
//   * the transposed spectral operators: a derivative block Q_k = M_k u_src contributes
//     M_k^T Qbar_k to ubar_src.  For the real operators here M^T has the symbol
//     conj(M(k)) = (-1)^order M(k), so the same FFT passes apply it with the entry
//     coefficients multiplied by (-1)^order.  Linear single-derivative terms C_t M_t u_s
//     are handled in the transposed pass only: ubar_s += C_t M_t^T w_field and
//     dL/dC_t = <M_t^T w_field, u_s>.
// Checkpoints: the state every K steps; each segment is recomputed from its
// checkpoint with the fused forward stages, keeping the stage states Y_1..Y_6.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "adjoint.h"

namespace rdcu {
namespace {

// dp45.cu:6-11 (a_{l,i} for l = 2..6, and b)
const double kA[8][6] = {
    {0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
    {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};

constexpr int kBlocks = 296;
constexpr int kThreads = 256;
constexpr int kMaxQ = 16;      // fields + derivative quantities in one term evaluation
constexpr int kMaxTerms = 64;  // terms with per-thread gradient accumulators
constexpr int kMaxGraphSteps = 512;  // longer segments are launched directly (graph size)

struct AdjTerm {
  int field, nf, off, orig;
  double C;
};
struct AdjFactor {
  int q, eta;  // q < n: field q; else derivative quantity q - n
};
struct AdjFold {
  int src, g, orig, field;
  double C;
};
struct AdjQ {
  int src, g;
};

__device__ __forceinline__ double pw(double x, int e) {
  switch (e) {
    case 0: return 1.0;
    case 1: return x;
    case 2: return x * x;
    case 3: return x * x * x;
    default: break;
  }
  const int a = e < 0 ? -e : e;
  double r = 1.0;
  for (int i = 0; i < a; ++i) r *= x;
  return e < 0 ? 1.0 / r : r;
}

__device__ __forceinline__ double block_reduce(double v) {
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kThreads / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

struct Coef7 {
  double c[7];
};

struct CombineArgs {
  int n, nfold, nq, final_stage;
  long long N, nN;
  const AdjFold* folds;
  const AdjQ* qs;
  const double* ubar;
  const double* G;   // transposed-operator outputs (ng channels)
  const double* u;   // stage state
  double* Yb;        // out: Ybar_i (n fields); stage 1: not stored
  double* lam;       // stage 1: lambda += sum_i Ybar_i
  double* part;
};

struct PointwiseArgs {
  int n, nq, nkept, nfac, stage;
  long long N, nN;
  const AdjTerm* terms;
  const AdjFactor* fac;
  const double* u;   // stage state Y_i (n fields)
  const double* Q;   // derivative quantities of Y_i (nq)
  const double* lam; // adjoint state after the step
  const double* Yb;  // stage adjoints, block l-1 for stage l
  double hb;         // h b_i
  Coef7 ha;          // ha.c[l] = h a_{l,i}
  double* w;         // out: kbar_i (n fields), input of the transposed operators
  double* ubar;      // out: pointwise field adjoint (n)
  double* Qbar;      // out: derivative-quantity adjoint (nq)
  double* part;      // [term][kBlocks] partial sums of dL/dC, accumulated
};

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Shared memory of k_adj_stage: per-thread slices [i][thread] of the quantities q,
// their adjoints qb and kbar (indexed by the dictionary's runtime factor lists, so they
// live in shared rather than local memory), then per-warp gradient sums [term][warp].
size_t pointwise_smem(int n, int nq, int nkept, int nfac) {
  return ((size_t)(2 * (n + nq) + n) * kThreads + (size_t)nkept * (kThreads / 32)) * sizeof(double) +
         (size_t)nkept * sizeof(AdjTerm) + (size_t)nfac * sizeof(AdjFactor);
}

// One kernel per stage of the reverse sweep, at every point:
//  (1) when do_cb: the end of the previous stage's adjoint (the "combine"):
//      Ybar_i = ubar + sum_folded C_t M_t^T kbar_field(t) + sum_q M_q^T Qbar_q, with partial
//      sums of dL/dC_t = <M_t^T kbar_field(t), u_src(t)> for the folded terms; at stage 1
//      the step ends: lambda_n = lambda_{n+1} + sum_{i=1..6} Ybar_i;
//  (2) when do_pw: this stage's start (the "pointwise" part): kbar_i = h b_i lambda +
//      h sum_{l > i} a_li Ybar_l (stored for the transposed operators), then the monomial
//      VJP ubar_f = sum_t kbar_field(t) dP_t/du_f, Qbar_q likewise, and per-block partial
//      sums of dL/dC_t = sum_x kbar_field(t) P_t.
// (2) reads the Ybar and lambda that (1) just wrote at the same point (same thread).
// Partial sums: warp sums, then warps in a fixed order (deterministic).
__global__ void __launch_bounds__(kThreads) k_adj_stage(PointwiseArgs a, CombineArgs cb, int do_pw, int do_cb) {
  extern __shared__ double psm[];
  constexpr int T = kThreads, NW = kThreads / 32;
  __shared__ double sgc[kMaxTerms * NW];
  __shared__ AdjFold sfold[kMaxTerms];
  __shared__ AdjQ sqs[kMaxQ];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nqt = a.n + a.nq;
  double* sq = psm;
  double* sqb = sq + nqt * T;
  double* swk = sqb + nqt * T;
  double* sg = swk + a.n * T;
  AdjTerm* sterm = reinterpret_cast<AdjTerm*>(sg + a.nkept * NW);
  AdjFactor* sfac = reinterpret_cast<AdjFactor*>(sterm + a.nkept);
  for (int i = tid; i < a.nkept * NW; i += T) sg[i] = 0.0;
  for (int i = tid; i < cb.nfold * NW; i += T) sgc[i] = 0.0;
  // the tables are read in every term iteration: stage them next to the slices
  for (int i = tid; i < a.nkept; i += T) sterm[i] = a.terms[i];
  for (int i = tid; i < a.nfac; i += T) sfac[i] = a.fac[i];
  for (int i = tid; i < cb.nfold; i += T) sfold[i] = cb.folds[i];
  for (int i = tid; i < cb.nq; i += T) sqs[i] = cb.qs[i];
  __syncthreads();
  for (long long base = (long long)blockIdx.x * T; base < a.N; base += (long long)gridDim.x * T) {
    const long long x = base + tid;
    const bool live = x < a.N;
    if (do_cb) {
      if (live) {
        for (int s = 0; s < cb.n; ++s) {
          const long long o = (long long)s * cb.N + x;
          double v = cb.ubar[o];
          for (int t = 0; t < cb.nfold; ++t)
            if (sfold[t].src == s) v += sfold[t].C * cb.G[(long long)sfold[t].g * cb.N + x];
          for (int q = 0; q < cb.nq; ++q)
            if (sqs[q].src == s) v += cb.G[(long long)sqs[q].g * cb.N + x];
          if (cb.final_stage) {
            double l = cb.lam[o] + v;
            for (int i = 2; i <= 6; ++i) l += cb.Yb[(long long)(i - 1) * cb.nN + o];
            cb.lam[o] = l;
          } else {
            cb.Yb[o] = v;
          }
        }
      }
      for (int t = 0; t < cb.nfold; ++t) {
        double g = live ? cb.G[(long long)sfold[t].g * cb.N + x] * cb.u[(long long)sfold[t].src * cb.N + x] : 0.0;
        g = warp_sum(g);
        if (lane == 0) sgc[t * NW + warp] += g;
      }
    }
    if (!do_pw) continue;
    if (live) {
      for (int f = 0; f < a.n; ++f) {
        const long long o = (long long)f * a.N + x;
        double v = a.hb * a.lam[o];
        for (int l = a.stage + 1; l <= 6; ++l) v += a.ha.c[l] * a.Yb[(long long)(l - 1) * a.nN + o];
        a.w[o] = v;
        swk[f * T + tid] = v;
      }
      for (int i = 0; i < nqt; ++i) {
        sq[i * T + tid] = i < a.n ? a.u[(long long)i * a.N + x] : a.Q[(long long)(i - a.n) * a.N + x];
        sqb[i * T + tid] = 0.0;
      }
    }
    for (int t = 0; t < a.nkept; ++t) {
      double g = 0.0;
      if (live) {
        const AdjTerm tm = sterm[t];
        const double w = swk[tm.field * T + tid];
        double P = 1.0;
        for (int j = 0; j < tm.nf; ++j) {
          const AdjFactor f = sfac[tm.off + j];
          P *= pw(sq[f.q * T + tid], f.eta);
        }
        g = w * P;
        for (int j = 0; j < tm.nf; ++j) {
          // product rule: eta_j Q_j^(eta_j - 1) * prod of the other factors
          double d = tm.C;
          for (int l = 0; l < tm.nf; ++l) {
            const AdjFactor f = sfac[tm.off + l];
            const double qv = sq[f.q * T + tid];
            d *= (l == j) ? f.eta * pw(qv, f.eta - 1) : pw(qv, f.eta);
          }
          sqb[sfac[tm.off + j].q * T + tid] += w * d;
        }
      }
      g = warp_sum(g);
      if (lane == 0) sg[t * NW + warp] += g;
    }
    if (live) {
      for (int i = 0; i < a.n; ++i) a.ubar[(long long)i * a.N + x] = sqb[i * T + tid];
      for (int i = 0; i < a.nq; ++i) a.Qbar[(long long)i * a.N + x] = sqb[(a.n + i) * T + tid];
    }
  }
  __syncthreads();
  if (do_pw) {
    for (int t = tid; t < a.nkept; t += T) {
      double s = 0.0;
      for (int w = 0; w < NW; ++w) s += sg[t * NW + w];
      a.part[(long long)sterm[t].orig * gridDim.x + blockIdx.x] += s;
    }
  }
  if (do_cb) {
    for (int t = tid; t < cb.nfold; t += T) {
      double s = 0.0;
      for (int w = 0; w < NW; ++w) s += sgc[t * NW + w];
      cb.part[(long long)sfold[t].orig * gridDim.x + blockIdx.x] += s;
    }
  }
}

// dL/dC_t = sum over the blocks' accumulated partials (fixed order: deterministic)
__global__ void k_adj_reduce(const double* part, int nterms, double* gC) {
  const int t = blockIdx.x;
  if (t >= nterms) return;
  double s = 0.0;
  for (int b = threadIdx.x; b < kBlocks; b += blockDim.x) s += part[(long long)t * kBlocks + b];
  s = block_reduce(s);
  if (threadIdx.x == 0) gC[t] = s;
}

ChanEntry op_entry(int k, int n, int ndim, int src_index, double coef) {
  ChanEntry e{};
  const int Yind = k / n;
  e.src = src_index;
  e.part = 0;
  e.coef = coef;
  if (Yind == 0) {
    e.nax = 0;
  } else if (Yind <= ndim) {
    e.nax = 1;
    e.ax0 = Yind - 1;
  } else {
    const int t = Yind - ndim - 1;
    e.nax = 2;
    e.ax0 = t / ndim;
    e.ax1 = t % ndim;
  }
  return e;
}

}  // namespace

struct AdjointEngine::Tables {
  AdjTerm* terms = nullptr;
  AdjFactor* fac = nullptr;
  AdjFold* folds = nullptr;
  AdjQ* qs = nullptr;
  int nkept = 0, nfac = 0, nfold = 0, nq = 0;
  std::vector<AdjTerm> h_terms;
  std::vector<AdjFold> h_folds;
};

#define RDCU_TRY(x)                   \
  do {                                \
    cudaError_t _e = (x);             \
    if (_e != cudaSuccess) return _e; \
  } while (0)

template <typename T>
static cudaError_t up(T** d, const std::vector<T>& v) {
  RDCU_TRY(cudaMalloc((void**)d, std::max<size_t>(1, v.size()) * sizeof(T)));
  if (!v.empty()) RDCU_TRY(cudaMemcpy(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return cudaSuccess;
}

bool AdjointEngine::init(SpectralPlan* fwd, DP45Engine* dp, const std::vector<HostTerm>& terms, int n, int ndim,
                         const int* Ns, const double* Ls, cudaStream_t st, std::string* msg) {
  release();
  fwd_ = fwd;
  dp_ = dp;
  st_ = st;
  n_ = n;
  terms_ = terms;
  nterms = (int)terms.size();
  N_ = 1;
  for (int a = 0; a < ndim; ++a) N_ *= Ns[a];
  nN_ = N_ * n;
  tab_ = new Tables;
  Tables& T = *tab_;
  // classify the terms exactly as the forward plan does
  std::vector<int> qk;  // derivative Y indices needed pointwise (nonlinear factors)
  struct Kept {
    int field, orig;
    double C;
    std::vector<std::pair<int, int>> fac;
  };
  std::vector<Kept> kept;
  struct Fold {
    int field, src, k, orig;
    double C;
  };
  std::vector<Fold> folds;
  for (int ti = 0; ti < nterms; ++ti) {
    const auto& t = terms[ti];
    const int field = t.ints.empty() ? 0 : t.ints[0];
    std::vector<std::pair<int, int>> fac;
    const int np = (int)t.ints.size();
    for (int j = 1; j < np; j += 2) {
      const int p = (j + 1 < np) ? t.ints[j + 1] : 0;
      if (p != 0) fac.push_back({t.ints[j], p});
    }
    if (fac.size() == 1 && fac[0].second == 1 && fac[0].first >= n) {
      folds.push_back({field, fac[0].first % n, fac[0].first, ti, t.C});
      continue;
    }
    for (auto& f : fac)
      if (f.first >= n && std::find(qk.begin(), qk.end(), f.first) == qk.end()) qk.push_back(f.first);
    kept.push_back({field, ti, t.C, fac});
  }
  std::sort(qk.begin(), qk.end());
  nq_ = (int)qk.size();
  if ((int)kept.size() > kMaxTerms || (int)folds.size() > kMaxTerms || n + nq_ > kMaxQ) {
    *msg = "dictionary too large for the adjoint kernels";
    return false;
  }
  // distinct (operator, cotangent field) pairs of the folded terms
  std::vector<std::pair<int, int>> pairs;  // (Yind, field)
  std::vector<int> fold_g(folds.size());
  for (size_t i = 0; i < folds.size(); ++i) {
    const std::pair<int, int> key{folds[i].k / n, folds[i].field};
    auto it = std::find(pairs.begin(), pairs.end(), key);
    fold_g[i] = (int)(it - pairs.begin());
    if (it == pairs.end()) pairs.push_back(key);
  }
  nfold_pairs_ = (int)pairs.size();
  ng_ = nfold_pairs_ + nq_;
  // transposed operators: inputs [kbar (n), Qbar (nq)], outputs G (ng)
  std::vector<std::vector<ChanEntry>> tch;
  for (auto& pr : pairs) {
    const int k = pr.first * n;  // Y index of the operator (field 0), source = cotangent field pr.second
    ChanEntry e = op_entry(k, n, ndim, pr.second, 1.0);
    if (e.nax & 1) e.coef = -1.0;  // transpose of an odd-order derivative
    tch.push_back({e});
  }
  for (int q = 0; q < nq_; ++q) {
    ChanEntry e = op_entry(qk[q], n, ndim, n + q, 1.0);
    if (e.nax & 1) e.coef = -1.0;
    tch.push_back({e});
  }
  if (ng_ > 0 && !planT_.init_linear(n + nq_, ndim, Ns, Ls, tch, msg)) return false;
  if (nq_ > 0) {
    std::vector<std::vector<ChanEntry>> qch;
    for (int q = 0; q < nq_; ++q) qch.push_back({op_entry(qk[q], n, ndim, qk[q] % n, 1.0)});
    if (!planQ_.init_linear(n, ndim, Ns, Ls, qch, msg)) return false;
    have_q_ = true;
  }
  // device tables
  std::vector<AdjFactor> fac;
  for (auto& k : kept) {
    AdjTerm t{};
    t.field = k.field;
    t.orig = k.orig;
    t.C = k.C;
    t.off = (int)fac.size();
    t.nf = (int)k.fac.size();
    for (auto& f : k.fac) {
      AdjFactor af{};
      af.q = f.first < n ? f.first : n + (int)(std::find(qk.begin(), qk.end(), f.first) - qk.begin());
      af.eta = f.second;
      fac.push_back(af);
    }
    T.h_terms.push_back(t);
  }
  for (size_t i = 0; i < folds.size(); ++i) {
    AdjFold f{};
    f.src = folds[i].src;
    f.g = fold_g[i];
    f.orig = folds[i].orig;
    f.field = folds[i].field;
    f.C = folds[i].C;
    T.h_folds.push_back(f);
  }
  std::vector<AdjQ> qs;
  for (int q = 0; q < nq_; ++q) qs.push_back({qk[q] % n, nfold_pairs_ + q});
  T.nkept = (int)T.h_terms.size();
  T.nfac = (int)fac.size();
  T.nfold = (int)T.h_folds.size();
  T.nq = nq_;
  pw_smem_ = pointwise_smem(n, nq_, T.nkept, T.nfac);
  if (pw_smem_ > 48 * 1024 &&
      cudaFuncSetAttribute(k_adj_stage, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pw_smem_) != cudaSuccess) {
    *msg = "adjoint set-up: dictionary too large for the pointwise kernel's shared memory";
    return false;
  }
  const size_t sb = (size_t)nN_ * sizeof(double);
  auto fail = [&](const char* w) {
    *msg = std::string("adjoint set-up: ") + w;
    return false;
  };
  if (up(&T.terms, T.h_terms) != cudaSuccess || up(&T.fac, fac) != cudaSuccess ||
      up(&T.folds, T.h_folds) != cudaSuccess || up(&T.qs, qs) != cudaSuccess)
    return fail("tables");
  if (cudaMalloc((void**)&lam_, sb) != cudaSuccess) return fail("out of device memory");
  if (cudaMalloc((void**)&Yb_, sb * 6) != cudaSuccess) return fail("out of device memory");
  if (cudaMalloc((void**)&tin_, (size_t)N_ * (n + nq_) * sizeof(double)) != cudaSuccess)
    return fail("out of device memory");
  if (cudaMalloc((void**)&tout_, (size_t)N_ * std::max(1, ng_) * sizeof(double)) != cudaSuccess)
    return fail("out of device memory");
  if (cudaMalloc((void**)&qv_, (size_t)N_ * std::max(1, nq_) * sizeof(double)) != cudaSuccess)
    return fail("out of device memory");
  if (cudaMalloc((void**)&ubar_, sb) != cudaSuccess) return fail("out of device memory");
  if (cudaMalloc((void**)&part_, sizeof(double) * std::max(1, nterms) * kBlocks) != cudaSuccess)
    return fail("out of device memory");
  if (cudaMalloc((void**)&gC_, sizeof(double) * std::max(1, nterms)) != cudaSuccess) return fail("out of device memory");
  device_bytes = sb * 8 + (size_t)N_ * (n + 2 * nq_ + ng_) * sizeof(double);
  return true;
}

void AdjointEngine::release() {
  drop_graphs();
  for (double* p : ckpt_pool_)
    if (p) cudaFree(p);
  ckpt_pool_.clear();
  ckpt_.clear();
  double* bufs[] = {store_, lam_, Yb_, tin_, tout_, qv_, ubar_, part_, gC_};
  for (double* p : bufs)
    if (p) cudaFree(p);
  store_ = lam_ = Yb_ = tin_ = tout_ = qv_ = ubar_ = part_ = gC_ = nullptr;
  store_steps_ = 0;
  if (tab_) {
    void* t[] = {tab_->terms, tab_->fac, tab_->folds, tab_->qs};
    for (void* p : t)
      if (p) cudaFree(p);
    delete tab_;
    tab_ = nullptr;
  }
}

cudaError_t AdjointEngine::set_coefficients(const std::vector<double>& C) {
  Tables& T = *tab_;
  for (auto& t : T.h_terms) t.C = C[t.orig];
  for (auto& f : T.h_folds) f.C = C[f.orig];
  if (!T.h_terms.empty())
    RDCU_TRY(cudaMemcpy(T.terms, T.h_terms.data(), T.h_terms.size() * sizeof(AdjTerm), cudaMemcpyHostToDevice));
  if (!T.h_folds.empty())
    RDCU_TRY(cudaMemcpy(T.folds, T.h_folds.data(), T.h_folds.size() * sizeof(AdjFold), cudaMemcpyHostToDevice));
  return cudaSuccess;
}

cudaError_t AdjointEngine::forward(const double* y0, const double* hs, int nsteps, int K, double* yT) {
  nsteps_ = std::max(0, nsteps);
  hs_.assign(hs, hs + nsteps_);
  uniform_h_ = true;
  for (int j = 1; j < nsteps_; ++j) uniform_h_ = uniform_h_ && hs_[j] == hs_[0];
  K_ = std::max(1, K);
  const int nseg = std::max(1, (nsteps_ + K_ - 1) / K_);
  const size_t sb = (size_t)nN_ * sizeof(double);
  // checkpoint buffers are kept across calls and only added to
  ckpt_.clear();
  while ((int)ckpt_pool_.size() < nseg) {
    double* p = nullptr;
    RDCU_TRY(cudaMalloc((void**)&p, sb));
    ckpt_pool_.push_back(p);
  }
  ckpt_.assign(ckpt_pool_.begin(), ckpt_pool_.begin() + nseg);
  RDCU_TRY(dp_->set_state(0.0, nsteps_ ? hs_[0] : 0.0, y0));
  for (int seg = 0; seg < nseg; ++seg) {
    RDCU_TRY(dp_->copy_current_y(ckpt_[seg]));
    const int j0 = seg * K_, steps = std::min(K_, nsteps_ - j0);
    if (steps <= 0) break;
    if (uniform_h_) {
      long long acc = 0;
      RDCU_TRY(dp_->advance(steps, 0.0, INFINITY, &acc));
    } else {
      const int cap = dp_->log_cap();  // a full attempt log stops the controller: re-arm
      for (int j = 0; j < steps; ++j) {
        if (j % cap == 0) RDCU_TRY(dp_->arm(1, INFINITY, 0.0, INFINITY, 0, 0, std::min(cap, steps - j)));
        if (seg == 0 && j == 0) RDCU_TRY(dp_->launch_k1());
        RDCU_TRY(dp_->set_h_async(hs_[j0 + j]));
        RDCU_TRY(dp_->launch_attempt());
      }
    }
  }
  if (yT) RDCU_TRY(dp_->get_state(nullptr, nullptr, yT, cudaMemcpyDefault));
  return cudaStreamSynchronize(st_);
}

cudaError_t AdjointEngine::ensure_store(int steps) {
  if (store_steps_ >= steps) return cudaSuccess;
  drop_graphs();  // the graphs hold store_ addresses
  if (store_) cudaFree(store_);
  store_ = nullptr;
  store_steps_ = 0;
  RDCU_TRY(cudaMalloc((void**)&store_, (size_t)nN_ * sizeof(double) * 6 * (size_t)steps));
  store_steps_ = steps;
  return cudaSuccess;
}

void AdjointEngine::drop_graphs() {
  for (auto& g : graphs_) {
    if (g.rec) cudaGraphExecDestroy(g.rec);
    if (g.rev) cudaGraphExecDestroy(g.rev);
  }
  graphs_.clear();
}

// Recomputes `steps` steps from the state in bufs.ybuf[0] (queued; capturable), storing
// the stage states Y_1..Y_6 of step j at store_ + 6 j nN.
cudaError_t AdjointEngine::launch_recompute(int j0, int steps) {
  const int cap = dp_->log_cap();
  RDCU_TRY(dp_->reset_async(0.0, hs_[j0]));
  for (int j = 0; j < steps; ++j) {
    if (j % cap == 0) RDCU_TRY(dp_->arm(1, INFINITY, 0.0, INFINITY, 0, 0, std::min(cap, steps - j)));
    if (j == 0) RDCU_TRY(dp_->launch_k1());
    double* base = store_ + (size_t)j * 6 * nN_;
    RDCU_TRY(dp_->copy_current_y(base));  // Y_1 = y_j
    double* outs[8] = {};
    for (int st = 2; st <= 6; ++st) outs[st] = base + (size_t)(st - 1) * nN_;
    if (!uniform_h_) RDCU_TRY(dp_->set_h_async(hs_[j0 + j]));
    RDCU_TRY(dp_->launch_attempt_capture(outs));
  }
  return cudaSuccess;
}

// Reverse sweep over `steps` recomputed steps (queued; capturable).  Each stage's
// combine runs in the kernel of the next stage's pointwise part; the last one alone.
cudaError_t AdjointEngine::launch_reverse(int j0, int steps) {
  bool pending = false;
  const double* Yprev = nullptr;
  int sprev = 0;
  for (int j = steps - 1; j >= 0; --j) {
    const double* Ystore = store_ + (size_t)j * 6 * nN_;
    const double h = hs_[j0 + j];
    for (int i = 6; i >= 1; --i) {
      const double* Y = Ystore + (size_t)(i - 1) * nN_;
      RDCU_TRY(stage_kernels(Y, i, h, pending ? Yprev : nullptr, sprev));
      pending = true;
      Yprev = Y;
      sprev = i;
    }
  }
  if (pending) RDCU_TRY(stage_kernels(nullptr, 0, 0.0, Yprev, sprev));
  return cudaSuccess;
}

// Launches the combine of stage sprev at state Yprev (if Yprev) fused with the pointwise
// part of stage `stage` at state Y (if Y), then stage's transposed operators.
cudaError_t AdjointEngine::stage_kernels(const double* Y, int stage, double h, const double* Yprev, int sprev) {
  Tables& T = *tab_;
  if (Y && have_q_) RDCU_TRY(planQ_.run_linear(Y, qv_, st_));
  PointwiseArgs pa{};
  pa.n = n_;
  pa.nq = nq_;
  pa.nkept = T.nkept;
  pa.nfac = T.nfac;
  pa.stage = stage;
  pa.N = N_;
  pa.nN = nN_;
  pa.terms = T.terms;
  pa.fac = T.fac;
  pa.u = Y;
  pa.Q = qv_;
  pa.lam = lam_;
  pa.Yb = Yb_;
  pa.hb = Y ? h * kA[7][stage - 1] : 0.0;
  if (Y)
    for (int l = stage + 1; l <= 6; ++l) pa.ha.c[l] = h * kA[l][stage - 1];
  pa.w = tin_;
  pa.ubar = ubar_;
  pa.Qbar = tin_ + (size_t)n_ * N_;
  pa.part = part_;
  CombineArgs ca{};
  ca.n = n_;
  ca.nfold = Yprev ? T.nfold : 0;
  ca.nq = Yprev ? nq_ : 0;
  ca.final_stage = sprev == 1;
  ca.N = N_;
  ca.nN = nN_;
  ca.folds = T.folds;
  ca.qs = T.qs;
  ca.ubar = ubar_;
  ca.G = tout_;
  ca.u = Yprev;
  ca.Yb = Yb_ + (size_t)(sprev > 0 ? sprev - 1 : 0) * nN_;
  ca.lam = lam_;
  ca.part = part_;
  k_adj_stage<<<kBlocks, kThreads, pw_smem_, st_>>>(pa, ca, Y ? 1 : 0, Yprev ? 1 : 0);
  RDCU_TRY(cudaGetLastError());
  if (Y && ng_ > 0) RDCU_TRY(planT_.run_linear(tin_, tout_, st_));
  return cudaSuccess;
}

template <typename F>
static cudaError_t capture(cudaStream_t st, cudaGraphExec_t* out, F&& body) {
  RDCU_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = body();
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(st, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
  if (g) cudaGraphDestroy(g);
  return e;
}

cudaError_t AdjointEngine::backward(const double* lambdaT, double* grad_y0, double* grad_C) {
  if (ckpt_.empty()) return cudaErrorInvalidValue;  // no forward run recorded
  const size_t sb = (size_t)nN_ * sizeof(double);
  RDCU_TRY(cudaMemcpyAsync(lam_, lambdaT, sb, cudaMemcpyDefault, st_));
  RDCU_TRY(cudaMemsetAsync(part_, 0, sizeof(double) * std::max(1, nterms) * kBlocks, st_));
  const int nseg = (nsteps_ + K_ - 1) / K_;
  if (nseg > 0) RDCU_TRY(ensure_store(std::min(K_, nsteps_)));
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int j0 = seg * K_, steps = std::min(K_, nsteps_ - j0);
    RDCU_TRY(cudaMemcpyAsync(dp_->bufs.ybuf[0], ckpt_[seg], sb, cudaMemcpyDeviceToDevice, st_));
    if (uniform_h_ && use_graphs && steps <= kMaxGraphSteps) {
      // segments of equal length and step size replay the same two graphs
      SegGraphs* g = nullptr;
      for (auto& e : graphs_)
        if (e.steps == steps && e.h == hs_[j0]) g = &e;
      if (!g) {
        SegGraphs e{};
        e.steps = steps;
        e.h = hs_[j0];
        RDCU_TRY(capture(st_, &e.rec, [&] { return launch_recompute(j0, steps); }));
        RDCU_TRY(capture(st_, &e.rev, [&] { return launch_reverse(j0, steps); }));
        graphs_.push_back(e);
        g = &graphs_.back();
      }
      RDCU_TRY(cudaGraphLaunch(g->rec, st_));
      RDCU_TRY(cudaGraphLaunch(g->rev, st_));
    } else {
      RDCU_TRY(launch_recompute(j0, steps));
      RDCU_TRY(launch_reverse(j0, steps));
    }
  }
  k_adj_reduce<<<std::max(1, nterms), kThreads, 0, st_>>>(part_, nterms, gC_);
  RDCU_TRY(cudaGetLastError());
  if (grad_y0) RDCU_TRY(cudaMemcpyAsync(grad_y0, lam_, sb, cudaMemcpyDefault, st_));
  std::vector<double> g(std::max(1, nterms));
  RDCU_TRY(cudaMemcpyAsync(g.data(), gC_, sizeof(double) * std::max(1, nterms), cudaMemcpyDeviceToHost, st_));
  RDCU_TRY(cudaStreamSynchronize(st_));
  if (grad_C)
    for (int t = 0; t < nterms; ++t) grad_C[t] = g[t];
  return cudaSuccess;
}

}  // namespace rdcu
