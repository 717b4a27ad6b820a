// Finite-difference Y blocks, RHS and analytic CSR Jacobian (BDF path).
//
// Stencils restate init_dY (rdcu.cu:385-596): d_a is (+-0.5/dx_a) at the +-1
// neighbours, d_a d_a is (1,-2,1)/dx_a^2, d_a d_b (a != b) is +-0.5/(dx_a dx_b) at the
// four diagonal neighbours (twice the textbook 1/4 stencil, as the reference has it),
// periodic, each row's entries in increasing column order (the reference sorts them
// with qsort_r).  The reference applies them as COO SpMVs per block and field
// (rdcu.cu:130-148); here each point evaluates the few stencil entries it needs
// directly, in the same column order.  The Jacobian keeps the reference's sparsity:
// the csrgeam2 union of every term/factor contribution (rdcu.cu:202-245), explicit
// zeros included, with values accumulated in term order; the pattern is built once on
// the host, the values by one thread per row.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fd.h"

namespace rdcu {
namespace {

struct Stencil {
  int m;
  long long col[4];
  double val[4];
};

// multi-index helpers (C order, last axis fastest)
__host__ __device__ inline void unravel(long long j, const int* Ns, int ndim, int* ns) {
  for (int d = ndim - 1; d >= 0; --d) {
    ns[d] = (int)(j % Ns[d]);
    j /= Ns[d];
  }
}
__host__ __device__ inline long long ravel(const int* ns, const int* Ns, int ndim) {
  long long j = 0, stride = 1;
  for (int d = ndim - 1; d >= 0; --d) {
    j += ns[d] * stride;
    stride *= Ns[d];
  }
  return j;
}

// Stencil of Y block yind at grid point j, sorted by column.
__host__ __device__ inline void stencil_at(const FDTables& T, int yind, long long j, Stencil* s) {
  int ns[3] = {0, 0, 0};
  unravel(j, T.Ns, T.ndim, ns);
  const int nd = T.ndim;
  if (yind == 0) {
    s->m = 1;
    s->col[0] = j;
    s->val[0] = 1.0;
    return;
  }
  if (yind <= nd) {
    const int a = yind - 1;
    int t[3] = {ns[0], ns[1], ns[2]};
    t[a] = (ns[a] + 1) % T.Ns[a];
    const long long jp = ravel(t, T.Ns, nd);
    t[a] = (ns[a] + T.Ns[a] - 1) % T.Ns[a];
    const long long jm = ravel(t, T.Ns, nd);
    s->m = 2;
    s->col[0] = jm;
    s->val[0] = -T.s1[a];
    s->col[1] = jp;
    s->val[1] = T.s1[a];
  } else {
    const int q = yind - nd - 1;
    const int a = q / nd, b = q % nd;
    const double sc = T.s2[a][b];
    if (a == b) {
      int t[3] = {ns[0], ns[1], ns[2]};
      t[a] = (ns[a] + 1) % T.Ns[a];
      const long long jp = ravel(t, T.Ns, nd);
      t[a] = (ns[a] + T.Ns[a] - 1) % T.Ns[a];
      const long long jm = ravel(t, T.Ns, nd);
      s->m = 3;
      s->col[0] = jm;
      s->val[0] = 1.0 / sc;
      s->col[1] = j;
      s->val[1] = -2.0 / sc;
      s->col[2] = jp;
      s->val[2] = 1.0 / sc;
    } else {
      int t[3] = {ns[0], ns[1], ns[2]};
      const int ap = (ns[a] + 1) % T.Ns[a], am = (ns[a] + T.Ns[a] - 1) % T.Ns[a];
      const int bp = (ns[b] + 1) % T.Ns[b], bm = (ns[b] + T.Ns[b] - 1) % T.Ns[b];
      t[a] = am; t[b] = bm;
      s->col[0] = ravel(t, T.Ns, nd);
      s->val[0] = 0.5 / sc;
      t[a] = am; t[b] = bp;
      s->col[1] = ravel(t, T.Ns, nd);
      s->val[1] = -0.5 / sc;
      t[a] = ap; t[b] = bm;
      s->col[2] = ravel(t, T.Ns, nd);
      s->val[2] = -0.5 / sc;
      t[a] = ap; t[b] = bp;
      s->col[3] = ravel(t, T.Ns, nd);
      s->val[3] = 0.5 / sc;
      s->m = 4;
    }
  }
  // insertion sort by column (stable; the reference's qsort_r order only differs for
  // duplicate columns, i.e. axes of length <= 2)
  for (int i = 1; i < s->m; ++i) {
    const long long c = s->col[i];
    const double v = s->val[i];
    int k = i - 1;
    while (k >= 0 && s->col[k] > c) {
      s->col[k + 1] = s->col[k];
      s->val[k + 1] = s->val[k];
      --k;
    }
    s->col[k + 1] = c;
    s->val[k + 1] = v;
  }
}

__device__ inline double fd_value(const FDTables& T, const double* y, int k, long long j) {
  const int yind = k / T.n, f = k % T.n;
  const double* u = y + (long long)f * T.N;
  if (yind == 0) return u[j];
  Stencil s;
  stencil_at(T, yind, j, &s);
  double acc = s.val[0] * u[s.col[0]];
  for (int e = 1; e < s.m; ++e) acc += s.val[e] * u[s.col[e]];
  return acc;
}

__device__ __forceinline__ double ipow0(double x, int e) {
  if (e == 0) return 1.0;  // pow(x, 0) == 1 for every x
  const int a = e < 0 ? -e : e;
  double r = x;
  for (int i = 1; i < a; ++i) r *= x;
  return e < 0 ? 1.0 / r : r;
}

__global__ void k_fd_rhs(FDTables T, const double* y, double* f) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= T.N) return;
  for (int i = 0; i < T.n; ++i) {
    double acc = 0.0;
    for (int t = T.field_begin[i]; t < T.field_begin[i + 1]; ++t) {
      const FDTerm tm = T.terms[t];
      double prod = 1.0;
      for (int q = 0; q < tm.nf; ++q) {
        const FDFactor fc = T.fac[tm.off + q];
        if (fc.eta == 0) continue;
        prod *= ipow0(fd_value(T, y, fc.k, j), fc.eta);
      }
      acc += tm.C * prod;
    }
    f[(long long)i * T.N + j] = acc;
  }
}

__global__ void k_fd_Y(FDTables T, const double* y, double* Y) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= T.N) return;
  for (int k = 0; k < T.nY * T.n; ++k) {
    const long long o = ((long long)k * T.N + j) * 2;
    Y[o] = fd_value(T, y, k, j);
    Y[o + 1] = 0.0;
  }
}

// One thread per Jacobian row (field i, point j).
__global__ void k_fd_jac(FDTables T, const double* y, const int* rows, const int* cols, double* vals) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)T.n * T.N) return;
  const int i = (int)(gid / T.N);
  const long long j = gid - (long long)i * T.N;
  const int b = rows[gid], e = rows[gid + 1];
  for (int p = b; p < e; ++p) vals[p] = 0.0;
  for (int c = T.contrib_begin[i]; c < T.contrib_begin[i + 1]; ++c) {
    const JacContrib cb = T.contrib[c];
    const FDTerm tm = T.terms[cb.term];
    double tv = 1.0;
    for (int q = 0; q < tm.nf; ++q) {
      const FDFactor fc = T.fac[tm.off + q];
      int pw = fc.eta;
      if (q == cb.jf) {
        const double coeff = tm.C * pw;
        tv = coeff * tv;
        pw -= 1;
      }
      tv = tv * ipow0(fd_value(T, y, fc.k, j), pw);
    }
    Stencil s;
    stencil_at(T, cb.yind, j, &s);
    const long long coff = (long long)cb.src * T.N;
    for (int q = 0; q < s.m; ++q) {
      const int col = (int)(s.col[q] + coff);
      // entries of a row are few and sorted: linear search
      int p = b;
      while (p < e && cols[p] != col) ++p;
      if (p < e) vals[p] += s.val[q] * tv;
    }
  }
}

}  // namespace

template <typename T>
static cudaError_t upload_vec(T** dst, const std::vector<T>& v, size_t* bytes) {
  const size_t b = std::max<size_t>(1, v.size()) * sizeof(T);
  cudaError_t e = cudaMalloc((void**)dst, b);
  if (e != cudaSuccess) return e;
  *bytes += b;
  if (!v.empty()) e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

bool FDProblem::init(int n_, int ndim_, const int* Ns_, const double* Ls_, const std::vector<HostTerm>& terms_,
                     cudaStream_t st_, std::string* msg) {
  release();
  n = n_;
  ndim = ndim_;
  st = st_;
  terms = terms_;
  N = 1;
  for (int a = 0; a < 3; ++a) {
    Ns[a] = a < ndim ? Ns_[a] : 1;
    Ls[a] = a < ndim ? Ls_[a] : 1.0;
  }
  for (int a = 0; a < ndim; ++a) N *= Ns[a];
  nN = N * n;
  if (nN >= (1LL << 31) - 1) {
    *msg = "state too large for 32-bit CSR indices";
    return false;
  }
  const int nY = 1 + ndim + ndim * ndim;
  FDTables T{};
  T.n = n;
  T.ndim = ndim;
  T.nY = nY;
  T.N = N;
  for (int a = 0; a < 3; ++a) T.Ns[a] = Ns[a];
  for (int a = 0; a < ndim; ++a) {
    const double scale = Ls[a] / Ns[a];  // rdcu.cu:442
    T.s1[a] = 0.5 / scale;
    T.inv_dx[a] = 1.0 / scale;
    for (int b = 0; b < ndim; ++b) T.s2[a][b] = (Ls[a] / Ns[a]) * (Ls[b] / Ns[b]);  // rdcu.cu:496
  }
  // term tables (all factors kept), grouped by field
  std::vector<FDTerm> dterms;
  std::vector<FDFactor> dfac;
  std::vector<int> field_begin(n + 1, 0);
  std::vector<int> term_index_of;  // original term index of each grouped entry
  std::vector<int> grouped_of(terms.size(), -1);
  for (int i = 0; i < n; ++i) {
    field_begin[i] = (int)dterms.size();
    for (size_t t = 0; t < terms.size(); ++t) {
      const auto& ht = terms[t];
      const int field = ht.ints.empty() ? 0 : ht.ints[0];
      if (field != i) continue;
      FDTerm d{};
      d.field = i;
      d.C = ht.C;
      d.off = (int)dfac.size();
      const int np = (int)ht.ints.size();
      for (int j = 1; j < np; j += 2) {
        FDFactor f{};
        f.k = ht.ints[j];
        f.eta = (j + 1 < np) ? ht.ints[j + 1] : 0;
        dfac.push_back(f);
      }
      d.nf = (int)dfac.size() - d.off;
      grouped_of[t] = (int)dterms.size();
      dterms.push_back(d);
    }
  }
  field_begin[n] = (int)dterms.size();
  // Jacobian contributions: reference order is term-major (all fields interleaved);
  // per row field the order is the term order restricted to that field.
  std::vector<JacContrib> contrib;
  std::vector<int> contrib_begin(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    contrib_begin[i] = (int)contrib.size();
    for (size_t t = 0; t < terms.size(); ++t) {
      const int gt = grouped_of[t];
      if (dterms[gt].field != i) continue;
      for (int q = 0; q < dterms[gt].nf; ++q) {
        JacContrib c{};
        c.term = gt;
        c.jf = q;
        c.yind = dfac[dterms[gt].off + q].k / n;
        c.src = dfac[dterms[gt].off + q].k % n;
        contrib.push_back(c);
      }
    }
  }
  contrib_begin[n] = (int)contrib.size();
  T.nterms = (int)dterms.size();
  T.ncontrib = (int)contrib.size();

  // CSR pattern: per row, the sorted union of the contributions' stencil columns
  std::vector<int> rows(nN + 1, 0);
  std::vector<int> cols;
  std::vector<int> diag(nN, -1);
  cols.reserve((size_t)nN * 6);
  std::vector<long long> buf;
  for (int i = 0; i < n; ++i) {
    for (long long j = 0; j < N; ++j) {
      buf.clear();
      for (int c = contrib_begin[i]; c < contrib_begin[i + 1]; ++c) {
        Stencil s;
        stencil_at(T, contrib[c].yind, j, &s);
        for (int q = 0; q < s.m; ++q) buf.push_back(s.col[q] + (long long)contrib[c].src * N);
      }
      std::sort(buf.begin(), buf.end());
      buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
      const long long r = (long long)i * N + j;
      for (long long c : buf) {
        if (c == r) diag[r] = (int)cols.size();
        cols.push_back((int)c);
      }
      rows[r + 1] = (int)cols.size();
      if (cols.size() > (size_t)INT32_MAX - 64) {
        *msg = "Jacobian too large for 32-bit CSR indices";
        return false;
      }
    }
  }
  nnz = (long long)cols.size();
  bool ok = true;
  auto chk = [&](cudaError_t e) {
    if (e != cudaSuccess && ok) {
      ok = false;
      *msg = std::string("out of device memory (FD tables): ") + cudaGetErrorString(e);
    }
  };
  chk(upload_vec(&d_terms_, dterms, &device_bytes));
  chk(upload_vec(&d_fac_, dfac, &device_bytes));
  chk(upload_vec(&d_field_begin_, field_begin, &device_bytes));
  chk(upload_vec(&d_contrib_, contrib, &device_bytes));
  chk(upload_vec(&d_contrib_begin_, contrib_begin, &device_bytes));
  chk(upload_vec(&rows_, rows, &device_bytes));
  chk(upload_vec(&cols_, cols, &device_bytes));
  chk(upload_vec(&diag_, diag, &device_bytes));
  if (ok) {
    chk(cudaMalloc((void**)&vals_, std::max<size_t>(1, (size_t)nnz) * sizeof(double)));
    device_bytes += (size_t)nnz * sizeof(double);
  }
  if (!ok) return false;
  T.terms = d_terms_;
  T.fac = d_fac_;
  T.field_begin = d_field_begin_;
  T.contrib = d_contrib_;
  T.contrib_begin = d_contrib_begin_;
  tab = T;
  return true;
}

void FDProblem::release() {
  void* p[] = {d_terms_, d_fac_, d_field_begin_, d_contrib_, d_contrib_begin_, rows_, cols_, vals_, diag_};
  for (void* q : p)
    if (q) cudaFree(q);
  d_terms_ = nullptr;
  d_fac_ = nullptr;
  d_field_begin_ = nullptr;
  d_contrib_ = nullptr;
  d_contrib_begin_ = nullptr;
  rows_ = nullptr;
  cols_ = nullptr;
  vals_ = nullptr;
  diag_ = nullptr;
  device_bytes = 0;
}

cudaError_t FDProblem::rhs(const double* y, double* f, double* Y) {
  const unsigned blocks = (unsigned)((N + 255) / 256);
  k_fd_rhs<<<blocks, 256, 0, st>>>(tab, y, f);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !Y) return e;
  k_fd_Y<<<blocks, 256, 0, st>>>(tab, y, Y);
  return cudaGetLastError();
}

cudaError_t FDProblem::jac_values(const double* y) {
  const unsigned blocks = (unsigned)((nN + 255) / 256);
  k_fd_jac<<<blocks, 256, 0, st>>>(tab, y, rows_, cols_, vals_);
  return cudaGetLastError();
}

cudaError_t FDProblem::jac_csr(const double* y, int* rows, int* cols, double* vals) {
  cudaError_t e = jac_values(y);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(rows, rows_, (size_t)(nN + 1) * sizeof(int), cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return e;
  if (nnz > 0) {
    e = cudaMemcpyAsync(cols, cols_, (size_t)nnz * sizeof(int), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(vals, vals_, (size_t)nnz * sizeof(double), cudaMemcpyDeviceToDevice, st);
  }
  return e;
}

}  // namespace rdcu
