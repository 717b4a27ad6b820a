// Defect lines of a 3D complex field on the GPU (the reference's post-processing of CGLE
// states, makelines.py): plaquette phase winding, line cubes, their face-neighbour graph,
// its connected components, and the distance matrix between the components of two frames.
//
// Passes of one frame (grid of N points, n line cubes):
//   k_phase     th = atan2(v, u) + pi                              16 B read, 8 B written /pt
//   k_faces     winding of the three plaquettes at every point     8 B read, 1 B written /pt
//   k_mark      line cubes (either side of a winding plaquette)    1 B read, 1 B written /pt
//   k_compact   ascending cube list and the grid -> node map       1 B read, 4 B written /pt
//   k_hook      union-find over face neighbours (lock-free CAS)    per node
//   k_flatten, k_roots, k_label  component of every node, numbered by smallest cube
//   radix passes: nodes stably sorted by component
//   k_edges     each component's edges (u < v ascending) as scaled coordinates
// The grid passes are HBM-bound streaming passes (one thread per point, coalesced along
// the last axis; neighbour reads hit L2).  The graph passes touch only the n line cubes.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <memory>
#include <string>
#include <vector>

#include "../../include/rdcu.h"
#include "internal.h"

namespace rdcu {
namespace {

constexpr double kPi = 3.141592653589793;  // the double nearest pi (numpy's np.pi)
constexpr double kTwoPi = 2.0 * kPi;
constexpr int kT = 256;                     // threads per block
constexpr int kChunk = 1024;                // items per block in counting, compaction, sorting
constexpr int kSlices = kChunk / kT;          // slices of kT items per chunk
constexpr int kUfLimit = 1 << 26;           // bound of a root walk (a path is shorter than the nodes)
constexpr int kUfRetries = 1 << 20;         // bound of the CAS retries of one union

struct Grid {
  int N[3];
  int s0, s1;  // strides of axes 0 and 1 (axis 2 is contiguous)
  int total;
  FastDiv d2, d1;  // by N[2], by N[1]
  double L[3];
};

__device__ __forceinline__ void coords(const Grid& g, int c, int& i, int& j, int& k) {
  const int ij = fdiv(c, g.d2);
  k = c - ij * g.N[2];
  i = fdiv(ij, g.d1);
  j = ij - i * g.N[1];
}

// numpy's floored float modulus of x + pi by 2 pi, minus pi (makelines.py:20-23):
// fmod, then the divisor added to a negative remainder, a zero remainder made +0.
// Differences of phases in [0, 2 pi] put a = x + pi in (-2 pi, 4 pi), where fmod needs no
// division: fmod(a, 2 pi) is a on (-2 pi, 2 pi) and a - 2 pi on [2 pi, 4 pi) (n = 1, and
// the subtraction is exact by Sterbenz's lemma), so both branches give fmod's bits.
__device__ __forceinline__ double wrap_pi(double x) {
  const double a = x + kPi;
  double m;
  if (a > -kTwoPi && a < kTwoPi)
    m = a;
  else if (a >= kTwoPi && a < 2.0 * kTwoPi)
    m = a - kTwoPi;
  else
    m = fmod(a, kTwoPi);
  if (m < 0.0)
    m += kTwoPi;
  else if (m == 0.0)
    m = 0.0;
  return m - kPi;
}

// Nonzero winding of the plaquette t0 -> t1 -> t2 -> t3 (makelines.py:19-24): the four
// wrapped differences summed in that order, over 2 pi, rounded half to even.
// Shortcut with the same answer: when every difference d is below 3 in magnitude, d + pi
// lies in (0.14, 6.15), no branch of wrap_pi adds or subtracts 2 pi, and each wrapped
// difference is d to within two roundings of pi-sized values (~1e-15); the exact
// differences sum to zero, so the rounded ones, and s, stay within ~1e-14 of zero and
// rint(s / 2 pi) is 0.  A NaN fails the comparisons and takes the full path.
__device__ __forceinline__ bool winds(double t0, double t1, double t2, double t3) {
  const double d0 = t1 - t0, d1 = t2 - t1, d2 = t3 - t2, d3 = t0 - t3;
  if (fabs(d0) < 3.0 && fabs(d1) < 3.0 && fabs(d2) < 3.0 && fabs(d3) < 3.0) return false;
  const double s = wrap_pi(d0) + wrap_pi(d1) + wrap_pi(d2) + wrap_pi(d3);
  return rint(s / kTwoPi) != 0.0;
}

__global__ void __launch_bounds__(kT) k_phase(const double* __restrict__ y, double* __restrict__ th, int n) {
  const int p = blockIdx.x * kT + threadIdx.x;
  if (p < n) th[p] = atan2(y[(long long)n + p], y[p]) + kPi;
}

// Face code of point p: bit 0 the (0,1) plaquette p, p+e0, p+e0+e1, p+e1; bit 1 the (1,2)
// plaquette; bit 2 the (2,0) plaquette (axis 2 first, then axis 0).  Periodic.
__global__ void __launch_bounds__(kT) k_faces(const double* __restrict__ th, unsigned char* __restrict__ face,
                                              Grid g) {
  const int p = blockIdx.x * kT + threadIdx.x;
  if (p >= g.total) return;
  int i, j, k;
  coords(g, p, i, j, k);
  const int di = (i + 1 < g.N[0]) ? g.s0 : -(g.N[0] - 1) * g.s0;
  const int dj = (j + 1 < g.N[1]) ? g.s1 : -(g.N[1] - 1) * g.s1;
  const int dk = (k + 1 < g.N[2]) ? 1 : -(g.N[2] - 1);
  const double t = th[p], ti = th[p + di], tj = th[p + dj], tk = th[p + dk];
  const double tij = th[p + di + dj], tjk = th[p + dj + dk], tki = th[p + dk + di];
  unsigned char f = 0;
  if (winds(t, ti, tij, tj)) f |= 1;
  if (winds(t, tj, tjk, tk)) f |= 2;
  if (winds(t, tk, tki, ti)) f |= 4;
  face[p] = f;
}

__device__ __forceinline__ int block_sum(int v, int* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  int s = 0;
  for (int w = 0; w < kT / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

// Line cube c: a winding plaquette on one of its six faces.  A (0,1) plaquette at p
// borders cubes p and p - e2, a (1,2) one p and p - e0, a (2,0) one p and p - e1
// (makelines.py:28-36), so cube c looks at its own three faces and at the (0,1) face of
// c + e2, the (1,2) face of c + e0 and the (2,0) face of c + e1.
__global__ void __launch_bounds__(kT) k_mark(const unsigned char* __restrict__ face, unsigned char* __restrict__ mark,
                                             int* __restrict__ counts, Grid g) {
  __shared__ int red[kT / 32];
  int cnt = 0;
  for (int r = 0; r < kSlices; ++r) {
    const int c = blockIdx.x * kChunk + r * kT + threadIdx.x;
    if (c < g.total) {
      int i, j, k;
      coords(g, c, i, j, k);
      const int di = (i + 1 < g.N[0]) ? g.s0 : -(g.N[0] - 1) * g.s0;
      const int dj = (j + 1 < g.N[1]) ? g.s1 : -(g.N[1] - 1) * g.s1;
      const int dk = (k + 1 < g.N[2]) ? 1 : -(g.N[2] - 1);
      const int m = ((face[c] & 7) | (face[c + dk] & 1) | (face[c + di] & 2) | (face[c + dj] & 4)) != 0;
      mark[c] = (unsigned char)m;
      cnt += m;
    }
  }
  const int s = block_sum(cnt, red);
  if (threadIdx.x == 0) counts[blockIdx.x] = s;
}

// Exclusive prefix of one slice's flags over the block, in index order; returns the
// block's total for the slice.
__device__ __forceinline__ int block_rank(bool f, int* wcnt, int* pre) {
  const unsigned b = __ballot_sync(0xffffffffu, f);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wcnt[w] = __popc(b);
  __syncthreads();
  int off = 0, tot = 0;
  for (int q = 0; q < kT / 32; ++q) {
    off += (q < w) ? wcnt[q] : 0;
    tot += wcnt[q];
  }
  *pre = off + __popc(b & ((1u << lane) - 1u));
  __syncthreads();
  return tot;
}

// Cubes in ascending index order (np.unique order of makelines.py:38-39), the grid ->
// node map (-1 off the lines) and the union-find forest's initial singletons.
__global__ void __launch_bounds__(kT) k_compact(const unsigned char* __restrict__ mark, const int* __restrict__ offs,
                                                int* __restrict__ cubes, int* __restrict__ node_of,
                                                int* __restrict__ parent, int total) {
  __shared__ int wcnt[kT / 32];
  int run = offs[blockIdx.x];
  for (int r = 0; r < kSlices; ++r) {
    const int c = blockIdx.x * kChunk + r * kT + threadIdx.x;
    const bool m = c < total && mark[c];
    int pre;
    const int tot = block_rank(m, wcnt, &pre);
    if (c < total) {
      if (m) {
        const int v = run + pre;
        cubes[v] = c;
        node_of[c] = v;
        parent[v] = v;
      } else {
        node_of[c] = -1;
      }
    }
    run += tot;
  }
}

// Face neighbours of cube c (periodic): up to two per axis of length >= 3, one per axis of
// length 2 (both steps reach the same cube) -- the cubes at per-axis distance
// ((d + N/2) mod N) - N/2 summing to 1 in absolute value (makelines.py:41-50).
__device__ __forceinline__ int face_neighbours(const Grid& g, int c, int* nb) {
  int i, j, k;
  coords(g, c, i, j, k);
  int n = 0;
  const int x[3] = {i, j, k};
  const int s[3] = {g.s0, g.s1, 1};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int N = g.N[a];
    nb[n++] = c + ((x[a] + 1 < N) ? s[a] : -(N - 1) * s[a]);
    if (N > 2) nb[n++] = c + ((x[a] > 0) ? -s[a] : (N - 1) * s[a]);
  }
  return n;
}

// Root of x's tree, or -1 (error flagged) past the iteration bound.  Parents only ever
// point to smaller nodes, so the walk ends; path halving rewrites x's parent to its
// grandparent (another ancestor, so racing writes keep the forest valid).
__device__ int uf_find(int* parent, int x, int* err) {
  volatile int* P = parent;
  for (int it = 0; it < kUfLimit; ++it) {
    const int p = P[x];
    if (p == x) return x;
    const int gp = P[p];
    if (gp != p) P[x] = gp;
    x = gp;
  }
  atomicExch(err, 1);
  return -1;
}

// Link the two roots, the larger under the smaller: every root is the smallest node of
// its tree, so a component's final root is its smallest cube.  A failed CAS means another
// thread linked that root first; retry from the new roots.
__device__ void uf_union(int* parent, int a, int b, int* err) {
  for (int it = 0; it < kUfRetries; ++it) {
    a = uf_find(parent, a, err);
    b = uf_find(parent, b, err);
    if (a < 0 || b < 0 || a == b) return;
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(parent + a, a, b) == a) return;
  }
  atomicExch(err, 1);
}

__global__ void __launch_bounds__(kT) k_hook(const int* __restrict__ cubes, const int* __restrict__ node_of,
                                             int* parent, int* __restrict__ deg, int n, Grid g, int* err,
                                             int* n_edges) {
  const int v = blockIdx.x * kT + threadIdx.x;
  int d = 0;
  if (v < n) {
    int nb[6];
    const int cnt = face_neighbours(g, cubes[v], nb);
    for (int q = 0; q < cnt; ++q) {
      const int u = node_of[nb[q]];
      if (u > v) {
        ++d;
        uf_union(parent, v, u, err);
      }
    }
    deg[v] = d;
  }
  for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
  if ((threadIdx.x & 31) == 0 && d) atomicAdd(n_edges, d);
}

__global__ void __launch_bounds__(kT) k_flatten(int* parent, int* __restrict__ label, int n, int* counts, int* err) {
  __shared__ int red[kT / 32];
  int cnt = 0;
  for (int r = 0; r < kSlices; ++r) {
    const int v = blockIdx.x * kChunk + r * kT + threadIdx.x;
    if (v < n) {
      int root = uf_find(parent, v, err);
      if (root < 0) root = v;  // error flagged; keeps the later passes in bounds
      label[v] = root;
      cnt += root == v;
    }
  }
  const int s = block_sum(cnt, red);
  if (threadIdx.x == 0) counts[blockIdx.x] = s;
}

// Component number of every root, in root order (= smallest-cube order, the order
// networkx's connected_components yields).
__global__ void __launch_bounds__(kT) k_roots(const int* __restrict__ label, const int* __restrict__ offs,
                                              int* __restrict__ comp_of_root, int n) {
  __shared__ int wcnt[kT / 32];
  int run = offs[blockIdx.x];
  for (int r = 0; r < kSlices; ++r) {
    const int v = blockIdx.x * kChunk + r * kT + threadIdx.x;
    const bool f = v < n && label[v] == v;
    int pre;
    const int tot = block_rank(f, wcnt, &pre);
    if (f) comp_of_root[v] = run + pre;
    run += tot;
  }
}

// The components of a frame with few line cubes in one CTA: the forest, its roots and
// their numbering in shared memory (atomics and root walks at shared-memory latency), the
// same union-find rules as k_hook / k_flatten / k_roots / k_label, so the labels and the
// component numbers are identical.  Writes deg, comp, key, order and the component count
// to *n_comp.
constexpr int kSmallThreads = 1024;
constexpr int kSmallNodes = 12288;  // 2 x 4 B per node of shared memory (96 KB)

__device__ int uf_find_s(int* parent, int x, int* err) {
  volatile int* P = parent;
  for (int it = 0; it < kUfLimit; ++it) {
    const int p = P[x];
    if (p == x) return x;
    const int gp = P[p];
    if (gp != p) P[x] = gp;
    x = gp;
  }
  atomicExch(err, 1);
  return -1;
}

__global__ void __launch_bounds__(kSmallThreads) k_components_small(const int* __restrict__ cubes,
                                                                     const int* __restrict__ node_of,
                                                                     int* __restrict__ deg, int* __restrict__ comp,
                                                                     int* __restrict__ key, int* __restrict__ order,
                                                                     int n, Grid g, int* err, int* n_comp,
                                                                     int* n_edges) {
  extern __shared__ int sm_int[];
  int* parent = sm_int;          // [n]
  int* croot = sm_int + n;       // [n]: label, then component of each root
  __shared__ int red[kSmallThreads / 32];
  __shared__ int run;
  for (int v = threadIdx.x; v < n; v += kSmallThreads) parent[v] = v;
  __syncthreads();
  int dsum = 0;
  for (int v = threadIdx.x; v < n; v += kSmallThreads) {
    int nb[6];
    const int cnt = face_neighbours(g, cubes[v], nb);
    int d = 0;
    for (int q = 0; q < cnt; ++q) {
      const int u = node_of[nb[q]];
      if (u <= v) continue;
      ++d;
      int a = v, b = u;
      for (int it = 0; it < kUfRetries; ++it) {
        a = uf_find_s(parent, a, err);
        b = uf_find_s(parent, b, err);
        if (a < 0 || b < 0 || a == b) break;
        if (a < b) {
          const int t = a;
          a = b;
          b = t;
        }
        if (atomicCAS(parent + a, a, b) == a) break;
        if (it == kUfRetries - 1) atomicExch(err, 1);
      }
    }
    deg[v] = d;
    dsum += d;
  }
  for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
  if ((threadIdx.x & 31) == 0 && dsum) atomicAdd(n_edges, dsum);
  __syncthreads();
  for (int v = threadIdx.x; v < n; v += kSmallThreads) {
    int r = uf_find_s(parent, v, err);
    croot[v] = r < 0 ? v : r;
  }
  __syncthreads();
  for (int v = threadIdx.x; v < n; v += kSmallThreads) parent[v] = croot[v];  // labels
  if (threadIdx.x == 0) run = 0;
  __syncthreads();
  // roots numbered in node order: ordered block scan over slices of kSmallThreads
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < n; base += kSmallThreads) {
    const int v = base + threadIdx.x;
    const bool f = v < n && parent[v] == v;
    const unsigned b = __ballot_sync(0xffffffffu, f);
    if (lane == 0) red[w] = __popc(b);
    __syncthreads();
    int off = 0, tot = 0;
    for (int q = 0; q < kSmallThreads / 32; ++q) {
      off += (q < w) ? red[q] : 0;
      tot += red[q];
    }
    if (f) croot[v] = run + off + __popc(b & ((1u << lane) - 1u));
    __syncthreads();
    if (threadIdx.x == 0) run += tot;
    __syncthreads();
  }
  for (int v = threadIdx.x; v < n; v += kSmallThreads) {
    const int c = croot[parent[v]];
    comp[v] = c;
    key[v] = c;
    order[v] = v;
  }
  if (threadIdx.x == 0) *n_comp = run;
}

__global__ void __launch_bounds__(kT) k_label(const int* __restrict__ label, const int* __restrict__ comp_of_root,
                                              int* __restrict__ comp, int* __restrict__ key, int* __restrict__ order,
                                              int n) {
  const int v = blockIdx.x * kT + threadIdx.x;
  if (v < n) {
    const int c = comp_of_root[label[v]];
    comp[v] = c;
    key[v] = c;
    order[v] = v;
  }
}

// ---- exclusive scan of an int array (two levels: chunk sums, one-block scan, chunk scan)
__device__ __forceinline__ int block_excl_scan(int v, int* red, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) red[w] = x;
  __syncthreads();
  int off = 0, tot = 0;
  for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
    off += (q < w) ? red[q] : 0;
    tot += red[q];
  }
  __syncthreads();
  *total = tot;
  return off + x - v;
}

__global__ void __launch_bounds__(kT) k_chunk_sums(const int* __restrict__ a, int n, int* __restrict__ sums) {
  __shared__ int red[kT / 32];
  int s = 0;
  for (int r = 0; r < kSlices; ++r) {
    const int i = blockIdx.x * kChunk + r * kT + threadIdx.x;
    if (i < n) s += a[i];
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) sums[blockIdx.x] = s;
}

// One block of 1024 threads: exclusive scan of a[0..n) in place; total to *total.
__global__ void __launch_bounds__(1024) k_scan_one(int* a, int n, int* total) {
  __shared__ int red[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < n ? a[i] : 0;
    int tot;
    const int e = block_excl_scan(v, red, &tot);
    if (i < n) a[i] = carry + e;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void __launch_bounds__(kT) k_chunk_scan(int* a, int n, const int* __restrict__ sums) {
  __shared__ int red[kT / 32];
  int run = sums[blockIdx.x];
  for (int r = 0; r < kSlices; ++r) {
    const int i = blockIdx.x * kChunk + r * kT + threadIdx.x;
    const int v = i < n ? a[i] : 0;
    int tot;
    const int e = block_excl_scan(v, red, &tot);
    if (i < n) a[i] = run + e;
    run += tot;
  }
}

// ---- stable LSD radix sort of (component, node) pairs by component, 8 bits a pass
__global__ void __launch_bounds__(kT) k_rs_hist(const int* __restrict__ key, int n, int shift, int* __restrict__ hist,
                                                int nblk) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  for (int r = 0; r < kSlices; ++r) {
    const int i = blockIdx.x * kChunk + r * kT + threadIdx.x;
    if (i < n) atomicAdd(&h[(key[i] >> shift) & 255], 1);
  }
  __syncthreads();
  hist[threadIdx.x * nblk + blockIdx.x] = h[threadIdx.x];
}

// Items of a chunk keep their order within a digit: each slice's lanes are ranked among
// equal digits of their warp (match_any), warps among the warps before them, slices after
// the slices before them.
__global__ void __launch_bounds__(kT) k_rs_scatter(const int* __restrict__ kin, const int* __restrict__ vin,
                                                   int* __restrict__ kout, int* __restrict__ vout, int n, int shift,
                                                   const int* __restrict__ hist, int nblk) {
  __shared__ int base[256];
  __shared__ int wc[kT / 32][256];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  base[threadIdx.x] = hist[threadIdx.x * nblk + blockIdx.x];
  for (int q = 0; q < kT / 32; ++q) wc[q][threadIdx.x] = 0;
  __syncthreads();
  for (int r = 0; r < kSlices; ++r) {
    const int i = blockIdx.x * kChunk + r * kT + threadIdx.x;
    const bool ok = i < n;
    const int key = ok ? kin[i] : 0;
    const int d = ok ? (key >> shift) & 255 : 256;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (ok && lane == __ffs(peers) - 1) wc[w][d] = __popc(peers);
    __syncthreads();
    if (ok) {
      int off = base[d] + rank;
      for (int q = 0; q < w; ++q) off += wc[q][d];
      kout[off] = key;
      vout[off] = vin[i];
    }
    __syncthreads();
    int add = 0;
    for (int q = 0; q < kT / 32; ++q) {
      add += wc[q][threadIdx.x];
      wc[q][threadIdx.x] = 0;
    }
    base[threadIdx.x] += add;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kT) k_edge_counts(const int* __restrict__ order, const int* __restrict__ deg,
                                                    int* __restrict__ edeg, int n) {
  const int p = blockIdx.x * kT + threadIdx.x;
  if (p < n) edeg[p] = deg[order[p]];
}

__device__ __forceinline__ double scaled(int c, int a, const Grid& g) {
  // (c * L) / (N - 1), in that order (makelines.py:56)
  return ((double)c * g.L[a]) / (double)(g.N[a] - 1);
}

// Node p of the component-sorted order writes its edges to the nodes above it, in
// ascending order, and the offsets of its component when it is the component's first.
__global__ void __launch_bounds__(kT) k_edges(const int* __restrict__ order, const int* __restrict__ eoff,
                                              const int* __restrict__ cubes, const int* __restrict__ node_of,
                                              const int* __restrict__ comp, Grid g, double* __restrict__ xyz,
                                              long long* __restrict__ comp_noff, long long* __restrict__ comp_eoff,
                                              int n, int n_comp, int n_edges) {
  const int p = blockIdx.x * kT + threadIdx.x;
  if (p >= n) return;
  const int v = order[p];
  const int c = cubes[v];
  int nb[6];
  const int cnt = face_neighbours(g, c, nb);
  int up[6], m = 0;
  for (int q = 0; q < cnt; ++q) {
    const int u = node_of[nb[q]];
    if (u > v) {
      int s = m++;
      while (s > 0 && up[s - 1] > u) {
        up[s] = up[s - 1];
        --s;
      }
      up[s] = u;
    }
  }
  int i, j, k;
  coords(g, c, i, j, k);
  const double xv[3] = {scaled(i, 0, g), scaled(j, 1, g), scaled(k, 2, g)};
  long long e = eoff[p];
  for (int q = 0; q < m; ++q, ++e) {
    int iu, ju, ku;
    coords(g, cubes[up[q]], iu, ju, ku);
    double* o = xyz + e * 6;
    o[0] = xv[0];
    o[1] = xv[1];
    o[2] = xv[2];
    o[3] = scaled(iu, 0, g);
    o[4] = scaled(ju, 1, g);
    o[5] = scaled(ku, 2, g);
  }
  const int cv = comp[v];
  if (p == 0 || comp[order[p - 1]] != cv) {
    comp_noff[cv] = p;
    comp_eoff[cv] = eoff[p];
  }
  if (p == n - 1) {
    comp_noff[n_comp] = n;
    comp_eoff[n_comp] = n_edges;
  }
}

// Cube coordinates of the component-sorted nodes for the distance matrix, as the
// reference's correlate recovers them from the scaled edge coordinates x:
// rint(x / s) for the earlier frame, trunc(x / s) for the later one, s = L / (N - 1)
// (makelines.py:115,120).
__global__ void __launch_bounds__(kT) k_pack(const int* __restrict__ order, const int* __restrict__ cubes,
                                             const int* __restrict__ comp, Grid g, double s0, double s1, double s2,
                                             int truncate, int4* __restrict__ out, int n) {
  const int p = blockIdx.x * kT + threadIdx.x;
  if (p >= n) return;
  const int v = order[p];
  int x[3];
  coords(g, cubes[v], x[0], x[1], x[2]);
  const double s[3] = {s0, s1, s2};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double q = scaled(x[a], a, g) / s[a];
    x[a] = truncate ? (int)q : (int)rint(q);
  }
  out[p] = make_int4(x[0], x[1], x[2], comp[v]);
}

__global__ void __launch_bounds__(kT) k_pack_sets(const long long* __restrict__ cubes, const long long* __restrict__ off,
                                                  int n_comp, Grid g, int4* __restrict__ out, int n, int* err) {
  const int p = blockIdx.x * kT + threadIdx.x;
  if (p >= n) return;
  const long long c = cubes[p];
  if (c < 0 || c >= g.total) {
    atomicExch(err, 1);
    out[p] = make_int4(0, 0, 0, -1);
    return;
  }
  int lo = 0, hi = n_comp - 1;  // component of p: last c with off[c] <= p
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= p)
      lo = mid;
    else
      hi = mid - 1;
  }
  int i, j, k;
  coords(g, (int)c, i, j, k);
  out[p] = make_int4(i, j, k, lo);
}

__global__ void k_fill(int* a, long long n, int v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = v;
}

__device__ __forceinline__ int axis_dist(int a, int b, int N) {
  // |((a - b + N/2) mod N) - N/2| with a floored modulus (makelines.py:133-134).  For
  // a, b in [0, N) that is the minimum image min(|a - b|, N - |a - b|): the modulus maps
  // a - b into [-N/2, N - N/2), where |t| is the shorter way round (both equal N/2 when
  // |a - b| = N/2).
  const int d = abs(a - b);
  return min(d, N - d);
}

// diffs[j][i] = min over cubes a of component i (frame A) and b of component j (frame B)
// of the periodic L1 distance.  One thread per cube of B, blockIdx.y picks a span of
// a_span cubes of A; A streams through shared memory in component order, so each thread
// keeps a running minimum per A component and flushes it with one atomicMin (one per warp
// when the warp's B cubes share a component).
__global__ void __launch_bounds__(kT) k_corr(const int4* __restrict__ A, int nA, const int4* __restrict__ B, int nB,
                                             Grid g, int* __restrict__ diffs, int n_comp_a, int a_span) {
  __shared__ int4 tile[kT];
  const unsigned full = 0xffffffffu;
  const int jb = blockIdx.x * kT + threadIdx.x;
  const bool ok = jb < nB;
  const int4 b = ok ? B[jb] : make_int4(0, 0, 0, -1);
  const int c0 = __shfl_sync(full, b.w, 0);
  const bool uniform = __all_sync(full, !ok || b.w == c0) && c0 >= 0;
  int cur = -1, best = INT_MAX;
  auto flush = [&]() {
    if (cur < 0) return;
    if (uniform) {
      int m = ok ? best : INT_MAX;
      for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(full, m, o));
      if ((threadIdx.x & 31) == 0) atomicMin(&diffs[(long long)c0 * n_comp_a + cur], m);
    } else if (ok) {
      atomicMin(&diffs[(long long)b.w * n_comp_a + cur], best);
    }
  };
  const int a0 = blockIdx.y * a_span, a1 = min(nA, a0 + a_span);
  for (int t0 = a0; t0 < a1; t0 += kT) {
    __syncthreads();
    if (t0 + threadIdx.x < a1) tile[threadIdx.x] = A[t0 + threadIdx.x];
    __syncthreads();
    const int cnt = min(kT, a1 - t0);
    for (int q = 0; q < cnt; ++q) {
      const int4 a = tile[q];
      if (a.w != cur) {
        flush();
        cur = a.w;
        best = INT_MAX;
      }
      const int d = axis_dist(a.x, b.x, g.N[0]) + axis_dist(a.y, b.y, g.N[1]) + axis_dist(a.z, b.z, g.N[2]);
      best = min(best, d);
    }
  }
  flush();
}

__global__ void __launch_bounds__(kT) k_gather_cubes(const int* __restrict__ order, const int* __restrict__ cubes,
                                                     long long* __restrict__ out, int n) {
  const int p = blockIdx.x * kT + threadIdx.x;
  if (p < n) out[p] = cubes[order[p]];
}

__global__ void k_widen(const int* __restrict__ a, long long* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i];
}

inline int nblocks(long long n, int per) { return (int)((n + per - 1) / per); }

// A device array that grows on demand (capacity 1.5x the request), counted in *bytes.
template <typename T>
struct Buf {
  T* p = nullptr;
  long long cap = 0;
  bool ensure(long long n, size_t* bytes, cudaStream_t st) {
    if (n <= cap && p) return true;
    if (p) {
      cudaStreamSynchronize(st);
      cudaFree(p);
      *bytes -= (size_t)cap * sizeof(T);
      p = nullptr;
      cap = 0;
    }
    const long long c = std::max<long long>(n + n / 2, 1024);
    if (cudaMalloc((void**)&p, (size_t)c * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return false;
    }
    cap = c;
    *bytes += (size_t)c * sizeof(T);
    return true;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace

// ------------------------------------------------------------------------------ engine
// Workspace and results of one frame of one grid.  Grid-sized buffers are allocated at
// init; node, component and edge buffers grow with the largest frame seen.
class LinesEngine {
 public:
  Grid g{};
  cudaStream_t st = nullptr;
  int device = 0;
  size_t device_bytes = 0;
  long long n_cubes = 0, n_edges = 0, n_comp = 0;  // of the last frame
  long long launches = 0;                          // kernels launched since init
  bool have = false;

  bool init(const int Ns[3], const double Ls[3], int dev, std::string* msg) {
    device = dev;
    long long total = 1;
    for (int a = 0; a < 3; ++a) {
      if (Ns[a] < 2) return fail(msg, "grid sizes must be >= 2 on every axis");
      if (!(Ls[a] != 0.0)) return fail(msg, "domain lengths must be nonzero");
      g.N[a] = Ns[a];
      g.L[a] = Ls[a];
      total *= Ns[a];
    }
    // edges (at most 3 per cube) are counted in int
    if (total > (1ll << 29)) return fail(msg, "grids above 2^29 points are not supported");
    g.total = (int)total;
    g.s1 = Ns[2];
    g.s0 = Ns[1] * Ns[2];
    g.d2 = make_fastdiv((unsigned)Ns[2]);
    g.d1 = make_fastdiv((unsigned)Ns[1]);
    if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&cst_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_main_, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_staged_, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return fail(msg, "cannot create a stream on the device");
    }
    if (cudaFuncSetAttribute(k_components_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSmallNodes * 2 * (int)sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      return fail(msg, "cannot configure shared memory");
    }
    const long long N = g.total;
    if (!th_.ensure(N, &device_bytes, st) || !src_.ensure(2 * N, &device_bytes, st) ||
        !face_.ensure(N, &device_bytes, st) || !mark_.ensure(N, &device_bytes, st) ||
        !node_of_.ensure(N, &device_bytes, st) || !counts_.ensure(nblocks(N, kChunk) + 1, &device_bytes, st) ||
        !flags_.ensure(4, &device_bytes, st) || cudaMallocHost((void**)&h_small_, 4 * sizeof(long long)) != cudaSuccess)
      return fail(msg, "device memory");
    return true;
  }

  void release() {
    for (Buf<int>* b : {&node_of_, &counts_, &sums_, &flags_, &cubes_, &parent_, &deg_, &label_, &root_comp_, &comp_,
                        &key_a_, &key_b_, &order_, &val_tmp_, &eoff_, &hist_, &diff32_})
      b->release();
    th_.release();
    src_.release();
    xyz_.release();
    face_.release();
    mark_.release();
    wide_.release();
    comp_noff_.release();
    comp_eoff_.release();
    diff64_.release();
    sets_.release();
    packed_.release();
    packed_b_.release();
    if (h_small_) cudaFreeHost(h_small_);
    h_small_ = nullptr;
    if (cst_) cudaStreamSynchronize(cst_);
    if (ev_main_) cudaEventDestroy(ev_main_);
    if (ev_staged_) cudaEventDestroy(ev_staged_);
    if (cst_) cudaStreamDestroy(cst_);
    if (st) cudaStreamDestroy(st);
    st = cst_ = nullptr;
    ev_main_ = ev_staged_ = nullptr;
  }
  ~LinesEngine() { release(); }

  // One frame from src: the 2-field state (RDCU_LINES_STATE, u block then v block) or the
  // phase field (RDCU_LINES_PHASE), on the device or the host.
  // Starts copying the next frame (host memory; pinned for the copy to overlap) into the
  // staging buffer on the copy stream, after this handle's queued work; find(nullptr)
  // then uses it.  The handle's current results are not touched.
  int prefetch(const double* src, int kind, std::string* msg) {
    const long long len = kind == RDCU_LINES_STATE ? 2ll * g.total : g.total;
    if (!ck(cudaEventRecord(ev_main_, st), msg) || !ck(cudaStreamWaitEvent(cst_, ev_main_, 0), msg) ||
        !ck(cudaMemcpyAsync(src_.p, src, len * sizeof(double), cudaMemcpyDefault, cst_), msg) ||
        !ck(cudaEventRecord(ev_staged_, cst_), msg))
      return RDCU_ERR_CUDA;
    staged_kind_ = kind;
    return RDCU_OK;
  }

  int find(const double* src, int kind, bool on_device, std::string* msg) {
    have = false;
    packed_mode_ = -1;
    const int N = g.total;
    const long long len = kind == RDCU_LINES_STATE ? 2ll * N : N;
    const double* d = src;
    if (src && staged_kind_ >= 0) {  // a prefetch still copying into the staging buffer
      if (!ck(cudaStreamWaitEvent(st, ev_staged_, 0), msg)) return RDCU_ERR_CUDA;
      staged_kind_ = -1;
    }
    if (!src) {  // the prefetched frame
      if (staged_kind_ != kind) return fail_code(msg, "no prefetched frame of this kind", RDCU_ERR_STATE);
      staged_kind_ = -1;
      if (!ck(cudaStreamWaitEvent(st, ev_staged_, 0), msg)) return RDCU_ERR_CUDA;
      d = src_.p;
    } else if (!on_device) {
      if (!ck(cudaMemcpyAsync(src_.p, src, len * sizeof(double), cudaMemcpyDefault, st), msg)) return RDCU_ERR_CUDA;
      d = src_.p;
    }
    const double* th = d;
    if (kind == RDCU_LINES_STATE) {
      launch(k_phase, nblocks(N, kT), kT, d, th_.p, N);
      th = th_.p;
    }
    const int nb = nblocks(N, kChunk);
    launch(k_faces, nblocks(N, kT), kT, th, face_.p, g);
    launch(k_mark, nb, kT, face_.p, mark_.p, counts_.p, g);
    int rc = scan(counts_.p, nb, msg);
    if (rc) return rc;
    const long long n = read_total(msg);
    if (n < 0) return RDCU_ERR_CUDA;
    n_cubes = n;
    n_edges = n_comp = 0;
    if (!ensure_nodes(n)) return fail_code(msg, "device memory", RDCU_ERR_NOMEM);
    if (!ck(cudaMemsetAsync(flags_.p, 0, 3 * sizeof(int), st), msg)) return RDCU_ERR_CUDA;
    launch(k_compact, nb, kT, mark_.p, counts_.p, cubes_.p, node_of_.p, parent_.p, N);
    if (n > 0) {
      const int nn = (int)n;
      const int nbn = nblocks(n, kChunk);
      if ((rc = components(nn, msg))) return rc;
      // one read: union-find error flag, component count, edge count
      int* hf = reinterpret_cast<int*>(h_small_);
      if (!ck(cudaMemcpyAsync(hf, flags_.p, 3 * sizeof(int), cudaMemcpyDeviceToHost, st), msg) ||
          !ck(cudaStreamSynchronize(st), msg))
        return RDCU_ERR_CUDA;
      if (hf[0] != 0) return fail_code(msg, "union-find iteration bound reached", RDCU_ERR_TIMEOUT);
      const long long nc = hf[1], ne = hf[2];
      n_comp = nc;
      n_edges = ne;
      if (!comp_noff_.ensure(nc + 1, &device_bytes, st) || !comp_eoff_.ensure(nc + 1, &device_bytes, st) ||
          !xyz_.ensure(ne * 6, &device_bytes, st))
        return fail_code(msg, "device memory", RDCU_ERR_NOMEM);
      // nodes stably sorted by component, 8 bits a pass; then the edges (no further host
      // reads: edges(), cubes() and correlate() synchronise before using the results)
      int *k0 = key_a_.p, *v0 = order_.p, *k1 = key_b_.p, *v1 = val_tmp_.p;
      for (int shift = 0; ((nc - 1) >> shift) > 0; shift += 8) {
        launch(k_rs_hist, nbn, kT, k0, nn, shift, hist_.p, nbn);
        if ((rc = scan(hist_.p, 256 * nbn, msg))) return rc;
        launch(k_rs_scatter, nbn, kT, k0, v0, k1, v1, nn, shift, hist_.p, nbn);
        std::swap(k0, k1);
        std::swap(v0, v1);
      }
      sorted_ = v0;
      launch(k_edge_counts, nblocks(n, kT), kT, sorted_, deg_.p, eoff_.p, nn);
      if ((rc = scan(eoff_.p, nn, msg))) return rc;
      launch(k_edges, nblocks(n, kT), kT, sorted_, eoff_.p, cubes_.p, node_of_.p, comp_.p, g, xyz_.p, comp_noff_.p,
             comp_eoff_.p, nn, (int)nc, (int)ne);
    }
    if (!ck(cudaGetLastError(), msg)) return RDCU_ERR_CUDA;
    have = true;
    return RDCU_OK;
  }

  // Times the passes of find on src: one find for the sizes, then `reps` runs of the same
  // launches (no host reads; the sizes are known) with CUDA events between the groups.
  // Each entry: name, mean ms, algorithmic bytes (grid passes: bytes per point x N; the
  // graph groups: the arrays they must read and write once per node or edge).
  struct PassTime {
    const char* name;
    double ms, bytes;
  };
  int profile(const double* src, int kind, bool on_device, int reps, std::vector<PassTime>* out, std::string* msg) {
    int rc = find(src, kind, on_device, msg);
    if (rc) return rc;
    const int N = g.total, nb = nblocks(N, kChunk);
    const int nn = (int)n_cubes, nbn = nblocks(n_cubes, kChunk), nc = (int)n_comp, ne = (int)n_edges;
    const double* d = on_device ? src : src_.p;
    const double* th = kind == RDCU_LINES_STATE ? th_.p : d;
    const char* names[7] = {"phase", "faces", "mark", "compact", "components", "sort", "edges"};
    int passes = 0;
    for (int shift = 0; nc > 1 && ((nc - 1) >> shift) > 0; shift += 8) ++passes;
    const double bytes[7] = {kind == RDCU_LINES_STATE ? 24.0 * N : 0.0, 9.0 * N, 2.0 * N,
                             5.0 * N + 12.0 * nn, 48.0 * nn, 16.0 * passes * nn, 28.0 * nn + 48.0 * ne};
    cudaEvent_t ev[8];
    for (auto& e : ev)
      if (!ck(cudaEventCreate(&e), msg)) return RDCU_ERR_CUDA;
    std::vector<double> acc(7, 0.0);
    for (int r = 0; r < reps && rc == RDCU_OK; ++r) {
      cudaEventRecord(ev[0], st);
      if (kind == RDCU_LINES_STATE) launch(k_phase, nblocks(N, kT), kT, d, th_.p, N);
      cudaEventRecord(ev[1], st);
      launch(k_faces, nblocks(N, kT), kT, th, face_.p, g);
      cudaEventRecord(ev[2], st);
      launch(k_mark, nb, kT, face_.p, mark_.p, counts_.p, g);
      rc = scan(counts_.p, nb, msg);
      cudaEventRecord(ev[3], st);
      launch(k_compact, nb, kT, mark_.p, counts_.p, cubes_.p, node_of_.p, parent_.p, N);
      cudaEventRecord(ev[4], st);
      if (nn > 0 && rc == RDCU_OK) {
        cudaMemsetAsync(flags_.p, 0, 3 * sizeof(int), st);
        rc = components(nn, msg);
      }
      cudaEventRecord(ev[5], st);
      int *k0 = key_a_.p, *v0 = order_.p, *k1 = key_b_.p, *v1 = val_tmp_.p;
      for (int shift = 0; nn > 0 && rc == RDCU_OK && ((nc - 1) >> shift) > 0; shift += 8) {
        launch(k_rs_hist, nbn, kT, k0, nn, shift, hist_.p, nbn);
        rc = scan(hist_.p, 256 * nbn, msg);
        launch(k_rs_scatter, nbn, kT, k0, v0, k1, v1, nn, shift, hist_.p, nbn);
        std::swap(k0, k1);
        std::swap(v0, v1);
      }
      cudaEventRecord(ev[6], st);
      if (nn > 0 && rc == RDCU_OK) {
        launch(k_edge_counts, nblocks(nn, kT), kT, v0, deg_.p, eoff_.p, nn);
        rc = scan(eoff_.p, nn, msg);
        launch(k_edges, nblocks(nn, kT), kT, v0, eoff_.p, cubes_.p, node_of_.p, comp_.p, g, xyz_.p, comp_noff_.p,
               comp_eoff_.p, nn, nc, ne);
      }
      cudaEventRecord(ev[7], st);
      if (!ck(cudaEventSynchronize(ev[7]), msg)) rc = RDCU_ERR_CUDA;
      for (int i = 0; i < 7 && rc == RDCU_OK; ++i) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
        acc[i] += ms;
      }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    if (!ck(cudaGetLastError(), msg)) return RDCU_ERR_CUDA;
    out->clear();
    for (int i = 0; i < 7; ++i)
      if (i > 0 || kind == RDCU_LINES_STATE) out->push_back({names[i], acc[i] / reps, bytes[i]});
    return RDCU_OK;
  }

  // edges (n_edges x 2 x 3 doubles) and the component offsets into them (n_comp + 1)
  int edges(double* xyz, long long* comp_off, std::string* msg) {
    if (!have) return fail_code(msg, "no frame found yet", RDCU_ERR_STATE);
    if (xyz && n_edges && !ck(cudaMemcpyAsync(xyz, xyz_.p, n_edges * 6 * sizeof(double), cudaMemcpyDefault, st), msg))
      return RDCU_ERR_CUDA;
    if (comp_off && !copy_offsets(comp_off, comp_eoff_.p, msg)) return RDCU_ERR_CUDA;
    return ck(cudaStreamSynchronize(st), msg) ? RDCU_OK : RDCU_ERR_CUDA;
  }

  // cubes grouped by component (ascending within each) and the component offsets into
  // them (n_comp + 1)
  int cubes(long long* idx, long long* comp_off, std::string* msg) {
    if (!have) return fail_code(msg, "no frame found yet", RDCU_ERR_STATE);
    const long long n = n_cubes;
    if (idx && n) {
      if (!wide_.ensure(n, &device_bytes, st)) return fail_code(msg, "device memory", RDCU_ERR_NOMEM);
      launch(k_gather_cubes, nblocks(n, kT), kT, sorted_, cubes_.p, wide_.p, (int)n);
      if (!ck(cudaMemcpyAsync(idx, wide_.p, n * sizeof(long long), cudaMemcpyDefault, st), msg)) return RDCU_ERR_CUDA;
    }
    if (comp_off && !copy_offsets(comp_off, comp_noff_.p, msg)) return RDCU_ERR_CUDA;
    return ck(cudaStreamSynchronize(st), msg) ? RDCU_OK : RDCU_ERR_CUDA;
  }

  // Component-sorted cube coordinates as correlate recovers them (truncate 0: the
  // earlier frame, rounded; 1: the later frame, truncated); kept until the next find.
  const int4* pack(int truncate, std::string* msg) {
    if (packed_mode_ == truncate) return packed_.p;
    if (!packed_.ensure(std::max<long long>(n_cubes, 1), &device_bytes, st)) {
      *msg = "device memory";
      return nullptr;
    }
    if (n_cubes) {
      const double s0 = g.L[0] / (double)(g.N[0] - 1), s1 = g.L[1] / (double)(g.N[1] - 1),
                   s2 = g.L[2] / (double)(g.N[2] - 1);
      launch(k_pack, nblocks(n_cubes, kT), kT, sorted_, cubes_.p, comp_.p, g, s0, s1, s2, truncate, packed_.p,
             (int)n_cubes);
      if (!ck(cudaGetLastError(), msg)) return nullptr;
    }
    packed_mode_ = truncate;
    return packed_.p;
  }

  // diffs[j][i] (int64, host or device) between components i of A and j of B
  int correlate_packed(const int4* A, long long nA, long long ncA, const int4* B, long long nB, long long ncB,
                       long long* diffs, std::string* msg) {
    const long long cells = ncA * ncB;
    if (cells == 0) return RDCU_OK;
    if (!diff32_.ensure(cells, &device_bytes, st) || !diff64_.ensure(cells, &device_bytes, st))
      return fail_code(msg, "device memory", RDCU_ERR_NOMEM);
    launch(k_fill, std::min(nblocks(cells, kT), 4096), kT, diff32_.p, cells, INT_MAX);
    if (nA && nB) {
      // enough blocks to fill the SMs a few times over: split A into spans
      const int bx = nblocks(nB, kT);
      const int want = std::max(1, (4 * 148 + bx - 1) / bx);
      const int span = kT * nblocks(nblocks(nA, want), kT);
      launch(k_corr, dim3(bx, nblocks(nA, span)), kT, A, (int)nA, B, (int)nB, g, diff32_.p, (int)ncA, span);
    }
    launch(k_widen, std::min(nblocks(cells, kT), 4096), kT, diff32_.p, diff64_.p, cells);
    if (!ck(cudaMemcpyAsync(diffs, diff64_.p, cells * sizeof(long long), cudaMemcpyDefault, st), msg) ||
        !ck(cudaStreamSynchronize(st), msg))
      return RDCU_ERR_CUDA;
    return RDCU_OK;
  }

  // explicit cube sets (C-order cube indices grouped by component; offsets n_comp + 1
  // starting at 0), host or device
  int correlate_sets(const long long* a, const long long* aoff, long long nca, const long long* b,
                     const long long* boff, long long ncb, long long* diffs, std::string* msg) {
    std::vector<long long> ha(nca + 1), hb(ncb + 1);
    if (!ck(cudaMemcpy(ha.data(), aoff, (nca + 1) * sizeof(long long), cudaMemcpyDefault), msg) ||
        !ck(cudaMemcpy(hb.data(), boff, (ncb + 1) * sizeof(long long), cudaMemcpyDefault), msg))
      return RDCU_ERR_CUDA;
    if (ha[0] != 0 || hb[0] != 0) return fail_code(msg, "component offsets must start at 0", RDCU_ERR_INVALID);
    for (long long c = 0; c < nca; ++c)
      if (ha[c + 1] < ha[c]) return fail_code(msg, "component offsets must not decrease", RDCU_ERR_INVALID);
    for (long long c = 0; c < ncb; ++c)
      if (hb[c + 1] < hb[c]) return fail_code(msg, "component offsets must not decrease", RDCU_ERR_INVALID);
    const long long nA = ha[nca], nB = hb[ncb];
    if (nA >= (1ll << 31) || nB >= (1ll << 31)) return fail_code(msg, "too many cubes", RDCU_ERR_UNSUPPORTED);
    if (!sets_.ensure(nA + nB + nca + ncb + 2, &device_bytes, st) || !packed_b_.ensure(nA + nB + 1, &device_bytes, st))
      return fail_code(msg, "device memory", RDCU_ERR_NOMEM);
    long long* da = sets_.p;
    long long* db = da + nA;
    long long* dao = db + nB;
    long long* dbo = dao + nca + 1;
    int4* pa = packed_b_.p;
    int4* pb = pa + nA;
    if ((nA && !ck(cudaMemcpyAsync(da, a, nA * sizeof(long long), cudaMemcpyDefault, st), msg)) ||
        (nB && !ck(cudaMemcpyAsync(db, b, nB * sizeof(long long), cudaMemcpyDefault, st), msg)) ||
        !ck(cudaMemcpyAsync(dao, ha.data(), (nca + 1) * sizeof(long long), cudaMemcpyHostToDevice, st), msg) ||
        !ck(cudaMemcpyAsync(dbo, hb.data(), (ncb + 1) * sizeof(long long), cudaMemcpyHostToDevice, st), msg) ||
        !ck(cudaMemsetAsync(flags_.p, 0, sizeof(int), st), msg))
      return RDCU_ERR_CUDA;
    if (nA) launch(k_pack_sets, nblocks(nA, kT), kT, da, dao, (int)nca, g, pa, (int)nA, flags_.p);
    if (nB) launch(k_pack_sets, nblocks(nB, kT), kT, db, dbo, (int)ncb, g, pb, (int)nB, flags_.p);
    if (!ck(cudaMemcpyAsync(h_small_, flags_.p, sizeof(int), cudaMemcpyDeviceToHost, st), msg) ||
        !ck(cudaStreamSynchronize(st), msg))
      return RDCU_ERR_CUDA;
    if (*(int*)h_small_ != 0) return fail_code(msg, "cube index outside the grid", RDCU_ERR_INVALID);
    return correlate_packed(pa, nA, nca, pb, nB, ncb, diffs, msg);
  }

 private:
  Buf<double> th_, src_, xyz_;
  Buf<unsigned char> face_, mark_;
  Buf<int> node_of_, counts_, sums_, flags_;  // flags_[0]: error, flags_[1]: scan total
  Buf<int> cubes_, parent_, deg_, label_, root_comp_, comp_, key_a_, key_b_, order_, val_tmp_, eoff_, hist_, diff32_;
  Buf<long long> wide_, comp_noff_, comp_eoff_, diff64_, sets_;
  Buf<int4> packed_, packed_b_;
  long long* h_small_ = nullptr;  // pinned
  cudaStream_t cst_ = nullptr;    // copy stream of prefetch
  cudaEvent_t ev_main_ = nullptr, ev_staged_ = nullptr;
  int staged_kind_ = -1;          // kind of the prefetched frame, -1: none
  int* sorted_ = nullptr;         // node order by component (order_ or val_tmp_)
  int packed_mode_ = -1;

  template <typename... KA, typename... A>
  void launch(void (*k)(KA...), dim3 grid, int block, A... args) {
    k<<<grid, block, 0, st>>>(args...);
    ++launches;
  }
  template <typename... KA, typename... A>
  void launch_smem(void (*k)(KA...), dim3 grid, int block, size_t smem, A... args) {
    k<<<grid, block, smem, st>>>(args...);
    ++launches;
  }
  static bool fail(std::string* msg, const char* m) {
    *msg = m;
    return false;
  }
  static int fail_code(std::string* msg, const char* m, int code) {
    *msg = m;
    return code;
  }
  static bool ck(cudaError_t e, std::string* msg) {
    if (e == cudaSuccess) return true;
    *msg = cudaGetErrorString(e);
    return false;
  }
  bool copy_offsets(long long* dst, const long long* dev, std::string* msg) {
    if (n_comp) return ck(cudaMemcpyAsync(dst, dev, (n_comp + 1) * sizeof(long long), cudaMemcpyDefault, st), msg);
    h_small_[1] = 0;  // no component: the single offset 0
    return ck(cudaMemcpyAsync(dst, h_small_ + 1, sizeof(long long), cudaMemcpyDefault, st), msg);
  }
  bool ensure_nodes(long long n) {
    for (Buf<int>* b : {&cubes_, &parent_, &deg_, &label_, &root_comp_, &comp_, &key_a_, &key_b_, &order_, &val_tmp_,
                        &eoff_})
      if (!b->ensure(n, &device_bytes, st)) return false;
    return hist_.ensure(256ll * (nblocks(n, kChunk) + 1), &device_bytes, st);
  }
  // components of the n >= 1 line cubes (after k_compact): deg, comp, key_a_ and order_,
  // the component count in flags_[1], the edge count added to flags_[2] (zeroed by the
  // caller).  One CTA in shared memory for small frames.
  int components(int n, std::string* msg) {
    if (n <= kSmallNodes) {
      launch_smem(k_components_small, 1, kSmallThreads, (size_t)n * 2 * sizeof(int), (const int*)cubes_.p,
                  (const int*)node_of_.p, deg_.p, comp_.p, key_a_.p, order_.p, n, g, flags_.p, flags_.p + 1,
                  flags_.p + 2);
      return ck(cudaGetLastError(), msg) ? RDCU_OK : RDCU_ERR_CUDA;
    }
    const int nbn = nblocks(n, kChunk);
    launch(k_hook, nblocks(n, kT), kT, cubes_.p, node_of_.p, parent_.p, deg_.p, n, g, flags_.p, flags_.p + 2);
    launch(k_flatten, nbn, kT, parent_.p, label_.p, n, counts_.p, flags_.p);
    if (int rc = scan(counts_.p, nbn, msg)) return rc;
    launch(k_roots, nbn, kT, label_.p, counts_.p, root_comp_.p, n);
    launch(k_label, nblocks(n, kT), kT, label_.p, root_comp_.p, comp_.p, key_a_.p, order_.p, n);
    return RDCU_OK;
  }
  // exclusive scan of a[0..n) in place; the total goes to flags_[1]
  int scan(int* a, int n, std::string* msg) {
    const int nb = nblocks(n, kChunk);
    if (n <= 8 * 1024) {  // a few rounds of one block beat three launches
      launch(k_scan_one, 1, 1024, a, n, flags_.p + 1);
    } else {
      if (!sums_.ensure(nb, &device_bytes, st)) return fail_code(msg, "device memory", RDCU_ERR_NOMEM);
      launch(k_chunk_sums, nb, kT, (const int*)a, n, sums_.p);
      launch(k_scan_one, 1, 1024, sums_.p, nb, flags_.p + 1);
      launch(k_chunk_scan, nb, kT, a, n, (const int*)sums_.p);
    }
    return ck(cudaGetLastError(), msg) ? RDCU_OK : RDCU_ERR_CUDA;
  }
  long long read_total(std::string* msg) {
    if (!ck(cudaMemcpyAsync(h_small_, flags_.p + 1, sizeof(int), cudaMemcpyDeviceToHost, st), msg) ||
        !ck(cudaStreamSynchronize(st), msg))
      return -1;
    return *(int*)h_small_;
  }
};

}  // namespace rdcu

// ------------------------------------------------------------------------------ C ABI
struct rdcu_lines {
  rdcu::LinesEngine eng;
  std::string err;
};

namespace {
thread_local std::string g_lines_create_error;

int lines_err(rdcu_lines_t* l, int code, const std::string& msg) {
  (l ? l->err : g_lines_create_error) = msg;
  return code;
}

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int lines_activate(rdcu_lines_t* l) {
  const cudaError_t e = cudaSetDevice(l->eng.device);
  return e == cudaSuccess ? RDCU_OK : lines_err(l, RDCU_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
}
}  // namespace

extern "C" {

int rdcu_lines_create(rdcu_lines_t** out, const int Ns[3], const double Ls[3], int device) {
  if (!out || !Ns || !Ls) return lines_err(nullptr, RDCU_ERR_INVALID, "null argument");
  *out = nullptr;
  std::unique_ptr<rdcu_lines> l(new rdcu_lines);
  std::string msg;
  if (!l->eng.init(Ns, Ls, device, &msg)) {
    const int code = msg.find("memory") != std::string::npos      ? RDCU_ERR_NOMEM
                     : msg.find("supported") != std::string::npos ? RDCU_ERR_UNSUPPORTED
                     : msg.find("stream") != std::string::npos    ? RDCU_ERR_CUDA
                                                                  : RDCU_ERR_INVALID;
    return lines_err(nullptr, code, msg);
  }
  *out = l.release();
  return RDCU_OK;
}

int rdcu_lines_destroy(rdcu_lines_t* l) {
  if (!l) return RDCU_OK;
  cudaSetDevice(l->eng.device);
  delete l;
  return RDCU_OK;
}

int rdcu_lines_prefetch(rdcu_lines_t* l, const double* src, int kind) {
  if (!l || !src) return lines_err(l, RDCU_ERR_INVALID, "null argument");
  if (kind != RDCU_LINES_STATE && kind != RDCU_LINES_PHASE) return lines_err(l, RDCU_ERR_INVALID, "unknown source kind");
  if (int rc = lines_activate(l)) return rc;
  std::string msg;
  const int rc = l->eng.prefetch(src, kind, &msg);
  return rc ? lines_err(l, rc, "rdcu_lines_prefetch: " + msg) : RDCU_OK;
}

int rdcu_lines_find(rdcu_lines_t* l, const double* src, int kind, long long* n_cubes, long long* n_edges,
                    long long* n_components) {
  if (!l) return lines_err(l, RDCU_ERR_INVALID, "null argument");
  if (kind != RDCU_LINES_STATE && kind != RDCU_LINES_PHASE) return lines_err(l, RDCU_ERR_INVALID, "unknown source kind");
  if (int rc = lines_activate(l)) return rc;
  std::string msg;
  const int rc = l->eng.find(src, kind, src && on_device(src), &msg);
  if (rc) return lines_err(l, rc, "rdcu_lines_find: " + msg);
  if (n_cubes) *n_cubes = l->eng.n_cubes;
  if (n_edges) *n_edges = l->eng.n_edges;
  if (n_components) *n_components = l->eng.n_comp;
  return RDCU_OK;
}

int rdcu_lines_edges(rdcu_lines_t* l, double* xyz, long long* comp_offsets) {
  if (!l) return lines_err(l, RDCU_ERR_INVALID, "null argument");
  if (int rc = lines_activate(l)) return rc;
  std::string msg;
  const int rc = l->eng.edges(xyz, comp_offsets, &msg);
  return rc ? lines_err(l, rc, "rdcu_lines_edges: " + msg) : RDCU_OK;
}

int rdcu_lines_cubes(rdcu_lines_t* l, long long* cubes, long long* comp_offsets) {
  if (!l) return lines_err(l, RDCU_ERR_INVALID, "null argument");
  if (int rc = lines_activate(l)) return rc;
  std::string msg;
  const int rc = l->eng.cubes(cubes, comp_offsets, &msg);
  return rc ? lines_err(l, rc, "rdcu_lines_cubes: " + msg) : RDCU_OK;
}

int rdcu_lines_correlate(rdcu_lines_t* prev, rdcu_lines_t* cur, long long* diffs) {
  if (!prev || !cur) return lines_err(cur, RDCU_ERR_INVALID, "null argument");
  if (prev == cur) return lines_err(cur, RDCU_ERR_INVALID, "rdcu_lines_correlate needs two handles");
  const rdcu::LinesEngine &a = prev->eng, &b = cur->eng;
  for (int q = 0; q < 3; ++q)
    if (a.g.N[q] != b.g.N[q] || a.g.L[q] != b.g.L[q])
      return lines_err(cur, RDCU_ERR_INVALID, "rdcu_lines_correlate: the handles' grids differ");
  if (a.device != b.device) return lines_err(cur, RDCU_ERR_INVALID, "rdcu_lines_correlate: different devices");
  if (!a.have || !b.have) return lines_err(cur, RDCU_ERR_STATE, "rdcu_lines_correlate: a handle has no frame");
  if (!diffs && a.n_comp * b.n_comp > 0) return lines_err(cur, RDCU_ERR_INVALID, "null argument");
  if (int rc = lines_activate(cur)) return rc;
  std::string msg;
  const int4* A = prev->eng.pack(0, &msg);
  if (!A || cudaStreamSynchronize(prev->eng.st) != cudaSuccess)
    return lines_err(cur, RDCU_ERR_CUDA, "rdcu_lines_correlate: " + msg);
  const int4* B = cur->eng.pack(1, &msg);
  if (!B) return lines_err(cur, RDCU_ERR_CUDA, "rdcu_lines_correlate: " + msg);
  const int rc = cur->eng.correlate_packed(A, a.n_cubes, a.n_comp, B, b.n_cubes, b.n_comp, diffs, &msg);
  return rc ? lines_err(cur, rc, "rdcu_lines_correlate: " + msg) : RDCU_OK;
}

int rdcu_lines_correlate_sets(rdcu_lines_t* l, const long long* prev_cubes, const long long* prev_offsets,
                              long long n_prev, const long long* cur_cubes, const long long* cur_offsets,
                              long long n_cur, long long* diffs) {
  if (!l || !prev_offsets || !cur_offsets || (n_prev && n_cur && !diffs) || n_prev < 0 || n_cur < 0)
    return lines_err(l, RDCU_ERR_INVALID, "null or negative argument");
  if (int rc = lines_activate(l)) return rc;
  std::string msg;
  const int rc = l->eng.correlate_sets(prev_cubes, prev_offsets, n_prev, cur_cubes, cur_offsets, n_cur, diffs, &msg);
  return rc ? lines_err(l, rc, "rdcu_lines_correlate_sets: " + msg) : RDCU_OK;
}

int rdcu_lines_profile(rdcu_lines_t* l, const double* src, int kind, int reps, rdcu_pass_timing* out, int max_passes,
                       int* npass) {
  if (!l || !src || !out || !npass || reps < 1) return lines_err(l, RDCU_ERR_INVALID, "bad argument");
  if (kind != RDCU_LINES_STATE && kind != RDCU_LINES_PHASE) return lines_err(l, RDCU_ERR_INVALID, "unknown source kind");
  if (int rc = lines_activate(l)) return rc;
  std::string msg;
  std::vector<rdcu::LinesEngine::PassTime> pt;
  const int rc = l->eng.profile(src, kind, on_device(src), reps, &pt, &msg);
  if (rc) return lines_err(l, rc, "rdcu_lines_profile: " + msg);
  const int m = std::min((int)pt.size(), max_passes);
  for (int i = 0; i < m; ++i) {
    out[i].name = pt[i].name;
    out[i].ms = pt[i].ms;
    out[i].bytes = pt[i].bytes;
  }
  *npass = m;
  return RDCU_OK;
}

int rdcu_lines_info(rdcu_lines_t* l, void** stream, long long* device_bytes, long long* launches) {
  if (!l) return lines_err(l, RDCU_ERR_INVALID, "null argument");
  if (stream) *stream = (void*)l->eng.st;
  if (device_bytes) *device_bytes = (long long)l->eng.device_bytes;
  if (launches) *launches = l->eng.launches;
  return RDCU_OK;
}

const char* rdcu_lines_last_error(rdcu_lines_t* l) { return l ? l->err.c_str() : g_lines_create_error.c_str(); }

}  // extern "C"
