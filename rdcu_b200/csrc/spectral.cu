// Fused pseudospectral RHS: f = sum_terms C prod_k Y_k^eta with Y from spectral
// derivatives (reference rdcu.cu:78-106,117-184), as 3-5 shared-memory passes.
//
// Passes (d = ndim, last axis x contiguous, M = N_x, Mh = M/2+1):
//   fwd_x : DP45 stage combination (y + h sum a_j k_j) fused with the real-to-complex
//           FFT along x; two real rows per complex line, separated after the FFT.
//   c2c   : complex FFT along a strided middle axis (3D only), in place.
//   mid   : FFT along axis 0, the derivative multipliers that build each inverse
//           channel, and the inverse FFT along axis 0 -- one kernel.
//   c2c   : inverse along the middle axis (3D).
//   inv_x : complex-to-real along x (two channels per complex line), then the
//           dictionary at every grid point, written as the stage slope k_s; the
//           stage-7 launch also forms the DP45 error estimate's partial sums.
//
// Channels.  Terms with a single derivative factor of power one are linear with
// constant coefficients; per output field they are summed in spectral space into one
// channel L_i (one inverse transform instead of one per derivative block).  Every
// other derivative Y_k a term needs gets its own channel.  Physical fields come from
// the stage state itself.
//
// Multipliers.  The reference keeps Re(IFFT(M_k FFT(u))) of a full complex transform,
// with the wavenumber map k(na) = na*2pi/L for na < N/2 else (na-N)*2pi/L, the Nyquist
// bin included (rdcu.cu:89-98).  With a real input, Re(IFFT(M U)) = IFFT(Mr U) where
// Mr(k) = (M(k) + conj(M(-k)))/2 is Hermitian, so a real-to-complex transform with Mr
// reproduces it exactly (zeroing first derivatives at their own Nyquist bin, and mixed
// derivatives where exactly one index is at Nyquist).  The imaginary part of the
// reference's block is IFFT(Mi U) with Mi(k) = (M(k) - conj(M(-k)))/(2i); Y.dat output
// uses both.
#include <algorithm>
#include <array>
#include <cmath>
#include <cudaTypedefs.h>
#include <cstdlib>
#include <cstring>
#include <map>
#include <type_traits>

#include "fft_line.cuh"
#include "pencil.cuh"
#include "spectral.h"

namespace rdcu {

// Stage-combination coefficients a_{s,j} (dp45.cu:6-11; row s = stage 2..7) and
// error coefficients e_j (dp45.cu:13).
__constant__ double c_a[8][6] = {
    {0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
    {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
__constant__ double c_e[7] = {-71.0 / 57600, 0, 71.0 / 16695, -71.0 / 1920,
                              17253.0 / 339200, -22.0 / 525, 1.0 / 40};

namespace {

struct Resolved {
  const double* y = nullptr;   // stage input state
  double* ytemp = nullptr;     // stage state written by fwd_x (nullptr: not written)
  const double* u = nullptr;   // physical fields read by inv_x
  double* f = nullptr;         // slope written by inv_x
  const double* k[7] = {};
  double h = 0, atol = 0, rtol = 0;
  int stage = 0;
  double* aux = nullptr;       // stage 7: the slope sums fwd_x writes (RhsIO::err_aux)
  long long nN = 0;            // n * N (set by the pass that uses it)
};

__device__ __forceinline__ Resolved resolve(const RhsIO& io) {
  Resolved r;
  if (io.mode == 0) {
    r.y = io.y;
    r.u = io.y;
    r.f = io.f;
    return r;
  }
  const DP45Ctl* c = io.ctl;
  r.stage = io.stage;
  r.h = c->h;
  r.atol = c->atol;
  r.rtol = c->rtol;
  r.y = io.bufs.ybuf[c->y_slot];
  r.k[0] = io.bufs.kbuf[c->k1_buf];
  for (int j = 1; j < 6; ++j) r.k[j] = io.bufs.kbuf[j];
  r.k[6] = io.bufs.kbuf[c->k7_buf];
  if (io.stage <= 1) {
    r.u = r.y;
    r.f = io.bufs.kbuf[c->k1_buf];
  } else {
    r.ytemp = io.ytemp_out ? io.ytemp_out : io.bufs.ybuf[c->yn_slot];
    r.u = r.ytemp;
    r.f = (io.stage == 7) ? io.bufs.kbuf[c->k7_buf] : io.bufs.kbuf[io.stage - 1];
    if (io.stage == 7) r.aux = io.err_aux;
  }
  return r;
}

// Stage 7's error term at point i from the slopes, in k_inv_x's operation order: the
// slope sum without e_7 k_7 (e_2 = 0).
__device__ __forceinline__ double stage7_slope_sum(long long i, const Resolved& r) {
  return c_e[0] * r.k[0][i] + c_e[2] * r.k[2][i] + c_e[3] * r.k[3][i] + c_e[4] * r.k[4][i] + c_e[5] * r.k[5][i];
}
// the error scale atol + rtol max(|y|, |y_new|) (dp45.cu:79-84); the inverse pass forms
// it from y and the stage-7 state it reads anyway, bitwise the value of the forward pass
__device__ __forceinline__ double stage7_scale(const Resolved& r, double y, double ynew) {
  return r.atol + r.rtol * fmax(fabs(y), fabs(ynew));
}

// Stage states follow the reference kernels' arithmetic order (dp45.cu:34-69): stage 2
// is y + h*a*k1, later stages y + h*(sum_j a_j k_j); b_2 = 0 (dp45.cu:11), so stage 7
// does not read k2 (stage_value_t below).
__device__ __forceinline__ double ipow(double x, int e) {
  // straight-line products for the small powers dictionaries use (e is warp-uniform)
  switch (e) {
    case 1: return x;
    case 2: return x * x;
    case 3: return x * x * x;
    case 0: return 1.0;  // pow(x, 0) == 1 for every x
    case -1: return 1.0 / x;
    case -2: return 1.0 / (x * x);
    default: break;
  }
  const int a = e < 0 ? -e : e;
  double r = x;
  for (int j = 1; j < a; ++j) r *= x;
  return e < 0 ? 1.0 / r : r;
}

// Multiplier of one channel entry applied to u at the multi-index nidx.
__device__ __forceinline__ double2 apply_entry(const ChanEntry& e, const int* nidx, const ChanTable& ct,
                                               double2 u) {
  double ap = 1.0, am = 1.0;
  if (e.nax >= 1) {
    const int a = e.ax0, na = nidx[a], nm = na == 0 ? 0 : ct.Ns[a] - na;
    ap *= ct.kv[ct.kv_off[a] + na];
    am *= ct.kv[ct.kv_off[a] + nm];
  }
  if (e.nax >= 2) {
    const int a = e.ax1, na = nidx[a], nm = na == 0 ? 0 : ct.Ns[a] - na;
    ap *= ct.kv[ct.kv_off[a] + na];
    am *= ct.kv[ct.kv_off[a] + nm];
  }
  // M(k) = i^p alpha(k); Mr = i^p (alpha(k) + (-1)^p alpha(-k))/2,
  // Mi = i^(p-1) (alpha(k) - (-1)^p alpha(-k))/2
  const double sgn = (e.nax & 1) ? -1.0 : 1.0;
  double beta;
  int q;
  if (e.part == 0) {
    q = e.nax;
    beta = 0.5 * (ap + sgn * am);
  } else {
    q = e.nax + 3;
    beta = 0.5 * (ap - sgn * am);
  }
  beta *= e.coef;
  const double2 r = make_double2(beta * u.x, beta * u.y);
  switch (q & 3) {
    case 0: return r;
    case 1: return make_double2(-r.y, r.x);
    case 2: return make_double2(-r.x, -r.y);
    default: return make_double2(r.y, -r.x);
  }
}

__device__ __forceinline__ double sel3(double a0, double a1, double a2, int i) {
  return i == 0 ? a0 : (i == 1 ? a1 : a2);
}

// apply_entry with the point's wavenumbers k(n_a), k(-n_a) already in registers
__device__ __forceinline__ double2 apply_entry_k(const ChanEntry& e, const double* kp, const double* km,
                                                 double2 u) {
  double ap = 1.0, am = 1.0;
  if (e.nax >= 1) {
    ap *= sel3(kp[0], kp[1], kp[2], e.ax0);
    am *= sel3(km[0], km[1], km[2], e.ax0);
  }
  if (e.nax >= 2) {
    ap *= sel3(kp[0], kp[1], kp[2], e.ax1);
    am *= sel3(km[0], km[1], km[2], e.ax1);
  }
  const double sgn = (e.nax & 1) ? -1.0 : 1.0;
  double beta;
  int q;
  if (e.part == 0) {
    q = e.nax;
    beta = 0.5 * (ap + sgn * am);
  } else {
    q = e.nax + 3;
    beta = 0.5 * (ap - sgn * am);
  }
  beta *= e.coef;
  const double2 r = make_double2(beta * u.x, beta * u.y);
  switch (q & 3) {
    case 0: return r;
    case 1: return make_double2(-r.y, r.x);
    case 2: return make_double2(-r.x, -r.y);
    default: return make_double2(r.y, -r.x);
  }
}

// ------------------------------------------------------------------------- kernels
struct FwdXArgs {
  int M, Mh, nrows, P, do_fft, tw_smem;
  FastDiv d2M, dM, d2Mh, dMh;  // invariant divisors (prep)
  LinePlan plan;
  const double2* tw;
  double2* S;
  RhsIO io;
};

// Largest block of the length-specialised kernels (the axis-0 pass is compiled for three
// resident 256-thread CTAs per SM, at most 85 registers per thread, to hide shared-memory
// and FP64 latency); a launch that needs more threads takes the general kernels.
constexpr int kSpecBlock = 256;

// Line stride (in double2) of the column tiles of the strided-axis passes: TW columns of
// one row are consecutive threads, so line c starts at c * LS; LS = L + 8/TW (at least
// L + 1) makes c * LS + z hit distinct 16-byte bank groups across a quarter warp.
__host__ __device__ __forceinline__ int tile_stride(int L, int TW) { return L + (TW >= 8 ? 1 : 8 / TW); }

// Division by an invariant divisor: the compile-time constant D when D > 0, else the
// precomputed FastDiv f.
template <int D>
__device__ __forceinline__ int fdivc(int n, FastDiv f) {
  if constexpr (D > 0)
    return (int)((unsigned)n / (unsigned)D);
  else
    return fdiv(n, f);
}

// Line FFTs of a pass: compile-time power-of-two length LX, or the plan's stages (LX = 0).
// twz: the twiddle table is in shared memory at swz8 positions (stage_twiddles).
template <int RS, int LX, bool INV>
__device__ __forceinline__ void fft_lines_x(double2* buf, int LS, int nlines, const LinePlan& p, const double2* tw,
                                            bool twz) {
  if constexpr (LX > 0 && (LX & (LX - 1)) == 0)
    fft_pow2_t<LX, INV>(buf, LS, nlines, tw, twz);
  else if constexpr (LX > 0)
    fft_fixed_t<LX, INV>(buf, LS, nlines, tw);
  else
    fft_lines<RS, INV>(buf, LS, nlines, p, tw);
}

// Copies the L-point twiddle table into shared memory; kernels specialised to a
// power-of-two length store it swizzled (see fft_pow2_t).  Returns whether it did.
template <int LX>
__device__ __forceinline__ bool stage_twiddles(double2* dst, const double2* src, int L) {
  constexpr bool swz = LX > 0 && (LX & (LX - 1)) == 0;
  for (int t = threadIdx.x; t < L; t += blockDim.x) dst[swz ? swz8(t) : t] = src[t];
  return swz;
}

// Stage state with the stage number known at compile time (slopes in registers).
template <int S>
__device__ __forceinline__ double stage_value_t(long long i, const Resolved& r) {
  const double yi = r.y[i];
  if (S <= 1) return yi;
  if (S == 2) return yi + r.h * c_a[2][0] * r.k[0][i];
  double acc = c_a[S][0] * r.k[0][i];
  if (S != 7) acc += c_a[S][1] * r.k[1][i];
#pragma unroll
  for (int j = 2; j < S - 1; ++j) acc += c_a[S][j] * r.k[j][i];
  return yi + r.h * acc;
}

// Loads (with the stage combination) the rows of P line pairs into the complex lines
// of buf, real row in .x, partner row in .y; writes the stage state when asked.  Each
// thread issues the loads of kUnroll elements before storing any of them.
template <int S, int LX>
__device__ __forceinline__ void fwd_load(const FwdXArgs& a, const Resolved& r, double2* buf, long long row0) {
  constexpr int kUnroll = 4;
  const int M = LX ? LX : a.M, T = blockDim.x, tid = threadIdx.x;
  const int nel = a.P * 2 * M;
  for (int e0 = tid; e0 < nel; e0 += T * kUnroll) {
    double v[kUnroll];
    long long gi[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int e = e0 + u * T;
      gi[u] = -1;
      v[u] = 0.0;
      if (e < nel) {
        const int pl = fdivc<2 * LX>(e, a.d2M);
        const int w = e - pl * 2 * M;
        const int half = fdivc<LX>(w, a.dM);
        const int x = w - half * M;
        const long long g = row0 + 2 * pl + half;
        if (g < a.nrows) {
          gi[u] = g * M + x;
          v[u] = stage_value_t<S>(gi[u], r);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int e = e0 + u * T;
      if (e >= nel) break;
      if (r.ytemp && gi[u] >= 0) r.ytemp[gi[u]] = v[u];
      if (S == 7 && r.aux && gi[u] >= 0) r.aux[gi[u]] = stage7_slope_sum(gi[u], r);
      if (a.do_fft) {
        const int pl = fdivc<2 * LX>(e, a.d2M);
        const int w = e - pl * 2 * M;
        const int half = fdivc<LX>(w, a.dM);
        const int x = w - half * M;
        reinterpret_cast<double*>(buf)[2 * (pl * M + x) + half] = v[u];
      }
    }
  }
}

// stage_value_t for the two consecutive points i, i+1 (i even) with 16-byte loads; the
// same arithmetic per component.
template <int S>
__device__ __forceinline__ double2 stage_value_t2(long long i, const Resolved& r) {
  const double2 yi = *reinterpret_cast<const double2*>(r.y + i);
  if (S <= 1) return yi;
  if (S == 2) {
    const double2 k0 = *reinterpret_cast<const double2*>(r.k[0] + i);
    return make_double2(yi.x + r.h * c_a[2][0] * k0.x, yi.y + r.h * c_a[2][0] * k0.y);
  }
  const double2 k0 = *reinterpret_cast<const double2*>(r.k[0] + i);
  double ax = c_a[S][0] * k0.x, ay = c_a[S][0] * k0.y;
  if (S != 7) {
    const double2 k1 = *reinterpret_cast<const double2*>(r.k[1] + i);
    ax += c_a[S][1] * k1.x;
    ay += c_a[S][1] * k1.y;
  }
#pragma unroll
  for (int j = 2; j < S - 1; ++j) {
    const double2 kj = *reinterpret_cast<const double2*>(r.k[j] + i);
    ax += c_a[S][j] * kj.x;
    ay += c_a[S][j] * kj.y;
  }
  return make_double2(yi.x + r.h * ax, yi.y + r.h * ay);
}

// Stage 7 at the two points i, i+1 with the error term from the same loads: the new
// state (stage_value_t2<7>'s arithmetic) and stage7_slope_sum's slope sum.
__device__ __forceinline__ double2 stage7_value_terms2(long long i, const Resolved& r, double2* es_p) {
  const double2 yi = *reinterpret_cast<const double2*>(r.y + i);
  const double2 k0 = *reinterpret_cast<const double2*>(r.k[0] + i);
  const double2 k2 = *reinterpret_cast<const double2*>(r.k[2] + i);
  const double2 k3 = *reinterpret_cast<const double2*>(r.k[3] + i);
  const double2 k4 = *reinterpret_cast<const double2*>(r.k[4] + i);
  const double2 k5 = *reinterpret_cast<const double2*>(r.k[5] + i);
  double ax = c_a[7][0] * k0.x, ay = c_a[7][0] * k0.y;
  ax += c_a[7][2] * k2.x;
  ay += c_a[7][2] * k2.y;
  ax += c_a[7][3] * k3.x;
  ay += c_a[7][3] * k3.y;
  ax += c_a[7][4] * k4.x;
  ay += c_a[7][4] * k4.y;
  ax += c_a[7][5] * k5.x;
  ay += c_a[7][5] * k5.y;
  const double2 v = make_double2(yi.x + r.h * ax, yi.y + r.h * ay);
  es_p->x = c_e[0] * k0.x + c_e[2] * k2.x + c_e[3] * k3.x + c_e[4] * k4.x + c_e[5] * k5.x;
  es_p->y = c_e[0] * k0.y + c_e[2] * k2.y + c_e[3] * k3.y + c_e[4] * k4.y + c_e[5] * k5.y;
  return v;
}

// fwd_load for a compile-time power-of-two row length: each thread moves pairs of
// consecutive points (16-byte loads and stores of the state arrays).
template <int S, int LX>
__device__ __forceinline__ void fwd_load2(const FwdXArgs& a, const Resolved& r, double2* buf, long long row0) {
  static_assert(LX % 2 == 0, "even compile-time row length");
  if constexpr (LX > 0) {
  constexpr int kUnroll = 4, H = LX / 2;
  const int T = blockDim.x, tid = threadIdx.x;
  const int npair = a.P * LX;  // P line pairs of two rows, LX/2 point pairs per row
  const bool terms = S == 7 && r.aux != nullptr;
  for (int e0 = tid; e0 < npair; e0 += T * kUnroll) {
    double2 v[kUnroll];
    long long gi[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int e = e0 + u * T;
      gi[u] = -1;
      v[u] = make_double2(0.0, 0.0);
      if (e < npair) {
        const int pl = (unsigned)e / LX;
        const int w = e - pl * LX;
        const int half = (unsigned)w / H;
        const int x = (w - half * H) * 2;
        const long long g = row0 + 2 * pl + half;
        if (g < a.nrows) {
          gi[u] = g * LX + x;
          if (terms) {
            // the error term leaves at once (no registers held across the unrolled loads)
            double2 es_p;
            v[u] = stage7_value_terms2(gi[u], r, &es_p);
            *reinterpret_cast<double2*>(r.aux + gi[u]) = es_p;
          } else {
            v[u] = stage_value_t2<S>(gi[u], r);
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int e = e0 + u * T;
      if (e >= npair) break;
      if (r.ytemp && gi[u] >= 0) *reinterpret_cast<double2*>(r.ytemp + gi[u]) = v[u];

      if (a.do_fft) {
        const int pl = (unsigned)e / LX;
        const int w = e - pl * LX;
        const int half = (unsigned)w / H;
        const int x = (w - half * H) * 2;
        double* b = reinterpret_cast<double*>(buf) + 2 * (pl * LX + x) + half;
        b[0] = v[u].x;
        b[2] = v[u].y;
      }
    }
  }
  }
}

// bx: the CTA's index within this plan's grid (blockIdx.x, or a work item of a batch).
// SF > 0: the stage is SF, known at compile time (a kernel per stage has the registers
// of its own stage combination, not those of the largest); SF = 0: the stage of a.io.
template <int RS, int LX, int SF = 0>
__device__ __forceinline__ void fwd_x_body(const FwdXArgs& a, int bx) {
  extern __shared__ double2 sm[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;
  Resolved r = resolve(a.io);
  r.nN = (long long)a.nrows * (LX ? LX : a.M);
  const int M = LX ? LX : a.M, T = blockDim.x, tid = threadIdx.x;
  const double2* tw = a.tw;
  double2* buf = sm;
  bool twz = false;
  if (a.do_fft && a.tw_smem) {
    twz = stage_twiddles<LX>(sm, a.tw, M);
    tw = sm;
    buf = sm + M;
  }
  const long long row0 = 2LL * bx * a.P;
  // 16-byte state loads need 16-byte aligned arrays (a caller's y may be offset)
  unsigned long long align = reinterpret_cast<unsigned long long>(r.y) | reinterpret_cast<unsigned long long>(r.ytemp);
  for (int j = 0; j < 7; ++j) align |= reinterpret_cast<unsigned long long>(r.k[j]);
  if (LX > 0 && (align & 15) == 0) {
    switch (SF > 0 ? SF : r.stage) {
      case 2: fwd_load2<2, LX>(a, r, buf, row0); break;
      case 3: fwd_load2<3, LX>(a, r, buf, row0); break;
      case 4: fwd_load2<4, LX>(a, r, buf, row0); break;
      case 5: fwd_load2<5, LX>(a, r, buf, row0); break;
      case 6: fwd_load2<6, LX>(a, r, buf, row0); break;
      case 7: fwd_load2<7, LX>(a, r, buf, row0); break;
      default: fwd_load2<1, LX>(a, r, buf, row0); break;
    }
  } else {
    switch (SF > 0 ? SF : r.stage) {
      case 2: fwd_load<2, LX>(a, r, buf, row0); break;
      case 3: fwd_load<3, LX>(a, r, buf, row0); break;
      case 4: fwd_load<4, LX>(a, r, buf, row0); break;
      case 5: fwd_load<5, LX>(a, r, buf, row0); break;
      case 6: fwd_load<6, LX>(a, r, buf, row0); break;
      case 7: fwd_load<7, LX>(a, r, buf, row0); break;
      default: fwd_load<1, LX>(a, r, buf, row0); break;
    }
  }
  if (!a.do_fft) return;
  __syncthreads();
  fft_lines_x<RS, LX, false>(buf, M, a.P, a.plan, tw, twz);
  const int Mh = LX ? LX / 2 + 1 : a.Mh;
  const int nout = a.P * 2 * Mh;
  for (int e = tid; e < nout; e += T) {
    const int pl = fdivc<LX ? 2 * (LX / 2 + 1) : 0>(e, a.d2Mh);
    const int w = e - pl * 2 * Mh;
    const int half = fdivc<LX ? LX / 2 + 1 : 0>(w, a.dMh);
    const int kx = w - half * Mh;
    const long long g = row0 + 2 * pl + half;
    if (g >= a.nrows) continue;
    const double2 z = buf[pl * M + kx];
    const double2 zm = buf[pl * M + (kx == 0 ? 0 : M - kx)];
    double2 o;
    if (half == 0)
      o = make_double2(0.5 * (z.x + zm.x), 0.5 * (z.y - zm.y));
    else
      o = make_double2(0.5 * (z.y + zm.y), -0.5 * (z.x - zm.x));
    a.S[g * Mh + kx] = o;
  }
}

// The CTAs take the rows from the last to the first: the previous stage's row kernel
// ended on the last rows of the slope this stage reads (still in L2), and the axis-1
// pass after it starts on the first planes, written last here.
template <int RS, int LX, int SF = 0>
__global__ void __launch_bounds__(LX > 0 ? kSpecBlock : kMaxBlock, LX > 0 ? (SF > 0 ? 4 : 2) : 1) k_fwd_x(FwdXArgs a) {
  fwd_x_body<RS, LX, SF>(a, gridDim.x - 1 - blockIdx.x);
}

struct C2CArgs {
  int La, I, TW;
  FastDiv dTW;
  LinePlan plan;
  const double2* tw;
  double2* S;
  RhsIO io;
};

template <int RS, bool INV, int LX>
__global__ void __launch_bounds__(LX > 0 ? kSpecBlock : kMaxBlock, LX > 0 ? 2 : 1) k_c2c(C2CArgs a) {
  extern __shared__ double2 sm[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;
  const int La = LX ? LX : a.La, TW = a.TW, LS = tile_stride(La, TW), T = blockDim.x, tid = threadIdx.x;
  double2* tw = sm;
  double2* buf = sm + La;
  const bool twz = stage_twiddles<LX>(tw, a.tw, La);
  const long long i0 = (long long)blockIdx.x * TW;
  double2* base = a.S + (long long)blockIdx.y * La * a.I;
  const int nel = La * TW;
  // the last tile of a plane may hold fewer columns (e.g. 1 of 16 when I = 129): only
  // its valid lines are loaded and transformed (lines are independent)
  const int nl = (int)min((long long)TW, a.I - i0);
  for (int e = tid; e < nel; e += T) {
    const int z = fdiv(e, a.dTW), c = e - z * TW;
    if (c < nl) cp_async16(&buf[c * LS + z], &base[(long long)z * a.I + i0 + c], true);
  }
  cp_async_wait_all();
  __syncthreads();
  fft_lines_x<RS, LX, INV>(buf, LS, nl, a.plan, tw, twz);
  for (int e = tid; e < nel; e += T) {
    const int z = fdiv(e, a.dTW), c = e - z * TW;
    const long long ii = i0 + c;
    if (ii < a.I) base[(long long)z * a.I + ii] = buf[c * LS + z];
  }
}

struct MidArgs {
  int L0, I, TW, nsrc, G, GB, ch0;
  int sorted;      // entries sorted by operator, .pad = local channel (all G <= 4 channels at once)
  FastDiv dTW, dL0, dMh;
  int ent0, nent;  // entries [ent0, ent0+nent) of the launched channels, staged in smem
  int ndim, D1, Mh;
  LinePlan plan;
  const double2* tw;
  const double2* Sf;
  double2* Sc;
  ChanTable chan;
  RhsIO io;
};

template <int RS, int LX>
__device__ __forceinline__ void mid_body(const MidArgs& a, int bx) {
  extern __shared__ double2 sm[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;
  const int L0 = LX ? LX : a.L0, TW = a.TW, LS = tile_stride(L0, TW), T = blockDim.x, tid = threadIdx.x;
  double2* tw = sm;
  double2* fb = sm + L0;
  // the all-channel path writes each point's channels over its own sources (every point
  // belongs to one thread), so its channel lines reuse the source lines
  const bool inplace = a.sorted && a.G <= a.nsrc;
  double2* cb = inplace ? fb : fb + a.nsrc * TW * LS;
  // channel entries, offsets (relative to ent0) and wavenumbers staged in shared memory
  ChanEntry* se = reinterpret_cast<ChanEntry*>(inplace ? fb + a.nsrc * TW * LS : cb + a.GB * TW * LS);
  double* skv = reinterpret_cast<double*>(se + a.nent);
  int* soff = reinterpret_cast<int*>(skv + a.chan.kv_total);
  const bool twz = stage_twiddles<LX>(tw, a.tw, L0);
  for (int t = tid; t < a.nent; t += T) se[t] = a.chan.ent[a.ent0 + t];
  for (int t = tid; t < a.chan.kv_total; t += T) skv[t] = a.chan.kv[t];
  for (int t = tid; t <= a.G; t += T) soff[t] = a.chan.off[a.ch0 + t] - a.ent0;
  const long long i0 = (long long)bx * TW;
  const int nload = a.nsrc * L0 * TW;
  for (int e = tid; e < nload; e += T) {
    const int q0 = fdiv(e, a.dTW), c = e - q0 * TW;
    const int f = fdivc<LX>(q0, a.dL0), z = q0 - f * L0;
    const long long ii = i0 + c;
    const bool in = ii < a.I;
    cp_async16(&fb[(f * TW + c) * LS + z], in ? (const void*)&a.Sf[((long long)f * L0 + z) * a.I + ii] : (const void*)a.Sf,
               in);
  }
  cp_async_wait_all();
  __syncthreads();
  fft_lines_x<RS, LX, false>(fb, LS, a.nsrc * TW, a.plan, tw, twz);
  if (a.sorted) {
    // Every channel at once in dense form.  The operator-sorted entries become groups of
    // one operator each with a coefficient matrix A[g][channel][source] (built once per
    // CTA); per point, each group's multiplier beta_g is formed once and
    //   channel c += i^q_g beta_g sum_s A[g][c][s] u_s.
    int* sng = soff + a.G + 1;
    ChanEntry* sgrp = reinterpret_cast<ChanEntry*>(reinterpret_cast<char*>(sm) +
                                                   ((reinterpret_cast<char*>(sng + 1) - reinterpret_cast<char*>(sm) + 15) / 16 * 16));
    double* sA = reinterpret_cast<double*>(sgrp + a.nent);
    __syncthreads();  // staged entries visible
    if (tid == 0) {
      int g = -1, last = -1;
      for (int qi = 0; qi < a.nent; ++qi) {
        const ChanEntry en = se[qi];
        const int key = en.nax | (en.ax0 << 2) | (en.ax1 << 4) | (en.part << 6);
        if (key != last) {
          last = key;
          ++g;
          sgrp[g] = en;
          for (int k = 0; k < 16; ++k) sA[g * 16 + k] = 0.0;
        }
        sA[g * 16 + en.pad * 4 + en.src] += en.coef;
      }
      *sng = g + 1;
    }
    __syncthreads();
    const int ngrp = *sng;
    const int npts = L0 * TW;
    for (int e = tid; e < npts; e += T) {
      const int z = fdiv(e, a.dTW), c = e - z * TW;
      const long long ii = i0 + c;
      double2 acc[4] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0),
                        make_double2(0.0, 0.0)};
      if (ii < a.I) {
        int nidx[3] = {z, 0, 0};
        if (a.ndim == 3) {
          nidx[1] = fdiv((int)ii, a.dMh);
          nidx[2] = (int)ii - nidx[1] * a.Mh;
        } else {
          nidx[1] = (int)ii;
        }
        double kp[3] = {0.0, 0.0, 0.0}, km[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          if (ax < a.ndim) {
            const int na = nidx[ax], nm = na == 0 ? 0 : a.chan.Ns[ax] - na;
            kp[ax] = skv[a.chan.kv_off[ax] + na];
            km[ax] = skv[a.chan.kv_off[ax] + nm];
          }
        }
        double2 u[4];
#pragma unroll
        for (int s4 = 0; s4 < 4; ++s4) u[s4] = s4 < a.nsrc ? fb[(s4 * TW + c) * LS + z] : make_double2(0.0, 0.0);
        for (int g = 0; g < ngrp; ++g) {
          const ChanEntry en = sgrp[g];
          double ap = 1.0, am = 1.0;
          if (en.nax >= 1) {
            ap *= sel3(kp[0], kp[1], kp[2], en.ax0);
            am *= sel3(km[0], km[1], km[2], en.ax0);
          }
          if (en.nax >= 2) {
            ap *= sel3(kp[0], kp[1], kp[2], en.ax1);
            am *= sel3(km[0], km[1], km[2], en.ax1);
          }
          const double sgn = (en.nax & 1) ? -1.0 : 1.0;
          int q;
          double beta;
          if (en.part == 0) {
            q = en.nax;
            beta = 0.5 * (ap + sgn * am);
          } else {
            q = en.nax + 3;
            beta = 0.5 * (ap - sgn * am);
          }
          const double* Ag = sA + g * 16;
#pragma unroll
          for (int c4 = 0; c4 < 4; ++c4) {
            if (c4 >= a.G) break;
            double2 sum = make_double2(0.0, 0.0);
#pragma unroll
            for (int s4 = 0; s4 < 4; ++s4) {
              if (s4 >= a.nsrc) break;
              const double w = Ag[c4 * 4 + s4];
              sum.x += w * u[s4].x;
              sum.y += w * u[s4].y;
            }
            double2 v = make_double2(beta * sum.x, beta * sum.y);
            switch (q & 3) {
              case 1: v = make_double2(-v.y, v.x); break;
              case 2: v = make_double2(-v.x, -v.y); break;
              case 3: v = make_double2(v.y, -v.x); break;
              default: break;
            }
            acc[c4].x += v.x;
            acc[c4].y += v.y;
          }
        }
      }
#pragma unroll
      for (int c4 = 0; c4 < 4; ++c4)
        if (c4 < a.G) cb[(c4 * TW + c) * LS + z] = acc[c4];
    }
    __syncthreads();
    fft_lines_x<RS, LX, true>(cb, LS, a.G * TW, a.plan, tw, twz);
    const int ncomp = a.G * L0 * TW;
    for (int e = tid; e < ncomp; e += T) {
      const int q0 = fdiv(e, a.dTW), c = e - q0 * TW;
      const int ch = fdivc<LX>(q0, a.dL0), z = q0 - ch * L0;
      const long long ii = i0 + c;
      if (ii < a.I) a.Sc[((long long)ch * L0 + z) * a.I + ii] = cb[(ch * TW + c) * LS + z];
    }
    return;
  }
  for (int g0 = 0; g0 < a.G; g0 += a.GB) {
    const int gc = min(a.GB, a.G - g0);
    const int ncomp = gc * L0 * TW;
    for (int e = tid; e < ncomp; e += T) {
      const int q0 = fdiv(e, a.dTW), c = e - q0 * TW;
      const int ch = fdivc<LX>(q0, a.dL0), z = q0 - ch * L0;
      const long long ii = i0 + c;
      double2 acc = make_double2(0.0, 0.0);
      if (ii < a.I) {
        int nidx[3] = {z, 0, 0};
        if (a.ndim == 3) {
          nidx[1] = fdiv((int)ii, a.dMh);
          nidx[2] = (int)ii - nidx[1] * a.Mh;
        } else {
          nidx[1] = (int)ii;
        }
        double kp[3] = {0.0, 0.0, 0.0}, km[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          if (ax < a.ndim) {
            const int na = nidx[ax], nm = na == 0 ? 0 : a.chan.Ns[ax] - na;
            kp[ax] = skv[a.chan.kv_off[ax] + na];
            km[ax] = skv[a.chan.kv_off[ax] + nm];
          }
        }
        const int lch = g0 + ch;
        for (int q = soff[lch]; q < soff[lch + 1]; ++q) {
          const ChanEntry en = se[q];
          const double2 u = fb[(en.src * TW + c) * LS + z];
          const double2 v = apply_entry_k(en, kp, km, u);
          acc.x += v.x;
          acc.y += v.y;
        }
      }
      cb[(ch * TW + c) * LS + z] = acc;
    }
    __syncthreads();
    fft_lines_x<RS, LX, true>(cb, LS, gc * TW, a.plan, tw, twz);
    for (int e = tid; e < ncomp; e += T) {
      const int q0 = fdiv(e, a.dTW), c = e - q0 * TW;
      const int ch = fdivc<LX>(q0, a.dL0), z = q0 - ch * L0;
      const long long ii = i0 + c;
      if (ii < a.I) a.Sc[((long long)(g0 + ch) * L0 + z) * a.I + ii] = cb[(ch * TW + c) * LS + z];
    }
    __syncthreads();
  }
}

template <int RS, int LX>
__global__ void __launch_bounds__(LX > 0 ? kSpecBlock : kMaxBlock, LX > 0 ? 3 : 1) k_mid(MidArgs a) {
  mid_body<RS, LX>(a, blockIdx.x);
}

// ---- axis-0 pass of 3D grids on TMA tiles (pencil.cuh): 128- or 256-point lines, at
// most two fields, channels written over their sources (the operator-grouped form of
// k_mid's multipliers, groups built at plan time).  Persistent CTAs of kPipeThreads:
// warp w transforms column (w & 7) of the tile (two half-warp columns for 128-point
// lines) for source / channel w >> 3.  Per tile: TMA loads of every source's boxes, the
// forward FFTs, the multipliers (each warp forms its channel at its points from all
// sources), the inverse FFTs in place, TMA stores of the channels.
struct MidPipeArgs {
  int I, nsrc, G, ntiles, ngrp, Mh;
  const double2* tw;      // axis-0 twiddle table (global)
  const ChanEntry* grp;   // one entry per operator group (its operator)
  const double* A;        // [ngrp][16]: A[g][channel * 4 + source]
  const double* kv;       // wavenumbers of every axis (ChanTable layout)
  int kv_off[3];
  int Ns[3];
  int kv_total;
  RhsIO io;
  int* err;
  // multiplier tables (TAB kernels): channel c at (z, column P) = sum_s (Mz[z][c][s] +
  // Mc[P][c][s]) U_s, the operator groups summed at plan time
  const double2* Mz;  // [G][nsrc][L0]
  const double2* Mc;  // [I][G][nsrc]
  // k_mid_pipe2: the groups on axis 0 alone as beta_g(z) and rotated matrices R_g
  const double* Bz;   // [NZ][L0]
  const double2* Rz;  // [NZ][G][nsrc]
};

constexpr int kPipeThreads = 512;
constexpr int kPipeSrcBytes = 32768;  // one source's tile: 8 columns x 256 rows or 16 x 128
constexpr int kPipeBufBytes = 2 * kPipeSrcBytes;  // one tile buffer (two sources, or two boxes)
constexpr int kPipeBufs = 3;  // tile ring: computing on one, storing from the one before, loading the next
constexpr int kPipeCols = 16;  // most columns of a tile (16 for 128-point lines, 8 for 256)

__host__ __device__ constexpr size_t mid_pipe_smem(int ngrp, int kv_total, int ztab) {
  return 1024 + kPipeBufs * (size_t)kPipeBufBytes + 8 * kPipeBufs + 8 + (size_t)ngrp * sizeof(ChanEntry) +
         (size_t)ngrp * 16 * 8 + (size_t)kv_total * 8 + (size_t)ngrp * kPipeCols * 3 * 8 + (size_t)ngrp * 4 + 16 +
         (size_t)ztab * 16 + 16 + (ztab ? kPipeBufs * kPipeCols * 4 * 16 : 0);
}

// TAB: the multipliers from the plan's tables (no operator group mixes axis 0 with
// another axis); otherwise k_mid's group arithmetic with per-tile column factors.
template <int L, bool TAB>
__global__ void __launch_bounds__(kPipeThreads, 1)
    k_mid_pipe(const __grid_constant__ CUtensorMap tmF, const __grid_constant__ CUtensorMap tmC, MidPipeArgs a) {
  extern __shared__ char smraw[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;
  constexpr int NB = 256 / L;  // boxes per source tile
  constexpr int LPL = L / 8;
  constexpr int BOXB = L * 128;
  char* sm = smraw + ((1024 - (smem_u32(smraw) & 1023)) & 1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kPipeBufs * kPipeBufBytes);
  ChanEntry* sgrp = reinterpret_cast<ChanEntry*>(full + kPipeBufs + 1);
  double* sA = reinterpret_cast<double*>(sgrp + a.ngrp);
  double* skv = sA + 16 * a.ngrp;
  // per tile: each group's column factors (kp and km products over the factors not on
  // axis 0) and, for groups without an axis-0 factor, its whole multiplier beta
  double* sgt = skv + a.kv_total;
  int* sgc = reinterpret_cast<int*>(sgt + a.ngrp * kPipeCols * 3);
  double2* smz = reinterpret_cast<double2*>(
      (reinterpret_cast<uintptr_t>(sgc + a.ngrp) + 15) & ~static_cast<uintptr_t>(15));  // TAB: Mz
  double2* smc = smz + L * a.G * a.nsrc;  // TAB: each buffer's column multipliers (Mc rows of its tile)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (TAB)
    for (int t = tid; t < L * a.G * a.nsrc; t += kPipeThreads) smz[t] = a.Mz[t];
  for (int t = tid; t < a.ngrp; t += kPipeThreads) sgrp[t] = a.grp[t];
  for (int t = tid; t < a.ngrp; t += kPipeThreads) {
    const ChanEntry en = a.grp[t];
    const int na0 = (en.nax >= 1 && en.ax0 == 0) + (en.nax >= 2 && en.ax1 == 0);
    const int q = en.part == 0 ? en.nax : en.nax + 3;
    sgc[t] = na0 | (en.nax << 2) | (en.part << 4) | ((q & 3) << 5);
  }
  for (int t = tid; t < 16 * a.ngrp; t += kPipeThreads) sA[t] = a.A[t];
  for (int t = tid; t < a.kv_total; t += kPipeThreads) skv[t] = a.kv[t];
  if (tid == 0) {
    for (int k = 0; k < kPipeBufs; ++k) mbar_init(&full[k], 1);
    mbar_fence_init();
    tma_prefetch(&tmF);
    tma_prefetch(&tmC);
  }
  __syncthreads();
  const int h = warp >> 3;                              // source (forward) / channel (inverse)
  const int cc = (warp & 7) * (32 / LPL) + lane / LPL;  // column of the tile
  const int coff = (cc >> 3) * BOXB;                    // offset of the column's box in a source tile
  const int c = cc & 7;
  WarpLine<L> wl;
  wl.init(a.tw, lane % LPL);
  auto issue = [&](int tile, int b) {
    const int P0 = tile * 8 * NB;
    const int ncol = min(8 * NB, a.I - P0);
    const unsigned mcb = TAB ? (unsigned)(ncol * a.G * a.nsrc * 16) : 0u;
    mbar_expect_tx(&full[b], (unsigned)(a.nsrc * kPipeSrcBytes) + mcb);
    char* dst = sm + b * kPipeBufBytes;
    for (int s = 0; s < a.nsrc; ++s)
      for (int bx = 0; bx < NB; ++bx)
        tma_load_2d(dst + s * kPipeSrcBytes + bx * BOXB, &tmF, 2 * (P0 + 8 * bx), s * L, &full[b]);
    if (TAB) bulk_load(smc + b * kPipeCols * 4, a.Mc + (long long)P0 * a.G * a.nsrc, mcb, &full[b]);
  };
  if (tid == 0) {
    if ((int)blockIdx.x < a.ntiles) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < a.ntiles) issue(blockIdx.x + gridDim.x, 1);
  }
  int it = 0, b = 0;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x, ++it, b = (b + 1 == kPipeBufs) ? 0 : b + 1) {
    const bool ok = mbar_wait(&full[b], (unsigned)((it / kPipeBufs) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(a.io.mode == 1 ? &a.io.ctl->pipe_err : a.err, kPipeErrTimeout);
        const int b1 = (b + 1) % kPipeBufs;  // bounded: the next buffer's loads
        if (tile + (int)gridDim.x < a.ntiles) mbar_wait(&full[b1], (unsigned)(((it + 1) / kPipeBufs) & 1));
        bulk_wait_all();
      }
      return;
    }
    char* tb = sm + b * kPipeBufBytes;
    const long long P = (long long)tile * 8 * NB + cc;
    // the tile's column factors (read after the barrier that ends the forward FFTs)
    for (int t = tid; !TAB && t < a.ngrp * 8 * NB; t += kPipeThreads) {
      const int g = t / (8 * NB), col = t - g * (8 * NB);
      const long long Pc = (long long)tile * 8 * NB + col;
      const int k1 = Pc < a.I ? (int)(Pc / a.Mh) : 0, kx = Pc < a.I ? (int)(Pc - (long long)k1 * a.Mh) : 0;
      const int m1 = k1 == 0 ? 0 : a.Ns[1] - k1, m2 = kx == 0 ? 0 : a.Ns[2] - kx;
      const double kpc[3] = {1.0, skv[a.kv_off[1] + k1], skv[a.kv_off[2] + kx]};
      const double kmc[3] = {1.0, skv[a.kv_off[1] + m1], skv[a.kv_off[2] + m2]};
      const ChanEntry en = sgrp[g];
      double cp = 1.0, cm = 1.0;  // k_mid's products, axis-0 factors left out
      if (en.nax >= 1 && en.ax0 != 0) {
        cp *= kpc[en.ax0];
        cm *= kmc[en.ax0];
      }
      if (en.nax >= 2 && en.ax1 != 0) {
        cp *= kpc[en.ax1];
        cm *= kmc[en.ax1];
      }
      const double sgn = (en.nax & 1) ? -1.0 : 1.0;
      double* gt = sgt + (g * kPipeCols + col) * 3;
      gt[0] = cp;
      gt[1] = cm;
      gt[2] = en.part == 0 ? 0.5 * (cp + sgn * cm) : 0.5 * (cp - sgn * cm);
    }
    double2 v[8];
    if (h < a.nsrc) {
      char* bx = tb + h * kPipeSrcBytes + coff;
      wl.load(v, bx, c);
      wl.template transform<false>(v, bx, c);
      wl.store(v, bx, c);
    }
    __syncthreads();
    if (TAB && h < a.G) {
      // channel h at this lane's points: (Mz[z] + Mc[P]) . U
      const bool inP = P < a.I;
      double2 mc[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
      if (inP)
        for (int s2 = 0; s2 < a.nsrc; ++s2) mc[s2] = smc[b * kPipeCols * 4 + (cc * a.G + h) * a.nsrc + s2];
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int z = wl.ml + LPL * p;
        double2 acc = make_double2(0.0, 0.0);
        if (inP) {
          const double2 u0 = *swz_col(tb + coff, c, z);
          const double2* mz = smz + h * a.nsrc * L + z;  // [h][s][z]: consecutive lanes, consecutive z
          const double2 m0 = c_add(mz[0], mc[0]);
          acc = c_mul(m0, u0);
          if (a.nsrc > 1) {
            const double2 u1 = *swz_col(tb + kPipeSrcBytes + coff, c, z);
            const double2 m1 = c_add(mz[L], mc[1]);
            acc = c_add(acc, c_mul(m1, u1));
          }
        }
        v[p] = acc;
      }
    } else if (!TAB && h < a.G) {
      // channel h at this lane's points z = ml + LPL p of column P: k_mid's arithmetic,
      // the factors off axis 0 taken from the tile's column table
      const bool inP = P < a.I;
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int z = wl.ml + LPL * p;
        double2 acc = make_double2(0.0, 0.0);
        if (inP) {
          const int m0 = z == 0 ? 0 : a.Ns[0] - z;
          const double kp0 = skv[a.kv_off[0] + z], km0 = skv[a.kv_off[0] + m0];
          double2 u[2];
          u[0] = *swz_col(tb + coff, c, z);
          u[1] = a.nsrc > 1 ? *swz_col(tb + kPipeSrcBytes + coff, c, z) : make_double2(0.0, 0.0);
          for (int g = 0; g < a.ngrp; ++g) {
            const int code = sgc[g];
            const int na0 = code & 3, nax = (code >> 2) & 3, part = (code >> 4) & 1, q = code >> 5;
            const double* gt = sgt + (g * kPipeCols + cc) * 3;
            double beta;
            if (na0 == 0) {
              beta = gt[2];
            } else {
              double ap, am;
              if (na0 == 2) {
                ap = kp0 * kp0;
                am = km0 * km0;
              } else if (nax == 1) {
                ap = kp0;
                am = km0;
              } else {
                ap = kp0 * gt[0];
                am = km0 * gt[1];
              }
              const double sgn = (nax & 1) ? -1.0 : 1.0;
              beta = part == 0 ? 0.5 * (ap + sgn * am) : 0.5 * (ap - sgn * am);
            }
            const double* Ag = sA + g * 16 + h * 4;
            double2 sum = make_double2(0.0, 0.0);
#pragma unroll
            for (int s4 = 0; s4 < 2; ++s4) {
              if (s4 >= a.nsrc) break;
              const double w = Ag[s4];
              sum.x += w * u[s4].x;
              sum.y += w * u[s4].y;
            }
            double2 vv = make_double2(beta * sum.x, beta * sum.y);
            switch (q) {
              case 1: vv = make_double2(-vv.y, vv.x); break;
              case 2: vv = make_double2(-vv.x, -vv.y); break;
              case 3: vv = make_double2(vv.y, -vv.x); break;
              default: break;
            }
            acc.x += vv.x;
            acc.y += vv.y;
          }
        }
        v[p] = acc;
      }
    }
    __syncthreads();  // every source read before the channels overwrite them
    if (h < a.G) {
      char* bx = tb + h * kPipeSrcBytes + coff;
      wl.template transform<true>(v, bx, c);
      wl.store(v, bx, c);
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      const int P0 = tile * 8 * NB;
      for (int ch = 0; ch < a.G; ++ch)
        for (int bx = 0; bx < NB; ++bx) tma_store_2d(&tmC, 2 * (P0 + 8 * bx), ch * L, tb + ch * kPipeSrcBytes + bx * BOXB);
      bulk_commit();
      const int nt = tile + 2 * (int)gridDim.x;
      if (nt < a.ntiles) {
        bulk_wait_read_1();  // the previous tile's stores have read the buffer the next load fills
        issue(nt, (b + 2) % kPipeBufs);
      }
    }
  }
  if (tid == 0) bulk_wait_all();
}

// ---- axis-0 pass, one column per warp (two per warp for 128-point lines): the lanes of a
// column transform every source, form every channel in registers and transform the
// channels back, so a tile needs no block barrier between its phases.  For
// multipliers that split into at most two groups on axis 0 alone (NZ) and groups off
// axis 0: channel c at (z, P) = sum_s (Mc[P][c][s] + sum_g beta_g(z) R_g[c][s]) U_s, with
// the lane's beta_g at its eight points and the R_g in registers and the tile's Mc rows
// bulk-copied with the tile.  kMid2Threads: one warp per column pair or column.
constexpr int kMid2Threads = 256;

__host__ __device__ constexpr size_t mid2_smem(int L0) {
  return 1024 + kPipeBufs * (size_t)kPipeBufBytes + 8 * kPipeBufs + 8 + kPipeBufs * kPipeCols * 4 * 16 +
         2 * (size_t)L0 * 8 + 2 * 4 * 16;
}

// REALM: every multiplier is real (the operator groups' i^q rotations are all even, as
// for the CGLE's second derivatives): each channel term is two products instead of a
// complex product, in the complex product's rounding (no contraction).
template <int L, int NZ, bool REALM>
__global__ void __launch_bounds__(kMid2Threads, 1)
    k_mid_pipe2(const __grid_constant__ CUtensorMap tmF, const __grid_constant__ CUtensorMap tmC, MidPipeArgs a) {
  extern __shared__ char smraw[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;
  constexpr int NB = 256 / L;  // boxes per source tile
  constexpr int LPL = L / 8;
  constexpr int BOXB = L * 128;
  char* sm = smraw + ((1024 - (smem_u32(smraw) & 1023)) & 1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kPipeBufs * kPipeBufBytes);
  double2* smc = reinterpret_cast<double2*>(full + kPipeBufs + 1);  // each buffer's Mc rows
  double2* srz = smc + kPipeBufs * kPipeCols * 4;                     // R_g[c][s], zero-padded to 2 x 2
  double* sbz = reinterpret_cast<double*>(srz + NZ * 4);              // beta_g(z)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = a.G, nsrc = a.nsrc;
  for (int t = tid; t < NZ * L; t += kMid2Threads) sbz[t] = a.Bz[t];
  for (int t = tid; t < NZ * 4; t += kMid2Threads) {
    const int g = t >> 2, ch = (t >> 1) & 1, s2 = t & 1;
    srz[t] = (ch < G && s2 < nsrc) ? a.Rz[(g * G + ch) * nsrc + s2] : make_double2(0.0, 0.0);
  }
  if (tid == 0) {
    for (int k = 0; k < kPipeBufs; ++k) mbar_init(&full[k], 1);
    mbar_fence_init();
    tma_prefetch(&tmF);
    tma_prefetch(&tmC);
  }
  __syncthreads();
  const int cc = warp * (32 / LPL) + lane / LPL;  // column of the tile
  const int coff = (cc >> 3) * BOXB;              // offset of the column's box in a source tile
  const int c = cc & 7;
  WarpLine<L> wl;
  wl.init(a.tw, lane % LPL);
  auto issue = [&](int tile, int b) {
    const int P0 = tile * 8 * NB;
    const int ncol = min(8 * NB, a.I - P0);
    const unsigned mcb = (unsigned)(ncol * G * nsrc * 16);
    mbar_expect_tx(&full[b], (unsigned)(nsrc * kPipeSrcBytes) + mcb);
    char* dst = sm + b * kPipeBufBytes;
    for (int s2 = 0; s2 < nsrc; ++s2)
      for (int bx = 0; bx < NB; ++bx)
        tma_load_2d(dst + s2 * kPipeSrcBytes + bx * BOXB, &tmF, 2 * (P0 + 8 * bx), s2 * L, &full[b]);
    bulk_load(smc + b * kPipeCols * 4, a.Mc + (long long)P0 * G * nsrc, mcb, &full[b]);
  };
  if (tid == 0) {
    if ((int)blockIdx.x < a.ntiles) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < a.ntiles) issue(blockIdx.x + gridDim.x, 1);
  }
  int it = 0, b = 0;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x, ++it, b = (b + 1 == kPipeBufs) ? 0 : b + 1) {
    const bool ok = mbar_wait(&full[b], (unsigned)((it / kPipeBufs) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(a.io.mode == 1 ? &a.io.ctl->pipe_err : a.err, kPipeErrTimeout);
        const int b1 = (b + 1) % kPipeBufs;  // bounded: the next buffer's loads
        if (tile + (int)gridDim.x < a.ntiles) mbar_wait(&full[b1], (unsigned)(((it + 1) / kPipeBufs) & 1));
        bulk_wait_all();
      }
      return;
    }
    char* tb = sm + b * kPipeBufBytes;
    const long long P = (long long)tile * 8 * NB + cc;
    const bool inP = P < a.I;
    double2 x[2][8];
#pragma unroll
    for (int s2 = 0; s2 < 2; ++s2) {
      if (s2 < nsrc) {
        char* bx = tb + s2 * kPipeSrcBytes + coff;
        wl.load(x[s2], bx, c);
        wl.template transform<false>(x[s2], bx, c);
      } else {
#pragma unroll
        for (int p = 0; p < 8; ++p) x[s2][p] = make_double2(0.0, 0.0);
      }
    }
    double2 mc[2][2];
#pragma unroll
    for (int ch = 0; ch < 2; ++ch)
#pragma unroll
      for (int s2 = 0; s2 < 2; ++s2)
        mc[ch][s2] = (inP && ch < G && s2 < nsrc) ? smc[b * kPipeCols * 4 + (cc * G + ch) * nsrc + s2]
                                                   : make_double2(0.0, 0.0);
    // every channel at the lane's points, over the sources in place
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      double2 out[2];
#pragma unroll
      for (int ch = 0; ch < 2; ++ch) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int s2 = 0; s2 < 2; ++s2) {
          if (REALM) {
            double m = mc[ch][s2].x;
#pragma unroll
            for (int g = 0; g < NZ; ++g) {
              const double bg = sbz[g * L + wl.ml + LPL * p];
              m += bg * srz[g * 4 + ch * 2 + s2].x;
            }
            acc.x = __dadd_rn(acc.x, __dmul_rn(m, x[s2][p].x));
            acc.y = __dadd_rn(acc.y, __dmul_rn(m, x[s2][p].y));
          } else {
            double2 m = mc[ch][s2];
#pragma unroll
            for (int g = 0; g < NZ; ++g) {
              const double bg = sbz[g * L + wl.ml + LPL * p];
              const double2 r = srz[g * 4 + ch * 2 + s2];
              m.x += bg * r.x;
              m.y += bg * r.y;
            }
            acc = c_add(acc, c_mul(m, x[s2][p]));
          }
        }
        out[ch] = inP ? acc : make_double2(0.0, 0.0);
      }
      x[0][p] = out[0];
      x[1][p] = out[1];
    }
#pragma unroll
    for (int ch = 0; ch < 2; ++ch) {
      if (ch < G) {
        char* bx = tb + ch * kPipeSrcBytes + coff;
        wl.template transform<true>(x[ch], bx, c);
        wl.store(x[ch], bx, c);
      }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      const int P0 = tile * 8 * NB;
      for (int ch = 0; ch < G; ++ch)
        for (int bx = 0; bx < NB; ++bx) tma_store_2d(&tmC, 2 * (P0 + 8 * bx), ch * L, tb + ch * kPipeSrcBytes + bx * BOXB);
      bulk_commit();
      const int nt = tile + 2 * (int)gridDim.x;
      if (nt < a.ntiles) {
        bulk_wait_read_1();  // the previous tile's stores have read the buffer the next load fills
        issue(nt, (b + 2) % kPipeBufs);
      }
    }
  }
  if (tid == 0) bulk_wait_all();
}

// ---- middle-axis pass of 3D grids on TMA tiles: FFT (forward or inverse) of every
// line along axis 1, in place.  A box is 8 consecutive x-wavenumber columns by the whole
// axis-1 line of one plane (field or channel, axis-0 index); a tile is c2c_boxes(L)
// consecutive boxes (32 KB), one line per warp (256 points) or half warp (128 points).
// Two CTAs of eight warps per SM, each with its own ring of three tiles, so that one
// CTA's barrier and store waits overlap the other's transforms.
struct C2CPipeArgs {
  int nbox, nchunk, ntiles;
  int rev;  // take the tiles from the last to the first
  const double2* tw;
  RhsIO io;
  int* err;
};

constexpr int kC2cThreads = 256;
constexpr int kC2cBufBytes = 32 * 1024;
constexpr int kC2cBufs = 3;
__host__ __device__ constexpr int c2c_boxes(int L) { return 256 / L; }
static_assert(c2c_boxes(256) * 256 * 128 == kC2cBufBytes && c2c_boxes(128) * 128 * 128 == kC2cBufBytes,
              "a tile fills one buffer");
static_assert((kC2cThreads / 32) * (32 / (256 / 8)) == 8 * c2c_boxes(256) &&
                  (kC2cThreads / 32) * (32 / (128 / 8)) == 8 * c2c_boxes(128),
              "one line of a tile per warp (256 points) or half warp (128 points)");
constexpr size_t kC2cPipeSmem = 1024 + kC2cBufs * (size_t)kC2cBufBytes + 8 * kC2cBufs + 8;

template <int L, bool INV>
__global__ void __launch_bounds__(kC2cThreads, 2)
    k_c2c_pipe(const __grid_constant__ CUtensorMap tm, C2CPipeArgs a) {
  extern __shared__ char smraw[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;
  constexpr int BPT = c2c_boxes(L);
  constexpr int LPL = L / 8;
  constexpr int BOXB = L * 128;
  char* sm = smraw + ((1024 - (smem_u32(smraw) & 1023)) & 1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kC2cBufs * kC2cBufBytes);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int k = 0; k < kC2cBufs; ++k) mbar_init(&full[k], 1);
    mbar_fence_init();
    tma_prefetch(&tm);
  }
  __syncthreads();
  const int li = warp * (32 / LPL) + lane / LPL;  // line of the tile
  const int coff = (li >> 3) * BOXB, c = li & 7;
  WarpLine<L> wl;
  wl.init(a.tw, lane % LPL);
  // the inverse pass takes its tiles in reverse order before a row kernel (it ends on
  // the planes the row kernel starts with, which are then still in L2) and in order
  // before a fused row kernel, which takes its rows from the last to the first
  auto order = [&](int tile) { return a.rev ? a.ntiles - 1 - tile : tile; };
  auto issue = [&](int tile, int b) {
    const int b0 = order(tile) * BPT, nb = min(BPT, a.nbox - b0);
    mbar_expect_tx(&full[b], (unsigned)(nb * BOXB));
    char* dst = sm + b * kC2cBufBytes;
    for (int k = 0; k < nb; ++k) {
      const int plane = (b0 + k) / a.nchunk, chunk = (b0 + k) - plane * a.nchunk;
      tma_load_3d(dst + k * BOXB, &tm, 16 * chunk, 0, plane, &full[b]);
    }
  };
  if (tid == 0) {
    if ((int)blockIdx.x < a.ntiles) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < a.ntiles) issue(blockIdx.x + gridDim.x, 1);
  }
  int it = 0, b = 0;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x, ++it, b = (b + 1 == kC2cBufs) ? 0 : b + 1) {
    const bool ok = mbar_wait(&full[b], (unsigned)((it / kC2cBufs) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(a.io.mode == 1 ? &a.io.ctl->pipe_err : a.err, kPipeErrTimeout);
        const int b1 = (b + 1) % kC2cBufs;
        if (tile + (int)gridDim.x < a.ntiles) mbar_wait(&full[b1], (unsigned)(((it + 1) / kC2cBufs) & 1));
        bulk_wait_all();
      }
      return;
    }
    char* tb = sm + b * kC2cBufBytes;
    char* bx = tb + coff;
    if (order(tile) * BPT + (li >> 3) < a.nbox) {
      double2 v[8];
      wl.load(v, bx, c);
      wl.template transform<INV>(v, bx, c);
      wl.store(v, bx, c);
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      const int b0 = order(tile) * BPT, nb = min(BPT, a.nbox - b0);
      for (int k = 0; k < nb; ++k) {
        const int plane = (b0 + k) / a.nchunk, chunk = (b0 + k) - plane * a.nchunk;
        tma_store_3d(&tm, 16 * chunk, 0, plane, tb + k * BOXB);
      }
      bulk_commit();
      const int nt = tile + 2 * (int)gridDim.x;
      if (nt < a.ntiles) {
        bulk_wait_read_1();
        issue(nt, (b + 2) % kC2cBufs);
      }
    }
  }
  if (tid == 0) bulk_wait_all();
}

struct Mult1DArgs {
  int Mh, nch, ch0;
  const double2* Sf;
  double2* Sc;
  ChanTable chan;
  RhsIO io;
};

__global__ void k_mult1d(Mult1DArgs a) {
  if (a.io.mode == 1 && !a.io.ctl->running) return;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)a.nch * a.Mh) return;
  const int ch = (int)(e / a.Mh), kx = (int)(e - (long long)ch * a.Mh);
  int nidx[3] = {kx, 0, 0};
  double2 acc = make_double2(0.0, 0.0);
  const int gch = a.ch0 + ch;
  for (int q = a.chan.off[gch]; q < a.chan.off[gch + 1]; ++q) {
    const ChanEntry en = a.chan.ent[q];
    const double2 v = apply_entry(en, nidx, a.chan, a.Sf[(long long)en.src * a.Mh + kx]);
    acc.x += v.x;
    acc.y += v.y;
  }
  a.Sc[(long long)ch * a.Mh + kx] = acc;
}

// Symbol of the constant-coefficient FD operator of one linear entry at multi-index
// nidx (see LinEntry): returns the complex value.
__device__ __forceinline__ double2 lin_symbol(const LinEntry& e, const int* nidx, const LinTable& t) {
  if (e.nax == 0) return make_double2(1.0, 0.0);
  const int a = e.ax0;
  const double sa = t.sinv[t.off[a] + nidx[a]];
  if (e.nax == 1) return make_double2(0.0, sa / t.dx[a]);
  if (e.ax0 == e.ax1) {
    const double ca = t.cosv[t.off[a] + nidx[a]];
    return make_double2((2.0 * ca - 2.0) / (t.dx[a] * t.dx[a]), 0.0);
  }
  const int b = e.ax1;
  const double sb = t.sinv[t.off[b] + nidx[b]];
  return make_double2(-2.0 * sa * sb / (t.dx[a] * t.dx[b]), 0.0);
}

// x = (I + alpha L(k))^-1 r at one mode, n <= kMaxPrecFields, Gaussian elimination
// with partial pivoting; a (numerically) singular mode is passed through unchanged.
__device__ __forceinline__ void mode_solve(const LinTable& t, const int* nidx, double2* v, int n) {
  double2 A[kMaxPrecFields][kMaxPrecFields];
  double2 b[kMaxPrecFields];
#pragma unroll
  for (int i = 0; i < kMaxPrecFields; ++i) {
#pragma unroll
    for (int j = 0; j < kMaxPrecFields; ++j) A[i][j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    b[i] = i < n ? v[i] : make_double2(0.0, 0.0);
  }
  const double alpha = t.alpha_dev ? *t.alpha_dev : t.alpha;
  for (int q = 0; q < t.nent; ++q) {
    const LinEntry e = t.ent[q];
    const double2 sy = lin_symbol(e, nidx, t);
    const double cf = alpha * e.coef;
#pragma unroll
    for (int i = 0; i < kMaxPrecFields; ++i)
#pragma unroll
      for (int j = 0; j < kMaxPrecFields; ++j)
        if (i == e.row && j == e.src) {
          A[i][j].x += cf * sy.x;
          A[i][j].y += cf * sy.y;
        }
  }
  bool ok = true;
#pragma unroll
  for (int k = 0; k < kMaxPrecFields; ++k) {
    if (k >= n) break;
    // pivot
    int p = k;
    double best = A[k][k].x * A[k][k].x + A[k][k].y * A[k][k].y;
#pragma unroll
    for (int i = k + 1; i < kMaxPrecFields; ++i) {
      if (i >= n) break;
      const double m2 = A[i][k].x * A[i][k].x + A[i][k].y * A[i][k].y;
      if (m2 > best) { best = m2; p = i; }
    }
    if (!(best > 1e-300)) { ok = false; break; }
#pragma unroll
    for (int i = 0; i < kMaxPrecFields; ++i)
      if (i == p && p != k) {
#pragma unroll
        for (int j = 0; j < kMaxPrecFields; ++j) { const double2 tmp = A[k][j]; A[k][j] = A[i][j]; A[i][j] = tmp; }
        const double2 tb = b[k]; b[k] = b[i]; b[i] = tb;
      }
    const double2 piv = A[k][k];
    const double inv = 1.0 / (piv.x * piv.x + piv.y * piv.y);
    const double2 ip = make_double2(piv.x * inv, -piv.y * inv);
#pragma unroll
    for (int i = k + 1; i < kMaxPrecFields; ++i) {
      if (i >= n) break;
      const double2 f = c_mul(A[i][k], ip);
#pragma unroll
      for (int j = k; j < kMaxPrecFields; ++j) A[i][j] = c_sub(A[i][j], c_mul(f, A[k][j]));
      b[i] = c_sub(b[i], c_mul(f, b[k]));
    }
  }
  if (!ok) return;
#pragma unroll
  for (int k = kMaxPrecFields - 1; k >= 0; --k) {
    if (k >= n) continue;
    double2 acc = b[k];
#pragma unroll
    for (int j = k + 1; j < kMaxPrecFields; ++j)
      if (j < n) acc = c_sub(acc, c_mul(A[k][j], b[j]));
    const double2 piv = A[k][k];
    const double inv = 1.0 / (piv.x * piv.x + piv.y * piv.y);
    b[k] = c_mul(acc, make_double2(piv.x * inv, -piv.y * inv));
  }
  for (int i = 0; i < n; ++i) v[i] = b[i];
}

struct MidSolveArgs {
  int L0, I, TW, n, ndim, Mh;
  FastDiv dTW, dL0, dMh;
  LinePlan plan;
  const double2* tw;
  const double2* Sf;
  double2* Sc;
  LinTable lin;
};

template <int RS>
__global__ void __launch_bounds__(kMaxBlock, 1) k_mid_solve(MidSolveArgs a) {
  extern __shared__ double2 sm[];
  const int L0 = a.L0, TW = a.TW, LS = L0 + 1, T = blockDim.x, tid = threadIdx.x, n = a.n;
  double2* tw = sm;
  double2* fb = sm + L0;
  for (int t = tid; t < L0; t += T) tw[t] = a.tw[t];
  const long long i0 = (long long)blockIdx.x * TW;
  const int nload = n * L0 * TW;
  for (int e = tid; e < nload; e += T) {
    const int q0 = fdiv(e, a.dTW), c = e - q0 * TW;
    const int f = fdiv(q0, a.dL0), z = q0 - f * L0;
    const long long ii = i0 + c;
    const bool in = ii < a.I;
    cp_async16(&fb[(f * TW + c) * LS + z], in ? (const void*)&a.Sf[((long long)f * L0 + z) * a.I + ii] : (const void*)a.Sf,
               in);
  }
  cp_async_wait_all();
  __syncthreads();
  fft_lines<RS, false>(fb, LS, n * TW, a.plan, tw);
  for (int e = tid; e < L0 * TW; e += T) {
    const int z = fdiv(e, a.dTW), c = e - z * TW;
    const long long ii = i0 + c;
    if (ii >= a.I) continue;
    int nidx[3];
    nidx[0] = z;
    if (a.ndim == 3) {
      nidx[1] = fdiv((int)ii, a.dMh);
      nidx[2] = (int)ii - nidx[1] * a.Mh;
    } else {
      nidx[1] = (int)ii;
    }
    double2 v[kMaxPrecFields];
    for (int f = 0; f < n; ++f) v[f] = fb[(f * TW + c) * LS + z];
    mode_solve(a.lin, nidx, v, n);
    for (int f = 0; f < n; ++f) fb[(f * TW + c) * LS + z] = v[f];
  }
  __syncthreads();
  fft_lines<RS, true>(fb, LS, n * TW, a.plan, tw);
  for (int e = tid; e < nload; e += T) {
    const int q0 = fdiv(e, a.dTW), c = e - q0 * TW;
    const int f = fdiv(q0, a.dL0), z = q0 - f * L0;
    const long long ii = i0 + c;
    if (ii < a.I) a.Sc[((long long)f * L0 + z) * a.I + ii] = fb[(f * TW + c) * LS + z];
  }
}

__global__ void k_mult1d_solve(int Mh, int n, const double2* Sf, double2* Sc, LinTable lin) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  if (kx >= Mh) return;
  int nidx[3] = {kx, 0, 0};
  double2 v[kMaxPrecFields];
  for (int f = 0; f < n; ++f) v[f] = Sf[(long long)f * Mh + kx];
  mode_solve(lin, nidx, v, n);
  for (int f = 0; f < n; ++f) Sc[(long long)f * Mh + kx] = v[f];
}

struct InvXArgs {
  int M, Mh, R, P, n, nch_run, npairs, do_fft, tw_smem;
  FastDiv dM, dnpM, dnhalf, dhalf, dnM, dncM;
  long long N;
  LinePlan plan;
  const double2* tw;
  const double2* Sc;
  DictTable dict;
  RhsIO io;
  double* Yout;       // Y mode: channel c -> complex block ydst[c]>>1, part ydst[c]&1
  const int* ydst;
  int yplain;         // 1: channel c -> real array Yout[c*N + point]
  int ch_base;        // first channel row of Sc this launch reads
};

template <int RS, int LX>
__device__ __forceinline__ void inv_x_body(const InvXArgs& a, int bx) {
  extern __shared__ double2 sm[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;
  const Resolved r = resolve(a.io);
  const int M = LX ? LX : a.M, Mh = LX ? LX / 2 + 1 : a.Mh, T = blockDim.x, tid = threadIdx.x;
  const int P = a.P, np = a.npairs, n = a.n;
  const double2* tw = a.tw;
  double2* lines = sm;
  bool twz = false;
  if (a.do_fft && a.tw_smem) {
    twz = stage_twiddles<LX>(sm, a.tw, M);
    tw = sm;
    lines = sm + M;
  }
  double* phys = reinterpret_cast<double*>(lines + (a.do_fft ? P * np * M : 0));
  const long long r0 = (long long)bx * P;
  // dictionary tables staged in shared memory (read by every point)
  double* spoly = phys + (long long)P * n * M;
  const int npoly = a.dict.poly_nf ? n * a.dict.poly_count : 0;
  DictTerm* sterm = reinterpret_cast<DictTerm*>(spoly + npoly);
  DictFactor* sfac = reinterpret_cast<DictFactor*>(sterm + a.dict.nterms);
  int* sfb = reinterpret_cast<int*>(sfac + a.dict.nfac);
  int* sfold = sfb + n + 1;
  if (!a.Yout) {
    for (int t = tid; t < npoly; t += T) spoly[t] = a.dict.poly[t];
    for (int t = tid; t < a.dict.nterms; t += T) sterm[t] = a.dict.terms[t];
    for (int t = tid; t < a.dict.nfac; t += T) sfac[t] = a.dict.fac[t];
    for (int t = tid; t <= n; t += T) sfb[t] = a.dict.field_begin[t];
    for (int t = tid; t < n; t += T) sfold[t] = a.dict.fold[t];
  }
  if (!a.Yout) {
    // physical fields of the P rows: asynchronous 16-byte copies where rows and the
    // array's alignment allow (a caller's y may be only 8-byte aligned)
    if ((M & 1) == 0 && (reinterpret_cast<unsigned long long>(r.u) & 15) == 0) {
      const int half = M / 2;
      const int nph = P * n * half;
      for (int e = tid; e < nph; e += T) {
        const int pr = fdiv(e, a.dnhalf);
        const int w = e - pr * n * half;
        const int fi = fdivc<LX / 2>(w, a.dhalf);
        const int x2 = (w - fi * half) * 2;
        const long long row = r0 + pr;
        const bool in = row < a.R;
        cp_async16(&phys[(pr * n + fi) * M + x2], in ? (const void*)&r.u[((long long)fi * a.R + row) * M + x2] : (const void*)r.u,
                   in);
      }
    } else {
      const int nph = P * n * M;
      for (int e = tid; e < nph; e += T) {
        const int pr = fdiv(e, a.dnM);
        const int w = e - pr * n * M;
        const int fi = fdivc<LX>(w, a.dM);
        const int x = w - fi * M;
        const long long row = r0 + pr;
        phys[(pr * n + fi) * M + x] = row < a.R ? r.u[((long long)fi * a.R + row) * M + x] : 0.0;
      }
    }
  }
  if (a.do_fft) {
    constexpr int kUnroll = 4;
    const int nel = P * np * M;
    for (int e0 = tid; e0 < nel; e0 += T * kUnroll) {
      double2 A[kUnroll], B[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const int e = e0 + u * T;
        A[u] = make_double2(0.0, 0.0);
        B[u] = make_double2(0.0, 0.0);
        if (e >= nel) continue;
        const int pr = fdiv(e, a.dnpM);
        const int w = e - pr * np * M;
        const int cp = fdivc<LX>(w, a.dM);
        const int kx = w - cp * M;
        const long long row = r0 + pr;
        if (row >= a.R) continue;
        const int c0 = 2 * cp, c1 = c0 + 1;
        const int kk = kx >= Mh ? M - kx : kx;
        A[u] = a.Sc[((long long)(a.ch_base + c0) * a.R + row) * Mh + kk];
        if (c1 < a.nch_run) B[u] = a.Sc[((long long)(a.ch_base + c1) * a.R + row) * Mh + kk];
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const int e = e0 + u * T;
        if (e >= nel) break;
        const int pr = fdiv(e, a.dnpM);
        const int w = e - pr * np * M;
        const int cp = fdivc<LX>(w, a.dM);
        const int kx = w - cp * M;
        double2 Av = A[u], Bv = B[u];
        if (kx == 0 || 2 * kx == M) {
          Av.y = 0.0;
          Bv.y = 0.0;
        }
        if (kx >= Mh) {
          Av.y = -Av.y;
          Bv.y = -Bv.y;
        }
        lines[(pr * np + cp) * M + kx] = make_double2(Av.x - Bv.y, Av.y + Bv.x);
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  if (a.do_fft) fft_lines_x<RS, LX, true>(lines, M, P * np, a.plan, tw, twz);

  if (a.Yout) {
    const int nel = P * a.nch_run * M;
    for (int e = tid; e < nel; e += T) {
      const int pr = fdiv(e, a.dncM);
      const int w = e - pr * a.nch_run * M;
      const int c = fdivc<LX>(w, a.dM);
      const int x = w - c * M;
      const long long row = r0 + pr;
      if (row >= a.R) continue;
      const double2 z = lines[(pr * np + (c >> 1)) * M + x];
      const double val = (c & 1) ? z.y : z.x;
      if (a.yplain) {
        a.Yout[(long long)c * a.N + row * M + x] = val;
      } else {
        const int d = a.ydst[c];
        a.Yout[(((long long)(d >> 1)) * a.N + row * M + x) * 2 + (d & 1)] = val;
      }
    }
    return;
  }

  const DictTable& D = a.dict;
  // stage-7 epilogue of adaptive steps only (fixed steps pass no partials buffer)
  const bool err = (a.io.mode == 1 && r.stage == 7 && a.io.err_part != nullptr);
  const int npts = P * M;
  // Each thread evaluates the dictionary at PPT points at once, so that the tables
  // (warp-uniform shared-memory reads, loop control, the power switch) are read once per
  // PPT points.  Points past the tile read a valid address and store nothing.  NF > 0: the
  // dense polynomial form (all monomials of the NF fields once per point, then one
  // multiply-add per monomial and field); NF = 0: the term list.
  auto points = [&](auto ppt, auto nf) {
    constexpr int PPT = decltype(ppt)::value, NF = decltype(nf)::value;
    for (int e0 = tid; e0 < npts; e0 += T * PPT) {
      int phoff[PPT], lnoff[PPT];
      long long gbase[PPT];
      bool live[PPT];
      double err2[PPT];
#pragma unroll
      for (int k = 0; k < PPT; ++k) {
        const int e = e0 + k * T;
        const int pr = fdivc<LX>(e, a.dM);
        const int x = e - pr * M;
        const long long row = r0 + pr;
        live[k] = e < npts && row < a.R;
        phoff[k] = live[k] ? pr * n * M + x : 0;
        lnoff[k] = live[k] ? pr * np * M + x : 0;
        gbase[k] = live[k] ? row * M + x : 0;
        err2[k] = 0.0;
      }
      double mono[PPT][NF > 0 ? Mono<(NF > 0 ? NF : 1)>::count : 1];
      if constexpr (NF > 0) {
        using MN = Mono<NF>;
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
          mono[k][0] = 1.0;
#pragma unroll
          for (int m = 1; m < MN::count; ++m) mono[k][m] = mono[k][MN::parent(m)] * phys[phoff[k] + MN::var(m) * M];
        }
      }
      for (int i = 0; i < n; ++i) {
        double acc[PPT];
        const int fc = sfold[i];
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
          acc[k] = 0.0;
          if (fc >= 0) {
            const double2 z = lines[lnoff[k] + (fc >> 1) * M];
            acc[k] = (fc & 1) ? z.y : z.x;
          }
        }
        if constexpr (NF > 0) {
          const double* ci = spoly + i * Mono<NF>::count;
#pragma unroll
          for (int m = 0; m < Mono<NF>::count; ++m) {
            const double c = ci[m];
#pragma unroll
            for (int k = 0; k < PPT; ++k) acc[k] += c * mono[k][m];
          }
        } else {
          for (int t = sfb[i]; t < sfb[i + 1]; ++t) {
            const DictTerm tm = sterm[t];
            double prod[PPT];
#pragma unroll
            for (int k = 0; k < PPT; ++k) prod[k] = 1.0;
            for (int q = 0; q < tm.nf; ++q) {
              const DictFactor fc2 = sfac[tm.off + q];
              if (fc2.q < n) {
#pragma unroll
                for (int k = 0; k < PPT; ++k) prod[k] *= ipow(phys[phoff[k] + fc2.q * M], fc2.eta);
              } else {
                const int c = fc2.q - n;
                const int co = (c >> 1) * M;
#pragma unroll
                for (int k = 0; k < PPT; ++k) {
                  const double2 z = lines[lnoff[k] + co];
                  prod[k] *= ipow((c & 1) ? z.y : z.x, fc2.eta);
                }
              }
            }
#pragma unroll
            for (int k = 0; k < PPT; ++k) acc[k] += tm.C * prod[k];
          }
        }
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
          if (!live[k]) continue;
          const long long gi = (long long)i * a.R * M + gbase[k];
          r.f[gi] = acc[k];
          if (err) {
            // error kernel of dp45.cu:79-84 (e_2 = 0 drops k2)
            const double ynew = phys[phoff[k] + i * M];
            const double yold = r.y[gi];
            const double es = c_e[0] * r.k[0][gi] + c_e[2] * r.k[2][gi] + c_e[3] * r.k[3][gi] +
                              c_e[4] * r.k[4][gi] + c_e[5] * r.k[5][gi] + c_e[6] * acc[k];
            const double ev = r.h * es / (r.atol + r.rtol * fmax(fabs(yold), fabs(ynew)));
            err2[k] += ev * ev;
          }
        }
      }
      if (err) {
        // a point's squared error replaces its own first field in the staging buffer (no
        // other thread reads that point)
#pragma unroll
        for (int k = 0; k < PPT; ++k)
          if (live[k]) phys[phoff[k]] = err2[k];
      }
    }
  };
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  switch (a.dict.poly_nf) {
    case 1: points(I2{}, I1{}); break;
    case 2: points(I2{}, I2{}); break;
    case 3: points(I1{}, std::integral_constant<int, 3>{}); break;
    default: points(std::integral_constant<int, 4>{}, std::integral_constant<int, 0>{}); break;
  }
  if (err) {
    // one partial sum per grid row, in an order fixed by the row alone (x = lane,
    // lane + 32, ..., then a butterfly over the lanes): the error norm does not depend
    // on how rows are tiled into CTAs or on the block size
    __syncthreads();
    const int lane = tid & 31, nw = T >> 5;
    for (int pr = tid >> 5; pr < P; pr += nw) {
      const long long row = r0 + pr;
      if (row >= a.R) break;
      double v = 0.0;
      for (int x = lane; x < M; x += 32) v += phys[pr * n * M + x];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) a.io.err_part[row] = v;
    }
  }
}

template <int RS, int LX>
__global__ void __launch_bounds__(LX > 0 ? kSpecBlock : kMaxBlock, LX > 0 ? 3 : 1) k_inv_x(InvXArgs a) {
  inv_x_body<RS, LX>(a, blockIdx.x);
}

// ---- x pass of 3D grids with 128- or 256-point rows and a dense-polynomial dictionary
// of at most two inverse channels (DP45 stages without the error epilogue, and plain
// RHS evaluations): one row per warp (two per warp for 128 points).  Each warp streams
// its rows through two staging slots in shared memory: while one row is transformed and
// evaluated, asynchronous copies (cp.async) bring the next row's channel half spectra
// and physical fields.  Per row: k_inv_x's Hermitian extension and two-channel packing
// from the staged spectra, the inverse transform in registers with its exchanges in the
// warp's line buffer (WarpLine), then the dictionary at the lane's points -- k_inv_x's
// arithmetic per point.  No block barriers after the table staging.
struct InvRowArgs {
  int R, n, nch, Mh;
  const double2* tw;
  const double2* Sc;
  DictTable dict;
  RhsIO io;
};
// Warps per CTA: ten for at most two fields (168 registers each; their staging fits),
// else eight; eight with the stage-7 error epilogue, which reads each row's slope sums
// and y straight into registers before the row's transform (255 registers).
__host__ __device__ constexpr int row_warps(bool err, int nf) { return err || nf > 2 ? 8 : 10; }
// one staging slot of a warp: 2 channels x (at most 129 + padding) spectral values and
// NF x 256 field values (two rows of 128 points take the same room)
constexpr int kRowSpec = 2 * 136;  // double2 per slot
__host__ __device__ constexpr int row_slot_doubles(int nf, bool) { return 2 * kRowSpec + nf * 256; }

__host__ __device__ constexpr size_t inv_row_smem(int n, int count, bool err) {
  return (size_t)row_warps(err, n) * (256 * 16 + 2 * (size_t)row_slot_doubles(n, err) * 8) + (size_t)n * count * 8 + 64;
}

template <int L, int NF, bool ERR>
__global__ void __launch_bounds__(row_warps(ERR, NF) * 32, 1) k_inv_row(InvRowArgs a) {
  extern __shared__ double2 sm[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;
  using MN = Mono<NF>;
  constexpr int kRowWarps = row_warps(ERR, NF), kRowThreads = kRowWarps * 32;
  constexpr int LPL = L / 8, RPW = 32 / LPL;  // lanes per row, rows per warp
  constexpr int SLOT = row_slot_doubles(NF, ERR);
  const Resolved r = resolve(a.io);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double* stage = reinterpret_cast<double*>(sm + kRowWarps * 256);
  double* spoly = stage + kRowWarps * 2 * SLOT;
  int* sfold = reinterpret_cast<int*>(spoly + NF * MN::count);
  for (int t = tid; t < NF * MN::count; t += kRowThreads) spoly[t] = a.dict.poly[t];
  for (int t = tid; t < NF; t += kRowThreads) sfold[t] = a.dict.fold[t];
  __syncthreads();
  const int sub = lane / LPL, ml = lane % LPL;
  double2* line = sm + warp * 256 + sub * L;
  WarpLine<L> wl;
  wl.init(a.tw, ml);
  const long long RL = (long long)a.R * L;
  // the row's spectra (both channels) and fields as 16-byte pieces, when aligned
  const bool a16 = ((reinterpret_cast<unsigned long long>(r.u) | reinterpret_cast<unsigned long long>(a.Sc)) & 15) == 0;
  const int Mh = a.Mh, nch = a.nch;
  const long long wstride = (long long)gridDim.x * kRowWarps * RPW;
  // slot k of this warp; the sub-row's part of it
  auto slot_spec = [&](int k) { return reinterpret_cast<double2*>(stage + (warp * 2 + k) * SLOT) + sub * (kRowSpec / RPW); };
  auto slot_u = [&](int k) { return stage + (warp * 2 + k) * SLOT + 2 * kRowSpec + sub * NF * L; };
  const long long nN = (long long)NF * RL;
  auto fetch = [&](long long row, int k) {
    if (row >= a.R) return;
    double2* sp = slot_spec(k);
    double* su = slot_u(k);
    if (a16) {
      for (int c = 0; c < nch; ++c)
        for (int e = ml; e < Mh; e += LPL) cp_async16(sp + c * Mh + e, a.Sc + ((long long)c * a.R + row) * Mh + e, true);
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int k2 = 0; k2 < L / 2 / LPL; ++k2) {
          const int x2 = 2 * (ml + LPL * k2);
          cp_async16(su + f * L + x2, r.u + f * RL + row * L + x2, true);
        }
    } else {
      for (int c = 0; c < nch; ++c)
        for (int e = ml; e < Mh; e += LPL) sp[c * Mh + e] = a.Sc[((long long)c * a.R + row) * Mh + e];
      for (int f = 0; f < NF; ++f)
        for (int k2 = 0; k2 < 8; ++k2) su[f * L + ml + LPL * k2] = r.u[f * RL + row * L + ml + LPL * k2];
    }
  };
  long long row0 = ((long long)blockIdx.x * kRowWarps + warp) * RPW;
  fetch(row0 + sub, 0);
  cp_async_commit();
  int k = 0;
  for (; row0 < a.R; row0 += wstride, k ^= 1) {
    const long long row = row0 + sub;
    const bool live = row < a.R;
    // the next row's copies go to the other slot (its last reads ended at the previous
    // row's final barrier)
    fetch(row0 + wstride + sub, k ^ 1);
    cp_async_commit();
    cp_async_wait_1();
    __syncwarp();  // this row's copies (every lane's) landed
    const double2* sp = slot_spec(k);
    const double* su = slot_u(k);
    // ERR: the row's slope sums and y at the lane's points, loaded before the transform
    // so that it covers their latency (y and the staged stage-7 state give the error
    // scale)
    double es_t[ERR ? 8 : 1][NF], y_t[ERR ? 8 : 1][NF];
    if (ERR && live) {
#pragma unroll
      for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int i = 0; i < NF; ++i) {
          const long long gi = i * RL + row * L + ml + LPL * p;
          es_t[ERR ? p : 0][i] = r.aux[gi];
          y_t[ERR ? p : 0][i] = r.y[gi];
        }
    }
    double2 v[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int kx = ml + LPL * p;
      const int kk = kx >= Mh ? L - kx : kx;
      double2 Av = make_double2(0.0, 0.0), Bv = make_double2(0.0, 0.0);
      if (live) {
        Av = sp[kk];
        if (nch > 1) Bv = sp[Mh + kk];
      }
      if (kx == 0 || 2 * kx == L) {
        Av.y = 0.0;
        Bv.y = 0.0;
      }
      if (kx >= Mh) {
        Av.y = -Av.y;
        Bv.y = -Bv.y;
      }
      v[p] = make_double2(Av.x - Bv.y, Av.y + Bv.x);
    }
    wl.template transform<true>(v, [line](int e) { return line + e; });
    // the lane's values back to its own line positions (the transform's last barrier has
    // passed), so the point loop holds no spectral registers
#pragma unroll
    for (int p = 0; p < 8; ++p) line[ml + LPL * p] = v[p];
    double es_even = 0.0, es_odd = 0.0;  // ERR, 128 points: the partials of lanes ml and ml + 16
    // (unrolled fully with the error epilogue: its terms stay in registers)
#pragma unroll(ERR ? 8 : 2)
    for (int p = 0; p < 8; ++p) {
      const int x = ml + LPL * p;
      const double2 z = line[x];
      double u[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) u[f] = su[f * L + x];
      double mono[MN::count];
      mono[0] = 1.0;
#pragma unroll
      for (int m = 1; m < MN::count; ++m) mono[m] = mono[MN::parent(m)] * u[MN::var(m)];
      double err2 = 0.0;
#pragma unroll
      for (int i = 0; i < NF; ++i) {
        const int fc = sfold[i];
        double acc = fc >= 0 ? ((fc & 1) ? z.y : z.x) : 0.0;
        const double* ci = spoly + i * MN::count;
#pragma unroll
        for (int m = 0; m < MN::count; ++m) acc += ci[m] * mono[m];
        if (live) r.f[i * RL + row * L + x] = acc;
        if (ERR) {
          // k_inv_x's error kernel (dp45.cu:79-84) from the forward pass's slope sum
          const double es = es_t[ERR ? p : 0][i] + c_e[6] * acc;
          const double ev = r.h * es / stage7_scale(r, y_t[ERR ? p : 0][i], su[i * L + x]);
          err2 += ev * ev;
        }
      }
      if (L == 256 || (p & 1) == 0)
        es_even += err2;
      else
        es_odd += err2;
    }
    if (ERR) {
      // one partial per row in k_inv_x's order: x = lane, lane + 32, ..., then the
      // butterfly over the lanes (for 128 points its first step pairs lanes ml, ml + 16)
      double sacc = es_even;
      if (L == 128) sacc = es_even + es_odd;
#pragma unroll
      for (int o = LPL / 2; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
      if (ml == 0 && live) a.io.err_part[row] = sacc;
    }
    __syncwarp();  // the next row's transform and the copies after it rewrite the line and this slot
  }
  cp_async_wait_all();
}

// ---- the inverse x pass of DP45 stage s fused with the forward x pass of stage s + 1
// (s = 2..5; 3D grids with 128- or 256-point rows, two fields, a dense-polynomial
// dictionary of at most two channels).  Per row, k_inv_row's steps (staged channel spectra
// and fields, inverse transform, dictionary, slope k_s written), then stage s + 1 at the
// lane's points: its state from y, the slopes before k_s (read while the inverse
// transform runs) and k_s still in registers -- the stage combination of dp45.cu:34-69
// with stage_value_t2's terms in its order --
// written out, then transformed forward as one complex line (field 0 real part, field 1
// imaginary part) and split into the two fields' half spectra with k_fwd_x's formulas.
// Against separate launches this saves reading k_s back and one launch per stage.
// k_fwd_x pairs two rows of one field in a line instead, so the spectra agree with its
// spectra to rounding; the stage states are the same arithmetic.  Stage 7's forward pass
// stays separate: with its error terms the fused kernel ran out of registers (spills;
// 256^3: 0.75 ms against 0.57 ms for the two kernels).
struct InvFwdRowArgs {
  InvRowArgs inv;  // stage s: channel spectra in, slope k_s out
  RhsIO io2;       // stage s + 1: its state out
  double2* Sf;     // stage s + 1's field half spectra [field][row][Mh]
};
constexpr int kFuseWarps = 8;
__host__ __device__ constexpr size_t inv_fwd_row_smem(int count) {
  return (size_t)kFuseWarps * (256 * 16 + 2 * (size_t)row_slot_doubles(2, false) * 8) + (size_t)2 * count * 8 + 64;
}

template <int L, int S2>
__global__ void __launch_bounds__(kFuseWarps * 32, 1) k_inv_fwd_row(const __grid_constant__ InvFwdRowArgs fa) {
  static_assert(S2 >= 3 && S2 <= 6, "the stage after an inverse pass of stages 2..5");
  extern __shared__ double2 sm[];
  const InvRowArgs& a = fa.inv;
  if (!a.io.ctl->running) return;
  constexpr int NF = 2;
  using MN = Mono<NF>;
  constexpr int LPL = L / 8, RPW = 32 / LPL;  // lanes per row, rows per warp
  constexpr int SLOT = row_slot_doubles(NF, false);
  constexpr int NEW = S2 - 2;  // slot of k_s among stage S2's slopes
  const Resolved r = resolve(a.io);
  const Resolved r2 = resolve(fa.io2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double* stage = reinterpret_cast<double*>(sm + kFuseWarps * 256);
  double* spoly = stage + kFuseWarps * 2 * SLOT;
  int* sfold = reinterpret_cast<int*>(spoly + NF * MN::count);
  for (int t = tid; t < NF * MN::count; t += kFuseWarps * 32) spoly[t] = a.dict.poly[t];
  for (int t = tid; t < NF; t += kFuseWarps * 32) sfold[t] = a.dict.fold[t];
  __syncthreads();
  const int sub = lane / LPL, ml = lane % LPL;
  double2* line = sm + warp * 256 + sub * L;
  WarpLine<L> wl;
  wl.init(a.tw, ml);
  const long long RL = (long long)a.R * L;
  const bool a16 = ((reinterpret_cast<unsigned long long>(r.u) | reinterpret_cast<unsigned long long>(a.Sc)) & 15) == 0;
  const int Mh = a.Mh, nch = a.nch;
  const long long wstride = (long long)gridDim.x * kFuseWarps * RPW;
  auto slot_spec = [&](int k) { return reinterpret_cast<double2*>(stage + (warp * 2 + k) * SLOT) + sub * (kRowSpec / RPW); };
  auto slot_u = [&](int k) { return stage + (warp * 2 + k) * SLOT + 2 * kRowSpec + sub * NF * L; };
  // the rows go from the last to the first (q counts them): the axis-1 pass after this
  // one starts on the first planes, which are then still in L2
  auto fetch = [&](long long q, int k) {
    if (q >= a.R) return;
    const long long row = a.R - 1 - q;
    double2* sp = slot_spec(k);
    double* su = slot_u(k);
    if (a16) {
      for (int c = 0; c < nch; ++c)
        for (int e = ml; e < Mh; e += LPL) cp_async16(sp + c * Mh + e, a.Sc + ((long long)c * a.R + row) * Mh + e, true);
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int k2 = 0; k2 < L / 2 / LPL; ++k2) {
          const int x2 = 2 * (ml + LPL * k2);
          cp_async16(su + f * L + x2, r.u + f * RL + row * L + x2, true);
        }
    } else {
      for (int c = 0; c < nch; ++c)
        for (int e = ml; e < Mh; e += LPL) sp[c * Mh + e] = a.Sc[((long long)c * a.R + row) * Mh + e];
      for (int f = 0; f < NF; ++f)
        for (int k2 = 0; k2 < 8; ++k2) su[f * L + ml + LPL * k2] = r.u[f * RL + row * L + ml + LPL * k2];
    }
  };
  long long row0 = ((long long)blockIdx.x * kFuseWarps + warp) * RPW;
  fetch(row0 + sub, 0);
  cp_async_commit();
  int k = 0;
  for (; row0 < a.R; row0 += wstride, k ^= 1) {
    const bool live = row0 + sub < a.R;
    const long long row = live ? a.R - 1 - (row0 + sub) : 0;
    fetch(row0 + wstride + sub, k ^ 1);
    cp_async_commit();
    // stage S2's sums over the slopes before k_s at the lane's points, issued before the
    // inverse transform so that it covers their latency
    double yv[8][NF], ax[8][NF];
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
      for (int i = 0; i < NF; ++i) {
        double yy = 0.0, s = 0.0;
        if (live) {
          const long long gi = i * RL + row * L + ml + LPL * p;
          yy = r2.y[gi];
          s = c_a[S2][0] * r2.k[0][gi];
          if (S2 >= 4) s += c_a[S2][1] * r2.k[1][gi];
#pragma unroll
          for (int j = 2; j < NEW; ++j) s += c_a[S2][j] * r2.k[j][gi];
        }
        yv[p][i] = yy;
        ax[p][i] = s;
      }
    cp_async_wait_1();
    __syncwarp();  // this row's copies (every lane's) landed
    const double2* sp = slot_spec(k);
    const double* su = slot_u(k);
    double2 v[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int kx = ml + LPL * p;
      const int kk = kx >= Mh ? L - kx : kx;
      double2 Av = make_double2(0.0, 0.0), Bv = make_double2(0.0, 0.0);
      if (live) {
        Av = sp[kk];
        if (nch > 1) Bv = sp[Mh + kk];
      }
      if (kx == 0 || 2 * kx == L) {
        Av.y = 0.0;
        Bv.y = 0.0;
      }
      if (kx >= Mh) {
        Av.y = -Av.y;
        Bv.y = -Bv.y;
      }
      v[p] = make_double2(Av.x - Bv.y, Av.y + Bv.x);
    }
    wl.template transform<true>(v, [line](int e) { return line + e; });
#pragma unroll
    for (int p = 0; p < 8; ++p) line[ml + LPL * p] = v[p];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int x = ml + LPL * p;
      const double2 z = line[x];
      double u[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) u[f] = su[f * L + x];
      double mono[MN::count];
      mono[0] = 1.0;
#pragma unroll
      for (int m = 1; m < MN::count; ++m) mono[m] = mono[MN::parent(m)] * u[MN::var(m)];
#pragma unroll
      for (int i = 0; i < NF; ++i) {
        const int fc = sfold[i];
        double acc = fc >= 0 ? ((fc & 1) ? z.y : z.x) : 0.0;
        const double* ci = spoly + i * MN::count;
#pragma unroll
        for (int m = 0; m < MN::count; ++m) acc += ci[m] * mono[m];
        const long long gi = i * RL + row * L + x;
        // stage S2 at this point: k_s is its last slope term
        double s = ax[p][i];
        s += c_a[S2][NEW] * acc;
        const double yn = yv[p][i] + r2.h * s;
        if (live) {
          r.f[gi] = acc;
          if (r2.ytemp) r2.ytemp[gi] = yn;
        }
        yv[p][i] = yn;
      }
    }
    __syncwarp();  // every lane's reads of the line are done before the forward transform
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = make_double2(yv[p][0], yv[p][1]);
    wl.template transform<false>(v, [line](int e) { return line + e; });
#pragma unroll
    for (int p = 0; p < 8; ++p) line[ml + LPL * p] = v[p];
    __syncwarp();
    if (live) {
#pragma unroll
      for (int p = 0; p < (L / 2 + LPL) / LPL; ++p) {
        const int kx = ml + LPL * p;
        if (kx < Mh) {
          const double2 z = line[kx];
          const double2 zm = line[kx == 0 ? 0 : L - kx];
          fa.Sf[row * Mh + kx] = make_double2(0.5 * (z.x + zm.x), 0.5 * (z.y - zm.y));
          fa.Sf[((long long)a.R + row) * Mh + kx] = make_double2(0.5 * (z.y + zm.y), -0.5 * (z.x - zm.x));
        }
      }
    }
    __syncwarp();  // the next row's transform and the copies after it rewrite the line and this slot
  }
  cp_async_wait_all();
}

// ---- 3D x passes that also transform along axis 1, one thread-block cluster per plane
// (an alternative to the axis-1 passes on TMA tiles, enabled by SpectralPlan::setup_planes
// on request).  For 3D grids whose x rows and axis-1 lines have 128 or 256 points, the
// forward x pass also does the forward axis-1 transform and the inverse x pass the
// inverse one, so the
// spectra of a stage cross HBM once each way between the x and axis-0 passes (the axis-1
// passes on TMA tiles read and write them once more each).  A cluster of C = N1/32 CTAs
// takes one axis-0 plane at a time (with one field, in the forward pass); CTA r of the
// cluster holds the 32 rows y = r + C q (q < 32) of the plane.  The axis-1 DFT of length
// N1 = 32 C splits as
//     X[a + 32 b] = sum_r W_C^(r b) W_N1^(r a) sum_q W_32^(q a) x[r + C q]   (a < 32, b < C):
// each CTA transforms its own rows over q -- a 32-point DFT per x wavenumber, as 8-point
// DFTs over q2, the twiddles W_32^(q1 k2), then 4-point DFTs over q1 (q = q1 + 4 q2,
// a = k2 + 8 k1) -- and applies W_N1^(r a); after a cluster barrier CTA j reads the
// values of its a-range (a = j 32/C + i) from every CTA of the cluster through
// distributed shared memory and finishes the C-point DFTs over r, writing the spectra
// in the layout the axis-0 pass reads.  The inverse pass takes the same steps backwards.
// The x transforms are the warp-per-line transforms of the row kernels (WarpLine),
// bitwise those of the other x passes; the axis-1 transform uses the line kernels'
// twiddle table in another factorisation, so it agrees with the tiled axis-1 pass to
// rounding.  Control flow is uniform over a cluster: every CTA takes the same planes and
// passes the same cluster barriers, and none leaves while another may read its shared
// memory.

__device__ __forceinline__ unsigned cl_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cl_id() {
  unsigned r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cl_count() {
  unsigned r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
// every thread of every CTA of the cluster arrives (release) and waits (acquire)
__device__ __forceinline__ void cl_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// the shared-memory address of p in CTA `rank` of the cluster
__device__ __forceinline__ unsigned cl_map(const void* p, unsigned rank) {
  unsigned d;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(d) : "r"(smem_u32(p)), "r"(rank));
  return d;
}
__device__ __forceinline__ double2 cl_load(unsigned addr) {
  double2 v;
  asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr) : "memory");
  return v;
}

struct PlaneArgs {
  int N0, n, nch;       // axis-0 planes, fields, inverse channels
  const double2* twx;   // x twiddles (LX-point table)
  const double2* twy;   // axis-1 twiddles (N1-point table)
  double2* S;           // forward: field half spectra [field][z][ky][kx] (written)
  const double2* Sc;    // inverse: channel half spectra [channel][z][ky][kx] (read)
  DictTable dict;
  RhsIO io;
};

constexpr int kPlaneFwdThreads = 512;
constexpr int kPlaneInvThreads = 256;
// forward: 16 complex lines of LX points, then 32 half-spectrum rows
__host__ __device__ constexpr size_t plane_fwd_smem(int LX) { return (size_t)(16 * LX + 32 * (LX / 2 + 1)) * 16; }
// inverse: the exchange block (32 half rows, later the warps' line buffers), two
// channels' 32 half rows, the dictionary's polynomial and fold tables
__host__ __device__ constexpr size_t plane_inv_smem(int LX, int nf, int count) {
  return (size_t)(3 * 32 * (LX / 2 + 1)) * 16 + (size_t)nf * count * 8 + 64;
}

// Stage values of the CTA's 32 rows of one (plane, field): row q of the CTA is global
// row grow0 + C q; rows 2l and 2l + 1 become the real and imaginary parts of line l.
// The stage state (and stage 7's slope sums) leave as fwd_load2 writes them.
template <int S, int LX, int C>
__device__ __forceinline__ void plane_load(const Resolved& r, double2* lines, long long grow0) {
  constexpr int kUnroll = 4, H = LX / 2, NP = 32 * H;
  static_assert(NP % (kPlaneFwdThreads * kUnroll) == 0, "whole unrolled rounds");
  const bool terms = S == 7 && r.aux != nullptr;
  for (int e0 = threadIdx.x; e0 < NP; e0 += kPlaneFwdThreads * kUnroll) {
    double2 v[kUnroll];
    long long gi[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int e = e0 + u * kPlaneFwdThreads;
      const int q = e / H, x = 2 * (e - q * H);
      gi[u] = (grow0 + (long long)C * q) * LX + x;
      if (terms) {
        double2 es_p;
        v[u] = stage7_value_terms2(gi[u], r, &es_p);
        *reinterpret_cast<double2*>(r.aux + gi[u]) = es_p;
      } else {
        v[u] = stage_value_t2<S>(gi[u], r);
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int e = e0 + u * kPlaneFwdThreads;
      const int q = e / H, x = 2 * (e - q * H);
      if (r.ytemp) *reinterpret_cast<double2*>(r.ytemp + gi[u]) = v[u];
      double* b = reinterpret_cast<double*>(lines) + 2 * ((q >> 1) * LX + x) + (q & 1);
      b[0] = v[u].x;
      b[2] = v[u].y;
    }
  }
}

template <int LX, int C>
__global__ void __launch_bounds__(kPlaneFwdThreads, 1) k_fwd_plane(PlaneArgs a) {
  extern __shared__ double2 smp[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;  // the same for every CTA
  constexpr int Mh = LX / 2 + 1, N1 = 32 * C, LPL = LX / 8, AC = 32 / C, T = kPlaneFwdThreads;
  double2* lines = smp;          // 16 lines of LX points
  double2* rows = smp + 16 * LX;  // 32 half rows of Mh points; the axis-1 stages in place
  Resolved r = resolve(a.io);
  r.nN = (long long)a.n * a.N0 * N1 * LX;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned rank = cl_rank();
  const int li = warp * (32 / LPL) + lane / LPL;  // the warp's line (two per warp for 128 points)
  WarpLine<LX> wl;
  wl.init(a.twx, lane % LPL);
  const int nitems = a.N0 * a.n;
  for (int it = (int)cl_id(); it < nitems; it += (int)cl_count()) {
    const int f = it / a.N0, z = it - f * a.N0;
    const long long grow0 = ((long long)f * a.N0 + z) * N1 + rank;
    switch (r.stage) {
      case 2: plane_load<2, LX, C>(r, lines, grow0); break;
      case 3: plane_load<3, LX, C>(r, lines, grow0); break;
      case 4: plane_load<4, LX, C>(r, lines, grow0); break;
      case 5: plane_load<5, LX, C>(r, lines, grow0); break;
      case 6: plane_load<6, LX, C>(r, lines, grow0); break;
      case 7: plane_load<7, LX, C>(r, lines, grow0); break;
      default: plane_load<1, LX, C>(r, lines, grow0); break;
    }
    __syncthreads();
    if (li < 16) {
      double2* line = lines + li * LX;
      double2 v[8];
#pragma unroll
      for (int p = 0; p < 8; ++p) v[p] = line[wl.ml + LPL * p];
      __syncwarp();
      wl.template transform<false>(v, [line](int e) { return line + e; });
#pragma unroll
      for (int p = 0; p < 8; ++p) line[wl.ml + LPL * p] = v[p];
    }
    // the cluster has read the previous item's rows; this CTA's lines are complete
    cl_sync();
    // the two real rows of each line (fwd_x_body's separation)
    for (int i = tid; i < 16 * Mh; i += T) {
      const int l = i / Mh, kx = i - l * Mh;
      const double2 zz = lines[l * LX + kx];
      const double2 zm = lines[l * LX + (kx == 0 ? 0 : LX - kx)];
      rows[(2 * l) * Mh + kx] = make_double2(0.5 * (zz.x + zm.x), 0.5 * (zz.y - zm.y));
      rows[(2 * l + 1) * Mh + kx] = make_double2(0.5 * (zz.y + zm.y), -0.5 * (zz.x - zm.x));
    }
    __syncthreads();
    // 8-point DFTs over q2, times W_32^(q1 k2), back to rows q1 + 4 k2
    for (int i = tid; i < 4 * Mh; i += T) {
      const int q1 = i / Mh, kx = i - q1 * Mh;
      double2 v[8];
#pragma unroll
      for (int q2 = 0; q2 < 8; ++q2) v[q2] = rows[(q1 + 4 * q2) * Mh + kx];
      Dft<8, false>::run(v, nullptr, 0);
      if (q1 > 0) {
#pragma unroll
        for (int k2 = 1; k2 < 8; ++k2) v[k2] = c_mul(v[k2], a.twy[C * q1 * k2]);
      }
#pragma unroll
      for (int k2 = 0; k2 < 8; ++k2) rows[(q1 + 4 * k2) * Mh + kx] = v[k2];
    }
    __syncthreads();
    // 4-point DFTs over q1: Y[k2 + 8 k1] times W_N1^(r a), at row 4 k2 + k1
    for (int i = tid; i < 8 * Mh; i += T) {
      const int k2 = i / Mh, kx = i - k2 * Mh;
      double2 w[4];
#pragma unroll
      for (int q1 = 0; q1 < 4; ++q1) w[q1] = rows[(q1 + 4 * k2) * Mh + kx];
      Dft<4, false>::run(w, nullptr, 0);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) {
        const int t = (int)rank * (k2 + 8 * k1);
        rows[(4 * k2 + k1) * Mh + kx] = t ? c_mul(w[k1], a.twy[t]) : w[k1];
      }
    }
    cl_sync();  // every CTA's values are visible to the cluster
    // C-point DFTs over r for this CTA's a-range, to the spectra
    for (int i = tid; i < AC * Mh; i += T) {
      const int al = i / Mh, kx = i - al * Mh;
      const int aa = (int)rank * AC + al;
      const double2* src = rows + (4 * (aa & 7) + (aa >> 3)) * Mh + kx;
      double2 v[C];
#pragma unroll
      for (int rr = 0; rr < C; ++rr) v[rr] = cl_load(cl_map(src, rr));
      Dft<C, false>::run(v, nullptr, 0);
      double2* dst = a.S + (((long long)f * a.N0 + z) * N1 + aa) * Mh + kx;
#pragma unroll
      for (int b = 0; b < C; ++b) dst[(long long)32 * b * Mh] = v[b];
    }
  }
  cl_sync();
}

template <int LX, int C, int NF, bool ERR>
__global__ void __launch_bounds__(kPlaneInvThreads, 1) k_inv_plane(PlaneArgs a) {
  extern __shared__ double2 smp[];
  if (a.io.mode == 1 && !a.io.ctl->running) return;  // the same for every CTA
  using MN = Mono<NF>;
  constexpr int Mh = LX / 2 + 1, N1 = 32 * C, LPL = LX / 8, RPW = 32 / LPL, AC = 32 / C, T = kPlaneInvThreads;
  constexpr int NW = T / 32;
  double2* zo = smp;              // [r][al] blocks of Mh values; later the warps' line buffers
  double2* rows = smp + 32 * Mh;  // two channels' 32 half rows
  double* spoly = reinterpret_cast<double*>(rows + 2 * 32 * Mh);
  int* sfold = reinterpret_cast<int*>(spoly + NF * MN::count);
  const Resolved r = resolve(a.io);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int t = tid; t < NF * MN::count; t += T) spoly[t] = a.dict.poly[t];
  for (int t = tid; t < NF; t += T) sfold[t] = a.dict.fold[t];
  const unsigned rank = cl_rank();
  const int sub = lane / LPL, ml = lane % LPL;
  WarpLine<LX> wl;
  wl.init(a.twx, ml);
  const long long RL = (long long)a.N0 * N1 * LX, nN = (long long)NF * RL;
  const int nch = a.nch;
  for (int z = (int)cl_id(); z < a.N0; z += (int)cl_count()) {
    for (int c = 0; c < nch; ++c) {
      // the cluster has read zo (previous channel); this CTA's line buffers are free
      cl_sync();
      // C-point inverse DFTs over b of this CTA's a-range, times conj W_N1^(r a), to zo[r][al]
      for (int i = tid; i < AC * Mh; i += T) {
        const int al = i / Mh, kx = i - al * Mh;
        const int aa = (int)rank * AC + al;
        const double2* src = a.Sc + (((long long)c * a.N0 + z) * N1 + aa) * Mh + kx;
        double2 v[C];
#pragma unroll
        for (int b = 0; b < C; ++b) v[b] = src[(long long)32 * b * Mh];
        Dft<C, true>::run(v, nullptr, 0);
#pragma unroll
        for (int rr = 0; rr < C; ++rr) {
          const int t = rr * aa;
          zo[(rr * AC + al) * Mh + kx] = t ? c_mul(v[rr], tw_get<true>(a.twy, t)) : v[rr];
        }
      }
      cl_sync();  // every CTA's values are visible to the cluster
      double2* rc = rows + c * 32 * Mh;
      // 4-point inverse DFTs over k1 (a = k2 + 8 k1) of this CTA's values, times
      // conj W_32^(k2 q1), at rows q1 + 4 k2
      for (int i = tid; i < 8 * Mh; i += T) {
        const int k2 = i / Mh, kx = i - k2 * Mh;
        double2 w[4];
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
          const int aa = k2 + 8 * k1;
          w[k1] = cl_load(cl_map(zo + ((int)rank * AC + aa % AC) * Mh + kx, aa / AC));
        }
        Dft<4, true>::run(w, nullptr, 0);
#pragma unroll
        for (int q1 = 0; q1 < 4; ++q1) {
          const int t = C * k2 * q1;
          rc[(q1 + 4 * k2) * Mh + kx] = t ? c_mul(w[q1], tw_get<true>(a.twy, t)) : w[q1];
        }
      }
      __syncthreads();
      // 8-point inverse DFTs over k2: row q1 + 4 q2
      for (int i = tid; i < 4 * Mh; i += T) {
        const int q1 = i / Mh, kx = i - q1 * Mh;
        double2 v[8];
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) v[k2] = rc[(q1 + 4 * k2) * Mh + kx];
        Dft<8, true>::run(v, nullptr, 0);
#pragma unroll
        for (int q2 = 0; q2 < 8; ++q2) rc[(q1 + 4 * q2) * Mh + kx] = v[q2];
      }
    }
    cl_sync();  // the cluster has read zo: it becomes the line buffers; every channel's rows are complete
    // k_inv_row's per-row work on this CTA's rows
    for (int q0 = warp * RPW; q0 < 32; q0 += NW * RPW) {
      const int q = q0 + sub;
      const long long row = (long long)z * N1 + rank + (long long)C * q;
      double2* line = zo + (warp * RPW + sub) * LX;
      double uu[8][NF];
#pragma unroll
      for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int f = 0; f < NF; ++f) uu[p][f] = r.u[f * RL + row * LX + ml + LPL * p];
      const double2* sa = rows + q * Mh;
      const double2* sb = rows + 32 * Mh + q * Mh;
      double2 v[8];
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int kx = ml + LPL * p;
        const int kk = kx >= Mh ? LX - kx : kx;
        double2 Av = sa[kk], Bv = nch > 1 ? sb[kk] : make_double2(0.0, 0.0);
        if (kx == 0 || 2 * kx == LX) {
          Av.y = 0.0;
          Bv.y = 0.0;
        }
        if (kx >= Mh) {
          Av.y = -Av.y;
          Bv.y = -Bv.y;
        }
        v[p] = make_double2(Av.x - Bv.y, Av.y + Bv.x);
      }
      wl.template transform<true>(v, [line](int e) { return line + e; });
      double es_even = 0.0, es_odd = 0.0;
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int x = ml + LPL * p;
        const double2 zz = v[p];
        double mono[MN::count];
        mono[0] = 1.0;
#pragma unroll
        for (int m = 1; m < MN::count; ++m) mono[m] = mono[MN::parent(m)] * uu[p][MN::var(m)];
        double err2 = 0.0;
#pragma unroll
        for (int i = 0; i < NF; ++i) {
          const int fc = sfold[i];
          double acc = fc >= 0 ? ((fc & 1) ? zz.y : zz.x) : 0.0;
          const double* ci = spoly + i * MN::count;
#pragma unroll
          for (int m = 0; m < MN::count; ++m) acc += ci[m] * mono[m];
          const long long gi = i * RL + row * LX + x;
          r.f[gi] = acc;
          if (ERR) {
            // k_inv_x's error kernel (dp45.cu:79-84) from the forward pass's slope sum
            const double es = r.aux[gi] + c_e[6] * acc;
            const double ev = r.h * es / stage7_scale(r, r.y[gi], uu[p][i]);
            err2 += ev * ev;
          }
        }
        if (LX == 256 || (p & 1) == 0)
          es_even += err2;
        else
          es_odd += err2;
      }
      if (ERR) {
        // one partial per row in k_inv_x's order (k_inv_row's butterfly)
        double sacc = es_even;
        if (LX == 128) sacc = es_even + es_odd;
#pragma unroll
        for (int o = LPL / 2; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
        if (ml == 0) a.io.err_part[row] = sacc;
      }
      __syncwarp();  // the next row's transform rewrites the line
    }
  }
  cl_sync();
}

// ---- batched passes: persistent CTAs over (problem, tile) work items
template <typename A>
__device__ __forceinline__ void load_args(A* dst, const A* src) {
  static_assert(sizeof(A) % 8 == 0, "argument blocks are copied as 8-byte words");
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int w = threadIdx.x; w < (int)(sizeof(A) / 8); w += blockDim.x) d[w] = s[w];
}

// Batched passes: persistent CTAs over (problem, tile) work items whose problems share one
// line length, with that length's specialised body inlined (LX = 0: the plan's stages) and
// the launch bounds of the single-problem kernels.  The groups of one pass run as
// concurrent branches (SpectralBatch::launch_stage).
template <int RS, int LX>
__global__ void __launch_bounds__(LX > 0 ? kSpecBlock : kMaxBlock, LX > 0 ? 2 : 1)
    k_fwd_x_group(const FwdXArgs* __restrict__ args, const int2* __restrict__ items, int nitems) {
  __shared__ __align__(16) FwdXArgs sa;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    load_args(&sa, args + w.x);
    __syncthreads();
    fwd_x_body<RS, LX>(sa, w.y);
    __syncthreads();
  }
}

template <int RS, int LX>
__global__ void __launch_bounds__(LX > 0 ? kSpecBlock : kMaxBlock, LX > 0 ? 3 : 1)
    k_mid_group(const MidArgs* __restrict__ args, const int2* __restrict__ items, int nitems) {
  __shared__ __align__(16) MidArgs sa;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    load_args(&sa, args + w.x);
    __syncthreads();
    mid_body<RS, LX>(sa, w.y);
    __syncthreads();
  }
}

template <int RS, int LX>
__global__ void __launch_bounds__(LX > 0 ? kSpecBlock : kMaxBlock, LX > 0 ? 3 : 1)
    k_inv_x_group(const InvXArgs* __restrict__ args, const int2* __restrict__ items, int nitems) {
  __shared__ __align__(16) InvXArgs sa;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    load_args(&sa, args + w.x);
    __syncthreads();
    inv_x_body<RS, LX>(sa, w.y);
    __syncthreads();
  }
}

// Kernel of pass k (0 fwd_x, 1 mid, 2 inv_x) for a group of line length L: the
// specialised lengths, else the plan's stages with radix set rs.
template <int RS, int LX>
const void* group_kernel(int k) {
  if (k == 0) return (const void*)k_fwd_x_group<RS, LX>;
  if (k == 1) return (const void*)k_mid_group<RS, LX>;
  return (const void*)k_inv_x_group<RS, LX>;
}
const void* group_kernel_for(int k, int L, int rs) {
  switch (L) {
    case 64: return group_kernel<kRadixPow2, 64>(k);
    case 128: return group_kernel<kRadixPow2, 128>(k);
    case 256: return group_kernel<kRadixPow2, 256>(k);
    case 512: return group_kernel<kRadixPow2, 512>(k);
    case 96: return group_kernel<kRadixAll, 96>(k);
    case 192: return group_kernel<kRadixAll, 192>(k);
    default: return rs == kRadixPow2 ? group_kernel<kRadixPow2, 0>(k) : group_kernel<kRadixAll, 0>(k);
  }
}
bool length_specialised(int L) { return L == 64 || L == 96 || L == 128 || L == 192 || L == 256 || L == 512; }

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Invariant divisors of each pass's index arithmetic, filled before every launch.
void prep(FwdXArgs& a) {
  a.d2M = make_fastdiv(2 * a.M);
  a.dM = make_fastdiv(a.M);
  a.d2Mh = make_fastdiv(2 * a.Mh);
  a.dMh = make_fastdiv(a.Mh);
}
void prep(C2CArgs& a) { a.dTW = make_fastdiv(a.TW); }
void prep(MidArgs& a) {
  a.dTW = make_fastdiv(a.TW);
  a.dL0 = make_fastdiv(a.L0);
  a.dMh = make_fastdiv(a.Mh > 0 ? a.Mh : 1);
}
void prep(MidSolveArgs& a) {
  a.dTW = make_fastdiv(a.TW);
  a.dL0 = make_fastdiv(a.L0);
  a.dMh = make_fastdiv(a.Mh > 0 ? a.Mh : 1);
}
void prep(InvXArgs& a) {
  const int half = a.M / 2;
  a.dM = make_fastdiv(a.M);
  a.dnpM = make_fastdiv(std::max(1, a.npairs) * a.M);
  a.dnhalf = make_fastdiv(std::max(1, a.n * half));
  a.dhalf = make_fastdiv(std::max(1, half));
  a.dnM = make_fastdiv(a.n * a.M);
  a.dncM = make_fastdiv(std::max(1, a.nch_run) * a.M);
}

// at most kMaxElems complex values per FFT pass CTA: kMaxBlock threads x kStageElems
constexpr int kMaxElems = kMaxBlock * kStageElems;

// Complex values a pass CTA aims to transform: 1024 (128 threads at 128 registers, four
// or more CTAs per SM so one CTA's loads overlap another's FFT stages).  A longer line
// takes one line per CTA.  RDCU_CTA_ELEMS overrides it (tuning experiments).
static int cta_elems() {
  static int v = [] {
    const char* e = getenv("RDCU_CTA_ELEMS");
    int x = e ? atoi(e) : 1024;
    if (x < 256) x = 256;
    if (x > kMaxElems) x = kMaxElems;
    return x;
  }();
  return v;
}

int block_for(const LinePlan& p, int elems);
int stage_threads(const LinePlan& p, int elems) {
  // each thread stages at most QMAX*R values per stage (see stockham_stage)
  int worst = kStageElems;
  for (int s = 0; s < p.nstages; ++s) {
    const int R = p.radix[s];
    const int per = (R >= kStageElems) ? R : (kStageElems / R) * R;
    worst = std::min(worst, per);
  }
  return (elems + worst - 1) / worst;
}

constexpr size_t kSmemBudget = 200 * 1024;
constexpr int kTargetCtas = 2 * 148;

}  // namespace

#define RDCU_TRY(x)                        \
  do {                                     \
    cudaError_t _e = (x);                  \
    if (_e != cudaSuccess) return _e;      \
  } while (0)

// Allows a kernel the largest dynamic shared memory the device grants next to its
// static shared memory.
static bool opt_in_smem(const void* func) {
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, func) != cudaSuccess) return false;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
  const int dyn = optin - (int)fa.sharedSizeBytes;
  return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) == cudaSuccess;
}

// Geometry of the inverse x pass for nch_run channels (with or without the
// physical-field staging): rows per CTA, grid, block and dynamic shared memory.
static void inv_geometry(int M, int R, int n, int nch_run, bool yout, const LinePlan& plan, PassCfg* c,
                         int* tw_smem, size_t extra = 0, int batch_elems = 0) {
  const bool spectral = nch_run > 0;
  const int np = (nch_run + 1) / 2;
  const int npm = std::max(1, np);
  // a single problem spreads its rows over the GPU; a batch member only sizes its tiles
  int P = batch_elems > 0 ? std::max(1, std::min(batch_elems / (M * npm), R))
                          : std::max(1, std::min(std::max(1, cta_elems() / (M * npm)), R / kTargetCtas));
  auto block_of = [&](int p) { return std::min(kMaxBlock, std::max(128, round_up(stage_threads(plan, p * npm * M), 32))); };
  auto bytes = [&](int p, bool tws) {
    return (size_t)((spectral && tws ? M : 0) + (spectral ? p * np * M : 0)) * 16 +
           (yout ? 0 : (size_t)p * n * M * 8 + extra);
  };
  while (P > 1 && bytes(P, true) > kSmemBudget) P /= 2;
  const bool tws = bytes(P, true) <= kSmemBudget;
  c->per_cta = P;
  c->grid = (R + P - 1) / P;
  c->block = block_of(P);
  c->smem = bytes(P, tws);
  *tw_smem = tws ? 1 : 0;
}

// Calls f(radix set, line length) with compile-time values for the plan's lengths:
// lines of 64..512 points (powers of two, and 96 and 192) get kernels specialised to
// their length, other power-of-two lines the shift-indexed kernels, every other length
// the general ones.
template <typename F>
static void by_length(const LinePlan& p, int block, F&& f) {
  using RP = std::integral_constant<int, kRadixPow2>;
  using RA = std::integral_constant<int, kRadixAll>;
  switch (block <= kSpecBlock ? p.L : 0) {
    case 64: f(RP{}, std::integral_constant<int, 64>{}); return;
    case 128: f(RP{}, std::integral_constant<int, 128>{}); return;
    case 256: f(RP{}, std::integral_constant<int, 256>{}); return;
    case 512: f(RP{}, std::integral_constant<int, 512>{}); return;
    case 96: f(RA{}, std::integral_constant<int, 96>{}); return;
    case 192: f(RA{}, std::integral_constant<int, 192>{}); return;
    default: break;
  }
  if (plan_is_pow2(p))
    f(RP{}, std::integral_constant<int, 0>{});
  else
    f(RA{}, std::integral_constant<int, 0>{});
}

// k_fwd_x on the plan's x lines: a kernel per stage (1..7; the stage of a DP45 launch, 1
// for a plain evaluation) for 128- and 256-point rows, the runtime-stage kernel
// otherwise.
static void launch_fwd_x(const LinePlan& plan, int block, int grid, size_t smem, cudaStream_t st,
                         const FwdXArgs& a) {
  const int stage = a.io.mode == 1 ? std::max(1, a.io.stage) : 1;
  by_length(plan, block, [&](auto rs, auto lx) {
    constexpr int RS = decltype(rs)::value, LX = decltype(lx)::value;
    if constexpr (LX == 128 || LX == 256) {
      switch (stage) {
        case 2: k_fwd_x<RS, LX, 2><<<grid, block, smem, st>>>(a); break;
        case 3: k_fwd_x<RS, LX, 3><<<grid, block, smem, st>>>(a); break;
        case 4: k_fwd_x<RS, LX, 4><<<grid, block, smem, st>>>(a); break;
        case 5: k_fwd_x<RS, LX, 5><<<grid, block, smem, st>>>(a); break;
        case 6: k_fwd_x<RS, LX, 6><<<grid, block, smem, st>>>(a); break;
        case 7: k_fwd_x<RS, LX, 7><<<grid, block, smem, st>>>(a); break;
        default: k_fwd_x<RS, LX, 1><<<grid, block, smem, st>>>(a); break;
      }
    } else {
      k_fwd_x<RS, LX><<<grid, block, smem, st>>>(a);
    }
  });
}

// ----------------------------------------------------------------------------- plan
ChanTable SpectralPlan::chan_table(const int* off, const ChanEntry* ent, int nchan) const {
  ChanTable t{};
  t.nch = nchan;
  t.off = off;
  t.ent = ent;
  t.kv = kv_;
  for (int a = 0; a < 3; ++a) {
    t.kv_off[a] = kv_off_[a];
    t.Ns[a] = Ns[a];
  }
  t.ndim = ndim;
  t.kv_total = kv_total_;
  return t;
}

size_t SpectralPlan::dict_smem_bytes() const {
  const size_t b = (size_t)(poly_nf_ ? n * poly_count_ : 0) * sizeof(double) + (size_t)nterms_dict_ * sizeof(DictTerm) +
                   (size_t)nfac_dict_ * sizeof(DictFactor) + (size_t)(2 * n + 1) * sizeof(int);
  return (b + 15) / 16 * 16;
}

std::vector<double> SpectralPlan::poly_table() const {
  std::vector<double> A((size_t)n * poly_count_, 0.0);
  for (size_t t = 0; t < h_dterms_.size(); ++t) A[(size_t)h_dterms_[t].field * poly_count_ + h_poly_mono_[t]] += h_dterms_[t].C;
  return A;
}

// Exponent vectors (up to 3 variables) of the Mono<nf> monomials.
static std::vector<std::array<int, 3>> mono_exponents(int nf) {
  std::vector<std::array<int, 3>> ex;
  auto build = [&](auto mn) {
    using MN = decltype(mn);
    ex.assign(MN::count, {0, 0, 0});
    for (int m = 1; m < MN::count; ++m) {
      ex[m] = ex[MN::parent(m)];
      ex[m][MN::var(m)] += 1;
    }
  };
  if (nf == 1) build(Mono<1>{});
  if (nf == 2) build(Mono<2>{});
  if (nf == 3) build(Mono<3>{});
  return ex;
}

DictTable SpectralPlan::dict_table() const {
  DictTable d{};
  d.n = n;
  d.nterms = nterms_dict_;
  d.terms = d_terms_;
  d.fac = d_fac_;
  d.field_begin = d_field_begin_;
  d.fold = d_fold_;
  d.nfac = nfac_dict_;
  d.poly = d_poly_;
  d.poly_nf = poly_nf_;
  d.poly_count = poly_count_;
  return d;
}

template <typename T>
static cudaError_t upload(T** dst, const std::vector<T>& v, size_t* bytes) {
  const size_t b = std::max<size_t>(1, v.size()) * sizeof(T);
  cudaError_t e = cudaMalloc((void**)dst, b);
  if (e != cudaSuccess) return e;
  *bytes += b;
  if (!v.empty()) e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

// Channel entries in operator order with the local channel index in .pad (the k_mid
// fast path computes each distinct multiplier once per point).
static std::vector<ChanEntry> sorted_entries(const std::vector<ChanEntry>& ent, const std::vector<int>& off, int nch) {
  std::vector<ChanEntry> srt;
  for (int c = 0; c < nch; ++c)
    for (int q = off[c]; q < off[c + 1]; ++q) {
      ChanEntry e = ent[q];
      e.pad = c;
      srt.push_back(e);
    }
  std::stable_sort(srt.begin(), srt.end(), [](const ChanEntry& x, const ChanEntry& y) {
    const int kx = x.nax | (x.ax0 << 2) | (x.ax1 << 4) | (x.part << 6);
    const int ky = y.nax | (y.ax0 << 2) | (y.ax1 << 4) | (y.part << 6);
    return kx < ky;
  });
  return srt;
}

// Operator groups of the operator-sorted hot entries, as k_mid forms them in each CTA:
// one group per distinct operator (its first entry), and A[g][channel * 4 + source] the
// sum of the group's coefficients in entry order.
static void operator_groups(const std::vector<ChanEntry>& srt, std::vector<ChanEntry>* grp, std::vector<double>* A) {
  grp->clear();
  A->clear();
  int last = -1;
  for (const ChanEntry& en : srt) {
    const int key = en.nax | (en.ax0 << 2) | (en.ax1 << 4) | (en.part << 6);
    if (key != last) {
      last = key;
      grp->push_back(en);
      A->resize(A->size() + 16, 0.0);
    }
    (*A)[(grp->size() - 1) * 16 + en.pad * 4 + en.src] += en.coef;
  }
}

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// A 2D view of `rows` rows of `row_doubles` doubles (rows contiguous), moved in boxes of
// 16 doubles (8 complex values, 128 bytes) by box_rows rows with the 128-byte swizzle.
static bool encode_rows(CUtensorMap* m, void* base, long long row_doubles, long long rows, int box_rows) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || !base) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)row_doubles, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)row_doubles * 8};
  const cuuint32_t box[2] = {16, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// A 3D view of `planes` planes of `rows` rows of `row_c` complex values (the half spectra
// [plane][axis 1][x]), moved in boxes of 8 complex values by `rows` rows of one plane
// with the 128-byte swizzle.
static bool encode_planes(CUtensorMap* m, void* base, long long row_c, long long rows, long long planes) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || !base || rows > 256) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)(2 * row_c), (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)(2 * row_c * 8), (cuuint64_t)(2 * row_c * 8 * rows)};
  const cuuint32_t box[3] = {16, (cuuint32_t)rows, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// Device memory of the plan: cudaMalloc, or the next 256-byte-aligned piece of the arena.
template <typename T>
cudaError_t SpectralPlan::dev_alloc(T** p, size_t bytes) {
  if (!arena_) return cudaMalloc((void**)p, bytes);
  const size_t off = (arena_->used + 255) / 256 * 256;
  if (off + bytes > arena_->size) return cudaErrorMemoryAllocation;
  *p = reinterpret_cast<T*>(arena_->base + off);
  arena_->used = off + bytes;
  return cudaSuccess;
}

template <typename T>
cudaError_t SpectralPlan::upload_vec(T** dst, const std::vector<T>& v) {
  if (!arena_) return upload(dst, v, &device_bytes);
  const size_t b = std::max<size_t>(1, v.size()) * sizeof(T);
  cudaError_t e = dev_alloc(dst, b);
  if (e != cudaSuccess) return e;
  if (!v.empty())
    e = cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, arena_->stream);
  return e;
}

bool SpectralPlan::init_in_arena(int n_, int ndim_, const int* Ns_, const double* Ls_,
                                 const std::vector<HostTerm>& terms, PlanArena* arena, std::string* msg) {
  release();
  arena_ = arena;
  const bool ok = init(n_, ndim_, Ns_, Ls_, terms, msg);
  return ok;
}

static ChanEntry entry_for(int k, int n, int ndim, int part, double coef) {
  ChanEntry e{};
  e.src = k % n;
  const int Yind = k / n;
  e.part = part;
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

bool SpectralPlan::init(int n_, int ndim_, const int* Ns_, const double* Ls_,
                        const std::vector<HostTerm>& terms, std::string* msg) {
  release();
  n = n_;
  ndim = ndim_;
  N = 1;
  for (int a = 0; a < 3; ++a) {
    Ns[a] = a < ndim ? Ns_[a] : 1;
    Ls[a] = a < ndim ? Ls_[a] : 1.0;
  }
  for (int a = 0; a < ndim; ++a) N *= Ns[a];
  M = Ns[ndim - 1];
  Mh = M / 2 + 1;
  R = (int)(N / M);
  const int nY = 1 + ndim + ndim * ndim;
  if (!make_line_plan(M, &plan_x_)) {
    *msg = "grid size " + std::to_string(M) + " along the last axis is not supported (radices 2,3,5,7,11,13; at most 8192)";
    return false;
  }
  for (int a = 0; a + 1 < ndim; ++a) {
    if (!make_line_plan(Ns[a], &plan_ax_[a])) {
      *msg = "grid size " + std::to_string(Ns[a]) + " along axis " + std::to_string(a) + " is not supported";
      return false;
    }
  }

  // ---- channels and dictionary (host)
  const double invN = 1.0 / (double)N;
  std::vector<std::vector<ChanEntry>> fold(n);
  std::vector<int> needY;  // Y indices (>= n) needed physically
  struct TermOut { int field; double C; std::vector<std::pair<int, int>> fac; };
  std::vector<TermOut> kept;
  std::vector<std::vector<int>> fold_term(n);  // term index of each fold entry
  std::vector<int> kept_term;                   // term index of each kept term
  for (size_t ti = 0; ti < terms.size(); ++ti) {
    const auto& t = terms[ti];
    const int field = t.ints.empty() ? 0 : t.ints[0];
    if (field < 0 || field >= n) {
      *msg = "coupling term field " + std::to_string(field) + " out of range";
      return false;
    }
    std::vector<std::pair<int, int>> fac;
    const int np = (int)t.ints.size();
    for (int j = 1; j < np; j += 2) {
      const int k = t.ints[j];
      const int p = (j + 1 < np) ? t.ints[j + 1] : 0;
      if (k < 0 || k >= nY * n) {
        *msg = "coupling term Y index " + std::to_string(k) + " out of range";
        return false;
      }
      if (p != 0) fac.push_back({k, p});  // pow(x, 0) == 1 for every x
    }
    if (fac.size() == 1 && fac[0].second == 1 && fac[0].first >= n) {
      fold[field].push_back(entry_for(fac[0].first, n, ndim, 0, t.C * invN));
      fold_term[field].push_back((int)ti);
      continue;
    }
    for (auto& f : fac)
      if (f.first >= n && std::find(needY.begin(), needY.end(), f.first) == needY.end()) needY.push_back(f.first);
    kept.push_back({field, t.C, fac});
    kept_term.push_back((int)ti);
  }
  std::sort(needY.begin(), needY.end());
  std::vector<int> ch_off{0};
  std::vector<ChanEntry> ch_ent;
  std::vector<int> fold_ch(n, -1);
  nch = 0;
  h_ent_term_.clear();
  std::vector<int> ych_of(nY * n, -1);
  if (explicit_channels_) {
    // a linear operator given channel by channel (adjoint passes): no dictionary
    for (auto& chn : *explicit_channels_) {
      for (ChanEntry e : chn) {
        e.coef *= invN;
        ch_ent.push_back(e);
        h_ent_term_.push_back(-1);
      }
      ch_off.push_back((int)ch_ent.size());
      ++nch;
    }
    kept.clear();
    kept_term.clear();
  } else {
    for (int i = 0; i < n; ++i) {
      if (fold[i].empty()) continue;
      fold_ch[i] = nch++;
      for (size_t q = 0; q < fold[i].size(); ++q) {
        ch_ent.push_back(fold[i][q]);
        h_ent_term_.push_back(fold_term[i][q]);
      }
      ch_off.push_back((int)ch_ent.size());
    }
    for (int k : needY) {
      ych_of[k] = nch++;
      ch_ent.push_back(entry_for(k, n, ndim, 0, invN));
      h_ent_term_.push_back(-1);
      ch_off.push_back((int)ch_ent.size());
    }
  }
  std::vector<DictTerm> dterms;
  std::vector<DictFactor> dfac;
  std::vector<int> field_begin(n + 1, 0);
  h_dict_term_.clear();
  for (int i = 0; i < n; ++i) {
    field_begin[i] = (int)dterms.size();
    for (size_t kt = 0; kt < kept.size(); ++kt) {
      auto& t = kept[kt];
      if (t.field != i) continue;
      h_dict_term_.push_back(kept_term[kt]);
      DictTerm dt{};
      dt.field = i;
      dt.C = t.C;
      dt.off = (int)dfac.size();
      dt.nf = (int)t.fac.size();
      for (auto& f : t.fac) {
        DictFactor df{};
        df.q = f.first < n ? f.first : n + ych_of[f.first];
        df.eta = f.second;
        dfac.push_back(df);
      }
      dterms.push_back(dt);
    }
  }
  field_begin[n] = (int)dterms.size();
  nterms_dict_ = (int)dterms.size();
  nfac_dict_ = (int)dfac.size();
  h_ch_off_ = ch_off;
  h_ch_ent_ = ch_ent;
  h_dterms_ = dterms;
  // dense polynomial form: every term a product of fields (no derivative quantity), total
  // degree <= 3, at most 3 fields
  poly_nf_ = 0;
  poly_count_ = 0;
  h_poly_mono_.clear();
  if (n <= 3 && !dterms.empty()) {
    const auto ex = mono_exponents(n);
    bool dense = true;
    std::vector<int> mono(dterms.size(), -1);
    for (size_t t = 0; t < dterms.size() && dense; ++t) {
      std::array<int, 3> e{0, 0, 0};
      for (int f = 0; f < dterms[t].nf; ++f) {
        const DictFactor& fc = dfac[dterms[t].off + f];
        if (fc.q >= n || fc.eta <= 0) {
          dense = false;
          break;
        }
        e[fc.q] += fc.eta;
      }
      if (!dense || e[0] + e[1] + e[2] > 3) {
        dense = false;
        break;
      }
      for (size_t m = 0; m < ex.size(); ++m)
        if (ex[m] == e) mono[t] = (int)m;
      dense = mono[t] >= 0;
    }
    if (dense) {
      poly_nf_ = n;
      poly_count_ = (int)ex.size();
      h_poly_mono_ = mono;
    }
  }
  inv_n_ = invN;

  // Y-mode channels: every block k, real and imaginary part
  std::vector<int> y_off{0};
  std::vector<ChanEntry> y_ent;
  std::vector<int> y_dst;
  for (int k = 0; k < nY * n; ++k)
    for (int part = 0; part < 2; ++part) {
      y_ent.push_back(entry_for(k, n, ndim, part, invN));
      y_off.push_back((int)y_ent.size());
      y_dst.push_back(k * 2 + part);
    }
  ych_ = (int)y_dst.size();
  h_ych_off_ = y_off;

  // wavenumbers exactly as d1 forms them (rdcu.cu:89-95)
  const double PI = 3.14159265358979323846;
  std::vector<double> kv;
  for (int a = 0; a < ndim; ++a) {
    kv_off_[a] = (int)kv.size();
    for (int na = 0; na < Ns[a]; ++na) {
      const int m2 = (na < Ns[a] / 2) ? na * 2 : (na - Ns[a]) * 2;
      kv.push_back(m2 * PI / Ls[a]);
    }
  }
  kv_total_ = (int)kv.size();
  h_kv_ = kv;

  // ---- device tables
  device_bytes = 0;
  std::vector<double2> tw;
  bool ok = true;
  auto chk = [&](cudaError_t e) {
    if (e != cudaSuccess && ok) {
      ok = false;
      *msg = std::string("CUDA error in spectral plan: ") + cudaGetErrorString(e);
    }
  };
  make_twiddles(M, tw);
  chk(upload_vec(&tw_x_, tw));
  for (int a = 0; a + 1 < ndim; ++a) {
    make_twiddles(Ns[a], tw);
    chk(upload_vec(&tw_ax_[a], tw));
  }
  chk(upload_vec(&kv_, kv));
  chk(upload_vec(&ch_off_, ch_off));
  chk(upload_vec(&ch_ent_, ch_ent));
  // operator-sorted copy of the hot entries with the local channel in .pad
  if (nch >= 1 && nch <= 4 && n <= 4) chk(upload_vec(&ch_sorted_, sorted_entries(ch_ent, ch_off, nch)));
  chk(upload_vec(&d_terms_, dterms));
  chk(upload_vec(&d_fac_, dfac));
  if (poly_nf_) chk(upload_vec(&d_poly_, poly_table()));
  chk(upload_vec(&d_field_begin_, field_begin));
  chk(upload_vec(&d_fold_, fold_ch));
  chk(upload_vec(&ych_off_, y_off));
  chk(upload_vec(&ych_ent_, y_ent));
  chk(upload_vec(&ych_dst_, y_dst));
  if (!ok) return false;

  // ---- launch configurations
  const int nrows = n * R;
  const int pairs = (nrows + 1) / 2;
  {
    int P = std::max(1, std::min(std::max(1, cta_elems() / M), pairs / kTargetCtas));
    const bool tws = (size_t)(M + P * M) * 16 <= kSmemBudget;
    fwd_.per_cta = P;
    fwd_.grid = (pairs + P - 1) / P;
    fwd_.block = std::min(kMaxBlock, std::max(128, round_up(stage_threads(plan_x_, P * M), 32)));
    fwd_.smem = (size_t)((tws ? M : 0) + P * M) * 16;
  }
  if (((nch + 1) / 2) * M > kMaxElems) {
    *msg = "the dictionary needs " + std::to_string(nch) + " inverse channels; with " + std::to_string(M) +
           " points along the last axis at most " + std::to_string(2 * (kMaxElems / M)) + " are supported";
    return false;
  }
  {
    int tws = 0;
    inv_geometry(M, R, n, nch, false, plan_x_, &inv_, &tws, dict_smem_bytes());
  }
  nparts_max = R;  // stage-7 error partials: one per grid row
  // Y-mode channel group
  const int GY = std::min(ych_, 8);
  sc_rows_ = std::max(nch, 1);
  if (ndim >= 2) {
    const int L0 = Ns[0];
    const int I = (ndim == 3) ? Ns[1] * Mh : Mh;
    for (int which = 0; which < 2; ++which) {
      const int G = which == 0 ? nch : GY;
      if (G == 0) continue;
      int TW = std::max(1, std::min(16, I / kTargetCtas));
      int GB = std::min(G, 4);
      while (TW > 1 && std::max(n, GB) * TW * L0 > cta_elems()) TW /= 2;
      while (GB > 1 && std::max(n, GB) * TW * L0 > kMaxElems) --GB;
      if (std::max(n, GB) * TW * L0 > kMaxElems) {
        *msg = "too many fields for one axis-0 pass (n * N0 must be <= " + std::to_string(kMaxElems) + ")";
        return false;
      }
      // plus the staged channel entries, wavenumbers and offsets (see k_mid)
      const int nent = which == 0 ? h_ch_off_[nch] : GY;
      // (+ the dense operator groups of the all-channel path, see k_mid)
      const size_t extra = (size_t)nent * sizeof(ChanEntry) + (size_t)kv_total_ * 8 + (size_t)(G + 2) * 4 + 16 +
                           (size_t)nent * (sizeof(ChanEntry) + 16 * 8);
      auto smem_of = [&](int tw_, int gb) { return (size_t)(L0 + (n + gb) * tw_ * tile_stride(L0, tw_)) * 16 + extra; };
      while (TW > 1 && smem_of(TW, GB) > kSmemBudget) TW /= 2;
      while (GB > 1 && smem_of(TW, GB) > kSmemBudget) --GB;
      if (smem_of(TW, GB) > 227 * 1024) {
        *msg = "grid too large for the shared-memory axis-0 pass";
        return false;
      }
      PassCfg& c = mid_[which];
      c.grid = (I + TW - 1) / TW;
      c.block = std::min(kMaxBlock, std::max(128, round_up(stage_threads(plan_ax_[0], std::max(n, GB) * TW * L0), 32)));
      c.smem = smem_of(TW, GB);
      if (which == 0 && ch_sorted_ && nch <= GB && nch <= n)  // in-place channel lines (k_mid)
        c.smem = (size_t)(L0 + n * TW * tile_stride(L0, TW)) * 16 + extra;
      c.per_cta = TW | (GB << 16);  // columns per CTA | channel lines held at once
    }
    if (ndim == 3) {
      const int La = Ns[1], I1 = Mh;
      int TW = std::min(16, I1);
      while (TW > 1 && ((size_t)(La + TW * tile_stride(La, TW)) * 16 > kSmemBudget || TW * La > cta_elems())) TW /= 2;
      c2c_f_.per_cta = TW;
      c2c_f_.grid = (I1 + TW - 1) / TW;
      c2c_f_.block = std::min(kMaxBlock, std::max(128, round_up(stage_threads(plan_ax_[1], TW * La), 32)));
      c2c_f_.smem = (size_t)(La + TW * tile_stride(La, TW)) * 16;
      c2c_i_ = c2c_f_;
    }
  }
  mult_.block = 256;

  // ---- buffers
  const size_t srow = (size_t)R * Mh * sizeof(double2);
  cudaError_t e = dev_alloc(&Sf_, std::max<size_t>(1, (size_t)n * srow));
  if (e != cudaSuccess) {
    *msg = "out of device memory (spectral buffers)";
    return false;
  }
  device_bytes += (size_t)n * srow;
  e = dev_alloc(&Sc_, (size_t)sc_rows_ * srow);
  if (e != cudaSuccess) {
    *msg = "out of device memory (spectral buffers)";
    return false;
  }
  device_bytes += (size_t)sc_rows_ * srow;

  // opt in to large dynamic shared memory (the limit is per block, static included)
  const int maxsm = 227 * 1024;
  bool optin_ok = true;
  auto optin_all = [&](const LinePlan& pl) {
    // the length-specialised kernels and the general ones larger blocks take
    for (int blk : {kSpecBlock, kMaxBlock}) {
      by_length(pl, blk, [&](auto rs, auto lx) {
        constexpr int RS = decltype(rs)::value, LX = decltype(lx)::value;
        optin_ok &= opt_in_smem((const void*)k_fwd_x<RS, LX>);
        if constexpr (LX == 128 || LX == 256) {
          optin_ok &= opt_in_smem((const void*)k_fwd_x<RS, LX, 1>);
          optin_ok &= opt_in_smem((const void*)k_fwd_x<RS, LX, 2>);
          optin_ok &= opt_in_smem((const void*)k_fwd_x<RS, LX, 3>);
          optin_ok &= opt_in_smem((const void*)k_fwd_x<RS, LX, 4>);
          optin_ok &= opt_in_smem((const void*)k_fwd_x<RS, LX, 5>);
          optin_ok &= opt_in_smem((const void*)k_fwd_x<RS, LX, 6>);
          optin_ok &= opt_in_smem((const void*)k_fwd_x<RS, LX, 7>);
        }
        optin_ok &= opt_in_smem((const void*)k_inv_x<RS, LX>);
        optin_ok &= opt_in_smem((const void*)k_mid<RS, LX>);
        optin_ok &= opt_in_smem((const void*)k_c2c<RS, false, LX>);
        optin_ok &= opt_in_smem((const void*)k_c2c<RS, true, LX>);
      });
    }
  };
  optin_all(plan_x_);
  for (int ax = 0; ax + 1 < ndim; ++ax) optin_all(plan_ax_[ax]);
  if (!optin_ok) {
    *msg = "cannot enable large shared memory for the FFT passes";
    return false;
  }
  if (fwd_.smem > (size_t)maxsm || inv_.smem > (size_t)maxsm) {
    *msg = "grid too large for the shared-memory x pass";
    return false;
  }
  setup_pipes();
  setup_planes();
  built_ = true;
  return true;
}

// Which 3D passes run as the specialised kernels: k_inv_row for 128- or 256-point rows
// with a dense-polynomial dictionary of at most two channels; k_mid_pipe for 128- or
// 256-point axis-0 lines with at most two fields and no more channels than fields
// (written over their sources); k_c2c_pipe with it for 128- or 256-point axis-1 lines.
// Every other plan keeps the general kernels.
using MidKernel = void (*)(const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, MidPipeArgs);

static MidKernel mid2_kernel(int L0, int nz, bool real) {
  if (L0 == 128) {
    if (nz == 2) return real ? k_mid_pipe2<128, 2, true> : k_mid_pipe2<128, 2, false>;
    return real ? k_mid_pipe2<128, 1, true> : k_mid_pipe2<128, 1, false>;
  }
  if (nz == 2) return real ? k_mid_pipe2<256, 2, true> : k_mid_pipe2<256, 2, false>;
  return real ? k_mid_pipe2<256, 1, true> : k_mid_pipe2<256, 1, false>;
}

void SpectralPlan::setup_pipes() {
  pipe_mid_ = pipe_c2c_ = inv_row_ = fuse_rows_ = false;
  if (ndim != 3) return;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  sms_ = std::max(1, sms);
  if ((M == 128 || M == 256) && poly_nf_ == n && n >= 1 && n <= 3 && nch >= 1 && nch <= 2 &&
      std::max(inv_row_smem(n, poly_count_, true), inv_row_smem(n, poly_count_, false)) <= 227 * 1024) {
    bool ok = true;
    auto attr = [&](const void* fn, bool err) {
      ok &= cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)inv_row_smem(n, poly_count_, err)) == cudaSuccess;
    };
    auto both = [&](auto lx, auto nf) {
      constexpr int LX = decltype(lx)::value, NF = decltype(nf)::value;
      attr((const void*)k_inv_row<LX, NF, false>, false);
      attr((const void*)k_inv_row<LX, NF, true>, true);
    };
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;
    using I3 = std::integral_constant<int, 3>;
    if (M == 128) {
      using L = std::integral_constant<int, 128>;
      n == 1 ? both(L{}, I1{}) : n == 2 ? both(L{}, I2{}) : both(L{}, I3{});
    } else {
      using L = std::integral_constant<int, 256>;
      n == 1 ? both(L{}, I1{}) : n == 2 ? both(L{}, I2{}) : both(L{}, I3{});
    }
    cudaGetLastError();
    inv_row_ = ok;
    // the inverse x pass of a stage fused with the next stage's forward x pass (two
    // fields); RDCU_FUSED_ROWS=0 keeps them separate
    const char* fz = getenv("RDCU_FUSED_ROWS");
    fuse_rows_ = inv_row_ && n == 2 && !(fz && fz[0] == '0') && inv_fwd_row_smem(poly_count_) <= 227 * 1024;
    if (fuse_rows_) {
      auto fattr = [&](auto lx) {
        constexpr int LX = decltype(lx)::value;
        const void* fns[] = {(const void*)k_inv_fwd_row<LX, 3>, (const void*)k_inv_fwd_row<LX, 4>,
                             (const void*)k_inv_fwd_row<LX, 5>, (const void*)k_inv_fwd_row<LX, 6>};
        for (const void* fn : fns)
          fuse_rows_ &= cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)inv_fwd_row_smem(poly_count_)) == cudaSuccess;
      };
      if (M == 128)
        fattr(std::integral_constant<int, 128>{});
      else
        fattr(std::integral_constant<int, 256>{});
      cudaGetLastError();
    }
  }
  if (!(Ns[0] == 128 || Ns[0] == 256) || !ch_sorted_ || nch < 1 || nch > n || n > 2) return;
  const long long I = (long long)Ns[1] * Mh;
  if (2 * I > 0x7fffffffLL) return;
  std::vector<ChanEntry> grp;
  std::vector<double> A;
  operator_groups(sorted_entries(h_ch_ent_, h_ch_off_, nch), &grp, &A);
  // multiplier tables unless an operator group mixes axis 0 with another axis
  mid_tab_ = true;
  for (const ChanEntry& en : grp) {
    const int na0 = (en.nax >= 1 && en.ax0 == 0) + (en.nax >= 2 && en.ax1 == 0);
    if (na0 > 0 && na0 < en.nax) mid_tab_ = false;
  }
  // one column per warp with register multipliers: at most two groups on axis 0 alone
  mid_nz_ = 0;
  for (const ChanEntry& en : grp) {
    const int na0 = (en.nax >= 1 && en.ax0 == 0) + (en.nax >= 2 && en.ax1 == 0);
    if (na0 > 0 && na0 == en.nax) ++mid_nz_;
  }
  mid2_ = mid_tab_ && mid_nz_ <= 2;
  if (mid2_) {
    for (bool real : {false, true})
      if (cudaFuncSetAttribute(mid2_kernel(Ns[0], mid_nz_, real), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)mid2_smem(Ns[0])) != cudaSuccess) {
        cudaGetLastError();
        mid2_ = false;
      }
  }
  const size_t smem = mid_pipe_smem((int)grp.size(), kv_total_, mid_tab_ ? Ns[0] * nch * n : 0);
  if (smem > 227 * 1024) return;
  if (!encode_rows(&tm_sf_, Sf_, 2 * I, (long long)n * Ns[0], Ns[0]) || !encode_sc_map()) return;
  const void* fn = Ns[0] == 128 ? (mid_tab_ ? (const void*)k_mid_pipe<128, true> : (const void*)k_mid_pipe<128, false>)
                                : (mid_tab_ ? (const void*)k_mid_pipe<256, true> : (const void*)k_mid_pipe<256, false>);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  if (mid_tab_ && build_mid_tables(grp, A) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  if (upload_vec(&mid_grp_, grp) != cudaSuccess || upload_vec(&mid_A_, A) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  if (!pipe_err_ && (dev_alloc(&pipe_err_, sizeof(int)) != cudaSuccess ||
                     cudaMemsetAsync(pipe_err_, 0, sizeof(int), arena_ ? arena_->stream : 0) != cudaSuccess)) {
    cudaGetLastError();
    pipe_err_ = nullptr;
    return;
  }
  const int cols = 8 * (256 / Ns[0]);  // columns per tile
  const int ntiles = (int)((I + cols - 1) / cols);
  pipe_grid_ = std::max(1, std::min(ntiles, sms_));
  mid_ngrp_ = (int)grp.size();
  pipe_mid_ = true;
  if (Ns[1] == 128 || Ns[1] == 256) {
    const void* ff = Ns[1] == 128 ? (const void*)k_c2c_pipe<128, false> : (const void*)k_c2c_pipe<256, false>;
    const void* fi = Ns[1] == 128 ? (const void*)k_c2c_pipe<128, true> : (const void*)k_c2c_pipe<256, true>;
    if (encode_planes(&tm_sf_c2c_, Sf_, Mh, Ns[1], (long long)n * Ns[0]) &&
        cudaFuncSetAttribute(ff, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kC2cPipeSmem) == cudaSuccess &&
        cudaFuncSetAttribute(fi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kC2cPipeSmem) == cudaSuccess)
      pipe_c2c_ = true;
    cudaGetLastError();
  }
}

// The multiplier of each channel and source summed over the operator groups, split by
// the axes the groups depend on: Mz[c][s][z] (groups on axis 0 only) and Mc[P][c][s]
// (the others; P = axis-1 index * Mh + x wavenumber).  Each group contributes
// i^q beta_g A_g[c][s], beta_g as k_mid forms it.
cudaError_t SpectralPlan::build_mid_tables(const std::vector<ChanEntry>& grp, const std::vector<double>& A) {
  const int G = nch, L0 = Ns[0];
  const long long I = (long long)Ns[1] * Mh;
  std::vector<double2> mz((size_t)L0 * G * n, make_double2(0.0, 0.0)), mc((size_t)I * G * n, make_double2(0.0, 0.0));
  auto kp = [&](int ax, int na) { return h_kv_[kv_off_[ax] + na]; };
  auto km = [&](int ax, int na) { return h_kv_[kv_off_[ax] + (na == 0 ? 0 : Ns[ax] - na)]; };
  // m[(c * n + s) * stride]: the (c, s) entry of the point's multiplier
  auto add = [&](double2* m, long long stride, const ChanEntry& en, const double* Ag, const int* nidx) {
    double ap = 1.0, am = 1.0;
    if (en.nax >= 1) {
      ap *= kp(en.ax0, nidx[en.ax0]);
      am *= km(en.ax0, nidx[en.ax0]);
    }
    if (en.nax >= 2) {
      ap *= kp(en.ax1, nidx[en.ax1]);
      am *= km(en.ax1, nidx[en.ax1]);
    }
    const double sgn = (en.nax & 1) ? -1.0 : 1.0;
    const double beta = en.part == 0 ? 0.5 * (ap + sgn * am) : 0.5 * (ap - sgn * am);
    const int q = (en.part == 0 ? en.nax : en.nax + 3) & 3;
    for (int c = 0; c < G; ++c)
      for (int s2 = 0; s2 < n; ++s2) {
        const double v = beta * Ag[c * 4 + s2];
        double2& d = m[(c * n + s2) * stride];
        switch (q) {
          case 0: d.x += v; break;
          case 1: d.y += v; break;
          case 2: d.x -= v; break;
          default: d.y -= v; break;
        }
      }
  };
  for (size_t g = 0; g < grp.size(); ++g) {
    const ChanEntry& en = grp[g];
    const int na0 = (en.nax >= 1 && en.ax0 == 0) + (en.nax >= 2 && en.ax1 == 0);
    if (na0 > 0) {
      for (int z = 0; z < L0; ++z) {
        const int nidx[3] = {z, 0, 0};
        add(&mz[z], L0, en, &A[g * 16], nidx);
      }
    } else {
      for (long long P = 0; P < I; ++P) {
        const int k1 = (int)(P / Mh), kx = (int)(P - (long long)k1 * Mh);
        const int nidx[3] = {0, k1, kx};
        add(&mc[(size_t)P * G * n], 1, en, &A[g * 16], nidx);
      }
    }
  }
  // the groups on axis 0 alone, for k_mid_pipe2: beta_g(z) and i^q A_g[c][s]
  const int NZ = std::max(1, mid_nz_);
  std::vector<double> bz((size_t)NZ * L0, 0.0);
  std::vector<double2> rz((size_t)NZ * G * n, make_double2(0.0, 0.0));
  int gz = 0;
  for (size_t g = 0; g < grp.size() && gz < NZ; ++g) {
    const ChanEntry& en = grp[g];
    const int na0 = (en.nax >= 1 && en.ax0 == 0) + (en.nax >= 2 && en.ax1 == 0);
    if (!(na0 > 0 && na0 == en.nax)) continue;
    for (int z = 0; z < L0; ++z) {
      const double ap = en.nax == 1 ? kp(0, z) : kp(0, z) * kp(0, z);
      const double am = en.nax == 1 ? km(0, z) : km(0, z) * km(0, z);
      const double sgn = (en.nax & 1) ? -1.0 : 1.0;
      bz[(size_t)gz * L0 + z] = en.part == 0 ? 0.5 * (ap + sgn * am) : 0.5 * (ap - sgn * am);
    }
    const int q = (en.part == 0 ? en.nax : en.nax + 3) & 3;
    for (int c = 0; c < G; ++c)
      for (int s2 = 0; s2 < n; ++s2) {
        const double v = A[g * 16 + c * 4 + s2];
        rz[((size_t)gz * G + c) * n + s2] = q == 0 ? make_double2(v, 0.0) : q == 1 ? make_double2(0.0, v)
                                           : q == 2 ? make_double2(-v, 0.0) : make_double2(0.0, -v);
      }
    ++gz;
  }
  // every multiplier real: the axis-0 pass's real form (the i^q rotations are fixed by the
  // operators, so later coefficients keep the form)
  bool real = true;
  for (const double2& v : rz) real &= v.y == 0.0;
  for (const double2& v : mc) real &= v.y == 0.0;
  if (!mid_tables_built_) {
    mid_real_ = real;
    mid_tables_built_ = true;
  } else if (mid_real_ && !real) {
    return cudaErrorInvalidValue;
  }
  if (!mid_bz_) RDCU_TRY(dev_alloc(&mid_bz_, bz.size() * sizeof(double)));
  if (!mid_rz_) RDCU_TRY(dev_alloc(&mid_rz_, rz.size() * sizeof(double2)));
  RDCU_TRY(cudaMemcpy(mid_bz_, bz.data(), bz.size() * sizeof(double), cudaMemcpyHostToDevice));
  RDCU_TRY(cudaMemcpy(mid_rz_, rz.data(), rz.size() * sizeof(double2), cudaMemcpyHostToDevice));
  if (!mid_mz_) RDCU_TRY(dev_alloc(&mid_mz_, mz.size() * sizeof(double2)));
  if (!mid_mc_) RDCU_TRY(dev_alloc(&mid_mc_, mc.size() * sizeof(double2)));
  RDCU_TRY(cudaMemcpy(mid_mz_, mz.data(), mz.size() * sizeof(double2), cudaMemcpyHostToDevice));
  RDCU_TRY(cudaMemcpy(mid_mc_, mc.data(), mc.size() * sizeof(double2), cudaMemcpyHostToDevice));
  return cudaSuccess;
}

bool SpectralPlan::encode_sc_map() {
  const long long I = (long long)Ns[1] * Mh;
  return encode_rows(&tm_sc_, Sc_, 2 * I, (long long)sc_rows_ * Ns[0], Ns[0]) &&
         (Ns[1] > 256 || encode_planes(&tm_sc_c2c_, Sc_, Mh, Ns[1], (long long)sc_rows_ * Ns[0]));
}

int SpectralPlan::take_pipe_error() {
  if (!pipe_err_) return 0;
  int e = 0;
  if (cudaMemcpy(&e, pipe_err_, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  if (e) cudaMemset(pipe_err_, 0, sizeof(int));
  return e;
}

cudaError_t SpectralPlan::launch_inv_row(const RhsIO& io, cudaStream_t st) {
  InvRowArgs a{};
  a.R = R;
  a.n = n;
  a.nch = nch;
  a.Mh = Mh;
  a.tw = tw_x_;
  a.Sc = Sc_;
  a.dict = dict_table();
  a.io = io;
  const bool err = io.mode == 1 && io.stage == 7 && io.err_part != nullptr && io.err_aux != nullptr;
  const size_t smem = inv_row_smem(n, poly_count_, err);
  const int rows_per_cta = row_warps(err, n) * (32 / (M / 8));
  const int grid = std::max(1, std::min((R + rows_per_cta - 1) / rows_per_cta, sms_));  // one resident CTA per SM
  const int threads = row_warps(err, n) * 32;
  auto go = [&](auto lx) {
    constexpr int LX = decltype(lx)::value;
    if (err) {
      switch (n) {
        case 1: k_inv_row<LX, 1, true><<<grid, threads, smem, st>>>(a); break;
        case 2: k_inv_row<LX, 2, true><<<grid, threads, smem, st>>>(a); break;
        default: k_inv_row<LX, 3, true><<<grid, threads, smem, st>>>(a); break;
      }
    } else {
      switch (n) {
        case 1: k_inv_row<LX, 1, false><<<grid, threads, smem, st>>>(a); break;
        case 2: k_inv_row<LX, 2, false><<<grid, threads, smem, st>>>(a); break;
        default: k_inv_row<LX, 3, false><<<grid, threads, smem, st>>>(a); break;
      }
    }
  };
  if (M == 128)
    go(std::integral_constant<int, 128>{});
  else
    go(std::integral_constant<int, 256>{});
  return cudaGetLastError();
}

bool SpectralPlan::fuse_ok(const RhsIO& io, const RhsIO& next) const {
  return fuse_rows_ && inv_row_ && io.mode == 1 && next.mode == 1 && io.ctl == next.ctl && io.stage >= 2 && io.stage <= 5 &&
         next.stage == io.stage + 1 && !plane_inv_ok(io) && !plane_fwd_ok(next);
}

cudaError_t SpectralPlan::launch_inv_fwd_row(const RhsIO& io, const RhsIO& next, cudaStream_t st) {
  InvFwdRowArgs f{};
  f.inv.R = R;
  f.inv.n = n;
  f.inv.nch = nch;
  f.inv.Mh = Mh;
  f.inv.tw = tw_x_;
  f.inv.Sc = Sc_;
  f.inv.dict = dict_table();
  f.inv.io = io;
  f.io2 = next;
  f.Sf = Sf_;
  const size_t smem = inv_fwd_row_smem(poly_count_);
  const int rows_per_cta = kFuseWarps * (32 / (M / 8));
  const int grid = std::max(1, std::min((R + rows_per_cta - 1) / rows_per_cta, sms_));  // one resident CTA per SM
  auto go = [&](auto lx) {
    constexpr int LX = decltype(lx)::value;
    switch (next.stage) {
      case 3: k_inv_fwd_row<LX, 3><<<grid, kFuseWarps * 32, smem, st>>>(f); break;
      case 4: k_inv_fwd_row<LX, 4><<<grid, kFuseWarps * 32, smem, st>>>(f); break;
      case 5: k_inv_fwd_row<LX, 5><<<grid, kFuseWarps * 32, smem, st>>>(f); break;
      default: k_inv_fwd_row<LX, 6><<<grid, kFuseWarps * 32, smem, st>>>(f); break;
    }
  };
  if (M == 128)
    go(std::integral_constant<int, 128>{});
  else
    go(std::integral_constant<int, 256>{});
  return cudaGetLastError();
}

cudaError_t SpectralPlan::launch_mid_pipe(const RhsIO& io, cudaStream_t st) {
  MidPipeArgs a{};
  a.I = Ns[1] * Mh;
  a.nsrc = n;
  a.G = nch;
  a.ntiles = (a.I + 8 * (256 / Ns[0]) - 1) / (8 * (256 / Ns[0]));
  a.ngrp = mid_ngrp_;
  a.Mh = Mh;
  a.tw = tw_ax_[0];
  a.grp = mid_grp_;
  a.A = mid_A_;
  a.kv = kv_;
  for (int ax = 0; ax < 3; ++ax) {
    a.kv_off[ax] = kv_off_[ax];
    a.Ns[ax] = Ns[ax];
  }
  a.kv_total = kv_total_;
  a.io = io;
  a.err = pipe_err_;
  a.Mz = mid_mz_;
  a.Mc = mid_mc_;
  a.Bz = mid_bz_;
  a.Rz = mid_rz_;
  if (mid2_) {
    const size_t sm2 = mid2_smem(Ns[0]);
    const int grid2 = std::max(1, std::min(a.ntiles, sms_));
    mid2_kernel(Ns[0], mid_nz_, mid_real_)<<<grid2, kMid2Threads, sm2, st>>>(tm_sf_, tm_sc_, a);
    return cudaGetLastError();
  }
  const size_t smem = mid_pipe_smem(mid_ngrp_, kv_total_, mid_tab_ ? Ns[0] * nch * n : 0);
  if (Ns[0] == 128) {
    if (mid_tab_)
      k_mid_pipe<128, true><<<pipe_grid_, kPipeThreads, smem, st>>>(tm_sf_, tm_sc_, a);
    else
      k_mid_pipe<128, false><<<pipe_grid_, kPipeThreads, smem, st>>>(tm_sf_, tm_sc_, a);
  } else {
    if (mid_tab_)
      k_mid_pipe<256, true><<<pipe_grid_, kPipeThreads, smem, st>>>(tm_sf_, tm_sc_, a);
    else
      k_mid_pipe<256, false><<<pipe_grid_, kPipeThreads, smem, st>>>(tm_sf_, tm_sc_, a);
  }
  return cudaGetLastError();
}

cudaError_t SpectralPlan::launch_c2c_pipe(bool inv, int nplanes, cudaStream_t st, const RhsIO& io, int rev) {
  C2CPipeArgs a{};
  a.rev = rev < 0 ? (inv ? 1 : 0) : rev;
  a.nchunk = (Mh + 7) / 8;
  a.nbox = nplanes * a.nchunk;
  const int bpt = c2c_boxes(Ns[1]);
  a.ntiles = (a.nbox + bpt - 1) / bpt;
  a.tw = tw_ax_[1];
  a.io = io;
  a.err = pipe_err_;
  const int grid = std::max(1, std::min(a.ntiles, 2 * sms_));  // two resident CTAs per SM
  if (!inv) {
    if (Ns[1] == 128)
      k_c2c_pipe<128, false><<<grid, kC2cThreads, kC2cPipeSmem, st>>>(tm_sf_c2c_, a);
    else
      k_c2c_pipe<256, false><<<grid, kC2cThreads, kC2cPipeSmem, st>>>(tm_sf_c2c_, a);
  } else {
    if (Ns[1] == 128)
      k_c2c_pipe<128, true><<<grid, kC2cThreads, kC2cPipeSmem, st>>>(tm_sc_c2c_, a);
    else
      k_c2c_pipe<256, true><<<grid, kC2cThreads, kC2cPipeSmem, st>>>(tm_sc_c2c_, a);
  }
  return cudaGetLastError();
}

// ---- 3D x passes that also transform along axis 1 (k_fwd_plane, k_inv_plane)
namespace {

using PlaneKernel = void (*)(PlaneArgs);

PlaneKernel plane_fwd_kernel(int M, int C) {
  if (M == 128) return C == 4 ? k_fwd_plane<128, 4> : k_fwd_plane<128, 8>;
  return C == 4 ? k_fwd_plane<256, 4> : k_fwd_plane<256, 8>;
}

template <int LX, int C>
PlaneKernel plane_inv_kernel_lc(int nf, bool err) {
  if (nf == 1) return err ? k_inv_plane<LX, C, 1, true> : k_inv_plane<LX, C, 1, false>;
  return err ? k_inv_plane<LX, C, 2, true> : k_inv_plane<LX, C, 2, false>;
}

PlaneKernel plane_inv_kernel(int M, int C, int nf, bool err) {
  if (M == 128) return C == 4 ? plane_inv_kernel_lc<128, 4>(nf, err) : plane_inv_kernel_lc<128, 8>(nf, err);
  return C == 4 ? plane_inv_kernel_lc<256, 4>(nf, err) : plane_inv_kernel_lc<256, 8>(nf, err);
}

cudaLaunchConfig_t cluster_config(int grid, int block, size_t smem, int C, cudaStream_t st, cudaLaunchAttribute* at) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3((unsigned)block, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

// Clusters of C CTAs of `kernel` that fit the GPU at once (0 when none does).
int plane_clusters(PlaneKernel kernel, int block, size_t smem, int C) {
  if (cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = cluster_config(C, block, smem, C, nullptr, at);
  int ncl = 0;
  if (cudaOccupancyMaxActiveClusters(&ncl, (const void*)kernel, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return ncl;
}

}  // namespace

// The fused axis-1 passes need 3D grids with 128- or 256-point x rows and axis-1 lines
// (clusters of N1/32 CTAs), the tiled axis-0 pass between them, and for the inverse the
// row kernel's dictionary form (a dense polynomial of at most two fields and two
// inverse channels).  They are used only when RDCU_PLANE_PASSES=1 is set in the
// environment at plan creation: on a B200 they are slower than the separate passes
// (3D CGLE 256^3: 7.4 vs 5.4 ms per DP45 attempt) -- at most 15 clusters of 8 CTAs are
// resident (120 of 148 SMs), and within a CTA the loads, the transforms and the
// cluster exchanges of a plane follow one another (DRAM 26% busy in the forward pass,
// 18% in the inverse), where the row and tile kernels overlap them.
void SpectralPlan::setup_planes() {
  plane_fwd_ = plane_inv_ = false;
  if (ndim != 3 || !pipe_mid_ || nch < 1 || n > 3) return;
  if (!(M == 128 || M == 256) || !(Ns[1] == 128 || Ns[1] == 256)) return;
  const char* env = std::getenv("RDCU_PLANE_PASSES");
  if (!env || std::strcmp(env, "1") != 0) return;
  const int C = Ns[1] / 32;
  const int nf = plane_clusters(plane_fwd_kernel(M, C), kPlaneFwdThreads, plane_fwd_smem(M), C);
  if (nf > 0) {
    plane_fwd_grid_ = C * std::min(nf, Ns[0] * n);
    plane_fwd_ = true;
  }
  if (!inv_row_ || nch > 2 || n > 2) return;
  const size_t ism = plane_inv_smem(M, n, poly_count_);
  if (ism > 227 * 1024) return;
  const int ni0 = plane_clusters(plane_inv_kernel(M, C, n, false), kPlaneInvThreads, ism, C);
  const int ni1 = plane_clusters(plane_inv_kernel(M, C, n, true), kPlaneInvThreads, ism, C);
  if (ni0 > 0 && ni1 > 0) {
    plane_inv_grid_ = C * std::min(std::min(ni0, ni1), Ns[0]);
    plane_inv_ = true;
  }
}

// the forward pass reads the state with 16-byte loads: its arrays must be 16-byte aligned
bool SpectralPlan::plane_fwd_ok(const RhsIO& io) const {
  if (!plane_fwd_ || nch < 1) return false;
  unsigned long long m = reinterpret_cast<unsigned long long>(io.ytemp_out);
  if (io.mode == 0) m |= reinterpret_cast<unsigned long long>(io.y);
  return (m & 15) == 0;
}

// the hot channel table in one launch; at stage 7 of an adaptive step with the forward
// pass's slope sums
bool SpectralPlan::plane_inv_ok(const RhsIO& io) const {
  if (!plane_inv_) return false;
  const bool err_epilogue = io.mode == 1 && io.stage == 7 && io.err_part != nullptr;
  return !err_epilogue || io.err_aux != nullptr;
}

cudaError_t SpectralPlan::launch_plane_fwd(const RhsIO& io, cudaStream_t st) {
  PlaneArgs a{};
  a.N0 = Ns[0];
  a.n = n;
  a.nch = nch;
  a.twx = tw_x_;
  a.twy = tw_ax_[1];
  a.S = Sf_;
  a.io = io;
  const int C = Ns[1] / 32;
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = cluster_config(plane_fwd_grid_, kPlaneFwdThreads, plane_fwd_smem(M), C, st, at);
  return cudaLaunchKernelEx(&cfg, plane_fwd_kernel(M, C), a);
}

cudaError_t SpectralPlan::launch_plane_inv(const RhsIO& io, cudaStream_t st) {
  PlaneArgs a{};
  a.N0 = Ns[0];
  a.n = n;
  a.nch = nch;
  a.twx = tw_x_;
  a.twy = tw_ax_[1];
  a.Sc = Sc_;
  a.dict = dict_table();
  a.io = io;
  const bool err = io.mode == 1 && io.stage == 7 && io.err_part != nullptr && io.err_aux != nullptr;
  const int C = Ns[1] / 32;
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg =
      cluster_config(plane_inv_grid_, kPlaneInvThreads, plane_inv_smem(M, n, poly_count_), C, st, at);
  return cudaLaunchKernelEx(&cfg, plane_inv_kernel(M, C, n, err), a);
}

cudaError_t SpectralPlan::ensure_channel_capacity(int rows) {
  if (rows <= sc_rows_) return cudaSuccess;
  const size_t srow = (size_t)R * Mh * sizeof(double2);
  double2* p = nullptr;
  RDCU_TRY(cudaMalloc((void**)&p, (size_t)rows * srow));
  cudaFree(Sc_);
  device_bytes += (size_t)(rows - sc_rows_) * srow;
  Sc_ = p;
  sc_rows_ = rows;
  ++buffers_gen;
  if ((pipe_mid_ || pipe_c2c_) && !encode_sc_map()) pipe_mid_ = pipe_c2c_ = false;
  return cudaSuccess;
}

void SpectralPlan::release() {
  if (ch_sorted_ && !arena_) cudaFree(ch_sorted_);
  ch_sorted_ = nullptr;
  void* ptrs[] = {tw_x_, tw_ax_[0], tw_ax_[1], tw_ax_[2], kv_, ch_off_, ch_ent_, d_terms_, d_fac_, d_poly_,
                  d_field_begin_, d_fold_, ych_off_, ych_ent_, ych_dst_, Sf_, Sc_, lin_ent_, sinv_, cosv_,
                  mid_grp_, mid_A_, pipe_err_, mid_mz_, mid_mc_, mid_bz_, mid_rz_};
  if (!arena_)  // arena memory belongs to the caller
    for (void* p : ptrs)
      if (p) cudaFree(p);
  tw_x_ = nullptr;
  for (auto& t : tw_ax_) t = nullptr;
  kv_ = nullptr;
  ch_off_ = nullptr;
  ch_ent_ = nullptr;
  d_terms_ = nullptr;
  d_fac_ = nullptr;
  d_poly_ = nullptr;
  d_field_begin_ = nullptr;
  d_fold_ = nullptr;
  ych_off_ = nullptr;
  ych_ent_ = nullptr;
  ych_dst_ = nullptr;
  Sf_ = nullptr;
  Sc_ = nullptr;
  lin_ent_ = nullptr;
  sinv_ = nullptr;
  cosv_ = nullptr;
  mid_grp_ = nullptr;
  mid_A_ = nullptr;
  mid_mz_ = nullptr;
  mid_mc_ = nullptr;
  mid_bz_ = nullptr;
  mid_rz_ = nullptr;
  mid2_ = false;
  pipe_err_ = nullptr;
  pipe_mid_ = pipe_c2c_ = inv_row_ = false;
  nlin_ = 0;
  built_ = false;
}

// Runs the passes for channels [g_first, g_first+nch_run) of table ct.  When Yout is
// set the inverse x pass writes channels to Y.dat layout instead of the dictionary.
cudaError_t SpectralPlan::launch_passes(const RhsIO& io, const ChanTable& ct, const std::vector<int>& hoff,
                                        int nch_run, int g_first, double* Yout, const int* ydst, cudaStream_t st,
                                        int yplain, const RhsIO* next, bool* fused) {
  const bool spectral = nch_run > 0;
  // the inverse x pass with the axis-1 transform: the hot table, every channel, no Y.dat
  const bool plane_inv = spectral && !Yout && ct.ent == ch_ent_ && g_first == 0 && nch_run == nch && plane_inv_ok(io);
  if (spectral && ndim >= 2) {
    const int which = (ct.ent == ch_ent_) ? 0 : 1;  // hot table or the Y-block table
    const PassCfg& c = mid_[which];
    MidArgs m{};
    m.L0 = Ns[0];
    m.I = (ndim == 3) ? Ns[1] * Mh : Mh;
    m.TW = c.per_cta & 0xffff;
    m.GB = c.per_cta >> 16;
    m.nsrc = n;
    m.G = nch_run;
    m.ch0 = g_first;
    m.ndim = ndim;
    m.D1 = Ns[1];
    m.Mh = Mh;
    m.plan = plan_ax_[0];
    m.tw = tw_ax_[0];
    m.Sf = Sf_;
    m.Sc = Sc_;
    m.chan = ct;
    m.io = io;
    m.ent0 = hoff[g_first];
    m.nent = hoff[g_first + nch_run] - m.ent0;
    if (ct.ent == ch_ent_ && ch_sorted_ && nch_run <= m.GB && g_first == 0) {
      m.sorted = 1;
      m.chan.ent = ch_sorted_;  // staged into shared memory in operator order
    }
    const size_t smem = c.smem;  // includes the staged tables
    if (which == 0 && pipe_mid_ && g_first == 0 && nch_run == nch) {
      RDCU_TRY(launch_mid_pipe(io, st));
    } else {
      prep(m);
      by_length(plan_ax_[0], c.block, [&](auto rs, auto lx) { k_mid<decltype(rs)::value, decltype(lx)::value><<<c.grid, c.block, smem, st>>>(m); });
      RDCU_TRY(cudaGetLastError());
    }
    if (ndim == 3 && !plane_inv) {
      C2CArgs a{};
      a.La = Ns[1];
      a.I = Mh;
      a.TW = c2c_i_.per_cta;
      a.plan = plan_ax_[1];
      a.tw = tw_ax_[1];
      a.S = Sc_;
      a.io = io;
      dim3 grid(c2c_i_.grid, nch_run * Ns[0]);
      if (pipe_c2c_) {
        // before a fused row kernel (rows from the last to the first) the tiles go in order
        const bool to_fused = next && fused && fuse_ok(io, *next);
        RDCU_TRY(launch_c2c_pipe(true, nch_run * Ns[0], st, io, to_fused ? 0 : 1));
      } else {
        prep(a);
        by_length(plan_ax_[1], c2c_i_.block, [&](auto rs, auto lx) { k_c2c<decltype(rs)::value, true, decltype(lx)::value><<<grid, c2c_i_.block, c2c_i_.smem, st>>>(a); });
        RDCU_TRY(cudaGetLastError());
      }
    }
  } else if (spectral) {
    Mult1DArgs m{};
    m.Mh = Mh;
    m.nch = nch_run;
    m.ch0 = g_first;
    m.Sf = Sf_;
    m.Sc = Sc_;
    m.chan = ct;
    m.io = io;
    const long long tot = (long long)nch_run * Mh;
    k_mult1d<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(m);
    RDCU_TRY(cudaGetLastError());
  }
  // inverse x pass: the dictionary needs every channel of a row in one CTA; the Y.dat
  // output is launched one channel pair at a time
  const int step = Yout ? 2 : std::max(1, nch_run);
  // stage 7 of an adaptive step: the row kernel's error epilogue reads the terms the
  // forward pass left in err_aux; without them k_inv_x forms the error from y and slopes
  const bool err_epilogue = io.mode == 1 && io.stage == 7 && io.err_part != nullptr;
  if (plane_inv) return launch_plane_inv(io, st);
  if (!Yout && inv_row_ && (!err_epilogue || io.err_aux) && ct.ent == ch_ent_ && g_first == 0 && nch_run == nch) {
    if (next && fused && fuse_ok(io, *next)) {
      *fused = true;
      return launch_inv_fwd_row(io, *next, st);
    }
    return launch_inv_row(io, st);
  }
  for (int c0 = 0; c0 < std::max(1, nch_run); c0 += step) {
    const int cnt = spectral ? std::min(step, nch_run - c0) : 0;
    InvXArgs a{};
    a.M = M;
    a.Mh = Mh;
    a.R = R;
    a.n = n;
    a.nch_run = cnt;
    a.npairs = (cnt + 1) / 2;
    a.do_fft = spectral ? 1 : 0;
    a.N = N;
    a.plan = plan_x_;
    a.tw = tw_x_;
    a.Sc = Sc_;
    a.dict = dict_table();
    a.io = io;
    a.Yout = (Yout && yplain) ? Yout + (long long)c0 * N : Yout;
    a.ydst = ydst ? ydst + c0 : nullptr;
    a.yplain = yplain;
    a.ch_base = c0;
    PassCfg g;
    int tws = 0;
    inv_geometry(M, R, n, cnt, Yout != nullptr, plan_x_, &g, &tws, Yout ? 0 : dict_smem_bytes());
    a.P = g.per_cta;
    a.tw_smem = tws;
    prep(a);
    by_length(plan_x_, g.block, [&](auto rs, auto lx) { k_inv_x<decltype(rs)::value, decltype(lx)::value><<<g.grid, g.block, g.smem, st>>>(a); });
    RDCU_TRY(cudaGetLastError());
    if (!spectral) break;
  }
  return cudaSuccess;
}

cudaError_t SpectralPlan::run(const RhsIO& io, cudaStream_t st, const RhsIO* next, bool fwd_done, bool* fused) {
  const bool spectral = nch > 0;
  const bool need_fwd = spectral || (io.mode == 1 && io.stage >= 2);
  if (fused) *fused = false;
  if (!fused) next = nullptr;
  if (spectral && plane_fwd_ok(io)) {
    RDCU_TRY(launch_plane_fwd(io, st));
    return launch_passes(io, chan_table(ch_off_, ch_ent_, nch), h_ch_off_, nch, 0, nullptr, nullptr, st);
  }
  if (need_fwd && !fwd_done) {
    FwdXArgs a{};
    a.M = M;
    a.Mh = Mh;
    a.nrows = n * R;
    a.P = fwd_.per_cta;
    a.do_fft = spectral ? 1 : 0;
    a.tw_smem = fwd_.smem >= (size_t)(M + a.P * M) * 16 ? 1 : 0;
    a.plan = plan_x_;
    a.tw = tw_x_;
    a.S = Sf_;
    a.io = io;
    const size_t smem = spectral ? fwd_.smem : 0;
    prep(a);
    launch_fwd_x(plan_x_, fwd_.block, fwd_.grid, smem, st, a);
    RDCU_TRY(cudaGetLastError());
  }
  if (spectral && ndim == 3) {
    C2CArgs a{};
    a.La = Ns[1];
    a.I = Mh;
    a.TW = c2c_f_.per_cta;
    a.plan = plan_ax_[1];
    a.tw = tw_ax_[1];
    a.S = Sf_;
    a.io = io;
    dim3 grid(c2c_f_.grid, n * Ns[0]);
    if (pipe_c2c_) {
      RDCU_TRY(launch_c2c_pipe(false, n * Ns[0], st, io));
    } else {
      prep(a);
      by_length(plan_ax_[1], c2c_f_.block, [&](auto rs, auto lx) { k_c2c<decltype(rs)::value, false, decltype(lx)::value><<<grid, c2c_f_.block, c2c_f_.smem, st>>>(a); });
      RDCU_TRY(cudaGetLastError());
    }
  }
  return launch_passes(io, chan_table(ch_off_, ch_ent_, nch), h_ch_off_, nch, 0, nullptr, nullptr, st, 0, next, fused);
}

cudaError_t SpectralPlan::run_Y(const double* y, double* Yout, cudaStream_t st) {
  const int GY = std::min(ych_, 8);
  RDCU_TRY(ensure_channel_capacity(GY));
  RhsIO io{};
  io.mode = 0;
  io.y = y;
  FwdXArgs a{};
  a.M = M;
  a.Mh = Mh;
  a.nrows = n * R;
  a.P = fwd_.per_cta;
  a.do_fft = 1;
  a.tw_smem = fwd_.smem >= (size_t)(M + a.P * M) * 16 ? 1 : 0;
  a.plan = plan_x_;
  a.tw = tw_x_;
  a.S = Sf_;
  a.io = io;
  prep(a);
  launch_fwd_x(plan_x_, fwd_.block, fwd_.grid, fwd_.smem, st, a);
  RDCU_TRY(cudaGetLastError());
  if (ndim == 3) {
    C2CArgs c{};
    c.La = Ns[1];
    c.I = Mh;
    c.TW = c2c_f_.per_cta;
    c.plan = plan_ax_[1];
    c.tw = tw_ax_[1];
    c.S = Sf_;
    c.io = io;
    dim3 grid(c2c_f_.grid, n * Ns[0]);
    prep(c);
    by_length(plan_ax_[1], c2c_f_.block, [&](auto rs, auto lx) { k_c2c<decltype(rs)::value, false, decltype(lx)::value><<<grid, c2c_f_.block, c2c_f_.smem, st>>>(c); });
    RDCU_TRY(cudaGetLastError());
  }
  const ChanTable ct = chan_table(ych_off_, ych_ent_, ych_);
  for (int g = 0; g < ych_; g += GY) {
    const int cnt = std::min(GY, ych_ - g);
    RDCU_TRY(launch_passes(io, ct, h_ych_off_, cnt, g, Yout, ych_dst_ + g, st));
  }
  return cudaSuccess;
}

bool SpectralPlan::init_precond(int n_, int ndim_, const int* Ns_, const double* Ls_,
                                const std::vector<LinEntry>& lin, std::string* msg) {
  if (n_ > kMaxPrecFields) {
    *msg = "preconditioner supports at most " + std::to_string(kMaxPrecFields) + " fields";
    return false;
  }
  if (!init(n_, ndim_, Ns_, Ls_, std::vector<HostTerm>(), msg)) return false;
  if (((n + 1) / 2) * M > kMaxElems) {
    *msg = "preconditioner: too many fields for the last-axis length";
    return false;
  }
  std::vector<double> sv, cv;
  const double PI = 3.14159265358979323846;
  for (int a = 0; a < ndim; ++a) {
    sc_off_[a] = (int)sv.size();
    for (int m = 0; m < Ns[a]; ++m) {
      const long double th = 2.0L * 3.141592653589793238462643383279502884L * m / Ns[a];
      sv.push_back((double)sinl(th));
      cv.push_back((double)cosl(th));
    }
  }
  (void)PI;
  nlin_ = (int)lin.size();
  cudaError_t e = upload(&lin_ent_, lin, &device_bytes);
  if (e == cudaSuccess) e = upload(&sinv_, sv, &device_bytes);
  if (e == cudaSuccess) e = upload(&cosv_, cv, &device_bytes);
  if (e == cudaSuccess) e = ensure_channel_capacity(n);
  if (e == cudaSuccess && !ych_dst_) e = cudaErrorInvalidValue;
  if (e != cudaSuccess) {
    *msg = std::string("preconditioner set-up: ") + cudaGetErrorString(e);
    return false;
  }
  if (ndim >= 2) {
    const int L0 = Ns[0];
    const int I = (ndim == 3) ? Ns[1] * Mh : Mh;
    int TW = std::max(1, std::min(16, I / kTargetCtas));
    auto smem_of = [&](int tw_) { return (size_t)(L0 + n * tw_ * (L0 + 1)) * 16; };
    while (TW > 1 && (smem_of(TW) > kSmemBudget || n * TW * L0 > cta_elems())) TW /= 2;
    if (smem_of(TW) > 227 * 1024 || n * TW * L0 > kMaxElems) {
      *msg = "grid too large for the preconditioner's axis-0 pass";
      return false;
    }
    midsolve_.per_cta = TW;
    midsolve_.grid = (I + TW - 1) / TW;
    midsolve_.block = std::min(kMaxBlock, std::max(128, round_up(stage_threads(plan_ax_[0], n * TW * L0), 32)));
    midsolve_.smem = smem_of(TW);
    if (!opt_in_smem((const void*)k_mid_solve<kRadixPow2>) || !opt_in_smem((const void*)k_mid_solve<kRadixAll>)) {
      *msg = "cannot enable large shared memory for the preconditioner pass";
      return false;
    }
  }
  return true;
}

cudaError_t SpectralPlan::launch_forward(const double* y, cudaStream_t st) {
  RhsIO io{};
  io.mode = 0;
  io.y = y;
  FwdXArgs a{};
  a.M = M;
  a.Mh = Mh;
  a.nrows = n * R;
  a.P = fwd_.per_cta;
  a.do_fft = 1;
  a.tw_smem = fwd_.smem >= (size_t)(M + a.P * M) * 16 ? 1 : 0;
  a.plan = plan_x_;
  a.tw = tw_x_;
  a.S = Sf_;
  a.io = io;
  prep(a);
  launch_fwd_x(plan_x_, fwd_.block, fwd_.grid, fwd_.smem, st, a);
  RDCU_TRY(cudaGetLastError());
  if (ndim == 3) {
    C2CArgs c{};
    c.La = Ns[1];
    c.I = Mh;
    c.TW = c2c_f_.per_cta;
    c.plan = plan_ax_[1];
    c.tw = tw_ax_[1];
    c.S = Sf_;
    c.io = io;
    dim3 grid(c2c_f_.grid, n * Ns[0]);
    prep(c);
    by_length(plan_ax_[1], c2c_f_.block, [&](auto rs, auto lx) { k_c2c<decltype(rs)::value, false, decltype(lx)::value><<<grid, c2c_f_.block, c2c_f_.smem, st>>>(c); });
    RDCU_TRY(cudaGetLastError());
  }
  return cudaSuccess;
}

cudaError_t SpectralPlan::precond(const double* r, double* z, double alpha, cudaStream_t st) {
  return precond(r, z, alpha, nullptr, st);
}

cudaError_t SpectralPlan::precond(const double* r, double* z, double alpha, const double* alpha_dev,
                                  cudaStream_t st) {
  RDCU_TRY(launch_forward(r, st));
  LinTable lt{};
  lt.n = n;
  lt.nent = nlin_;
  lt.ndim = ndim;
  lt.ent = lin_ent_;
  lt.sinv = sinv_;
  lt.cosv = cosv_;
  lt.alpha = alpha;
  lt.alpha_dev = alpha_dev;
  for (int a = 0; a < 3; ++a) {
    lt.off[a] = sc_off_[a];
    lt.Ns[a] = Ns[a];
    lt.dx[a] = Ls[a] / Ns[a];
  }
  if (ndim >= 2) {
    MidSolveArgs m{};
    m.L0 = Ns[0];
    m.I = (ndim == 3) ? Ns[1] * Mh : Mh;
    m.TW = midsolve_.per_cta;
    m.n = n;
    m.ndim = ndim;
    m.Mh = Mh;
    m.plan = plan_ax_[0];
    m.tw = tw_ax_[0];
    m.Sf = Sf_;
    m.Sc = Sc_;
    m.lin = lt;
    prep(m);
    if (plan_is_pow2(plan_ax_[0]))
      k_mid_solve<kRadixPow2><<<midsolve_.grid, midsolve_.block, midsolve_.smem, st>>>(m);
    else
      k_mid_solve<kRadixAll><<<midsolve_.grid, midsolve_.block, midsolve_.smem, st>>>(m);
    RDCU_TRY(cudaGetLastError());
    if (ndim == 3) {
      C2CArgs a{};
      a.La = Ns[1];
      a.I = Mh;
      a.TW = c2c_i_.per_cta;
      a.plan = plan_ax_[1];
      a.tw = tw_ax_[1];
      a.S = Sc_;
      a.io = RhsIO{};
      dim3 grid(c2c_i_.grid, n * Ns[0]);
      prep(a);
      by_length(plan_ax_[1], c2c_i_.block, [&](auto rs, auto lx) { k_c2c<decltype(rs)::value, true, decltype(lx)::value><<<grid, c2c_i_.block, c2c_i_.smem, st>>>(a); });
      RDCU_TRY(cudaGetLastError());
    }
  } else {
    k_mult1d_solve<<<(Mh + 127) / 128, 128, 0, st>>>(Mh, n, Sf_, Sc_, lt);
    RDCU_TRY(cudaGetLastError());
  }
  // inverse x pass of the n solved fields straight into z
  InvXArgs a{};
  a.M = M;
  a.Mh = Mh;
  a.R = R;
  a.n = n;
  a.nch_run = n;
  a.npairs = (n + 1) / 2;
  a.do_fft = 1;
  a.N = N;
  a.plan = plan_x_;
  a.tw = tw_x_;
  a.Sc = Sc_;
  a.dict = dict_table();
  a.io = RhsIO{};
  a.Yout = z;
  a.ydst = nullptr;
  a.yplain = 1;
  a.ch_base = 0;
  PassCfg g;
  int tws = 0;
  inv_geometry(M, R, n, n, true, plan_x_, &g, &tws);
  a.P = g.per_cta;
  a.tw_smem = tws;
  prep(a);
  by_length(plan_x_, g.block, [&](auto rs, auto lx) { k_inv_x<decltype(rs)::value, decltype(lx)::value><<<g.grid, g.block, g.smem, st>>>(a); });
  return cudaGetLastError();
}

cudaError_t SpectralPlan::profile(const RhsIO& io, int reps, cudaStream_t st, std::vector<PassTime>* out,
                                  const RhsIO* next) {
  // Each round runs the stage's passes once in an attempt's order (forward x, axis 1,
  // axis 0, axis 1, inverse x), so that every pass reads what the pass before it wrote
  // from the stage's own inputs (the axis passes and the fused row pass work in place:
  // repeating one of them alone would feed it its own output); one untimed round, then
  // `reps` rounds with a pair of events around each launch.  With next, each round also
  // runs the passes again up to the axis-1 pass and then the fused inverse/forward pass.
  out->clear();
  const double spec_row = (double)R * Mh * 16.0;  // one field's half spectrum
  const double arr = (double)N * 8.0;             // one field's physical array
  const int s = io.stage >= 2 ? io.stage : 1;
  const int nk = s >= 2 ? (s == 7 ? s - 2 : s - 1) : 0;  // slopes the stage combination reads
  const bool spectral = nch > 0;
  const bool plane_fwd = spectral && plane_fwd_ok(io);
  const bool plane_inv = spectral && plane_inv_ok(io);
  const bool fused = next && fuse_ok(io, *next);
  FwdXArgs fa{};
  fa.M = M;
  fa.Mh = Mh;
  fa.nrows = n * R;
  fa.P = fwd_.per_cta;
  fa.do_fft = spectral ? 1 : 0;
  fa.tw_smem = fwd_.smem >= (size_t)(M + fa.P * M) * 16 ? 1 : 0;
  fa.plan = plan_x_;
  fa.tw = tw_x_;
  fa.S = Sf_;
  fa.io = io;
  prep(fa);
  C2CArgs cf{};
  cf.La = Ns[1];
  cf.I = Mh;
  cf.TW = c2c_f_.per_cta;
  cf.plan = plan_ax_[1];
  cf.tw = tw_ax_[1];
  cf.S = Sf_;
  cf.io = io;
  prep(cf);
  const dim3 gcf(c2c_f_.grid, n * Ns[0]);
  C2CArgs ci{};
  ci.La = Ns[1];
  ci.I = Mh;
  ci.TW = c2c_i_.per_cta;
  ci.plan = plan_ax_[1];
  ci.tw = tw_ax_[1];
  ci.S = Sc_;
  ci.io = io;
  prep(ci);
  const dim3 gci(c2c_i_.grid, nch * Ns[0]);
  const PassCfg& mc = mid_[0];
  MidArgs m{};
  m.L0 = Ns[0];
  m.I = (ndim == 3) ? Ns[1] * Mh : Mh;
  m.TW = mc.per_cta & 0xffff;
  m.GB = mc.per_cta >> 16;
  m.nsrc = n;
  m.G = nch;
  m.ch0 = 0;
  m.ndim = ndim;
  m.D1 = Ns[1];
  m.Mh = Mh;
  m.plan = plan_ax_[0];
  m.tw = tw_ax_[0];
  m.Sf = Sf_;
  m.Sc = Sc_;
  m.chan = chan_table(ch_off_, ch_ent_, nch);
  m.io = io;
  m.ent0 = 0;
  m.nent = h_ch_off_[nch];
  if (ch_sorted_ && nch <= m.GB) {
    m.sorted = 1;
    m.chan.ent = ch_sorted_;
  }
  prep(m);
  InvXArgs a{};
  a.M = M;
  a.Mh = Mh;
  a.R = R;
  a.n = n;
  a.nch_run = nch;
  a.npairs = (nch + 1) / 2;
  a.do_fft = spectral ? 1 : 0;
  a.N = N;
  a.plan = plan_x_;
  a.tw = tw_x_;
  a.Sc = Sc_;
  a.dict = dict_table();
  a.io = io;
  PassCfg g;
  int tws = 0;
  inv_geometry(M, R, n, nch, false, plan_x_, &g, &tws, dict_smem_bytes());
  a.P = g.per_cta;
  a.tw_smem = tws;
  prep(a);

  // stage 7 with err_aux also writes each point's slope sum
  const double aux_w = (io.mode == 1 && io.stage == 7 && io.err_part && io.err_aux) ? 1.0 : 0.0;
  const double fwd_bytes = n * ((1 + nk) * arr + (s >= 2 ? arr : 0) + spec_row + aux_w * arr);
  // stage 7 of an adaptive step also reads y and five slopes for the error estimate, or
  // y and the slope sums the forward pass wrote (err_aux)
  const bool err_epilogue = io.mode == 1 && io.stage == 7 && io.err_part != nullptr;
  const double err_arrays = err_epilogue ? (io.err_aux ? 2.0 : 6.0) : 0.0;
  const double inv_bytes = nch * spec_row + 2.0 * n * arr + err_arrays * n * arr;
  // the fused pass: the inverse part's bytes, then the next stage's combination without
  // the slope k_s (in registers)
  const double fused_bytes =
      fused ? nch * spec_row + 2.0 * n * arr + n * ((next->stage - 1) * arr + arr + spec_row) : 0.0;

  auto go_fwd = [&]() -> cudaError_t {
    if (plane_fwd) return launch_plane_fwd(io, st);
    launch_fwd_x(plan_x_, fwd_.block, fwd_.grid, fwd_.smem, st, fa);
    return cudaGetLastError();
  };
  auto go_c2c_f = [&]() -> cudaError_t {
    if (pipe_c2c_) return launch_c2c_pipe(false, n * Ns[0], st, io);
    by_length(plan_ax_[1], c2c_f_.block, [&](auto rs, auto lx) { k_c2c<decltype(rs)::value, false, decltype(lx)::value><<<gcf, c2c_f_.block, c2c_f_.smem, st>>>(cf); });
    return cudaGetLastError();
  };
  auto go_mid = [&]() -> cudaError_t {
    if (pipe_mid_) return launch_mid_pipe(io, st);
    by_length(plan_ax_[0], mc.block, [&](auto rs, auto lx) { k_mid<decltype(rs)::value, decltype(lx)::value><<<mc.grid, mc.block, mc.smem, st>>>(m); });
    return cudaGetLastError();
  };
  // rev: the axis-1 inverse pass's tile order (in order before the fused row pass)
  auto go_c2c_i = [&](int rev) -> cudaError_t {
    if (pipe_c2c_) return launch_c2c_pipe(true, nch * Ns[0], st, io, rev);
    by_length(plan_ax_[1], c2c_i_.block, [&](auto rs, auto lx) { k_c2c<decltype(rs)::value, true, decltype(lx)::value><<<gci, c2c_i_.block, c2c_i_.smem, st>>>(ci); });
    return cudaGetLastError();
  };
  auto go_inv = [&]() -> cudaError_t {
    if (plane_inv) return launch_plane_inv(io, st);
    if (inv_row_ && !(io.mode == 1 && io.stage == 7 && io.err_part != nullptr && !io.err_aux))
      return launch_inv_row(io, st);
    by_length(plan_x_, g.block, [&](auto rs, auto lx) { k_inv_x<decltype(rs)::value, decltype(lx)::value><<<g.grid, g.block, g.smem, st>>>(a); });
    return cudaGetLastError();
  };

  // the passes reported, in order
  std::vector<PassTime> tab;
  tab.push_back({plane_fwd ? "fwd_plane" : "fwd_x", 0.0, fwd_bytes});
  const int i_c2c_f = (spectral && ndim == 3 && !plane_fwd) ? (int)tab.size() : -1;
  if (i_c2c_f >= 0) tab.push_back({"c2c_axis1_fwd", 0.0, 2.0 * n * spec_row});
  const int i_mid = (spectral && ndim >= 2) ? (int)tab.size() : -1;
  if (i_mid >= 0) tab.push_back({"mid_axis0", 0.0, (double)(n + nch) * spec_row});
  const int i_c2c_i = (spectral && ndim == 3 && !plane_inv) ? (int)tab.size() : -1;
  if (i_c2c_i >= 0) tab.push_back({"c2c_axis1_inv", 0.0, 2.0 * nch * spec_row});
  const int i_inv = (int)tab.size();
  tab.push_back({plane_inv ? "inv_plane" : "inv_x_dictionary", 0.0, inv_bytes});
  const int i_fused = fused ? (int)tab.size() : -1;
  if (fused) tab.push_back({"inv_fwd_row", 0.0, fused_bytes});

  std::vector<cudaEvent_t> ev;
  std::vector<int> which;
  cudaError_t err = cudaSuccess;
  // one launch: untimed (idx < 0 or a warm-up round) or between two new events
  auto one = [&](bool rec, int idx, auto&& go) -> cudaError_t {
    if (!rec || idx < 0) return go();
    cudaEvent_t e0, e1;
    RDCU_TRY(cudaEventCreate(&e0));
    ev.push_back(e0);
    RDCU_TRY(cudaEventCreate(&e1));
    ev.push_back(e1);
    which.push_back(idx);
    RDCU_TRY(cudaEventRecord(e0, st));
    RDCU_TRY(go());
    return cudaEventRecord(e1, st);
  };
  auto round = [&](bool rec) -> cudaError_t {
    RDCU_TRY(one(rec, 0, go_fwd));
    if (i_c2c_f >= 0) RDCU_TRY(one(rec, i_c2c_f, go_c2c_f));
    if (i_mid >= 0) RDCU_TRY(one(rec, i_mid, go_mid));
    if (i_c2c_i >= 0) RDCU_TRY(one(rec, i_c2c_i, [&]() { return go_c2c_i(-1); }));
    RDCU_TRY(one(rec, i_inv, go_inv));
    if (fused) {
      RDCU_TRY(go_fwd());
      if (i_c2c_f >= 0) RDCU_TRY(go_c2c_f());
      if (i_mid >= 0) RDCU_TRY(go_mid());
      if (i_c2c_i >= 0) RDCU_TRY(go_c2c_i(0));
      RDCU_TRY(one(rec, i_fused, [&]() { return launch_inv_fwd_row(io, *next, st); }));
    }
    return cudaSuccess;
  };
  err = round(false);
  for (int r = 0; r < reps && err == cudaSuccess; ++r) err = round(true);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  for (size_t k = 0; k < which.size() && err == cudaSuccess; ++k) {
    float ms = 0;
    err = cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]);
    tab[which[k]].ms += ms / reps;
  }
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  if (err != cudaSuccess) return err;
  *out = tab;
  return cudaSuccess;
}

bool SpectralPlan::init_linear(int n_in, int ndim_, const int* Ns_, const double* Ls_,
                               const std::vector<std::vector<ChanEntry>>& channels, std::string* msg) {
  explicit_channels_ = &channels;
  const bool ok = init(n_in, ndim_, Ns_, Ls_, std::vector<HostTerm>(), msg);
  explicit_channels_ = nullptr;
  return ok;
}

cudaError_t SpectralPlan::set_coefficients(const std::vector<double>& C) {
  std::vector<ChanEntry> ent = h_ch_ent_;
  for (size_t q = 0; q < ent.size(); ++q)
    if (h_ent_term_[q] >= 0) ent[q].coef = C[h_ent_term_[q]] * inv_n_;
  std::vector<DictTerm> dt = h_dterms_;
  for (size_t q = 0; q < dt.size(); ++q) dt[q].C = C[h_dict_term_[q]];
  if (!ent.empty()) RDCU_TRY(cudaMemcpy(ch_ent_, ent.data(), ent.size() * sizeof(ChanEntry), cudaMemcpyHostToDevice));
  if (ch_sorted_ && nch >= 1 && nch <= 4) {
    const std::vector<ChanEntry> srt = sorted_entries(ent, h_ch_off_, nch);
    RDCU_TRY(cudaMemcpy(ch_sorted_, srt.data(), srt.size() * sizeof(ChanEntry), cudaMemcpyHostToDevice));
    if (pipe_mid_) {
      std::vector<ChanEntry> grp;
      std::vector<double> A;
      operator_groups(srt, &grp, &A);
      if ((int)grp.size() != mid_ngrp_) return cudaErrorInvalidValue;
      RDCU_TRY(cudaMemcpy(mid_grp_, grp.data(), grp.size() * sizeof(ChanEntry), cudaMemcpyHostToDevice));
      RDCU_TRY(cudaMemcpy(mid_A_, A.data(), A.size() * sizeof(double), cudaMemcpyHostToDevice));
      if (mid_tab_) RDCU_TRY(build_mid_tables(grp, A));
    }
  }
  if (!dt.empty()) RDCU_TRY(cudaMemcpy(d_terms_, dt.data(), dt.size() * sizeof(DictTerm), cudaMemcpyHostToDevice));
  h_ch_ent_ = ent;
  h_dterms_ = dt;
  if (poly_nf_) {
    const std::vector<double> A = poly_table();
    RDCU_TRY(cudaMemcpy(d_poly_, A.data(), A.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  return cudaSuccess;
}

cudaError_t SpectralPlan::run_linear(const double* in, double* out, cudaStream_t st) {
  RDCU_TRY(launch_forward(in, st));
  RhsIO io{};
  io.mode = 0;
  io.y = in;
  return launch_passes(io, chan_table(ch_off_, ch_ent_, nch), h_ch_off_, nch, 0, out, nullptr, st, 1);
}

// ----------------------------------------------------------------------------- batch
struct SpectralBatch::Impl {
  int nm = 0;
  FwdXArgs* fwd[8] = {};
  MidArgs* mid[8] = {};
  InvXArgs* inv[8] = {};
  int2* items[3] = {};
  int nitems[3] = {0, 0, 0};
  // work items of one pass whose problems share a line length: [off, off + count) of items
  struct Group {
    int L = 0, rs = 0, off = 0, count = 0, grid = 0, block = 0;
    size_t smem = 0;
    const void* kern = nullptr;
  };
  std::vector<Group> groups[3];
  static constexpr int kMaxSide = 8;  // side streams of concurrent groups
  cudaStream_t side[kMaxSide] = {};
  cudaEvent_t fork = nullptr, join[kMaxSide] = {};
};

void SpectralBatch::release() {
  if (!impl_) return;
  for (int s = 0; s < 8; ++s) {
    if (impl_->fwd[s]) cudaFree(impl_->fwd[s]);
    if (impl_->mid[s]) cudaFree(impl_->mid[s]);
    if (impl_->inv[s]) cudaFree(impl_->inv[s]);
  }
  for (auto* p : impl_->items)
    if (p) cudaFree(p);
  for (int g = 0; g < Impl::kMaxSide; ++g) {
    if (impl_->side[g]) cudaStreamDestroy(impl_->side[g]);
    if (impl_->join[g]) cudaEventDestroy(impl_->join[g]);
  }
  if (impl_->fork) cudaEventDestroy(impl_->fork);
  delete impl_;
  impl_ = nullptr;
  device_bytes = 0;
}

bool SpectralBatch::init(const std::vector<BatchMember>& members, int elems_, std::string* msg) {
  release();
  impl_ = new Impl;
  Impl& B = *impl_;
  B.nm = (int)members.size();
  elems = std::max(128, std::min(elems_, kMaxElems));
  if (B.nm == 0) {
    *msg = "empty batch";
    return false;
  }
  std::vector<std::vector<FwdXArgs>> hf(8);
  std::vector<std::vector<MidArgs>> hmid(8);
  std::vector<std::vector<InvXArgs>> hi(8);
  // per pass: group key (line length, radix set) -> its items and largest block / smem
  struct Acc {
    std::vector<int2> items;
    int block = 0;
    size_t smem = 0;
  };
  std::map<std::pair<int, int>, Acc> acc[3];
  auto add = [&](int k, int L, const LinePlan& plan, int block, size_t smem, int m, int ntiles) {
    Acc& g = acc[k][{L, plan_is_pow2(plan) ? kRadixPow2 : kRadixAll}];
    g.block = std::max(g.block, block);
    g.smem = std::max(g.smem, smem);
    for (int j = 0; j < ntiles; ++j) g.items.push_back(make_int2(m, j));
  };
  // a specialised length keeps its blocks within the specialised kernels' 256 threads
  auto elems_for = [&](int L) { return length_specialised(L) ? std::min(elems, kSpecBlock * kStageElems) : elems; };
  for (int m = 0; m < B.nm; ++m) {
    const SpectralPlan& p = *members[m].plan;
    if (p.ndim != 2) {
      *msg = "batched problems must be two-dimensional";
      return false;
    }
    const int M = p.M, Mh = p.Mh, R = p.R, n = p.n, nch = p.nch;
    const bool spectral = nch > 0;
    // fwd_x tiles: P line pairs per item
    const int pairs = (n * R + 1) / 2;
    const int Pf = std::max(1, std::min(elems_for(M) / M, pairs));
    const bool ftws = (size_t)(M + Pf * M) * 16 <= kSmemBudget;
    const int gf = (pairs + Pf - 1) / Pf;
    add(0, M, p.plan_x_, std::min(kMaxBlock, std::max(128, round_up(stage_threads(p.plan_x_, Pf * M), 32))),
        spectral ? (size_t)((ftws ? M : 0) + Pf * M) * 16 : 0, m, gf);
    // mid tiles: TW columns per item, every channel at once when the plan does so
    const int L0 = p.Ns[0], I = Mh;
    const int GBp = p.mid_[0].per_cta >> 16;
    const bool sorted = p.ch_sorted_ && nch <= GBp;
    int GB = sorted ? nch : std::min(std::max(nch, 1), 4);
    int TW = std::max(1, std::min(elems_for(L0) / (std::max(n, GB) * L0), I));
    const size_t extra = (size_t)p.h_ch_off_[nch] * sizeof(ChanEntry) + (size_t)p.kv_total_ * 8 + (size_t)(nch + 2) * 4 +
                         16 + (size_t)p.h_ch_off_[nch] * (sizeof(ChanEntry) + 16 * 8);
    auto smem_of = [&](int tw_, int gb) { return (size_t)(L0 + (n + gb) * tw_ * tile_stride(L0, tw_)) * 16 + extra; };
    while (TW > 1 && (smem_of(TW, GB) > kSmemBudget || std::max(n, GB) * TW * L0 > kMaxElems)) TW /= 2;
    while (!sorted && GB > 1 && (smem_of(TW, GB) > kSmemBudget || std::max(n, GB) * TW * L0 > kMaxElems)) --GB;
    if (spectral && (smem_of(TW, GB) > 227 * 1024 || std::max(n, GB) * TW * L0 > kMaxElems)) {
      *msg = "batch member too large for the shared-memory axis-0 pass";
      return false;
    }
    const int gm = (I + TW - 1) / TW;
    if (spectral)
      add(1, L0, p.plan_ax_[0],
          std::min(kMaxBlock, std::max(128, round_up(stage_threads(p.plan_ax_[0], std::max(n, GB) * TW * L0), 32))),
          sorted && nch <= n ? (size_t)(L0 + n * TW * tile_stride(L0, TW)) * 16 + extra : smem_of(TW, GB), m, gm);
    // inv_x tiles
    PassCfg gi;
    int itws = 0;
    inv_geometry(M, R, n, nch, false, p.plan_x_, &gi, &itws, p.dict_smem_bytes(), elems_for(M));
    add(2, M, p.plan_x_, gi.block, gi.smem, m, gi.grid);
    for (int st = 1; st <= 7; ++st) {
      RhsIO io{};
      io.mode = 1;
      io.stage = st;
      io.bufs = members[m].bufs;
      io.ctl = members[m].ctl;
      io.err_part = st == 7 ? members[m].err_part : nullptr;
      FwdXArgs a{};
      a.M = M;
      a.Mh = Mh;
      a.nrows = n * R;
      a.P = Pf;
      a.do_fft = spectral ? 1 : 0;
      a.tw_smem = ftws ? 1 : 0;
      a.plan = p.plan_x_;
      a.tw = p.tw_x_;
      a.S = p.Sf_;
      a.io = io;
      prep(a);
      hf[st].push_back(a);
      MidArgs md{};
      md.L0 = L0;
      md.I = I;
      md.TW = TW;
      md.GB = GB;
      md.nsrc = n;
      md.G = nch;
      md.ch0 = 0;
      md.ndim = 2;
      md.D1 = p.Ns[1];
      md.Mh = Mh;
      md.plan = p.plan_ax_[0];
      md.tw = p.tw_ax_[0];
      md.Sf = p.Sf_;
      md.Sc = p.Sc_;
      md.chan = p.chan_table(p.ch_off_, p.ch_ent_, nch);
      md.io = io;
      md.ent0 = 0;
      md.nent = p.h_ch_off_[nch];
      if (sorted) {
        md.sorted = 1;
        md.chan.ent = p.ch_sorted_;
      }
      prep(md);
      hmid[st].push_back(md);
      InvXArgs v{};
      v.M = M;
      v.Mh = Mh;
      v.R = R;
      v.n = n;
      v.nch_run = nch;
      v.npairs = (nch + 1) / 2;
      v.do_fft = spectral ? 1 : 0;
      v.N = p.N;
      v.plan = p.plan_x_;
      v.tw = p.tw_x_;
      v.Sc = p.Sc_;
      v.dict = p.dict_table();
      v.io = io;
      v.P = gi.per_cta;
      v.tw_smem = itws;
      prep(v);
      hi[st].push_back(v);
    }
  }
  auto put = [&](auto** dst, const auto& v) -> bool {
    using T = typename std::remove_reference<decltype(v[0])>::type;
    const size_t b = std::max<size_t>(1, v.size()) * sizeof(T);
    if (cudaMalloc((void**)dst, b) != cudaSuccess) return false;
    device_bytes += b;
    return v.empty() || cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
  };
  bool ok = true;
  for (int st = 1; st <= 7; ++st) ok = ok && put(&B.fwd[st], hf[st]) && put(&B.mid[st], hmid[st]) && put(&B.inv[st], hi[st]);
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  for (int k = 0; k < 3 && ok; ++k) {
    std::vector<int2> all;
    for (auto& kv : acc[k]) {
      Impl::Group g;
      g.L = kv.first.first;
      g.rs = kv.first.second;
      g.off = (int)all.size();
      g.count = (int)kv.second.items.size();
      g.block = std::max(kv.second.block, 128);
      g.smem = kv.second.smem;
      // a block wider than the specialised kernels allow takes the plan's stages
      g.kern = group_kernel_for(k, g.block <= kSpecBlock ? g.L : 0, g.rs);
      if (!opt_in_smem(g.kern)) {
        *msg = "cannot enable large shared memory for the batched passes";
        return false;
      }
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g.kern, g.block, g.smem) != cudaSuccess ||
          per_sm < 1) {
        cudaGetLastError();
        *msg = "batched pass does not fit on an SM";
        return false;
      }
      g.grid = std::max(1, std::min(g.count, per_sm * nsm));
      all.insert(all.end(), kv.second.items.begin(), kv.second.items.end());
      B.groups[k].push_back(g);
    }
    ok = put(&B.items[k], all);
    B.nitems[k] = nitems[k] = (int)all.size();
  }
  if (!ok) {
    *msg = "out of device memory (batch tables)";
    return false;
  }
  // side streams and events of the concurrent groups
  if (cudaEventCreateWithFlags(&B.fork, cudaEventDisableTiming) != cudaSuccess) {
    *msg = "cannot create events";
    return false;
  }
  for (int g = 0; g < Impl::kMaxSide; ++g)
    if (cudaStreamCreateWithFlags(&B.side[g], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&B.join[g], cudaEventDisableTiming) != cudaSuccess) {
      *msg = "cannot create streams";
      return false;
    }
  return true;
}

cudaError_t SpectralBatch::launch_stage(int stage, cudaStream_t st) {
  Impl& B = *impl_;
  if (stage < 1 || stage > 7) return cudaErrorInvalidValue;
  const void* args[3] = {B.fwd[stage], B.mid[stage], B.inv[stage]};
  for (int k = 0; k < 3; ++k) {
    const std::vector<Impl::Group>& G = B.groups[k];
    if (G.empty()) continue;
    auto launch = [&](const Impl::Group& g, cudaStream_t s) {
      const void* a = args[k];
      const int2* items = B.items[k] + g.off;
      int cnt = g.count;
      void* params[3] = {(void*)&a, (void*)&items, (void*)&cnt};
      return cudaLaunchKernel(g.kern, dim3(g.grid), dim3(g.block), params, g.smem, s);
    };
    // group 0 on the stream, the others on side streams forked from it and joined back
    const int nside = std::min((int)G.size() - 1, (int)Impl::kMaxSide);
    if (nside > 0) RDCU_TRY(cudaEventRecord(B.fork, st));
    for (int i = 0; i < nside; ++i) RDCU_TRY(cudaStreamWaitEvent(B.side[i], B.fork, 0));
    for (size_t gi = 1; gi < G.size(); ++gi) RDCU_TRY(launch(G[gi], B.side[(gi - 1) % Impl::kMaxSide]));
    RDCU_TRY(launch(G[0], st));
    for (int i = 0; i < nside; ++i) {
      RDCU_TRY(cudaEventRecord(B.join[i], B.side[i]));
      RDCU_TRY(cudaStreamWaitEvent(st, B.join[i], 0));
    }
  }
  return cudaGetLastError();
}

}  // namespace rdcu
