// Shared-memory FP64 Stockham FFT over a batch of complex lines (device code).
//
// Method: the Stockham autosort formulation (Van Loan, "Computational Frameworks for
// the Fast Fourier Transform", SIAM 1992, ch. 1.7) with mixed radices 2, 3, 4, 5, 7, 8,
// 11, 13.  Stage s with radix R and span Ns (product of earlier radices) maps butterfly
// j of a line of length L (m = L/R butterflies) as
//     in:  x[j + r*m] * w^(r * (j mod Ns) * L/(Ns*R)),   r < R
//     out: y[(j/Ns)*Ns*R + (j mod Ns) + r*Ns]  = R-point DFT of the inputs,
// which leaves the result in natural order.  Twiddles w^t = exp(-2 pi i t/L) come from
// a table in shared memory.  Each stage stages its butterflies in registers, so one
// buffer suffices (two barriers per stage).
#pragma once
#include <cuda_runtime.h>

#include "internal.h"

namespace rdcu {

__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ double2 c_rot(double2 a) {
  return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ double2 tw_get(const double2* tw, int t) {
  double2 w = tw[t];
  if (INV) w.y = -w.y;
  return w;
}

// 16-byte asynchronous global->shared copy (zero-filled when pred is false; the source
// address is then not read).  Completion: cp_async_wait_all() and a barrier.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// commit the copies issued so far as a group; wait until at most one group is pending
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// In-register R-point DFT of v (forward: exp(-2 pi i rk/R); inverse: conjugate).
template <int R, bool INV>
struct Dft {
  __device__ __forceinline__ static void run(double2 (&v)[R], const double2* tw, int L) {
    // generic small prime: O(R^2) with the line's twiddle table (R divides L)
    double2 out[R];
    const int step = L / R;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      double2 acc = v[0];
#pragma unroll
      for (int r = 1; r < R; ++r) acc = c_add(acc, c_mul(v[r], tw_get<INV>(tw, ((r * k) % R) * step)));
      out[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = out[k];
  }
};

template <bool INV>
struct Dft<2, INV> {
  __device__ __forceinline__ static void run(double2 (&v)[2], const double2*, int) {
    double2 a = v[0], b = v[1];
    v[0] = c_add(a, b);
    v[1] = c_sub(a, b);
  }
};

template <bool INV>
struct Dft<4, INV> {
  __device__ __forceinline__ static void run(double2 (&v)[4], const double2*, int) {
    double2 t0 = c_add(v[0], v[2]), t1 = c_sub(v[0], v[2]);
    double2 t2 = c_add(v[1], v[3]), t3 = c_rot<INV>(c_sub(v[1], v[3]));
    v[0] = c_add(t0, t2);
    v[2] = c_sub(t0, t2);
    v[1] = c_add(t1, t3);
    v[3] = c_sub(t1, t3);
  }
};

template <bool INV>
struct Dft<8, INV> {
  __device__ __forceinline__ static void run(double2 (&v)[8], const double2*, int) {
    // X[k] = E[k] + W^k O[k], X[k+4] = E[k] - W^k O[k]; E, O = 4-point DFTs of the
    // even and odd inputs; W = exp(-+ 2 pi i / 8).
    double2 e[4] = {v[0], v[2], v[4], v[6]};
    double2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, INV>::run(e, nullptr, 0);
    Dft<4, INV>::run(o, nullptr, 0);
    const double s = 0.70710678118654752440;  // sqrt(1/2)
    // W^1 = s(1 -+ i), W^2 = -+ i, W^3 = s(-1 -+ i)
    double2 w1o = INV ? make_double2(s * (o[1].x - o[1].y), s * (o[1].x + o[1].y))
                      : make_double2(s * (o[1].x + o[1].y), s * (o[1].y - o[1].x));
    double2 w2o = c_rot<INV>(o[2]);
    double2 w3o = INV ? make_double2(-s * (o[3].x + o[3].y), s * (o[3].x - o[3].y))
                      : make_double2(s * (o[3].y - o[3].x), -s * (o[3].x + o[3].y));
    v[0] = c_add(e[0], o[0]);
    v[4] = c_sub(e[0], o[0]);
    v[1] = c_add(e[1], w1o);
    v[5] = c_sub(e[1], w1o);
    v[2] = c_add(e[2], w2o);
    v[6] = c_sub(e[2], w2o);
    v[3] = c_add(e[3], w3o);
    v[7] = c_sub(e[3], w3o);
  }
};

// Complex values a thread holds per stage (register budget of the staging), and the
// largest block of an FFT pass (kMaxBlock x 128 registers fills the register file).
constexpr int kStageElems = 8;
constexpr int kMaxBlock = 512;

// Position of line element i under the swizzle of a radix-8 first stage: the low three
// bits are XORed with the 8-element block index, so the eight consecutive outputs of a
// butterfly land in eight different bank groups across a quarter warp.
__device__ __forceinline__ int swz8(int i) { return i ^ ((i >> 3) & 7); }

// One Stockham stage over nlines lines (stride LS) held in shared memory `buf`.
// Requires blockDim.x * QMAX >= nlines*L/R; the caller sizes the block for that.
// POW2: L and Ns are powers of two (index arithmetic by shifts); otherwise the
// plan's precomputed invariant divisors are used.
// SWZ: bit 0 writes the outputs at swz8 positions (a first stage, Ns = 1, R = 8: its
// stride-8 stores otherwise put a quarter warp on one bank group); bit 1 reads the
// inputs from swz8 positions (the stage after it).  twz: the twiddle table is stored at
// swz8 positions (the span-8 stage reads twiddles r*kk*L/64 for kk = 0..7, which
// otherwise share a bank group).  Values are unchanged.
template <int R, bool INV, bool POW2, int SWZ = 0>
__device__ __forceinline__ void stockham_stage(double2* buf, int LS, int nlines, int L, int Ns, FastDiv dm,
                                               FastDiv dns, const double2* tw, bool twz = false) {
  constexpr int QMAX = (R >= kStageElems) ? 1 : (kStageElems / R);
  const int m = L / R;
  const int nb = nlines * m;
  const int T = blockDim.x;
  const int tstride = L / (Ns * R);
  const int lm = POW2 ? __ffs(m) - 1 : 0;
  const int lns = POW2 ? __ffs(Ns) - 1 : 0;
  double2 v[QMAX][R];
  int dst[QMAX], dbase[QMAX];
#pragma unroll
  for (int q = 0; q < QMAX; ++q) {
    const int g = threadIdx.x + q * T;
    dst[q] = -1;
    dbase[q] = 0;
    if (g < nb) {
      const int line = POW2 ? (g >> lm) : fdiv(g, dm);
      const int j = g - line * m;
      const int jd = POW2 ? (j >> lns) : fdiv(j, dns);
      const int kk = j - jd * Ns;
      const double2* src = buf + line * LS;
      const int tstep = kk * tstride;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        double2 x = src[(SWZ & 2) ? swz8(j + r * m) : j + r * m];
        if (r > 0 && tstep != 0) x = c_mul(x, tw_get<INV>(tw, twz ? swz8(r * tstep) : r * tstep));
        v[q][r] = x;
      }
      Dft<R, INV>::run(v[q], tw, L);
      dbase[q] = line * LS;
      dst[q] = jd * Ns * R + kk;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < QMAX; ++q) {
    if (dst[q] >= 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) buf[dbase[q] + ((SWZ & 1) ? swz8(dst[q] + r * Ns) : dst[q] + r * Ns)] = v[q][r];
    }
  }
  __syncthreads();
}

// A stage of the runtime-planned transform as a called function: the plan's stage loop
// then holds one stage's registers at a time (inlined, the union of every radix's
// registers exceeds the budget and spills).
template <int R, bool INV, bool POW2>
__device__ __noinline__ void stockham_stage_call(double2* buf, int LS, int nlines, int L, int Ns, FastDiv dm,
                                                 FastDiv dns, const double2* tw) {
  stockham_stage<R, INV, POW2>(buf, LS, nlines, L, Ns, dm, dns, tw);
}

// Radix sets a kernel is compiled for: power-of-two lengths use radices 8, 4, 2 only
// (no register spills); any other supported length uses the general set.
constexpr int kRadixPow2 = 0;
constexpr int kRadixAll = 1;

inline bool plan_is_pow2(const LinePlan& p) {
  for (int s = 0; s < p.nstages; ++s)
    if (p.radix[s] != 2 && p.radix[s] != 4 && p.radix[s] != 8) return false;
  return true;
}

// Full transform of nlines lines.  All threads of the block must call it; the data
// must be visible (a barrier before the call).  Returns after a barrier.
template <int RS, bool INV>
__device__ void fft_lines(double2* buf, int LS, int nlines, const LinePlan& p, const double2* tw) {
  int Ns = 1;
  for (int s = 0; s < p.nstages; ++s) {
    const int R = p.radix[s];
    const FastDiv dm = p.div_m[s], dns = p.div_ns[s];
    if (RS == kRadixPow2) {
      if (R == 8)
        stockham_stage_call<8, INV, true>(buf, LS, nlines, p.L, Ns, dm, dns, tw);
      else if (R == 4)
        stockham_stage_call<4, INV, true>(buf, LS, nlines, p.L, Ns, dm, dns, tw);
      else
        stockham_stage_call<2, INV, true>(buf, LS, nlines, p.L, Ns, dm, dns, tw);
    } else {
      switch (R) {
        case 2: stockham_stage_call<2, INV, false>(buf, LS, nlines, p.L, Ns, dm, dns, tw); break;
        case 3: stockham_stage_call<3, INV, false>(buf, LS, nlines, p.L, Ns, dm, dns, tw); break;
        case 4: stockham_stage_call<4, INV, false>(buf, LS, nlines, p.L, Ns, dm, dns, tw); break;
        case 5: stockham_stage_call<5, INV, false>(buf, LS, nlines, p.L, Ns, dm, dns, tw); break;
        case 7: stockham_stage_call<7, INV, false>(buf, LS, nlines, p.L, Ns, dm, dns, tw); break;
        case 8: stockham_stage_call<8, INV, false>(buf, LS, nlines, p.L, Ns, dm, dns, tw); break;
        case 11: stockham_stage_call<11, INV, false>(buf, LS, nlines, p.L, Ns, dm, dns, tw); break;
        case 13: stockham_stage_call<13, INV, false>(buf, LS, nlines, p.L, Ns, dm, dns, tw); break;
        default: break;  // plans only contain the radices above
      }
    }
    Ns *= R;
  }
}

// The same transform for a power-of-two length L known at compile time: the stage
// sequence of make_line_plan (radix 8 while 8 divides what is left, then 4 or 2) with
// every length, span and stride a constant.  Bitwise equal to fft_lines on that plan.
template <int L, bool INV, int NS = 1>
__device__ __forceinline__ void fft_pow2_t(double2* buf, int LS, int nlines, const double2* tw, bool twz) {
  if constexpr (NS < L) {
    constexpr int REM = L / NS;
    constexpr int R = (REM % 8 == 0) ? 8 : REM;  // REM is 8^a times 1, 2 or 4
    static_assert(R == 2 || R == 4 || R == 8, "power-of-two lengths only");
    // a radix-8 first stage writes swizzled when a second stage reads it back
    constexpr int SWZ = (NS == 1 && R == 8 && L > 8) ? 1 : (NS == 8 ? 2 : 0);
    stockham_stage<R, INV, true, SWZ>(buf, LS, nlines, L, NS, FastDiv{}, FastDiv{}, tw, twz);
    fft_pow2_t<L, INV, NS * R>(buf, LS, nlines, tw, twz);
  }
}

// Radix of the next stage when `rem` points of the line remain to be factored, in
// make_line_plan's order (all 8s, then 4s, 2s, 3s, 5s, 7s, 11s, 13s).
__host__ __device__ constexpr int plan_radix(int rem) {
  return rem % 8 == 0 ? 8 : rem % 4 == 0 ? 4 : rem % 2 == 0 ? 2 : rem % 3 == 0 ? 3 : rem % 5 == 0 ? 5
         : rem % 7 == 0 ? 7 : rem % 11 == 0 ? 11 : 13;
}

// The transform for any supported length L known at compile time (the plan's stage
// sequence, constant spans and divisors; bitwise equal to fft_lines on that plan).  A
// radix-8 first stage writes swizzled for the stage after it; twiddles are read plainly.
template <int L, bool INV, int NS = 1>
__device__ __forceinline__ void fft_fixed_t(double2* buf, int LS, int nlines, const double2* tw) {
  if constexpr (NS < L) {
    constexpr int R = plan_radix(L / NS);
    constexpr int R0 = plan_radix(L);
    constexpr int SWZ = (NS == 1 && R == 8 && L > 8) ? 1 : (NS == 8 && R0 == 8 ? 2 : 0);
    stockham_stage<R, INV, false, SWZ>(buf, LS, nlines, L, NS, make_fastdiv_c(L / R), make_fastdiv_c(NS), tw);
    fft_fixed_t<L, INV, NS * R>(buf, LS, nlines, tw);
  }
}

}  // namespace rdcu
