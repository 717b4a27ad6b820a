// Strided-axis passes of 3D grids on TMA tiles, and warp-per-line transforms (device code).
//
// A tile is a box of 8 consecutive columns (16-byte complex values) by one whole line
// of the transformed axis, moved between global and shared memory by the tensor memory
// accelerator (cp.async.bulk.tensor) with the 128-byte swizzle: row z of the box is 128
// bytes, and column c of it sits at byte z*128 + ((c ^ (z & 7)) << 4) from the box base
// (1024-byte aligned).  Each CTA is persistent and keeps a ring of three tile buffers:
// while one tile is transformed, the stores of the one before leave from its buffer and
// the loads of the one after complete on an mbarrier; results leave by TMA stores from
// the buffer they were computed in.
//
// Each line is transformed by one warp (256 points) or one half warp (128 points), its
// eight values per lane held in registers; the Stockham stages of the plan (8, 8, then
// 4 or 2: make_line_plan's sequence for these lengths) exchange through the line's own
// storage (a column of a tile, or a contiguous line), in the same element order and with
// the same arithmetic as fft_pow2_t, so results are bitwise those of the shared-memory
// line kernels.  Every 8-lane phase of an exchange touches 8 different 16-byte bank
// groups (under the tile swizzle, or the swz8 placement of a contiguous line): no bank
// conflicts.  Twiddles live in registers.
//
// Waits are bounded: a wait that does not complete within kWaitNs sets the pass's
// error word and the kernel returns (after waiting, again bounded, for its own copies).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fft_line.cuh"

namespace rdcu {

constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s
constexpr int kPipeErrTimeout = 1;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of `parity` to complete; false after kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_test(bar, parity))
    if (global_ns() - t0 > kWaitNs) return false;
  return true;
}

// Generic-proxy writes to shared memory become visible to the async proxy (TMA store).
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tma_prefetch(const CUtensorMap* m) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(m)) : "memory");
}
// 2D / 3D tile loads completing on `bar` (no multicast: the tensor maps cover this GPU's
// own buffers) and stores from shared memory (bulk group of the issuing thread).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* m, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* m, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// Plain bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from
// global to shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* m, int x, int y, const void* src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(m)),
               "r"(x), "r"(y), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* m, int x, int y, int z, const void* src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                   reinterpret_cast<uint64_t>(m)),
               "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the stores issued so far have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// every store group but the most recent one has finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
// ... and have completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Column c of a swizzled 128-byte-row box: row z.
__device__ __forceinline__ double2* swz_col(char* box, int c, int z) {
  return reinterpret_cast<double2*>(box + (z << 7) + (((c ^ z) & 7) << 4));
}

// One line of length L (128 or 256) per L/8 lanes; lane `ml` of the line holds values
// ml + (L/8) p, p < 8, in v[p] before and after a transform.
template <int L>
struct WarpLine {
  static_assert(L == 128 || L == 256, "128- and 256-point lines");
  static constexpr int LPL = L / 8;   // lanes per line
  static constexpr int R3 = L / 64;   // radix of the last stage
  static constexpr int QB3 = 8 / R3;  // last-stage butterflies per lane
  static constexpr int TS2 = L / 64;  // twiddle stride of stage 2 (span 8, radix 8)
  double2 w2[7];
  double2 w3[QB3][R3 - 1];
  int ml;

  // twiddles of this lane's butterflies (the plan's table, exp(-2 pi i t / L))
  __device__ __forceinline__ void init(const double2* tw, int ml_) {
    ml = ml_;
    const int kk2 = ml & 7;
#pragma unroll
    for (int r = 1; r < 8; ++r) w2[r - 1] = __ldg(&tw[r * kk2 * TS2]);
#pragma unroll
    for (int q = 0; q < QB3; ++q) {
      const int j = ml + LPL * q;
#pragma unroll
      for (int r = 1; r < R3; ++r) w3[q][r - 1] = __ldg(&tw[r * j]);
    }
  }

  template <bool INV>
  __device__ __forceinline__ static double2 twid(double2 x, double2 w) {
    if (INV) w.y = -w.y;
    return c_mul(x, w);
  }

  // Transform of v (natural order in, natural order out) using the line's storage as
  // the exchange space: at(e) is the address of line element e.  The storage is
  // overwritten.  Lanes of a line must have finished reading it before the call (the
  // first stage writes it).
  template <bool INV, typename At>
  __device__ __forceinline__ void transform(double2 (&v)[8], At at) const {
    // stage 1: radix 8, span 1: inputs v[r] = x[ml + LPL r]; outputs 8 ml + r, swizzled
    Dft<8, INV>::run(v, nullptr, 0);
#pragma unroll
    for (int r = 0; r < 8; ++r) *at(swz8(8 * ml + r)) = v[r];
    __syncwarp();
    // stage 2: radix 8, span 8: inputs ml + LPL r (swizzled), twiddles r * (ml % 8) * L/64
    {
      const bool tw_on = (ml & 7) != 0;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        double2 x = *at(swz8(ml + LPL * r));
        if (r > 0 && tw_on) x = twid<INV>(x, w2[r - 1]);
        v[r] = x;
      }
      Dft<8, INV>::run(v, nullptr, 0);
      __syncwarp();
      const int d0 = (ml >> 3) * 64 + (ml & 7);
#pragma unroll
      for (int r = 0; r < 8; ++r) *at(d0 + 8 * r) = v[r];
      __syncwarp();
    }
    // stage 3: radix R3, span 64: butterfly j = ml + LPL q reads j + 64 r
    double2 t[QB3][R3];
#pragma unroll
    for (int q = 0; q < QB3; ++q) {
      const int j = ml + LPL * q;
#pragma unroll
      for (int r = 0; r < R3; ++r) {
        double2 x = *at(j + 64 * r);
        if (r > 0 && j != 0) x = twid<INV>(x, w3[q][r - 1]);
        t[q][r] = x;
      }
      Dft<R3, INV>::run(t[q], nullptr, 0);
    }
    // output j + 64 r = ml + LPL (q + QB3 r)
#pragma unroll
    for (int q = 0; q < QB3; ++q)
#pragma unroll
      for (int r = 0; r < R3; ++r) v[q + QB3 * r] = t[q][r];
    __syncwarp();  // later writes to the line come after every lane's stage-3 reads
  }

  // column c of a swizzled 128-byte-row box
  template <bool INV>
  __device__ __forceinline__ void transform(double2 (&v)[8], char* box, int c) const {
    transform<INV>(v, [box, c](int e) { return swz_col(box, c, e); });
  }
  __device__ __forceinline__ void load(double2 (&v)[8], char* box, int c) const {
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = *swz_col(box, c, ml + LPL * p);
    __syncwarp();
  }
  __device__ __forceinline__ void store(const double2 (&v)[8], char* box, int c) const {
#pragma unroll
    for (int p = 0; p < 8; ++p) *swz_col(box, c, ml + LPL * p) = v[p];
  }
};

}  // namespace rdcu
