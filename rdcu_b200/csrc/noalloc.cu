// Allocation-free pseudospectral RHS (rdcu_rhs_noalloc in include/rdcu.h).
//
// The same fused passes as rdcu_rhs, with the plan's device memory carved from one
// file-scope __device__ array instead of cudaMalloc.  Host code must not take the
// array's address directly (in host code its name is a host-side stand-in, not a device
// address); the device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, and cached.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/rdcu.h"
#include "internal.h"
#include "spectral.h"

namespace {

__device__ __align__(256) unsigned char g_rhs_scratch[RDCU_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

int fail(int code, const std::string& msg) {
  rdcu::set_thread_error(msg);
  return code;
}

// Device address of g_rhs_scratch on the current device (looked up once per device).
cudaError_t scratch_address(int dev, void** out) {
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_rhs_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

// Makes `dev` current for the call and puts the caller's current device back on every
// return path (callers embedded in another framework keep their device selection).
struct DeviceGuard {
  int prev = -1;
  cudaError_t set(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    return cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int rdcu_rhs_noalloc(const rdcu_spec* spec, const double* y, double* f, void* stream) {
  if (!spec || !y || !f) return fail(RDCU_ERR_INVALID, "null argument");
  if (spec->method != RDCU_METHOD_DP45)
    return fail(RDCU_ERR_UNSUPPORTED, "rdcu_rhs_noalloc evaluates pseudospectral (DP45) problems only");
  if (spec->n < 1 || spec->ndim < 1 || spec->ndim > 3) return fail(RDCU_ERR_INVALID, "bad n or ndim");
  if (spec->device < 0 || spec->device >= kMaxDevices) return fail(RDCU_ERR_INVALID, "bad device ordinal");
  for (int a = 0; a < spec->ndim; ++a)
    if (spec->Ns[a] < 1 || !(spec->Ls[a] > 0 || spec->Ls[a] < 0))
      return fail(RDCU_ERR_INVALID, "bad grid size or length");
  if (spec->nterms < 0 || (spec->nterms > 0 && (!spec->C || !spec->nprods || !spec->c)))
    return fail(RDCU_ERR_INVALID, "bad coupling-term arrays");
  const int nY = 1 + spec->ndim + spec->ndim * spec->ndim;
  std::vector<rdcu::HostTerm> terms;
  for (int i = 0; i < spec->nterms; ++i) {
    rdcu::HostTerm t;
    t.C = spec->C[i];
    const int np = spec->nprods[i];
    if (np < 0 || (np > 0 && !spec->c[i])) return fail(RDCU_ERR_INVALID, "bad coupling term list");
    t.ints.assign(spec->c[i], spec->c[i] + np);
    const int field = np > 0 ? t.ints[0] : 0;
    if (field < 0 || field >= spec->n) return fail(RDCU_ERR_INVALID, "coupling term field out of range");
    for (int j = 1; j < np; j += 2)
      if (t.ints[j] < 0 || t.ints[j] >= nY * spec->n) return fail(RDCU_ERR_INVALID, "coupling term Y index out of range");
    terms.push_back(std::move(t));
  }
  DeviceGuard dg;
  cudaError_t e = dg.set(spec->device);
  if (e != cudaSuccess) return fail(RDCU_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  if (!on_device(y) || !on_device(f)) return fail(RDCU_ERR_INVALID, "y and f must be device pointers");
  void* base = nullptr;
  e = scratch_address(spec->device, &base);
  if (e != cudaSuccess) return fail(RDCU_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  rdcu::PlanArena arena;
  arena.base = static_cast<char*>(base);
  arena.size = RDCU_NOALLOC_SCRATCH_BYTES;
  arena.stream = st;
  rdcu::SpectralPlan plan;
  std::string msg;
  if (!plan.init_in_arena(spec->n, spec->ndim, spec->Ns, spec->Ls, terms, &arena, &msg)) {
    if (msg.find("memory") != std::string::npos)
      return fail(RDCU_ERR_UNSUPPORTED,
                  "problem needs more than the " + std::to_string(RDCU_NOALLOC_SCRATCH_BYTES >> 20) +
                      " MiB of scratch the allocation-free entry point has");
    return fail(RDCU_ERR_UNSUPPORTED, msg);
  }
  rdcu::RhsIO io{};
  io.mode = 0;
  io.y = y;
  io.f = f;
  e = plan.run(io, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(RDCU_ERR_CUDA, std::string("rdcu_rhs_noalloc: ") + cudaGetErrorString(e));
  return RDCU_OK;
}
