// Allocation-free entry point for the excluded / modified (1-4) pair
// corrections: nbk_exclusion_force_noalloc (declared in include/nbk.h).
//
// Some callers cannot call cudaMalloc: code running inside a host framework
// that owns every device allocation through its own pool, callers that must
// not touch the allocator between two captured regions, and embedded runtimes
// whose device heap is fixed at start-up. For them this entry point takes no
// handle and allocates nothing. Its scratch memory -- the 64-bit fixed-point
// force accumulators, the energy/virial accumulators and a staging copy of the
// tuples -- lives in the file-scope device array below, sized for at most
// kNoAllocMaxSlots atom slots and kNoAllocMaxTuples tuples. Every GPU that
// loads this library holds that array (about 11 MB) until the process exits.
//
// The array's host-side name is only a stand-in, not a device address: the
// kernels receive the address that cudaGetSymbolAddress returns for the
// current device, looked up once per device on the first call made with that
// device current (so make that first call before any stream capture).
//
// All calls share the one array: a call clears the parts it uses before its
// kernels run, and calls whose work overlaps on the GPU (different streams,
// different host threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "nbk.h"
#include "nbk_internal.cuh"
#include "nbk_launch.h"

using namespace nbk;

namespace {

constexpr int kNoAllocMaxSlots = 65536;
constexpr int kNoAllocMaxTuples = 4 * kNoAllocMaxSlots;
constexpr int kMaxDevices = 64;

// [6 * kNoAllocMaxSlots] force accumulators, [kAccCount] energy/virial
// accumulators, then the tuple staging area; 8-byte words throughout.
constexpr size_t kForceWords = 6 * (size_t)kNoAllocMaxSlots;
constexpr size_t kTupleWords = (size_t)kNoAllocMaxTuples * sizeof(nbk_exclusion) / 8;
constexpr size_t kScratchWords = kForceWords + kAccCount + kTupleWords;

static __device__ __align__(256) long long g_noallocScratch[kScratchWords];

std::mutex g_setupMutex;
long long* g_scratchPtr[kMaxDevices] = {};

thread_local std::string g_noallocErr;

int fail(int code, const std::string& msg) {
  g_noallocErr = msg;
  return code;
}

// Device address of the scratch array on the current device (looked up once).
int scratchFor(int device, long long** out) {
  if (device < 0 || device >= kMaxDevices) return fail(NBK_ERR_DEVICE, "device index out of range");
  std::lock_guard<std::mutex> lock(g_setupMutex);
  if (!g_scratchPtr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
    if (e != cudaSuccess)
      return fail(NBK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratchPtr[device] = static_cast<long long*>(p);
  }
  *out = g_scratchPtr[device];
  return NBK_OK;
}

}  // namespace

extern "C" NBK_API const char* nbk_noalloc_last_error(void) { return g_noallocErr.c_str(); }

extern "C" NBK_API int nbk_exclusion_force_noalloc(
    const nbk_params* params, const float* d_ljExclTable, int ljDim, int atomStorageSize,
    const nbk_float4* d_xyzq, int numModified, const nbk_exclusion* h_modified, int numExcluded,
    const nbk_exclusion* h_excluded, nbk_float3 lata, nbk_float3 latb, nbk_float3 latc,
    unsigned flags, nbk_float4* d_forces, nbk_float4* d_forcesSlow, nbk_virial_energy* d_ve,
    void* stream) {
  if (!params || !d_ljExclTable || !d_xyzq || !d_forces)
    return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: NULL argument");
  if (flags & ~(unsigned)(NBK_ENERGY | NBK_VIRIAL | NBK_SLOW))
    return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: only NBK_ENERGY, NBK_VIRIAL and NBK_SLOW apply");
  if ((flags & NBK_SLOW) && !d_forcesSlow)
    return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: NBK_SLOW needs d_forcesSlow");
  if ((flags & (NBK_ENERGY | NBK_VIRIAL)) && !d_ve)
    return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: energies/virials need d_ve");
  if (atomStorageSize <= 0 || atomStorageSize > kNoAllocMaxSlots)
    return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: atomStorageSize must be in 1.." +
                                 std::to_string(kNoAllocMaxSlots) + " (the static scratch limit)");
  // each count on its own, then the sum in 64 bits, so no overflow can pass
  if (numModified < 0 || numExcluded < 0 || numModified > kNoAllocMaxTuples ||
      numExcluded > kNoAllocMaxTuples ||
      (long long)numModified + (long long)numExcluded > (long long)kNoAllocMaxTuples)
    return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: more than " +
                                 std::to_string(kNoAllocMaxTuples) +
                                 " tuples (the static scratch limit)");
  if ((numModified && !h_modified) || (numExcluded && !h_excluded))
    return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: NULL tuple array");
  const int dim = ljDim;
  if (dim <= 0) return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: ljDim must be positive");
  if (!(params->cutoff > 0) || params->switchdist <= 0)
    return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: need 0 < switchdist, 0 < cutoff");
  for (int k = 0; k < numModified; ++k) {
    const nbk_exclusion& e = h_modified[k];
    if (e.pswitch || e.i < 0 || e.j < 0 || e.i >= atomStorageSize || e.j >= atomStorageSize ||
        e.vdwtypei < 0 || e.vdwtypei >= dim || e.vdwtypej < 0 || e.vdwtypej >= dim)
      return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: bad modified tuple " + std::to_string(k));
  }
  for (int k = 0; k < numExcluded; ++k) {
    const nbk_exclusion& e = h_excluded[k];
    if (e.pswitch || e.i < 0 || e.j < 0 || e.i >= atomStorageSize || e.j >= atomStorageSize)
      return fail(NBK_ERR_ARG, "nbk_exclusion_force_noalloc: bad excluded tuple " + std::to_string(k));
  }
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return fail(NBK_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  long long* scratch = nullptr;
  int rc = scratchFor(device, &scratch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = atomStorageSize;
  long long* force = scratch;
  long long* acc = scratch + kForceWords;
  nbk_exclusion* tuples = reinterpret_cast<nbk_exclusion*>(acc + kAccCount);
  // clear what must start at zero: the force and energy/virial accumulators
  e = cudaMemsetAsync(force, 0, sizeof(long long) * 6 * (size_t)n, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, sizeof(long long) * kAccCount, st);
  if (e == cudaSuccess && numModified)
    e = cudaMemcpyAsync(tuples, h_modified, sizeof(nbk_exclusion) * numModified,
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && numExcluded)
    e = cudaMemcpyAsync(tuples + numModified, h_excluded, sizeof(nbk_exclusion) * numExcluded,
                        cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return fail(NBK_ERR_CUDA, std::string("staging: ") + cudaGetErrorString(e));
  CorrArgs ca{};
  ca.modified = tuples;
  ca.numModified = numModified;
  ca.excluded = tuples + numModified;
  ca.numExcluded = numExcluded;
  ca.xyzq = reinterpret_cast<const float4*>(d_xyzq);
  ca.ljExclTable = reinterpret_cast<const float2*>(d_ljExclTable);
  ca.lata = make_float3(lata.x, lata.y, lata.z);
  ca.latb = make_float3(latb.x, latb.y, latb.z);
  ca.latc = make_float3(latc.x, latc.y, latc.z);
  makeConstants(*params, dim, ca.c, ca.c64);
  ca.force = force;
  ca.stride = n;
  ca.acc = acc;
  int numSM = 148;
  cudaDeviceGetAttribute(&numSM, cudaDevAttrMultiProcessorCount, device);
  e = launchCorrections(ca, flags, st);
  if (e == cudaSuccess)
    e = launchFinalizeForces(n, force, n, ca.xyzq, reinterpret_cast<float4*>(d_forces),
                             (flags & NBK_SLOW) ? reinterpret_cast<float4*>(d_forcesSlow) : nullptr,
                             flags, acc, numSM, st);
  if (e == cudaSuccess && (flags & (NBK_ENERGY | NBK_VIRIAL))) e = launchEnergyVirial(acc, d_ve, st);
  if (e != cudaSuccess) return fail(NBK_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return NBK_OK;
}
