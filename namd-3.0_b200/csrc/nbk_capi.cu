// C-ABI of the B200 nonbonded path (include/nbk.h): handle, device buffers and
// the call sequence that mirrors CudaTileListKernel / CudaComputeNonbondedKernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "nbk.h"
#include "nbk_internal.cuh"
#include "nbk_launch.h"

using namespace nbk;

// Strides the reference's arrays of these records have (CUDA's int2 and
// float4 are 8- and 16-byte aligned), so its buffers pass through unchanged.
static_assert(sizeof(nbk_compute_record) == 24, "CudaComputeRecord is 24 bytes");
static_assert(sizeof(nbk_tile_list) == 48, "TileList is 48 bytes");
static_assert(sizeof(nbk_patch_record) == 16, "CudaPatchRecord (with patchID) is 16 bytes");
static_assert(sizeof(nbk_tile_excl) == 128, "TileExcl is 128 bytes");
static_assert(sizeof(nbk_exclusion) == 32, "CudaExclusion is 32 bytes");
static_assert(sizeof(nbk_virial_energy) == sizeof(double) * 31, "VirialEnergy is 31 doubles");
static_assert(sizeof(nbk_local_record) == 128, "CudaLocalRecord is 128 bytes");

namespace {

thread_local std::string g_err;

int setErr(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// A failed CUDA call becomes NBK_ERR_NOMEM when it was an allocation that
// ran out of memory, else NBK_ERR_CUDA.
#define NBK_CUDA(call, what)                                                              \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return setErr(e_ == cudaErrorMemoryAllocation ? NBK_ERR_NOMEM : NBK_ERR_CUDA,       \
                    std::string(what) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

// Allocation-failure injection for tests (nbk_debug_fail_alloc): when > 0,
// counts down on every device allocation of a handle's buffers, and the
// allocation that takes it to 0 fails as an out-of-memory cudaMalloc would.
std::atomic<int> g_failAllocCountdown{0};

// Grow-only device buffer (over-allocates by 20% like the reference's
// reallocate_device with OVERALLOC, src/CudaTileListKernel.cu:30).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    int c = g_failAllocCountdown.load();
    while (c > 0 && !g_failAllocCountdown.compare_exchange_weak(c, c - 1)) {
    }
    if (c == 1) return cudaErrorMemoryAllocation;
    const size_t want = std::max<size_t>(n + n / 5, 32);
    cudaError_t e = cudaMalloc(&p, want * sizeof(T));
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace

struct nbk_context {
  int device = 0;
  int numSM = 148;
  nbk_params prm{};
  NbkConst c{};
  NbkConst64 c64{};
  int ljDim = 0;
  DBuf<float2> ljTable, ljExclTable;
  DBuf<double2> slowTable;  // FP64 phi_s rows (buildSlowTable)
  int slowTableRows = 0;
  double slowStep = 2.0;
  DBuf<unsigned> exclBits;
  int numExclWords = 0;
  // set-up data
  std::vector<nbk_compute_record> hComputes;
  DBuf<nbk_compute_record> computes;
  int numComputes = 0;
  DBuf<int> vdwTypes, atomIndex;
  DBuf<int2> exclIndexMaxDiff;
  DBuf<int2> exclByAtom;  // GPU-resident marshaling: (maxdiff, base) per global atom id
  int numExclByAtom = 0;
  int atomDataSize = 0;
  // positions
  DBuf<float4> xyzqOwn;
  const float4* xyzq = nullptr;
  int atomStorageSize = 0;
  // tile lists: sparse build output
  std::vector<nbk_patch_record> hPatches;
  DBuf<nbk_patch_record> patches;
  int numPatches = 0;
  std::vector<ListSeed> hSeeds;
  DBuf<ListSeed> seeds;
  int numLists = 0;
  int jcap = 0;
  bool seedsValid = false;
  DBuf<BBox> bboxes;
  DBuf<nbk_tile_list> lists1;
  DBuf<PatchPair> patchPairs;
  DBuf<int> jatom1;
  DBuf<nbk_tile_excl> excl1;
  DBuf<int> jtileActive, listActive;
  // compacted lists for steady-state evaluations
  DBuf<nbk_tile_list> lists2;      // refined, compacted lists, longest first
  DBuf<nbk_tile_list> listsCompact;  // the compaction's output before the sort
  // Batched replicas skip the sort: lists in compaction order stay grouped by
  // replica (per-replica LJ rows and accumulators stay hot), and a launch
  // over many replicas holds enough lists that its tail is short anyway.
  bool listsSorted = false;
  const nbk_tile_list* refinedLists() const { return listsSorted ? lists2.p : listsCompact.p; }
  DBuf<int> lenHist;                 // list-length histogram / cursors of the sort
  int maxListLen = 0;                // most j tiles a culled list can hold
  DBuf<int> jatom2;
  DBuf<nbk_tile_excl> excl2;
  DBuf<int> counters;  // [0] lists kept, [1] j tiles kept, [2] force / [3] refine / [4] precise work counters
  DBuf<unsigned> live;  // [j tiles][32] interacting-pair words of the last energy / virial evaluation
  bool built = false;     // tile lists built (sparse)
  bool refined = false;   // compacted lists valid
  bool tilesSizeExceeded = false;  // the last build was refused for a size limit
  float3 lata{}, latb{}, latc{};
  // accumulators
  DBuf<long long> force;
  int forceStride = 0;
  DBuf<long long> acc;
  DBuf<nbk_virial_energy> ve;
  // correction tuples
  DBuf<nbk_exclusion> modTuples, excTuples;
  int numMod = 0, numExc = 0;
  int maxTupleSlot = -1;  // largest atom slot named by a correction tuple
  unsigned lastFlags = 0;
  // batched replicas (0 = single system)
  int nrep = 0;
  DBuf<int> compRep, slotRep;
  DBuf<float3> repLat;
  DBuf<float2> repLJ, repLJExcl;
  int slotRepSize = 0;
  // adjoint
  DBuf<long long> adjGrad;
  DBuf<int> typeMask;
  int adjStride = 0;
  // launch shape of the force kernel per flag combination (tuneKey): CTAs per
  // SM and log2 of the work items per list; set by nbk_autotune
  int tuneMinBlocks[32];
  int tuneSplitLog2[32];
  float tuneMs[32];
  float lastCutoff2 = 0.f;
  // [numComputes][6] i-force sums per compute (shift virial): the tail of the
  // force buffer, cleared by the same memset
  long long* compF = nullptr;
  int compFComputes = 0;
  // measurement
  long long launches = 0;
  bool timing = false;
  std::vector<cudaEvent_t> evStart, evMid, evStop;
  int numTimed = 0;
  // second stream for the work that does not wait for the precise kernel
  // (corrections, force finalize, output copies), forked from and joined
  // back into the caller's stream within each evaluation
  cudaStream_t side = nullptr;
  cudaEvent_t evFork = nullptr, evJoin = nullptr;
};

namespace {
// Default launch shape of the force kernel: 4 CTAs per SM (a 128-register
// cap), one warp per tile list; measured fastest at 92k atoms for the energy
// and slow-force evaluations under flushed-L2 conditions (0.405 vs 0.411 ms
// at 5 CTAs per SM for energy + virial + slow).
constexpr int kDefaultMinBlocks = 4;
constexpr int kMaxTimed = 4096;

// Records the events of one evaluation when timing is on: before the force
// kernel (and the pairlist work before it), between the force kernel and the
// precise energy / virial kernel, and after that.
enum TimedPoint { kTimedStart = 0, kTimedMid = 1, kTimedStop = 2 };
cudaError_t timedEvent(nbk_context* h, TimedPoint which, cudaStream_t st) {
  if (!h->timing) return cudaSuccess;
  const int k = h->numTimed % kMaxTimed;
  std::vector<cudaEvent_t>& v =
      which == kTimedStart ? h->evStart : (which == kTimedMid ? h->evMid : h->evStop);
  if ((int)v.size() <= k) {
    cudaEvent_t e;
    cudaError_t r = cudaEventCreate(&e);
    if (r != cudaSuccess) return r;
    v.push_back(e);
  }
  cudaError_t r = cudaEventRecord(v[k], st);
  if (which == kTimedStop) ++h->numTimed;
  return r;
}

// The handle's side stream and its fork / join events, made on first use.
cudaError_t ensureSideStream(nbk_context* h) {
  if (h->side) return cudaSuccess;
  cudaError_t r = cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&h->evJoin, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
  if (r != cudaSuccess) {
    if (h->evFork) cudaEventDestroy(h->evFork);
    if (h->evJoin) cudaEventDestroy(h->evJoin);
    h->evFork = h->evJoin = nullptr;
    h->side = nullptr;
  }
  return r;
}
}  // namespace

namespace {

float3 f3(nbk_float3 v) { return make_float3(v.x, v.y, v.z); }

// Index of a flag combination in the tuning tables (the force kernel variant).
int tuneKey(const nbk_context* h, unsigned flags) {
  return (h->nrep > 0 ? 8 : 0) | ((flags & NBK_ENERGY) ? 4 : 0) | ((flags & NBK_VIRIAL) ? 2 : 0) |
         ((flags & NBK_SLOW) ? 1 : 0);
}

// Force-kernel arguments for the handle's compacted lists, positions, lattice,
// constants and replicas.
ForceArgs refinedForceArgs(nbk_context* h, float cutoff2) {
  ForceArgs a{};
  a.xyzq = h->xyzq;
  a.vdwTypes = h->vdwTypes.p;
  a.atomIndex = h->atomIndex.p;
  a.exclIndexMaxDiff = h->exclIndexMaxDiff.p;
  a.exclBits = h->exclBits.p;
  a.numExclWords = h->numExclWords;
  a.ljTable = h->ljTable.p;
  a.lata = h->lata;
  a.latb = h->latb;
  a.latc = h->latc;
  a.c = h->c;
  a.c.cutoff2 = cutoff2;
  a.force = h->force.p;
  a.stride = h->atomStorageSize;
  a.acc = h->acc.p;
  a.workCounter = h->counters.p + 2;
  a.slowTable = h->slowTable.p;
  a.slowTableRows = h->slowTableRows;
  a.slowStep = h->slowStep;
  a.slowInvStep = 1.0 / h->slowStep;
  if (h->nrep > 0) {
    a.compRep = h->compRep.p;
    a.repLat = h->repLat.p;
    a.repLJ = h->repLJ.p;
  }
  a.lists = h->refinedLists();
  a.numListsDev = h->counters.p;
  a.numListsHost = 0;
  a.tileJatomStart = h->jatom2.p;
  a.tileExcls = h->excl2.p;
  a.compF = h->compF;
  return a;
}

int checkHandle(nbk_handle h, const char* fn) {
  if (!h) return setErr(NBK_ERR_ARG, std::string(fn) + ": NULL handle");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return setErr(NBK_ERR_CUDA, std::string(fn) + ": cudaSetDevice: " +
                                                        cudaGetErrorString(e));
  return NBK_OK;
}

// Positions: copy a host array into the handle's buffer, or keep a device pointer.
int bindPositions(nbk_handle h, const nbk_float4* xyzq, int onDevice, int n, cudaStream_t st,
                  const char* fn) {
  if (!xyzq) {
    if (!h->xyzq) return setErr(NBK_ERR_STATE, std::string(fn) + ": no positions bound");
    return NBK_OK;
  }
  if (onDevice) {
    if (reinterpret_cast<const float4*>(xyzq) == h->xyzq) return NBK_OK;  // already bound
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, xyzq) != cudaSuccess || at.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      return setErr(NBK_ERR_ARG, std::string(fn) + ": xyzq is not a device pointer");
    }
    h->xyzq = reinterpret_cast<const float4*>(xyzq);
  } else {
    NBK_CUDA(h->xyzqOwn.ensure(n), fn);
    NBK_CUDA(cudaMemcpyAsync(h->xyzqOwn.p, xyzq, sizeof(float4) * (size_t)n,
                             cudaMemcpyHostToDevice, st), fn);
    h->xyzq = h->xyzqOwn.p;
  }
  return NBK_OK;
}

}  // namespace

int nbk::setLastError(int code, const std::string& msg) { return setErr(code, msg); }

extern "C" {

NBK_API const char* nbk_last_error(void) { return g_err.c_str(); }

NBK_API int nbk_debug_fail_alloc(int countdown) {
  if (countdown < 0) return setErr(NBK_ERR_ARG, "nbk_debug_fail_alloc: countdown must be >= 0");
  g_failAllocCountdown.store(countdown);
  return NBK_OK;
}
NBK_API int nbk_version(void) { return 1; }

NBK_API int nbk_create(int deviceID, const nbk_params* p, nbk_handle* out) {
  if (!p || !out) return setErr(NBK_ERR_ARG, "nbk_create: NULL argument");
  *out = nullptr;
  if (p->vdwTableDim <= 0 || !p->ljA || !p->ljB)
    return setErr(NBK_ERR_ARG, "nbk_create: LJ table missing");
  if (!(p->cutoff > 0) || p->pairlistdist < p->cutoff || p->switchdist <= 0)
    return setErr(NBK_ERR_ARG, "nbk_create: need 0 < switchdist, 0 < cutoff <= pairlistdist");
  if ((size_t)p->vdwTableDim * p->vdwTableDim * sizeof(float2) > 96 * 1024)
    return setErr(NBK_ERR_ARG, "nbk_create: LJ table larger than 96 KB of shared memory");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || deviceID < 0 || deviceID >= ndev) {
    cudaGetLastError();
    return setErr(NBK_ERR_DEVICE, "nbk_create: no such CUDA device");
  }
  cudaDeviceProp prop;
  NBK_CUDA(cudaGetDeviceProperties(&prop, deviceID), "nbk_create");
  if (prop.major != 10)
    return setErr(NBK_ERR_DEVICE, std::string("nbk_create: kernels are built for sm_100a, device is ") +
                                      prop.name);
  NBK_CUDA(cudaSetDevice(deviceID), "nbk_create");
  nbk_context* h = new (std::nothrow) nbk_context;
  if (!h) return setErr(NBK_ERR_NOMEM, "nbk_create: out of memory");
  h->device = deviceID;
  h->numSM = prop.multiProcessorCount;
  h->prm = *p;
  h->prm.ljA = h->prm.ljB = h->prm.ljA14 = h->prm.ljB14 = nullptr;
  h->ljDim = p->vdwTableDim;
  makeConstants(*p, p->vdwTableDim, h->c, h->c64);
  for (int k = 0; k < 32; ++k) {
    h->tuneMinBlocks[k] = kDefaultMinBlocks;
    h->tuneSplitLog2[k] = 0;
    h->tuneMs[k] = 0.f;
  }
  // LJ tables (CudaNonbondedTables::buildVdwCoefTable, src/CudaNonbondedTables.C:110-148)
  const int dim = h->ljDim;
  std::vector<float2> t(dim * dim), te(dim * dim);
  for (int k = 0; k < dim * dim; ++k) {
    t[k] = make_float2((float)(p->ljA[k] * p->scaling), (float)(p->ljB[k] * p->scaling));
    const double a14 = p->ljA14 ? p->ljA14[k] : p->ljA[k];
    const double b14 = p->ljB14 ? p->ljB14[k] : p->ljB[k];
    te[k] = make_float2((float)((a14 - p->ljA[k]) * p->scaling),
                        (float)((b14 - p->ljB[k]) * p->scaling));
  }
  int rc = NBK_OK;
  auto fin = [&](cudaError_t e, const char* what) {
    if (rc == NBK_OK && e != cudaSuccess)
      rc = setErr(e == cudaErrorMemoryAllocation ? NBK_ERR_NOMEM : NBK_ERR_CUDA,
                  std::string(what) + ": " + cudaGetErrorString(e));
  };
  fin(h->ljTable.ensure(dim * dim), "nbk_create: alloc");
  fin(h->ljExclTable.ensure(dim * dim), "nbk_create: alloc");
  if (rc == NBK_OK) fin(cudaMemcpy(h->ljTable.p, t.data(), sizeof(float2) * t.size(), cudaMemcpyHostToDevice), "nbk_create: copy");
  if (rc == NBK_OK) fin(cudaMemcpy(h->ljExclTable.p, te.data(), sizeof(float2) * te.size(), cudaMemcpyHostToDevice), "nbk_create: copy");
  // FP64 slow-term table over s in [0, pairlistdist^2 + 2]: the runtime cutoff
  // can be anything up to the pairlist cutoff
  std::vector<double> slow;
  h->slowTableRows = buildSlowTable(p->ewaldcof, p->cutoff, p->pairlistdist, slow, &h->slowStep);
  fin(h->slowTable.ensure(slow.size() / 2), "nbk_create: alloc");
  if (rc == NBK_OK) fin(cudaMemcpy(h->slowTable.p, slow.data(), sizeof(double) * slow.size(), cudaMemcpyHostToDevice), "nbk_create: copy");
  fin(h->acc.ensure(kAccCount), "nbk_create: alloc");
  fin(h->counters.ensure(8), "nbk_create: alloc");
  fin(h->ve.ensure(1), "nbk_create: alloc");
  if (rc == NBK_OK) fin(cudaMemset(h->acc.p, 0, sizeof(long long) * kAccCount), "nbk_create: memset");
  if (rc == NBK_OK) fin(cudaMemset(h->counters.p, 0, sizeof(int) * 8), "nbk_create: memset");
  if (rc != NBK_OK) {
    nbk_destroy(h);
    return rc;
  }
  *out = h;
  return NBK_OK;
}

NBK_API int nbk_destroy(nbk_handle h) {
  if (!h) return NBK_OK;
  cudaSetDevice(h->device);
  h->ljTable.release();
  h->ljExclTable.release();
  h->slowTable.release();
  h->exclBits.release();
  h->computes.release();
  h->vdwTypes.release();
  h->atomIndex.release();
  h->exclIndexMaxDiff.release();
  h->exclByAtom.release();
  h->xyzqOwn.release();
  h->patches.release();
  h->seeds.release();
  h->bboxes.release();
  h->lists1.release();
  h->patchPairs.release();
  h->jatom1.release();
  h->excl1.release();
  h->jtileActive.release();
  h->listActive.release();
  h->lists2.release();
  h->listsCompact.release();
  h->lenHist.release();
  h->jatom2.release();
  h->excl2.release();
  h->counters.release();
  h->live.release();
  h->force.release();
  h->acc.release();
  h->ve.release();
  h->modTuples.release();
  h->excTuples.release();
  h->adjGrad.release();
  h->typeMask.release();
  h->compRep.release();
  h->slotRep.release();
  h->repLat.release();
  h->repLJ.release();
  h->repLJExcl.release();
  for (cudaEvent_t e : h->evStart) cudaEventDestroy(e);
  for (cudaEvent_t e : h->evMid) cudaEventDestroy(e);
  for (cudaEvent_t e : h->evStop) cudaEventDestroy(e);
  if (h->side) {
    cudaStreamDestroy(h->side);
    cudaEventDestroy(h->evFork);
    cudaEventDestroy(h->evJoin);
  }
  delete h;
  return NBK_OK;
}

NBK_API int nbk_update_computes(nbk_handle h, int numComputes, const nbk_compute_record* hc,
                                void* stream) {
  int rc = checkHandle(h, "nbk_update_computes");
  if (rc) return rc;
  if (numComputes < 0 || (numComputes > 0 && !hc))
    return setErr(NBK_ERR_ARG, "nbk_update_computes: bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  h->hComputes.assign(hc, hc + numComputes);
  h->numComputes = numComputes;
  NBK_CUDA(h->computes.ensure(std::max(numComputes, 1)), "nbk_update_computes");
  if (numComputes)
    NBK_CUDA(cudaMemcpyAsync(h->computes.p, hc, sizeof(nbk_compute_record) * numComputes,
                             cudaMemcpyHostToDevice, st), "nbk_update_computes");
  h->seedsValid = false;
  h->built = h->refined = false;
  return NBK_OK;
}

NBK_API int nbk_bind_exclusions(nbk_handle h, int numExclusions, const unsigned int* bits) {
  int rc = checkHandle(h, "nbk_bind_exclusions");
  if (rc) return rc;
  if (numExclusions < 0 || (numExclusions > 0 && !bits))
    return setErr(NBK_ERR_ARG, "nbk_bind_exclusions: bad argument");
  NBK_CUDA(h->exclBits.ensure(std::max(numExclusions, 1)), "nbk_bind_exclusions");
  if (numExclusions)
    NBK_CUDA(cudaMemcpy(h->exclBits.p, bits, sizeof(unsigned) * numExclusions, cudaMemcpyHostToDevice),
             "nbk_bind_exclusions");
  h->numExclWords = numExclusions;
  return NBK_OK;
}

NBK_API int nbk_update_vdw_types_excl(nbk_handle h, int n, const int* vdwTypes,
                                      const nbk_int2* exclIndexMaxDiff, const int* atomIndex,
                                      void* stream) {
  int rc = checkHandle(h, "nbk_update_vdw_types_excl");
  if (rc) return rc;
  if (n <= 0 || (n & 31) || !vdwTypes || !exclIndexMaxDiff || !atomIndex)
    return setErr(NBK_ERR_ARG, "nbk_update_vdw_types_excl: bad argument (size must be a positive multiple of 32)");
  for (int k = 0; k < n; ++k)
    if (vdwTypes[k] < 0 || vdwTypes[k] >= h->ljDim)
      return setErr(NBK_ERR_ARG, "nbk_update_vdw_types_excl: vdw type out of range of the LJ table");
  cudaStream_t st = (cudaStream_t)stream;
  NBK_CUDA(h->vdwTypes.ensure(n), "nbk_update_vdw_types_excl");
  NBK_CUDA(h->atomIndex.ensure(n), "nbk_update_vdw_types_excl");
  NBK_CUDA(h->exclIndexMaxDiff.ensure(n), "nbk_update_vdw_types_excl");
  NBK_CUDA(cudaMemcpyAsync(h->vdwTypes.p, vdwTypes, sizeof(int) * n, cudaMemcpyHostToDevice, st),
           "nbk_update_vdw_types_excl");
  NBK_CUDA(cudaMemcpyAsync(h->atomIndex.p, atomIndex, sizeof(int) * n, cudaMemcpyHostToDevice, st),
           "nbk_update_vdw_types_excl");
  NBK_CUDA(cudaMemcpyAsync(h->exclIndexMaxDiff.p, exclIndexMaxDiff, sizeof(int2) * n,
                           cudaMemcpyHostToDevice, st), "nbk_update_vdw_types_excl");
  h->atomDataSize = n;
  return NBK_OK;
}

NBK_API int nbk_set_exclusion_tuples(nbk_handle h, int numModified, const nbk_exclusion* hm,
                                     int numExcluded, const nbk_exclusion* he, void* stream) {
  int rc = checkHandle(h, "nbk_set_exclusion_tuples");
  if (rc) return rc;
  if (numModified < 0 || numExcluded < 0 || (numModified && !hm) || (numExcluded && !he))
    return setErr(NBK_ERR_ARG, "nbk_set_exclusion_tuples: bad argument");
  int maxSlot = -1;
  for (int k = 0; k < numModified; ++k) {
    if (hm[k].pswitch != 0 || hm[k].vdwtypei < 0 || hm[k].vdwtypei >= h->ljDim ||
        hm[k].vdwtypej < 0 || hm[k].vdwtypej >= h->ljDim || hm[k].i < 0 || hm[k].j < 0)
      return setErr(NBK_ERR_ARG, "nbk_set_exclusion_tuples: bad tuple (alchemy, slot or vdw type)");
    maxSlot = std::max(maxSlot, std::max(hm[k].i, hm[k].j));
  }
  for (int k = 0; k < numExcluded; ++k) {
    if (he[k].pswitch != 0 || he[k].i < 0 || he[k].j < 0)
      return setErr(NBK_ERR_ARG, "nbk_set_exclusion_tuples: bad tuple (alchemy or slot)");
    maxSlot = std::max(maxSlot, std::max(he[k].i, he[k].j));
  }
  cudaStream_t st = (cudaStream_t)stream;
  NBK_CUDA(h->modTuples.ensure(std::max(numModified, 1)), "nbk_set_exclusion_tuples");
  NBK_CUDA(h->excTuples.ensure(std::max(numExcluded, 1)), "nbk_set_exclusion_tuples");
  if (numModified)
    NBK_CUDA(cudaMemcpyAsync(h->modTuples.p, hm, sizeof(nbk_exclusion) * numModified,
                             cudaMemcpyHostToDevice, st), "nbk_set_exclusion_tuples");
  if (numExcluded)
    NBK_CUDA(cudaMemcpyAsync(h->excTuples.p, he, sizeof(nbk_exclusion) * numExcluded,
                             cudaMemcpyHostToDevice, st), "nbk_set_exclusion_tuples");
  h->numMod = numModified;
  h->numExc = numExcluded;
  h->maxTupleSlot = maxSlot;
  return NBK_OK;
}

NBK_API int nbk_build_tile_lists(nbk_handle h, int numPatches, int atomStorageSize,
                                 int maxTileListLen, nbk_float3 lata, nbk_float3 latb,
                                 nbk_float3 latc, const nbk_patch_record* hp,
                                 const nbk_float4* xyzq, int xyzqOnDevice, float plcutoff2,
                                 void* stream) {
  int rc = checkHandle(h, "nbk_build_tile_lists");
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (numPatches <= 0 || !hp || atomStorageSize <= 0 || (atomStorageSize & 31))
    return setErr(NBK_ERR_ARG, "nbk_build_tile_lists: bad argument");
  if (maxTileListLen >= 65536) {
    h->tilesSizeExceeded = true;
    return setErr(NBK_ERR_OVERFLOW, "nbk_build_tile_lists: maximum number of tiles per tile list (65536) blown");
  }
  if (maxTileListLen <= 0) return setErr(NBK_ERR_ARG, "nbk_build_tile_lists: maxTileListLen must be positive");
  if (h->atomDataSize < atomStorageSize)
    return setErr(NBK_ERR_STATE, "nbk_build_tile_lists: nbk_update_vdw_types_excl not called for this atom storage size");
  if (!h->numComputes) return setErr(NBK_ERR_STATE, "nbk_build_tile_lists: no computes");
  // validate the patch layout and rebuild the list seeds when it changed
  bool same = h->seedsValid && numPatches == h->numPatches;
  for (int p = 0; p < numPatches; ++p) {
    const nbk_patch_record& r = hp[p];
    if (r.numAtoms < 0 || r.numFreeAtoms < 0 || r.numFreeAtoms > r.numAtoms || (r.atomStart & 31) ||
        r.atomStart < 0 || r.atomStart + ((r.numAtoms + 31) / 32) * 32 > atomStorageSize)
      return setErr(NBK_ERR_ARG, "nbk_build_tile_lists: patch record out of range of the atom storage");
    if ((r.numAtoms + 31) / 32 > maxTileListLen) {
      h->tilesSizeExceeded = true;
      return setErr(NBK_ERR_OVERFLOW, "nbk_build_tile_lists: a patch has more tiles than maxTileListLen");
    }
    if (same && (r.numAtoms != h->hPatches[p].numAtoms || r.atomStart != h->hPatches[p].atomStart ||
                 r.numFreeAtoms != h->hPatches[p].numFreeAtoms))
      same = false;
  }
  NBK_CUDA(h->patches.ensure(numPatches), "nbk_build_tile_lists");
  if (!same) {
    h->hPatches.assign(hp, hp + numPatches);
    h->numPatches = numPatches;
    NBK_CUDA(cudaMemcpyAsync(h->patches.p, h->hPatches.data(), sizeof(nbk_patch_record) * numPatches,
                             cudaMemcpyHostToDevice, st), "nbk_build_tile_lists");
    h->hSeeds.clear();
    long long jcap = 0;
    int maxT2 = 0;
    for (int ci = 0; ci < h->numComputes; ++ci) {
      const nbk_compute_record& cr = h->hComputes[ci];
      if (cr.patchInd.x < 0 || cr.patchInd.x >= numPatches || cr.patchInd.y < 0 ||
          cr.patchInd.y >= numPatches)
        return setErr(NBK_ERR_ARG, "nbk_build_tile_lists: compute refers to a missing patch");
      const int t1 = (hp[cr.patchInd.x].numAtoms + 31) / 32;
      const int t2 = (hp[cr.patchInd.y].numAtoms + 31) / 32;
      maxT2 = std::max(maxT2, t2);
      for (int it = 0; it < t1; ++it) {
        h->hSeeds.push_back(ListSeed{ci, it, (int)jcap, 0});
        jcap += t2;
      }
    }
    if (jcap > (1LL << 30))
      return setErr(NBK_ERR_OVERFLOW, "nbk_build_tile_lists: j-tile capacity exceeds 2^30");
    h->numLists = (int)h->hSeeds.size();
    h->jcap = (int)jcap;
    h->maxListLen = maxT2;
    NBK_CUDA(h->seeds.ensure(std::max(h->numLists, 1)), "nbk_build_tile_lists");
    if (h->numLists)
      NBK_CUDA(cudaMemcpyAsync(h->seeds.p, h->hSeeds.data(), sizeof(ListSeed) * h->numLists,
                               cudaMemcpyHostToDevice, st), "nbk_build_tile_lists");
    h->seedsValid = true;
  }
  rc = bindPositions(h, xyzq, xyzqOnDevice, atomStorageSize, st, "nbk_build_tile_lists");
  if (rc) return rc;
  if (!h->xyzq) return setErr(NBK_ERR_ARG, "nbk_build_tile_lists: xyzq is NULL");
  h->atomStorageSize = atomStorageSize;
  h->lata = f3(lata);
  h->latb = f3(latb);
  h->latc = f3(latc);
  const int nl = std::max(h->numLists, 1), nj = std::max(h->jcap, 1);
  NBK_CUDA(h->bboxes.ensure(atomStorageSize / 32), "nbk_build_tile_lists");
  NBK_CUDA(h->lists1.ensure(nl), "nbk_build_tile_lists");
  NBK_CUDA(h->patchPairs.ensure(nl), "nbk_build_tile_lists");
  NBK_CUDA(h->listActive.ensure(nl), "nbk_build_tile_lists");
  NBK_CUDA(h->jatom1.ensure(nj), "nbk_build_tile_lists");
  NBK_CUDA(h->excl1.ensure(nj), "nbk_build_tile_lists");
  NBK_CUDA(h->jtileActive.ensure(nj), "nbk_build_tile_lists");
  NBK_CUDA(launchBBoxes(atomStorageSize / 32, h->xyzq, h->bboxes.p, st), "bounding boxes");
  h->launches += 2;
  // culling distance: the pairlist cutoff inflated by a relative 1e-5 so FP32
  // rounding in the boxes can never drop a pair the exact pair test keeps
  const float cull2 = plcutoff2 * 1.00002f + 1e-6f;
  if (h->nrep > 0 && h->slotRepSize != atomStorageSize)
    return setErr(NBK_ERR_STATE, "nbk_build_tile_lists: atomStorageSize differs from the replica layout");
  NBK_CUDA(launchBuildLists(h->numLists, h->seeds.p, h->computes.p, h->patches.p, h->bboxes.p,
                            h->lata, h->latb, h->latc, h->nrep ? h->compRep.p : nullptr,
                            h->nrep ? h->repLat.p : nullptr, cull2, h->lists1.p, h->patchPairs.p,
                            h->jatom1.p, st), "tile-list build");
  h->c.plcutoff2 = plcutoff2;
  h->built = true;
  h->refined = false;
  h->tilesSizeExceeded = false;
  return NBK_OK;
}

NBK_API int nbk_nonbonded_force(nbk_handle h, int atomStorageSize, unsigned flags,
                                nbk_float3 lata, nbk_float3 latb, nbk_float3 latc,
                                const nbk_float4* xyzq, int xyzqOnDevice, float cutoff2,
                                nbk_float4* d_forces, nbk_float4* d_forcesSlow,
                                nbk_float4* h_forces, nbk_float4* h_forcesSlow,
                                long long* d_forcesFixed, void* stream) {
  int rc = checkHandle(h, "nbk_nonbonded_force");
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (flags & ~63u) return setErr(NBK_ERR_ARG, "nbk_nonbonded_force: unknown flag bits");
  const bool pairlist = flags & NBK_PAIRLIST;
  if (!h->built) return setErr(NBK_ERR_STATE, "nbk_nonbonded_force: tile lists not built");
  if (!pairlist && !h->refined)
    return setErr(NBK_ERR_STATE, "nbk_nonbonded_force: the first evaluation after a build needs NBK_PAIRLIST");
  if (atomStorageSize != h->atomStorageSize)
    return setErr(NBK_ERR_ARG, "nbk_nonbonded_force: atomStorageSize differs from the tile-list build");
  if (!(cutoff2 > 0.f) || cutoff2 > h->c.plcutoff2)
    return setErr(NBK_ERR_ARG, "nbk_nonbonded_force: cutoff2 must be in (0, plcutoff2]");
  rc = bindPositions(h, xyzq, xyzqOnDevice, atomStorageSize, st, "nbk_nonbonded_force");
  if (rc) return rc;
  const int n = atomStorageSize;
  if (h->forceStride != n || h->compFComputes != h->numComputes) {
    NBK_CUDA(h->force.ensure(6 * ((size_t)n + (size_t)h->numComputes)), "nbk_nonbonded_force");
    h->forceStride = n;
    h->compFComputes = h->numComputes;
  }
  h->compF = h->force.p + 6 * (size_t)n;
  NBK_CUDA(cudaMemsetAsync(h->force.p, 0,
                           sizeof(long long) * 6 * ((size_t)n + (size_t)h->numComputes), st),
           "nbk_nonbonded_force");
  const int accBlocks = h->nrep > 0 ? h->nrep : 1;
  NBK_CUDA(cudaMemsetAsync(h->acc.p, 0, sizeof(long long) * kAccCount * (size_t)accBlocks, st),
           "nbk_nonbonded_force");
  h->lata = f3(lata);
  h->latb = f3(latb);
  h->latc = f3(latc);

  h->lastCutoff2 = cutoff2;
  const bool shiftVirial = flags & NBK_VIRIAL;
  ForceArgs a = refinedForceArgs(h, cutoff2);
  const int key = tuneKey(h, flags);
  a.splitLog2 = h->tuneSplitLog2[key];
  NBK_CUDA(timedEvent(h, kTimedStart, st), "timing event");
  if (pairlist) {
    // refinement of the culled lists (the pairlist pass), then their
    // compaction (reSortTileLists), both on the device
    ForceArgs r = a;
    r.lists = h->lists1.p;
    r.numListsDev = nullptr;
    r.numListsHost = h->numLists;
    r.tileJatomStart = h->jatom1.p;
    r.tileExcls = h->excl1.p;
    r.jtileActive = h->jtileActive.p;
    r.listActive = h->listActive.p;
    r.patchPairs = h->patchPairs.p;
    r.workCounter = h->counters.p + 3;
    NBK_CUDA(cudaMemsetAsync(h->counters.p + 3, 0, sizeof(int), st), "nbk_nonbonded_force");
    NBK_CUDA(launchRefine(r, h->numSM, st), "pairlist refinement");
    const int nl = std::max(h->numLists, 1), nj = std::max(h->jcap, 1);
    NBK_CUDA(h->lists2.ensure(nl), "nbk_nonbonded_force");
    NBK_CUDA(h->listsCompact.ensure(nl), "nbk_nonbonded_force");
    NBK_CUDA(h->lenHist.ensure((size_t)h->maxListLen + 1), "nbk_nonbonded_force");
    NBK_CUDA(h->jatom2.ensure(nj), "nbk_nonbonded_force");
    NBK_CUDA(h->excl2.ensure(nj), "nbk_nonbonded_force");
    NBK_CUDA(cudaMemsetAsync(h->counters.p, 0, sizeof(int) * 2, st), "nbk_nonbonded_force");
    NBK_CUDA(launchCompact(h->numLists, h->lists1.p, h->listActive.p, h->jtileActive.p, h->jatom1.p,
                           h->excl1.p, h->listsCompact.p, h->jatom2.p, h->excl2.p, h->counters.p,
                           h->numSM, st), "tile-list compaction");
    h->listsSorted = h->nrep == 0;
    if (h->listsSorted) {
      NBK_CUDA(launchSortLists(h->numLists, h->listsCompact.p, h->counters.p, h->maxListLen,
                               h->lenHist.p, h->lists2.p, h->numSM, st), "tile-list sort");
      h->launches += 3;
    }
    h->launches += 2;
    h->refined = true;
  }
  // compacted lists (the pairlist block above may have grown these buffers)
  a.lists = h->refinedLists();
  a.tileJatomStart = h->jatom2.p;
  a.tileExcls = h->excl2.p;
  NBK_CUDA(cudaMemsetAsync(h->counters.p + 2, 0, sizeof(int) * 3, st), "nbk_nonbonded_force");
  if (needsPrecise(flags)) {
    NBK_CUDA(h->live.ensure((size_t)std::max(h->jcap, 1) * 32), "nbk_nonbonded_force");
    a.liveOut = h->live.p;
  }
  NBK_CUDA(launchForce(a, flags, h->tuneMinBlocks[key], h->numSM, st), "force kernel");
  h->launches += 1;
  NBK_CUDA(timedEvent(h, kTimedMid, st), "timing event");
  const bool corrections = (flags & NBK_CORRECTIONS) && (h->numMod || h->numExc);
  if (corrections && h->maxTupleSlot >= n)
    return setErr(NBK_ERR_ARG, "nbk_nonbonded_force: a correction tuple names a slot beyond atomStorageSize");
  if ((h_forces && !d_forces) || (h_forcesSlow && !d_forcesSlow))
    return setErr(NBK_ERR_ARG, "nbk_nonbonded_force: host force output needs the matching device buffer");
  // With a precise kernel to run, the corrections, the force finalize and the
  // output copies (which need only the forces) go to the side stream and run
  // beside it; the caller's stream waits for both before it goes on.
  const bool fork = needsPrecise(flags);
  cudaStream_t fs = st;
  if (fork) {
    NBK_CUDA(ensureSideStream(h), "nbk_nonbonded_force: side stream");
    NBK_CUDA(cudaEventRecord(h->evFork, st), "nbk_nonbonded_force: fork");
    NBK_CUDA(cudaStreamWaitEvent(h->side, h->evFork, 0), "nbk_nonbonded_force: fork");
    fs = h->side;
    ForceArgs pa = a;
    pa.workCounter = h->counters.p + 4;
    NBK_CUDA(launchPrecise(pa, flags, h->numSM, st), "precise energy / virial kernel");
    h->launches += 1;
  }
  NBK_CUDA(timedEvent(h, kTimedStop, st), "timing event");
  if (corrections) {
    CorrArgs ca{};
    ca.modified = h->modTuples.p;
    ca.numModified = h->numMod;
    ca.excluded = h->excTuples.p;
    ca.numExcluded = h->numExc;
    ca.xyzq = h->xyzq;
    ca.ljExclTable = h->ljExclTable.p;
    ca.lata = h->lata;
    ca.latb = h->latb;
    ca.latc = h->latc;
    ca.c = h->c;
    ca.c.cutoff2 = cutoff2;
    ca.force = h->force.p;
    ca.stride = n;
    ca.acc = h->acc.p;
    ca.c64 = h->c64;
    if (h->nrep > 0) {
      ca.slotRep = h->slotRep.p;
      ca.repLat = h->repLat.p;
      ca.repLJExcl = h->repLJExcl.p;
    }
    NBK_CUDA(launchCorrections(ca, flags, fs), "exclusion corrections");
    h->launches += 1;
  }
  ShiftVirialArgs sv{};
  if (shiftVirial) {
    sv.numComputes = h->numComputes;
    sv.compF = h->compF;
    sv.computes = h->computes.p;
    sv.lata = h->lata;
    sv.latb = h->latb;
    sv.latc = h->latc;
    sv.compRep = h->nrep ? h->compRep.p : nullptr;
    sv.repLat = h->nrep ? h->repLat.p : nullptr;
  }
  // page-locked host outputs are written by the finalize kernel itself;
  // other host memory gets a copy after it
  float4* hF = static_cast<float4*>(mappedHostPointer(h_forces));
  float4* hS = (flags & NBK_SLOW) ? static_cast<float4*>(mappedHostPointer(h_forcesSlow)) : nullptr;
  NBK_CUDA(launchFinalizeForces(n, h->force.p, n, h->xyzq, reinterpret_cast<float4*>(d_forces),
                                (flags & NBK_SLOW) ? reinterpret_cast<float4*>(d_forcesSlow) : nullptr,
                                flags, h->acc.p, h->numSM, fs, h->nrep ? h->slotRep.p : nullptr,
                                &sv, hF, hS),
           "force finalize");
  if ((flags & NBK_VIRIAL) || d_forces || d_forcesSlow) h->launches += 1;
  if (d_forcesFixed)
    NBK_CUDA(cudaMemcpyAsync(d_forcesFixed, h->force.p, sizeof(long long) * 6 * (size_t)n,
                             cudaMemcpyDeviceToDevice, fs), "nbk_nonbonded_force: fixed-point copy");
  if (h_forces && !hF)
    NBK_CUDA(cudaMemcpyAsync(h_forces, d_forces, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost, fs),
             "nbk_nonbonded_force: D2H");
  if (h_forcesSlow && (flags & NBK_SLOW) && !hS)
    NBK_CUDA(cudaMemcpyAsync(h_forcesSlow, d_forcesSlow, sizeof(float4) * (size_t)n,
                             cudaMemcpyDeviceToHost, fs), "nbk_nonbonded_force: D2H");
  if (fork) {
    NBK_CUDA(cudaEventRecord(h->evJoin, fs), "nbk_nonbonded_force: join");
    NBK_CUDA(cudaStreamWaitEvent(st, h->evJoin, 0), "nbk_nonbonded_force: join");
  }
  h->lastFlags = flags;
  return NBK_OK;
}

NBK_API int nbk_reduce_virial_energy(nbk_handle h, unsigned flags, nbk_virial_energy* ve,
                                     int veOnDevice, void* stream) {
  int rc = checkHandle(h, "nbk_reduce_virial_energy");
  if (rc) return rc;
  (void)flags;
  if (!ve) return setErr(NBK_ERR_ARG, "nbk_reduce_virial_energy: NULL output");
  if (h->nrep > 0)
    return setErr(NBK_ERR_STATE, "nbk_reduce_virial_energy: the handle holds replicas; use nbk_reduce_virial_energy_batch");
  cudaStream_t st = (cudaStream_t)stream;
  // page-locked host output: the read-out kernel writes it directly
  nbk_virial_energy* mapped = veOnDevice ? nullptr : static_cast<nbk_virial_energy*>(mappedHostPointer(ve));
  nbk_virial_energy* dst = veOnDevice ? ve : (mapped ? mapped : h->ve.p);
  NBK_CUDA(launchEnergyVirial(h->acc.p, dst, st), "energy/virial read-out");
  h->launches += 1;
  if (!veOnDevice && !mapped)
    NBK_CUDA(cudaMemcpyAsync(ve, h->ve.p, sizeof(nbk_virial_energy), cudaMemcpyDeviceToHost, st),
             "nbk_reduce_virial_energy: D2H");
  return NBK_OK;
}

NBK_API int nbk_get_tile_list_stat(nbk_handle h, nbk_tile_list_stat* out, void* stream) {
  int rc = checkHandle(h, "nbk_get_tile_list_stat");
  if (rc) return rc;
  if (!out) return setErr(NBK_ERR_ARG, "nbk_get_tile_list_stat: NULL output");
  cudaStream_t st = (cudaStream_t)stream;
  int cnt[2] = {0, 0};
  const int accBlocks = h->nrep > 0 ? h->nrep : 1;
  std::vector<long long> accHost((size_t)kAccCount * accBlocks);
  NBK_CUDA(cudaMemcpyAsync(cnt, h->counters.p, sizeof(int) * 2, cudaMemcpyDeviceToHost, st), "stat");
  NBK_CUDA(cudaMemcpyAsync(accHost.data(), h->acc.p, sizeof(long long) * accHost.size(),
                           cudaMemcpyDeviceToHost, st), "stat");
  NBK_CUDA(cudaStreamSynchronize(st), "stat");
  long long nex = 0;
  for (int r = 0; r < accBlocks; ++r) nex += accHost[(size_t)r * kAccCount + kAccNumExcl];
  std::memset(out, 0, sizeof(*out));
  out->tilesSizeExceeded = h->tilesSizeExceeded ? 1 : 0;
  out->numTileLists = h->refined ? cnt[0] : h->numLists;
  out->numTileListsGBIS = out->numTileLists;
  out->numJtiles = h->refined ? cnt[1] : h->jcap;
  out->numExcluded = (int)nex;
  return NBK_OK;
}

NBK_API int nbk_export_tile_lists(nbk_handle h, int* numTileLists, int* numJtiles,
                                  nbk_tile_list* tl, int* jatom, nbk_tile_excl* excl, void* stream) {
  int rc = checkHandle(h, "nbk_export_tile_lists");
  if (rc) return rc;
  if (!numTileLists || !numJtiles) return setErr(NBK_ERR_ARG, "nbk_export_tile_lists: NULL counts");
  if (!h->refined) return setErr(NBK_ERR_STATE, "nbk_export_tile_lists: no refined tile lists");
  cudaStream_t st = (cudaStream_t)stream;
  int cnt[2] = {0, 0};
  NBK_CUDA(cudaMemcpyAsync(cnt, h->counters.p, sizeof(int) * 2, cudaMemcpyDeviceToHost, st), "export");
  NBK_CUDA(cudaStreamSynchronize(st), "export");
  *numTileLists = cnt[0];
  *numJtiles = cnt[1];
  if (tl && cnt[0])
    NBK_CUDA(cudaMemcpy(tl, h->refinedLists(), sizeof(nbk_tile_list) * cnt[0], cudaMemcpyDeviceToHost), "export");
  if (jatom && cnt[1])
    NBK_CUDA(cudaMemcpy(jatom, h->jatom2.p, sizeof(int) * cnt[1], cudaMemcpyDeviceToHost), "export");
  if (excl && cnt[1])
    NBK_CUDA(cudaMemcpy(excl, h->excl2.p, sizeof(nbk_tile_excl) * cnt[1], cudaMemcpyDeviceToHost), "export");
  return NBK_OK;
}

NBK_API int nbk_adjoint(nbk_handle h, unsigned flags, const nbk_float4* d_wF, const nbk_float4* d_wS,
                        double cV, double cE, double cS, const int* h_typeMask,
                        nbk_float4* d_gradXQ, long long* d_gradFixed, double* d_gradAB,
                        void* stream) {
  int rc = checkHandle(h, "nbk_adjoint");
  if (rc) return rc;
  if (!d_wF || !d_gradAB) return setErr(NBK_ERR_ARG, "nbk_adjoint: NULL argument");
  if (flags & ~(unsigned)NBK_SLOW) return setErr(NBK_ERR_ARG, "nbk_adjoint: only NBK_SLOW applies");
  const bool slow = flags & NBK_SLOW;
  if (slow && !d_wS) return setErr(NBK_ERR_ARG, "nbk_adjoint: NBK_SLOW needs d_wS");
  if (!h->refined || !h->xyzq)
    return setErr(NBK_ERR_STATE, "nbk_adjoint: needs refined tile lists (an NBK_PAIRLIST evaluation) first");
  if (h->nrep > 0) return setErr(NBK_ERR_STATE, "nbk_adjoint: not available with replicas");
  cudaStream_t st = (cudaStream_t)stream;
  const int n = h->atomStorageSize, dim = h->ljDim;
  std::vector<int> mask(dim, 1);
  if (h_typeMask)
    for (int t = 0; t < dim; ++t) mask[t] = h_typeMask[t] ? 1 : 0;
  NBK_CUDA(h->typeMask.ensure(dim), "nbk_adjoint");
  NBK_CUDA(cudaMemcpyAsync(h->typeMask.p, mask.data(), sizeof(int) * dim, cudaMemcpyHostToDevice, st),
           "nbk_adjoint");
  if (h->adjStride != n) {
    NBK_CUDA(h->adjGrad.ensure(4 * (size_t)n), "nbk_adjoint");
    h->adjStride = n;
  }
  NBK_CUDA(cudaMemsetAsync(h->adjGrad.p, 0, sizeof(long long) * 4 * (size_t)n, st), "nbk_adjoint");
  NBK_CUDA(cudaMemsetAsync(d_gradAB, 0, sizeof(double) * 2 * (size_t)dim * dim, st), "nbk_adjoint");
  NBK_CUDA(cudaMemsetAsync(h->counters.p + 2, 0, sizeof(int), st), "nbk_adjoint");
  AdjArgs a{};
  a.lists = h->refinedLists();
  a.numListsDev = h->counters.p;
  a.tileJatomStart = h->jatom2.p;
  a.tileExcls = h->excl2.p;
  a.xyzq = h->xyzq;
  a.vdwTypes = h->vdwTypes.p;
  a.ljTable = h->ljTable.p;
  a.typeMask = h->typeMask.p;
  a.wF = reinterpret_cast<const float4*>(d_wF);
  a.wS = reinterpret_cast<const float4*>(d_wS);
  a.cV = (float)cV;
  a.cE = (float)cE;
  a.cS = (float)cS;
  a.lata = h->lata;
  a.latb = h->latb;
  a.latc = h->latc;
  a.c = h->c;
  a.grad = h->adjGrad.p;
  a.stride = n;
  a.gradAB = d_gradAB;
  a.workCounter = h->counters.p + 2;
  NBK_CUDA(timedEvent(h, kTimedStart, st), "timing event");
  NBK_CUDA(launchAdjoint(a, slow, h->numSM, n, reinterpret_cast<float4*>(d_gradXQ), st), "adjoint kernel");
  NBK_CUDA(timedEvent(h, kTimedMid, st), "timing event");
  NBK_CUDA(timedEvent(h, kTimedStop, st), "timing event");
  h->launches += d_gradXQ ? 2 : 1;
  if (d_gradFixed)
    NBK_CUDA(cudaMemcpyAsync(d_gradFixed, h->adjGrad.p, sizeof(long long) * 4 * (size_t)n,
                             cudaMemcpyDeviceToDevice, st), "nbk_adjoint: fixed-point copy");
  return NBK_OK;
}

NBK_API int nbk_set_replicas(nbk_handle h, int numReplicas, const int* repOfCompute,
                             const int* slotStart, const nbk_float3* lattices, const double* ljA,
                             const double* ljB, const double* ljA14, const double* ljB14,
                             void* stream) {
  int rc = checkHandle(h, "nbk_set_replicas");
  if (rc) return rc;
  if (numReplicas <= 0 || !repOfCompute || !slotStart || !lattices || !ljA || !ljB)
    return setErr(NBK_ERR_ARG, "nbk_set_replicas: bad argument");
  if (!h->numComputes) return setErr(NBK_ERR_STATE, "nbk_set_replicas: call nbk_update_computes first");
  cudaStream_t st = (cudaStream_t)stream;
  for (int c = 0; c < h->numComputes; ++c)
    if (repOfCompute[c] < 0 || repOfCompute[c] >= numReplicas)
      return setErr(NBK_ERR_ARG, "nbk_set_replicas: replica index of a compute out of range");
  if (slotStart[0] != 0) return setErr(NBK_ERR_ARG, "nbk_set_replicas: replicaSlotStart[0] must be 0");
  for (int r = 0; r < numReplicas; ++r)
    if (slotStart[r + 1] < slotStart[r] || (slotStart[r] & 31))
      return setErr(NBK_ERR_ARG, "nbk_set_replicas: replica slot ranges must increase in multiples of 32");
  const int n = slotStart[numReplicas];
  std::vector<int> slotRep(n);
  for (int r = 0; r < numReplicas; ++r)
    for (int k = slotStart[r]; k < slotStart[r + 1]; ++k) slotRep[k] = r;
  const int dim = h->ljDim, d2 = dim * dim;
  std::vector<float2> t((size_t)numReplicas * d2), te((size_t)numReplicas * d2);
  const double sc = h->prm.scaling;
  for (size_t k = 0; k < t.size(); ++k) {
    t[k] = make_float2((float)(ljA[k] * sc), (float)(ljB[k] * sc));
    const double a14 = ljA14 ? ljA14[k] : ljA[k], b14 = ljB14 ? ljB14[k] : ljB[k];
    te[k] = make_float2((float)((a14 - ljA[k]) * sc), (float)((b14 - ljB[k]) * sc));
  }
  NBK_CUDA(h->compRep.ensure(h->numComputes), "nbk_set_replicas");
  NBK_CUDA(h->slotRep.ensure(std::max(n, 1)), "nbk_set_replicas");
  NBK_CUDA(h->repLat.ensure(3 * (size_t)numReplicas), "nbk_set_replicas");
  NBK_CUDA(h->repLJ.ensure(t.size()), "nbk_set_replicas");
  NBK_CUDA(h->repLJExcl.ensure(te.size()), "nbk_set_replicas");
  NBK_CUDA(h->acc.ensure((size_t)kAccCount * numReplicas), "nbk_set_replicas");
  NBK_CUDA(h->ve.ensure(numReplicas), "nbk_set_replicas");
  NBK_CUDA(cudaMemcpy(h->compRep.p, repOfCompute, sizeof(int) * h->numComputes, cudaMemcpyHostToDevice),
           "nbk_set_replicas");
  if (n) NBK_CUDA(cudaMemcpy(h->slotRep.p, slotRep.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "nbk_set_replicas");
  NBK_CUDA(cudaMemcpy(h->repLat.p, lattices, sizeof(float3) * 3 * (size_t)numReplicas, cudaMemcpyHostToDevice),
           "nbk_set_replicas");
  NBK_CUDA(cudaMemcpy(h->repLJ.p, t.data(), sizeof(float2) * t.size(), cudaMemcpyHostToDevice), "nbk_set_replicas");
  NBK_CUDA(cudaMemcpy(h->repLJExcl.p, te.data(), sizeof(float2) * te.size(), cudaMemcpyHostToDevice),
           "nbk_set_replicas");
  NBK_CUDA(cudaMemsetAsync(h->acc.p, 0, sizeof(long long) * kAccCount * (size_t)numReplicas, st),
           "nbk_set_replicas");
  h->nrep = numReplicas;
  h->slotRepSize = n;
  h->built = h->refined = false;
  return NBK_OK;
}

NBK_API int nbk_reduce_virial_energy_batch(nbk_handle h, unsigned flags, nbk_virial_energy* ve,
                                           int veOnDevice, void* stream) {
  int rc = checkHandle(h, "nbk_reduce_virial_energy_batch");
  if (rc) return rc;
  (void)flags;
  if (!ve) return setErr(NBK_ERR_ARG, "nbk_reduce_virial_energy_batch: NULL output");
  const int nr = h->nrep > 0 ? h->nrep : 1;
  cudaStream_t st = (cudaStream_t)stream;
  nbk_virial_energy* dst = veOnDevice ? ve : h->ve.p;
  NBK_CUDA(h->ve.ensure(nr), "nbk_reduce_virial_energy_batch");
  dst = veOnDevice ? ve : h->ve.p;
  NBK_CUDA(launchEnergyVirial(h->acc.p, dst, st, nr), "energy/virial read-out");
  h->launches += 1;
  if (!veOnDevice)
    NBK_CUDA(cudaMemcpyAsync(ve, h->ve.p, sizeof(nbk_virial_energy) * nr, cudaMemcpyDeviceToHost, st),
             "nbk_reduce_virial_energy_batch: D2H");
  return NBK_OK;
}

NBK_API int nbk_get_pair_counts(nbk_handle h, long long* counts, int maxCount, void* stream) {
  int rc = checkHandle(h, "nbk_get_pair_counts");
  if (rc) return rc;
  if (!counts || maxCount <= 0) return setErr(NBK_ERR_ARG, "nbk_get_pair_counts: bad output");
  if (!(h->lastFlags & NBK_ENERGY))
    return setErr(NBK_ERR_STATE, "nbk_get_pair_counts: the last evaluation did not compute energies");
  const int nr = h->nrep > 0 ? h->nrep : 1;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<long long> accHost((size_t)kAccCount * nr);
  NBK_CUDA(cudaMemcpyAsync(accHost.data(), h->acc.p, sizeof(long long) * accHost.size(),
                           cudaMemcpyDeviceToHost, st), "nbk_get_pair_counts");
  NBK_CUDA(cudaStreamSynchronize(st), "nbk_get_pair_counts");
  for (int r = 0; r < nr && r < maxCount; ++r) counts[r] = accHost[(size_t)r * kAccCount + kAccNumPairs];
  return NBK_OK;
}

NBK_API int nbk_set_kernel_timing(nbk_handle h, int enable) {
  int rc = checkHandle(h, "nbk_set_kernel_timing");
  if (rc) return rc;
  h->timing = enable != 0;
  h->numTimed = 0;
  return NBK_OK;
}

namespace {
int timesBetween(nbk_handle h, const std::vector<cudaEvent_t>& from,
                 const std::vector<cudaEvent_t>& to, float* ms, int maxCount, int* count,
                 const char* fn) {
  int rc = checkHandle(h, fn);
  if (rc) return rc;
  if (!count || (maxCount > 0 && !ms)) return setErr(NBK_ERR_ARG, std::string(fn) + ": NULL output");
  const int n = std::min(h->numTimed, kMaxTimed);
  *count = n;
  const int first = h->numTimed - n;
  for (int k = 0; k < n && k < maxCount; ++k) {
    const int slot = (first + k) % kMaxTimed;
    NBK_CUDA(cudaEventSynchronize(to[slot]), fn);
    NBK_CUDA(cudaEventElapsedTime(&ms[k], from[slot], to[slot]), fn);
  }
  return NBK_OK;
}
}  // namespace

NBK_API int nbk_get_kernel_times(nbk_handle h, float* ms, int maxCount, int* count) {
  if (!h) return setErr(NBK_ERR_ARG, "nbk_get_kernel_times: NULL handle");
  return timesBetween(h, h->evStart, h->evMid, ms, maxCount, count, "nbk_get_kernel_times");
}

NBK_API int nbk_get_precise_times(nbk_handle h, float* ms, int maxCount, int* count) {
  if (!h) return setErr(NBK_ERR_ARG, "nbk_get_precise_times: NULL handle");
  return timesBetween(h, h->evMid, h->evStop, ms, maxCount, count, "nbk_get_precise_times");
}

NBK_API long long nbk_launch_count(nbk_handle h) { return h ? h->launches : -1; }

NBK_API int nbk_get_pair_count(nbk_handle h, long long* pairs, void* stream) {
  int rc = checkHandle(h, "nbk_get_pair_count");
  if (rc) return rc;
  if (!pairs) return setErr(NBK_ERR_ARG, "nbk_get_pair_count: NULL output");
  if (!(h->lastFlags & NBK_ENERGY))
    return setErr(NBK_ERR_STATE, "nbk_get_pair_count: the last evaluation did not compute energies");
  cudaStream_t st = (cudaStream_t)stream;
  const int nr = h->nrep > 0 ? h->nrep : 1;
  std::vector<long long> accHost((size_t)kAccCount * nr);
  NBK_CUDA(cudaMemcpyAsync(accHost.data(), h->acc.p, sizeof(long long) * accHost.size(),
                           cudaMemcpyDeviceToHost, st), "nbk_get_pair_count");
  NBK_CUDA(cudaStreamSynchronize(st), "nbk_get_pair_count");
  long long tot = 0;
  for (int r = 0; r < nr; ++r) tot += accHost[(size_t)r * kAccCount + kAccNumPairs];
  *pairs = tot;
  return NBK_OK;
}

}  // extern "C"

namespace {
// Register-resident FMA chains: 8 independent chains per thread keep the FP32
// pipe busy without memory traffic.
__global__ void fmaPeakKernel(int iters, float seed, float* out) {
  float a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5,
        a6 = a0 + 6, a7 = a0 + 7;
  const float m = 0.999999f, c = 1e-7f;
  for (int k = 0; k < iters; ++k) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
      a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
    }
  }
  const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678f) out[0] = s;  // never true; keeps the chains alive
}
}  // namespace

namespace {
// The same with FP64 FMAs.
__global__ void dfmaPeakKernel(int iters, double seed, double* out) {
  double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4,
         a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const double m = 0.999999, c = 1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
      a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
  }
  if (a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7 == -1.0) *out = a0;  // keeps the chains live
}
}  // namespace

extern "C" NBK_API int nbk_measure_fp64_peak(int deviceID, double* tflops) {
  if (!tflops) return setErr(NBK_ERR_ARG, "nbk_measure_fp64_peak: NULL output");
  NBK_CUDA(cudaSetDevice(deviceID), "nbk_measure_fp64_peak");
  cudaDeviceProp prop;
  NBK_CUDA(cudaGetDeviceProperties(&prop, deviceID), "nbk_measure_fp64_peak");
  double* out = nullptr;
  NBK_CUDA(cudaMalloc(&out, sizeof(double)), "nbk_measure_fp64_peak");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 1024;
  dfmaPeakKernel<<<blocks, threads>>>(16, 1.0, out);  // warm-up
  double best = 0;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0);
    dfmaPeakKernel<<<blocks, threads>>>(iters, 1.0, out);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      cudaFree(out);
      return setErr(NBK_ERR_CUDA, std::string("nbk_measure_fp64_peak: ") + cudaGetErrorString(e));
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *tflops = best;
  return NBK_OK;
}

extern "C" NBK_API int nbk_measure_fp32_peak(int deviceID, double* tflops) {
  if (!tflops) return setErr(NBK_ERR_ARG, "nbk_measure_fp32_peak: NULL output");
  NBK_CUDA(cudaSetDevice(deviceID), "nbk_measure_fp32_peak");
  cudaDeviceProp prop;
  NBK_CUDA(cudaGetDeviceProperties(&prop, deviceID), "nbk_measure_fp32_peak");
  float* out = nullptr;
  NBK_CUDA(cudaMalloc(&out, sizeof(float)), "nbk_measure_fp32_peak");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 4096;
  fmaPeakKernel<<<blocks, threads>>>(64, 1.0f, out);  // warm-up
  double best = 0;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0);
    fmaPeakKernel<<<blocks, threads>>>(iters, 1.0f, out);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      cudaFree(out);
      return setErr(NBK_ERR_CUDA, std::string("nbk_measure_fp32_peak: ") + cudaGetErrorString(e));
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *tflops = best;
  return NBK_OK;
}

NBK_API int nbk_autotune(nbk_handle h, unsigned flags, int iterations, void* stream) {
  int rc = checkHandle(h, "nbk_autotune");
  if (rc) return rc;
  if (!h->refined)
    return setErr(NBK_ERR_STATE, "nbk_autotune: needs refined tile lists (an NBK_PAIRLIST evaluation) first");
  if (flags & ~63u) return setErr(NBK_ERR_ARG, "nbk_autotune: unknown flag bits");
  if (iterations < 1) iterations = 1;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned kflags = flags & ~(unsigned)(NBK_PAIRLIST | NBK_CORRECTIONS);
  const int key = tuneKey(h, kflags);
  const int n = h->atomStorageSize;
  const int accBlocks = h->nrep > 0 ? h->nrep : 1;
  ForceArgs a = refinedForceArgs(h, h->lastCutoff2);
  if (needsPrecise(kflags)) {  // the timed force kernel stores live words
    NBK_CUDA(h->live.ensure((size_t)std::max(h->jcap, 1) * 32), "nbk_autotune");
    a.liveOut = h->live.p;
  }
  const int maxSplitLog2 = 2;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  NBK_CUDA(cudaEventCreate(&e0), "nbk_autotune");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return setErr(NBK_ERR_CUDA, "nbk_autotune: event");
  }
  // shapes are timed back to back on a warm L2; another shape replaces the
  // default (kDefaultMinBlocks CTAs per SM, one warp per list) only when it is
  // at least 3% faster, so that timing noise does not pick a shape that loses
  // in use
  float bestMs = 1e30f, defaultMs = 1e30f;
  int bestB = kDefaultMinBlocks, bestS = 0;
  cudaError_t err = cudaSuccess;
  const int shapes[3] = {4, 5, 6};
  for (int bi = 0; bi < 3 && err == cudaSuccess; ++bi) {
    for (int sl = 0; sl <= maxSplitLog2 && err == cudaSuccess; ++sl) {
      a.splitLog2 = sl;
      for (int it = -1; it < iterations && err == cudaSuccess; ++it) {  // it = -1: untimed
        if (it == 0) err = cudaEventRecord(e0, st);
        if (err == cudaSuccess) err = cudaMemsetAsync(h->force.p, 0, sizeof(long long) * 6 * (size_t)n, st);
        if (err == cudaSuccess)
          err = cudaMemsetAsync(h->acc.p, 0, sizeof(long long) * kAccCount * (size_t)accBlocks, st);
        if (err == cudaSuccess) err = cudaMemsetAsync(h->counters.p + 2, 0, sizeof(int), st);
        if (err == cudaSuccess) err = launchForce(a, kflags, shapes[bi], h->numSM, st);
        h->launches += 1;
      }
      if (err == cudaSuccess) err = cudaEventRecord(e1, st);
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
      if (err == cudaSuccess) {
        const float t = ms / iterations;
        if (shapes[bi] == kDefaultMinBlocks && sl == 0) defaultMs = t;
        if (t < bestMs) {
          bestMs = t;
          bestB = shapes[bi];
          bestS = sl;
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return setErr(NBK_ERR_CUDA, std::string("nbk_autotune: ") + cudaGetErrorString(err));
  if (!(bestMs < 0.97f * defaultMs)) {
    bestB = kDefaultMinBlocks;
    bestS = 0;
    bestMs = defaultMs;
  }
  h->tuneMinBlocks[key] = bestB;
  h->tuneSplitLog2[key] = bestS;
  h->tuneMs[key] = bestMs;
  return NBK_OK;
}

NBK_API int nbk_get_tuning(nbk_handle h, unsigned flags, int* minBlocksPerSM, int* listSplit,
                           float* ms) {
  int rc = checkHandle(h, "nbk_get_tuning");
  if (rc) return rc;
  const int key = tuneKey(h, flags & ~(unsigned)(NBK_PAIRLIST | NBK_CORRECTIONS));
  if (minBlocksPerSM) *minBlocksPerSM = h->tuneMinBlocks[key];
  if (listSplit) *listSplit = 1 << h->tuneSplitLog2[key];
  if (ms) *ms = h->tuneMs[key];
  return NBK_OK;
}

NBK_API int nbk_set_tuning(nbk_handle h, unsigned flags, int minBlocksPerSM, int listSplit) {
  int rc = checkHandle(h, "nbk_set_tuning");
  if (rc) return rc;
  if (minBlocksPerSM < 4 || minBlocksPerSM > 6)
    return setErr(NBK_ERR_ARG, "nbk_set_tuning: minBlocksPerSM must be 4, 5 or 6");
  int sl = -1;
  for (int k = 0; k <= 2; ++k)
    if (listSplit == (1 << k)) sl = k;
  if (sl < 0) return setErr(NBK_ERR_ARG, "nbk_set_tuning: listSplit must be 1, 2 or 4");
  const int key = tuneKey(h, flags & ~(unsigned)(NBK_PAIRLIST | NBK_CORRECTIONS));
  h->tuneMinBlocks[key] = minBlocksPerSM;
  h->tuneSplitLog2[key] = sl;
  h->tuneMs[key] = 0.f;
  return NBK_OK;
}

// ---- GPU-resident input marshaling -----------------------------------------

NBK_API int nbk_set_exclusions_by_atom(nbk_handle h, int numAtoms, const nbk_int2* hx) {
  int rc = checkHandle(h, "nbk_set_exclusions_by_atom");
  if (rc) return rc;
  if (numAtoms <= 0 || !hx) return setErr(NBK_ERR_ARG, "nbk_set_exclusions_by_atom: bad argument");
  NBK_CUDA(h->exclByAtom.ensure(numAtoms), "nbk_set_exclusions_by_atom");
  NBK_CUDA(cudaMemcpy(h->exclByAtom.p, hx, sizeof(int2) * numAtoms, cudaMemcpyHostToDevice),
           "nbk_set_exclusions_by_atom");
  h->numExclByAtom = numAtoms;
  return NBK_OK;
}

NBK_API int nbk_update_vdw_types_excl_device(nbk_handle h, int numPatches, int n,
                                             const nbk_local_record* rec, const int* vdw,
                                             const int* id, const int* sortOrder, int* status,
                                             void* stream) {
  int rc = checkHandle(h, "nbk_update_vdw_types_excl_device");
  if (rc) return rc;
  if (numPatches < 0 || n <= 0 || (n & 31) || (numPatches && (!rec || !vdw || !id || !sortOrder)))
    return setErr(NBK_ERR_ARG, "nbk_update_vdw_types_excl_device: bad argument (size must be a "
                               "positive multiple of 32)");
  if (!h->numExclByAtom)
    return setErr(NBK_ERR_STATE, "nbk_update_vdw_types_excl_device: nbk_set_exclusions_by_atom first");
  cudaStream_t st = (cudaStream_t)stream;
  NBK_CUDA(h->vdwTypes.ensure(n), "nbk_update_vdw_types_excl_device");
  NBK_CUDA(h->atomIndex.ensure(n), "nbk_update_vdw_types_excl_device");
  NBK_CUDA(h->exclIndexMaxDiff.ensure(n), "nbk_update_vdw_types_excl_device");
  NBK_CUDA(launchUpdateVdwTypesExclDevice(numPatches, rec, vdw, id, sortOrder, h->exclByAtom.p,
                                          h->numExclByAtom, h->ljDim, n, h->vdwTypes.p,
                                          h->atomIndex.p, h->exclIndexMaxDiff.p, status, st),
           "nbk_update_vdw_types_excl_device");
  h->atomDataSize = n;
  return NBK_OK;
}

NBK_API int nbk_accumulate_forces_to_soa(nbk_handle h, int maxForceNumber, int numPatches,
                                         const nbk_local_record* rec, const int* sortOrder,
                                         const double* fBond, const double* fBondNbond,
                                         const double* fBondSlow, int forceStride,
                                         const nbk_float3* fPme, double* nx, double* ny,
                                         double* nz, double* bx, double* by, double* bz,
                                         double* sx, double* sy, double* sz, void* stream) {
  int rc = checkHandle(h, "nbk_accumulate_forces_to_soa");
  if (rc) return rc;
  if (maxForceNumber < 0 || maxForceNumber > 2 || numPatches < 0 ||
      (numPatches && (!rec || !sortOrder || !nx || !ny || !nz)) ||
      (maxForceNumber >= 1 && (!bx || !by || !bz)) || (maxForceNumber >= 2 && (!sx || !sy || !sz)) ||
      ((fBond || fBondNbond || fBondSlow) && forceStride <= 0))
    return setErr(NBK_ERR_ARG, "nbk_accumulate_forces_to_soa: bad argument");
  if (!h->force.p || h->forceStride <= 0)
    return setErr(NBK_ERR_STATE, "nbk_accumulate_forces_to_soa: no nbk_nonbonded_force evaluation yet");
  AccumulateArgs a;
  a.numPatches = numPatches;
  a.maxForceNumber = maxForceNumber;
  a.stride = h->forceStride;
  a.forceStride = forceStride;
  a.rec = rec;
  a.sortOrder = sortOrder;
  a.fixed = h->force.p;
  a.fBond = fBond;
  a.fBondNbond = fBondNbond;
  a.fBondSlow = fBondSlow;
  a.fPme = reinterpret_cast<const float3*>(fPme);
  a.fNormal[0] = nx;
  a.fNormal[1] = ny;
  a.fNormal[2] = nz;
  a.fNbond[0] = bx;
  a.fNbond[1] = by;
  a.fNbond[2] = bz;
  a.fSlow[0] = sx;
  a.fSlow[1] = sy;
  a.fSlow[2] = sz;
  NBK_CUDA(launchAccumulateForces(a, (cudaStream_t)stream), "nbk_accumulate_forces_to_soa");
  return NBK_OK;
}
