// Test harness around the reference's own CUDA nonbonded kernels.
//
// The Makefile beside this file compiles the reference's
// src/CudaTileListKernel.cu and src/CudaComputeNonbondedKernel.cu in place
// (never copied) together with this file into oracle/_ref/libref_nbgpu.so.
// This file supplies what those two translation units need from the rest of
// NAMD, written here from the declarations in the reference headers:
//
//   - the CudaUtils allocation / copy / clear helpers and cudaDie
//     (declared in src/CudaUtils.h:206-383),
//   - NAMD_die / NAMD_bug (they throw; the C entry points below turn the
//     exception into an error status),
//   - the per-thread `deviceCUDA` object and DeviceCUDA::getMaxNumBlocks
//     (src/DeviceCUDA.h:148; the device's maximum grid x dimension),
//   - a CudaNonbondedTables built from plain parameters instead of the
//     ComputeNonbondedUtil statics (src/CudaNonbondedTables.C:10-34):
//       * the LJ table, width rounded up to an odd multiple of 16, entries
//         A*scaling and B*scaling (src/CudaNonbondedTables.C:110-148);
//       * the float4 force / energy textures of the table mode, 4096 texels
//         sampled at r = 4096/(i+0.5), components (fast elec, -vdwB, vdwA,
//         slow correction), force texel = 2 dE/d(r^2), zero beyond the
//         cutoff, texel 0 force 0 and energy = texel 1, normalised
//         coordinates with linear filtering (src/CudaNonbondedTables.C:
//         158-303). The reference fills these texels from its cubic r^2
//         interpolation tables (src/ComputeNonbondedUtil.C:607-1337); this
//         harness evaluates the same functions analytically in FP64
//         (C1 splitting, energy switching, PME erfc), which differs from the
//         cubic tables far below the texture's own linear-filter error.
//
// It then drives the reference objects in the order CudaComputeNonbonded::
// launchWork uses (src/CudaComputeNonbonded.C:1440-1530): buildTileLists,
// prepareTileList, clearTileListStat, updateVdwTypesExcl, nonbondedForce,
// finishTileList, reduceVirialEnergy, and reSortTileLists once the pairlist
// step has finished (src/CudaComputeNonbonded.C:1975-2040).
//
// Test infrastructure only: the product library never links this.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "CudaUtils.h"
#include "CudaTileListKernel.h"
#include "CudaNonbondedTables.h"
#include "CudaComputeNonbondedKernel.h"
#include "DeviceCUDA.h"

// ---------------------------------------------------------------------------
// NAMD runtime pieces the reference kernels call.

static void throwCuda(const char* what, cudaError_t err) {
  std::string m = what ? what : "cuda error";
  if (err != cudaSuccess) {
    m += ": ";
    m += cudaGetErrorString(err);
  }
  throw std::runtime_error(m);
}

void NAMD_die(const char* msg) { throw std::runtime_error(std::string("NAMD_die: ") + msg); }
void NAMD_bug(const char* msg) { throw std::runtime_error(std::string("NAMD_bug: ") + msg); }
void cudaDie(const char* msg, cudaError_t err) { throwCuda(msg, err); }
void cudaNAMD_bug(const char* msg) { throw std::runtime_error(std::string("cudaNAMD_bug: ") + msg); }

static void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throwCuda(what, e);
}

void clear_device_array_async_T(void* data, const size_t ndata, cudaStream_t stream,
                                const size_t sizeofT) {
  if (ndata) ck(cudaMemsetAsync(data, 0, ndata * sizeofT, stream), "clear_device_array_async_T");
}
// The synchronous clear and the zeroing of new buffers below run on the legacy
// default stream, which does not order itself with the harness's non-blocking
// stream: each waits for its memset, so no kernel queued afterwards can run
// before it (a kernel that did would have its output zeroed after the fact).
void clear_device_array_T(void* data, const size_t ndata, const size_t sizeofT) {
  if (!ndata) return;
  ck(cudaMemset(data, 0, ndata * sizeofT), "clear_device_array_T");
  ck(cudaDeviceSynchronize(), "clear_device_array_T sync");
}
void allocate_host_T(void** pp, const size_t len, const size_t sizeofT) {
  ck(cudaMallocHost(pp, len * sizeofT), "allocate_host_T");
  std::memset(*pp, 0, len * sizeofT);
}
void allocate_device_T(void** pp, const size_t len, const size_t sizeofT) {
  ck(cudaMalloc(pp, len * sizeofT), "allocate_device_T");
  ck(cudaMemset(*pp, 0, len * sizeofT), "allocate_device_T memset");
  ck(cudaDeviceSynchronize(), "allocate_device_T sync");
}
void deallocate_device_T(void** pp) {
  if (*pp) ck(cudaFree(*pp), "deallocate_device_T");
  *pp = nullptr;
}
void deallocate_host_T(void** pp) {
  if (*pp) ck(cudaFreeHost(*pp), "deallocate_host_T");
  *pp = nullptr;
}
// Grow-only: a new buffer of max(newlen*fac, newlen) elements when the
// current one is missing or shorter than newlen; old contents are dropped.
bool reallocate_device_T(void** pp, size_t* curlen, const size_t newlen, const float fac,
                         const size_t sizeofT) {
  if (*pp != nullptr && *curlen >= newlen) return false;
  if (*pp) ck(cudaFree(*pp), "reallocate_device_T free");
  *pp = nullptr;
  size_t n = (size_t)((double)newlen * (double)fac);
  if (n < newlen) n = newlen;
  if (n == 0) n = 1;
  ck(cudaMalloc(pp, n * sizeofT), "reallocate_device_T");
  ck(cudaMemset(*pp, 0, n * sizeofT), "reallocate_device_T memset");
  ck(cudaDeviceSynchronize(), "reallocate_device_T sync");
  *curlen = n;
  return true;
}
bool reallocate_host_T(void** pp, size_t* curlen, const size_t newlen, const float fac,
                       const unsigned int flag, const size_t sizeofT) {
  if (*pp != nullptr && *curlen >= newlen) return false;
  if (*pp) ck(cudaFreeHost(*pp), "reallocate_host_T free");
  *pp = nullptr;
  size_t n = (size_t)((double)newlen * (double)fac);
  if (n < newlen) n = newlen;
  if (n == 0) n = 1;
  ck(cudaHostAlloc(pp, n * sizeofT, flag), "reallocate_host_T");
  std::memset(*pp, 0, n * sizeofT);
  *curlen = n;
  return true;
}
// A source equal to the destination is skipped: the harness passes the
// kernel's own device xyzq as "host" positions to time the kernels alone.
void copy_HtoD_async_T(const void* h_array, void* d_array, size_t array_len, cudaStream_t stream,
                       const size_t sizeofT) {
  if (array_len == 0 || h_array == d_array) return;
  ck(cudaMemcpyAsync(d_array, h_array, array_len * sizeofT, cudaMemcpyDefault, stream),
     "copy_HtoD_async_T");
}
void copy_HtoD_T(const void* h_array, void* d_array, size_t array_len, const size_t sizeofT) {
  if (array_len == 0 || h_array == d_array) return;
  ck(cudaMemcpy(d_array, h_array, array_len * sizeofT, cudaMemcpyDefault), "copy_HtoD_T");
}
void copy_DtoH_async_T(const void* d_array, void* h_array, const size_t array_len,
                       cudaStream_t stream, const size_t sizeofT) {
  if (array_len == 0) return;
  ck(cudaMemcpyAsync(h_array, d_array, array_len * sizeofT, cudaMemcpyDefault, stream),
     "copy_DtoH_async_T");
}
void copy_DtoH_T(const void* d_array, void* h_array, const size_t array_len, const size_t sizeofT) {
  if (array_len == 0) return;
  ck(cudaMemcpy(h_array, d_array, array_len * sizeofT, cudaMemcpyDefault), "copy_DtoH_T");
}

__thread DeviceCUDA* deviceCUDA = nullptr;
DeviceCUDA::DeviceCUDA() {}
DeviceCUDA::~DeviceCUDA() {}
int DeviceCUDA::getMaxNumBlocks() {
  int dev = 0, v = 0;
  ck(cudaGetDevice(&dev), "getMaxNumBlocks");
  ck(cudaDeviceGetAttribute(&v, cudaDevAttrMaxGridDimX, dev), "getMaxNumBlocks attr");
  return v;
}

// ---------------------------------------------------------------------------
// Tables.

namespace {

struct TableParams {
  double cutoff, switchdist, ewaldcof, scaling;
  int dim;
  std::vector<double> A, B;
};

thread_local const TableParams* g_tableParams = nullptr;

// Functions of r held by the texture tables (per unit charge product / per
// unit A or B): energy and dE/d(r^2).
void tableFunctions(const TableParams& p, double r, double e[4], double g[4]) {
  const double rc = p.cutoff, rc2 = rc * rc, r2 = r * r;
  const double beta = p.ewaldcof;
  const double rinv = 1.0 / r, r2inv = rinv * rinv;
  // C1 splitting: slow part 0.5/rc (3 - r^2/rc^2), fast = 1/r - slow,
  // scor = slow + (erfc(beta r) - 1)/r.
  const double slowE = 0.5 / rc * (3.0 - r2 / rc2);
  const double slowDr = -r / (rc2 * rc);
  const double erfcv = std::erfc(beta * r);
  const double gauss = 2.0 * beta / std::sqrt(M_PI) * std::exp(-beta * beta * r2);
  const double fastE = rinv - slowE;
  const double fastDr = -r2inv - slowDr;
  const double scorE = slowE + (erfcv - 1.0) * rinv;
  const double scorDr = slowDr - gauss * rinv - (erfcv - 1.0) * r2inv;
  // Energy switching of LJ.
  const double rs2 = p.switchdist * p.switchdist;
  double S = 1.0, dS = 0.0;  // dS/d(r^2)
  if (r2 > rs2 && rc2 > rs2) {
    const double den = 1.0 / ((rc2 - rs2) * (rc2 - rs2) * (rc2 - rs2));
    const double D = rc2 - r2;
    S = D * D * (rc2 + 2.0 * r2 - 3.0 * rs2) * den;
    dS = (-2.0 * D * (rc2 + 2.0 * r2 - 3.0 * rs2) + 2.0 * D * D) * den;
  }
  const double r6 = r2inv * r2inv * r2inv, r12 = r6 * r6;
  const double vaE = S * r12, vbE = S * r6;
  const double vaG = dS * r12 - 6.0 * S * r12 * r2inv;
  const double vbG = dS * r6 - 3.0 * S * r6 * r2inv;
  e[0] = fastE;
  g[0] = fastDr * 0.5 * rinv;
  e[1] = -vbE;
  g[1] = -vbG;
  e[2] = vaE;
  g[2] = vaG;
  e[3] = scorE;
  g[3] = scorDr * 0.5 * rinv;
}

void makeTexture(const float* host, int n, cudaArray_t* arr, cudaTextureObject_t* tex,
                 float4** lin) {
  ck(cudaMalloc(lin, sizeof(float4) * n), "table linear");
  ck(cudaMemcpy(*lin, host, sizeof(float4) * n, cudaMemcpyHostToDevice), "table linear copy");
  cudaChannelFormatDesc desc = cudaCreateChannelDesc(32, 32, 32, 32, cudaChannelFormatKindFloat);
  ck(cudaMallocArray(arr, &desc, n, 0), "table array");
  ck(cudaMemcpy2DToArray(*arr, 0, 0, host, sizeof(float4) * n, sizeof(float4) * n, 1,
                         cudaMemcpyHostToDevice),
     "table array copy");
  cudaResourceDesc rd;
  std::memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = *arr;
  cudaTextureDesc td;
  std::memset(&td, 0, sizeof(td));
  td.addressMode[0] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModeLinear;
  td.normalizedCoords = 1;
  td.readMode = cudaReadModeElementType;
  ck(cudaCreateTextureObject(tex, &rd, &td, nullptr), "table texture");
}

}  // namespace

CudaNonbondedTables::CudaNonbondedTables(const int deviceID_) : deviceID(deviceID_) {
  const TableParams& p = *g_tableParams;
  vdwCoefTable = nullptr;
  exclusionVdwCoefTable = nullptr;
  vdwCoefTableTex = 0;
  exclusionVdwCoefTableTex = 0;
  forceTableTex = energyTableTex = 0;
  modifiedExclusionForceTableTex = modifiedExclusionEnergyTableTex = 0;
  forceArray = energyArray = nullptr;
  modifiedExclusionForceArray = modifiedExclusionEnergyArray = nullptr;
  forceTable = energyTable = nullptr;
  modifiedExclusionForceTable = modifiedExclusionEnergyTable = nullptr;
  exclusionTable = nullptr;
  r2_table = nullptr;
  exclusionTableTex = 0;
  r2_table_tex = 0;
  ck(cudaSetDevice(deviceID), "tables set device");

  // LJ table, width = the smallest odd multiple of 16 not below dim.
  int tsize = 16;
  while (tsize < p.dim) tsize += 32;
  vdwCoefTableWidth = tsize;
  std::vector<float2> t((size_t)tsize * tsize, make_float2(0.f, 0.f));
  for (int i = 0; i < p.dim; ++i)
    for (int j = 0; j < p.dim; ++j)
      t[(size_t)i * tsize + j] = make_float2((float)(p.A[(size_t)i * p.dim + j] * p.scaling),
                                             (float)(p.B[(size_t)i * p.dim + j] * p.scaling));
  ck(cudaMalloc(&vdwCoefTable, sizeof(float2) * t.size()), "vdw table");
  ck(cudaMemcpy(vdwCoefTable, t.data(), sizeof(float2) * t.size(), cudaMemcpyHostToDevice),
     "vdw table copy");

  // Force / energy textures.
  const int n = FORCE_ENERGY_TABLE_SIZE;
  forceAndEnergyTableSize = n;
  std::vector<float> ft((size_t)4 * n, 0.f), et((size_t)4 * n, 0.f);
  for (int i = 1; i < n; ++i) {
    const double r = (double)n / ((double)i + 0.5);
    if (r > p.cutoff) continue;
    double e[4], g[4];
    tableFunctions(p, r, e, g);
    for (int k = 0; k < 4; ++k) {
      ft[(size_t)4 * i + k] = (float)(2.0 * g[k]);
      et[(size_t)4 * i + k] = (float)e[k];
    }
  }
  for (int k = 0; k < 4; ++k) {
    ft[k] = 0.f;
    et[k] = et[4 + k];
  }
  makeTexture(ft.data(), n, &forceArray, &forceTableTex, &forceTable);
  makeTexture(et.data(), n, &energyArray, &energyTableTex, &energyTable);
}

CudaNonbondedTables::~CudaNonbondedTables() {
  cudaSetDevice(deviceID);
  if (forceTableTex) cudaDestroyTextureObject(forceTableTex);
  if (energyTableTex) cudaDestroyTextureObject(energyTableTex);
  if (forceArray) cudaFreeArray(forceArray);
  if (energyArray) cudaFreeArray(energyArray);
  if (forceTable) cudaFree(forceTable);
  if (energyTable) cudaFree(energyTable);
  if (vdwCoefTable) cudaFree(vdwCoefTable);
}

// ---------------------------------------------------------------------------
// C entry points (ctypes).

namespace {

thread_local std::string g_err;

struct RefGpu {
  int device = 0;
  TableParams tp;
  CudaNonbondedTables* tables = nullptr;
  CudaTileListKernel* tl = nullptr;
  CudaComputeNonbondedKernel* nb = nullptr;
  DeviceCUDA* dc = nullptr;
  cudaStream_t stream = nullptr;
  bool ownStream = true;
  CudaNBConstants c;
  float cutoff2 = 0.f, plcutoff2 = 0.f;
  int doTable = 1;
  int numPatches = 0, numComputes = 0, atomStorageSize = 0, maxTileListLen = 0;
  int numTileListsPrev = 0;
  std::vector<CudaPatchRecord> patches;
  float4* d_forces = nullptr;
  float4* d_forcesSlow = nullptr;
  VirialEnergy* d_ve = nullptr;
  size_t maxShmem = 0;
  bool listsReady = false;
};

template <class F>
int guarded(RefGpu* h, F&& f) {
  try {
    if (h) {
      ck(cudaSetDevice(h->device), "set device");
      deviceCUDA = h->dc;
    }
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char* refgpu_last_error(void) { return g_err.c_str(); }

// params: cutoff, switchdist, pairlistdist, ewaldcof, scaling, slowScale.
// A, B: [dim*dim] unscaled LJ table. doTable: 1 = texture tables (the
// reference's choice whenever slow forces are on), 0 = direct math.
int refgpu_create(int device, const double* params, int dim, const double* A, const double* B,
                  int doTable, void** out) {
  RefGpu* h = new RefGpu();
  h->device = device;
  const int rc = guarded(nullptr, [&] {
    ck(cudaSetDevice(device), "set device");
    h->dc = new DeviceCUDA();
    deviceCUDA = h->dc;
    h->tp.cutoff = params[0];
    h->tp.switchdist = params[1];
    h->tp.ewaldcof = params[3];
    h->tp.scaling = params[4];
    h->tp.dim = dim;
    h->tp.A.assign(A, A + (size_t)dim * dim);
    h->tp.B.assign(B, B + (size_t)dim * dim);
    h->doTable = doTable;
    g_tableParams = &h->tp;
    h->tables = new CudaNonbondedTables(device);
    g_tableParams = nullptr;
    h->tl = new CudaTileListKernel(device, false);
    h->nb = new CudaComputeNonbondedKernel(device, *h->tables, false);
    ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
    cudaDeviceProp prop;
    ck(cudaGetDeviceProperties(&prop, device), "props");
    h->maxShmem = prop.sharedMemPerBlock;
    // CudaNBConstants as CudaComputeNonbonded::getNonbondedCoef fills them
    // (field meanings in src/CudaUtils.h:574-590).
    const float cutoff = (float)params[0];
    const float cutoff2 = cutoff * cutoff;
    const float cutoffInv = 1.0f / cutoff;
    const float cutoff2Inv = 1.0f / cutoff2;
    const float sw2 = (float)(params[1] * params[1]);
    const double dd = params[0] * params[0] - params[1] * params[1];
    const float denom = (float)(1.0 / (dd * dd * dd));
    const float slowScale = (float)params[5];
    const float beta = (float)params[3];
    h->c.lj_0 = denom * cutoff2 - 3.0f * sw2 * denom;
    h->c.lj_1 = denom * 2.0f;
    h->c.lj_2 = denom * -12.0f;
    h->c.lj_3 = 12.0f * denom * sw2;
    h->c.lj_4 = cutoff2;
    h->c.lj_5 = sw2;
    h->c.e_0 = cutoff2Inv * cutoffInv;
    h->c.e_0_slow = cutoff2Inv * cutoffInv * (1.0f - slowScale);
    h->c.e_1 = cutoff2Inv;
    h->c.e_2 = cutoffInv;
    h->c.ewald_0 = beta;
    h->c.ewald_1 = (float)(2.0 * params[3] / std::sqrt(M_PI));
    h->c.ewald_2 = beta * beta;
    h->c.ewald_3_slow = beta * beta * beta * slowScale;
    h->c.slowScale = slowScale;
    h->cutoff2 = cutoff2;
    h->plcutoff2 = (float)(params[2] * params[2]);
  });
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return 0;
}

// patches4: [4*numPatches] (numAtoms, numFreeAtoms, atomStart, patchID).
// computes: [numComputes] CudaComputeRecord (int2 patchInd, float3 offsetXYZ; 24 B).
// exclIndexMaxDiff: [2*atomStorageSize].
int refgpu_setup(void* hp, int numPatches, const int* patches4, int numComputes,
                 const void* computes, int atomStorageSize, int maxTileListLen,
                 const int* vdwTypes, const int* exclIndexMaxDiff, const int* atomIndex,
                 int numExclWords, const unsigned int* exclBits) {
  RefGpu* h = (RefGpu*)hp;
  return guarded(h, [&] {
    h->numPatches = numPatches;
    h->numComputes = numComputes;
    h->atomStorageSize = atomStorageSize;
    h->maxTileListLen = maxTileListLen;
    h->patches.resize(numPatches);
    for (int i = 0; i < numPatches; ++i) {
      h->patches[i].numAtoms = patches4[4 * i];
      h->patches[i].numFreeAtoms = patches4[4 * i + 1];
      h->patches[i].atomStart = patches4[4 * i + 2];
    }
    const CudaComputeRecord* cr = (const CudaComputeRecord*)computes;
    int nl = 0;
    for (int i = 0; i < numComputes; ++i) {
      const int na = h->patches[cr[i].patchInd.x].numAtoms;
      nl += (na - 1) / WARPSIZE + 1;
    }
    h->numTileListsPrev = nl;
    h->tl->updateComputes(numComputes, cr, h->stream);
    h->nb->bindExclusions(numExclWords, const_cast<unsigned int*>(exclBits));
    h->nb->reallocate_forceSOA(atomStorageSize);
    h->nb->updateVdwTypesExcl(atomStorageSize, vdwTypes, (const int2*)exclIndexMaxDiff, atomIndex,
                              h->stream);
    if (h->d_forces) cudaFree(h->d_forces);
    if (h->d_forcesSlow) cudaFree(h->d_forcesSlow);
    ck(cudaMalloc(&h->d_forces, sizeof(float4) * atomStorageSize), "forces");
    ck(cudaMalloc(&h->d_forcesSlow, sizeof(float4) * atomStorageSize), "forcesSlow");
    if (!h->d_ve) ck(cudaMalloc(&h->d_ve, sizeof(VirialEnergy)), "ve");
    ck(cudaMemset(h->d_ve, 0, sizeof(VirialEnergy)), "ve clear");
    ck(cudaStreamSynchronize(h->stream), "setup sync");
    h->listsReady = false;
  });
}

// One evaluation. lat: [9] a, b, c. xyzq: host (pinned or pageable) positions,
// or NULL to use the positions already on the device (the kernels alone).
// A pairlist step builds and refines the tile lists (it needs host xyzq) and
// re-sorts them afterwards, synchronising the stream as the reference does.
int refgpu_eval(void* hp, int doPairlist, int doEnergy, int doVirial, int doSlow,
                const float* lat, const float* xyzq) {
  RefGpu* h = (RefGpu*)hp;
  return guarded(h, [&] {
    const float3 a = make_float3(lat[0], lat[1], lat[2]);
    const float3 b = make_float3(lat[3], lat[4], lat[5]);
    const float3 c = make_float3(lat[6], lat[7], lat[8]);
    if (!doPairlist && !h->listsReady) throw std::runtime_error("refgpu_eval: no tile lists yet");
    if (doPairlist && !xyzq) throw std::runtime_error("refgpu_eval: pairlist step needs xyzq");
    const float4* hx = xyzq ? (const float4*)xyzq : h->tl->get_xyzq();
    if (doPairlist) {
      h->tl->buildTileLists(h->numTileListsPrev, h->numPatches, h->atomStorageSize,
                            h->maxTileListLen, a, b, c, h->patches.data(), hx, h->plcutoff2,
                            h->maxShmem, h->stream, true, false, false, false);
      h->tl->prepareTileList(h->stream);
      h->tl->clearTileListStat(h->stream);
    }
    const bool table = h->doTable || doSlow;
    h->nb->nonbondedForce(*h->tl, h->atomStorageSize, doPairlist != 0, false, doPairlist != 0,
                          doEnergy != 0, doVirial != 0, doSlow != 0, false, false, false, false,
                          table, a, b, c, hx, h->cutoff2, h->c, h->d_forces, h->d_forcesSlow,
                          nullptr, nullptr, nullptr, false, nullptr, false, false, h->stream);
    if (doPairlist) h->tl->finishTileList(h->stream);
    h->nb->reduceVirialEnergy(*h->tl, h->atomStorageSize, doEnergy != 0, doVirial != 0,
                              doSlow != 0, false, h->d_forces, h->d_forcesSlow, h->d_ve,
                              h->stream);
    if (doPairlist) {
      h->tl->reSortTileLists(false, h->stream);
      h->listsReady = true;
    }
    ck(cudaGetLastError(), "eval launch");
  });
}

int refgpu_sync(void* hp) {
  RefGpu* h = (RefGpu*)hp;
  return guarded(h, [&] { ck(cudaStreamSynchronize(h->stream), "sync"); });
}

void* refgpu_stream(void* hp) { return ((RefGpu*)hp)->stream; }

// Runs this instance on a caller's stream from now on (NULL: back to its
// own). Several instances on one stream evaluate one after another.
int refgpu_set_stream(void* hp, void* stream) {
  RefGpu* h = (RefGpu*)hp;
  return guarded(h, [&] {
    ck(cudaStreamSynchronize(h->stream), "set_stream sync");
    if (stream) {
      if (h->ownStream) ck(cudaStreamDestroy(h->stream), "own stream destroy");
      h->stream = (cudaStream_t)stream;
      h->ownStream = false;
    } else if (!h->ownStream) {
      ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
      h->ownStream = true;
    }
  });
}
void* refgpu_device_xyzq(void* hp) { return ((RefGpu*)hp)->tl->get_xyzq(); }
void* refgpu_device_forces(void* hp, int slow) {
  RefGpu* h = (RefGpu*)hp;
  return slow ? (void*)h->d_forcesSlow : (void*)h->d_forces;
}

// forces / forcesSlow: [4*atomStorageSize] host; ve: [21] = virial[9],
// virialSlow[9], energyVdw, energyElec, energySlow. Synchronises.
int refgpu_results(void* hp, float* forces, float* forcesSlow, double* ve) {
  RefGpu* h = (RefGpu*)hp;
  return guarded(h, [&] {
    ck(cudaStreamSynchronize(h->stream), "results sync");
    if (forces)
      ck(cudaMemcpy(forces, h->d_forces, sizeof(float4) * h->atomStorageSize,
                    cudaMemcpyDeviceToHost),
         "forces copy");
    if (forcesSlow)
      ck(cudaMemcpy(forcesSlow, h->d_forcesSlow, sizeof(float4) * h->atomStorageSize,
                    cudaMemcpyDeviceToHost),
         "forcesSlow copy");
    if (ve) {
      VirialEnergy v;
      ck(cudaMemcpy(&v, h->d_ve, sizeof(v), cudaMemcpyDeviceToHost), "ve copy");
      for (int k = 0; k < 9; ++k) ve[k] = v.virial[k];
      for (int k = 0; k < 9; ++k) ve[9 + k] = v.virialSlow[k];
      ve[18] = v.energyVdw;
      ve[19] = v.energyElec;
      ve[20] = v.energySlow;
    }
  });
}

// Sizes of the refined, re-sorted tile lists: [0] lists, [1] j tiles,
// [2] excluded pairs counted by the refinement.
int refgpu_tile_list_sizes(void* hp, int* out3) {
  RefGpu* h = (RefGpu*)hp;
  return guarded(h, [&] {
    out3[0] = h->tl->getNumTileLists();
    out3[1] = h->tl->getNumJtiles();
    out3[2] = h->tl->getNumExcluded();
  });
}

// lists: [numLists] TileList (48 B); jatom: [numJtiles]; excl: [numJtiles] TileExcl.
int refgpu_tile_lists(void* hp, void* lists, int* jatom, void* excl) {
  RefGpu* h = (RefGpu*)hp;
  return guarded(h, [&] {
    ck(cudaStreamSynchronize(h->stream), "lists sync");
    const int nl = h->tl->getNumTileLists(), nj = h->tl->getNumJtiles();
    if (lists)
      ck(cudaMemcpy(lists, h->tl->getTileLists(), sizeof(TileList) * nl, cudaMemcpyDeviceToHost),
         "lists copy");
    if (jatom)
      ck(cudaMemcpy(jatom, h->tl->getTileJatomStart(), sizeof(int) * nj, cudaMemcpyDeviceToHost),
         "jatom copy");
    if (excl)
      ck(cudaMemcpy(excl, h->tl->getTileExcls(), sizeof(TileExcl) * nj, cudaMemcpyDeviceToHost),
         "excl copy");
  });
}

int refgpu_destroy(void* hp) {
  RefGpu* h = (RefGpu*)hp;
  if (!h) return 0;
  const int rc = guarded(h, [&] {
    cudaStreamSynchronize(h->stream);
    delete h->nb;
    delete h->tl;
    delete h->tables;
    if (h->d_forces) cudaFree(h->d_forces);
    if (h->d_forcesSlow) cudaFree(h->d_forcesSlow);
    if (h->d_ve) cudaFree(h->d_ve);
    if (h->ownStream) cudaStreamDestroy(h->stream);
    delete h->dc;
  });
  deviceCUDA = nullptr;
  delete h;
  return rc;
}

}  // extern "C"
