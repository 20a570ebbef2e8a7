// GPU-resident input marshaling: the patch sort, the patch-centred xyzq and
// the per-slot vdW types / exclusion indices built on the device from the
// integrator's per-atom arrays (declared in include/nbk.h).
//
// The reference does this work on the host for the non-resident path
// (src/SortAtoms.C:45-133, src/HomePatch.C:1054-1131,
// src/CudaComputeNonbonded.C:836-930) and with the GPU-resident integrator in
// setComputePositionsKernel (src/SequencerCUDAKernel.cu:1950-2041) and
// updateVdwTypesExclKernel (src/CudaComputeNonbondedKernel.cu:3648-3724).
// Here one block handles one patch for all three; the sort keeps the whole
// patch in shared memory and ranks atoms by counting, so it needs no global
// scratch and no host round trip.
#include <cuda_runtime.h>

#include <string>

#include "nbk.h"
#include "nbk_internal.cuh"
#include "nbk_launch.h"

namespace nbk {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
// every part that is split straddles an 8-atom block boundary of its own, so a
// level splits at most N/8 parts into at most N/4
constexpr int kMaxRanges = NBK_MAX_PATCH_ATOMS / 4;

struct Lattice12 {
  double ax, ay, az, bx, by, bz, cx, cy, cz, ox, oy, oz;
};

// Split point of the part [begin, end) of a patch (positions within the
// patch): the first of 32, 16, 8 whose blocks the part straddles, at the
// block boundary nearest the middle; -1 when the part is not split further.
__device__ __forceinline__ int splitPoint(int begin, int end) {
  int W = 0;
  if (begin / 32 < (end - 1) / 32) W = 32;
  else if (begin / 16 < (end - 1) / 16) W = 16;
  else if (begin / 8 < (end - 1) / 8) W = 8;
  if (W == 0) return -1;
  int split = ((begin + end + W) / (2 * W)) * W;
  if (split <= begin) split += W;
  if (split >= end) split -= W;
  if (split <= begin || split >= end) return -1;
  return split;
}

// One block per patch. Shared memory (dynamic) per atom for maxN atoms: x, y,
// z and the current sort key (double), id, ord, tmp and the key's id (int).
__global__ void __launch_bounds__(kSortThreads)
    sortPatchAtomsKernel(int numPatches, const nbk_local_record* __restrict__ rec, int maxN,
                         const double* __restrict__ px, const double* __restrict__ py,
                         const double* __restrict__ pz, const int* __restrict__ gid,
                         int* __restrict__ sortOrder, int* __restrict__ status) {
  extern __shared__ double s_dyn[];
  double* s_x = s_dyn;
  double* s_y = s_x + maxN;
  double* s_z = s_y + maxN;
  double* s_key = s_z + maxN;  // by position: the coordinate the position's part is split on
  int* s_id = reinterpret_cast<int*>(s_key + maxN);
  int* s_ord = s_id + maxN;
  int* s_tmp = s_ord + maxN;
  int* s_kid = s_tmp + maxN;   // by position: the atom id (tie break)
  __shared__ int s_rb[kMaxRanges], s_re[kMaxRanges], s_rs[kMaxRanges], s_ax[kMaxRanges];
  __shared__ int s_split[kMaxRanges / 2];
  __shared__ int s_numRanges, s_numNext;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  for (int p = blockIdx.x; p < numPatches; p += gridDim.x) {
    const int n = rec[p].numAtoms, off = rec[p].bufferOffset;
    if (n <= 0) continue;  // block-uniform
    if (n > maxN) {
      for (int k = threadIdx.x; k < n; k += blockDim.x) sortOrder[off + k] = k;
      if (threadIdx.x == 0 && status) atomicAdd(status, 1);
      continue;
    }
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      s_x[k] = px[off + k];
      s_y[k] = py[off + k];
      s_z[k] = pz[off + k];
      s_id[k] = gid[off + k];
      s_ord[k] = k;
    }
    if (threadIdx.x == 0) {
      s_rb[0] = 0;
      s_re[0] = n;
      s_numRanges = 1;
    }
    __syncthreads();
    for (;;) {  // one level of the bisection per pass; every split part is ordered by rank
      const int nr = s_numRanges;
      if (nr == 0) break;  // block-uniform
      // split point and longest axis of every part (a warp per part)
      for (int r = wib; r < nr; r += kSortWarps) {
        const int b = s_rb[r], e = s_re[r];
        const int sp = splitPoint(b, e);
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        if (sp >= 0) {
          for (int k = b + lane; k < e; k += 32) {
            const int a = s_ord[k];
            lo[0] = fmin(lo[0], s_x[a]);
            hi[0] = fmax(hi[0], s_x[a]);
            lo[1] = fmin(lo[1], s_y[a]);
            hi[1] = fmax(hi[1], s_y[a]);
            lo[2] = fmin(lo[2], s_z[a]);
            hi[2] = fmax(hi[2], s_z[a]);
          }
#pragma unroll
          for (int o = 16; o >= 1; o >>= 1)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
              hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
            }
        }
        if (lane == 0) {
          int axis = 0;
          if (hi[1] - lo[1] > hi[0] - lo[0]) axis = 1;
          if (hi[2] - lo[2] > hi[axis] - lo[axis]) axis = 2;
          s_rs[r] = sp;
          s_ax[r] = axis;
        }
      }
      __syncthreads();
      // the split key of every position of a split part, stored by position so
      // that the ranking reads it without indirection
      for (int r = 0; r < nr; ++r) {
        const int b = s_rb[r], e = s_re[r];
        if (s_rs[r] < 0) continue;
        const double* key = s_ax[r] == 0 ? s_x : (s_ax[r] == 1 ? s_y : s_z);
        for (int k = b + threadIdx.x; k < e; k += blockDim.x) {
          const int a = s_ord[k];
          s_key[k] = key[a];
          s_kid[k] = s_id[a];
        }
      }
      __syncthreads();
      // rank every atom of a split part by (coordinate on the part's axis, id)
      for (int r = 0; r < nr; ++r) {
        const int b = s_rb[r], e = s_re[r];
        if (s_rs[r] < 0) continue;
        for (int k = b + threadIdx.x; k < e; k += blockDim.x) {
          const double ka = s_key[k];
          const int ia = s_kid[k];
          int rank = 0;
          for (int m = b; m < e; ++m) {
            const double kc = s_key[m];
            rank += (kc < ka || (kc == ka && s_kid[m] < ia)) ? 1 : 0;
          }
          s_tmp[b + rank] = s_ord[k];
        }
      }
      __syncthreads();
      for (int r = 0; r < nr; ++r) {
        if (s_rs[r] < 0) continue;
        for (int k = s_rb[r] + threadIdx.x; k < s_re[r]; k += blockDim.x) s_ord[k] = s_tmp[k];
      }
      // the next level's parts: both halves of every split part
      if (threadIdx.x == 0) {
        int m = 0;
        for (int r = 0; r < nr; ++r)
          if (s_rs[r] >= 0) s_split[m++] = r;
        s_numNext = m;
      }
      __syncthreads();
      const int m = s_numNext;  // at most kMaxRanges / 2 = kSortThreads
      int nb = 0, ne = 0, nsp = 0;
      if (threadIdx.x < m) {
        const int r = s_split[threadIdx.x];
        nb = s_rb[r];
        ne = s_re[r];
        nsp = s_rs[r];
      }
      __syncthreads();
      if (threadIdx.x < m) {
        s_rb[2 * threadIdx.x] = nb;
        s_re[2 * threadIdx.x] = nsp;
        s_rb[2 * threadIdx.x + 1] = nsp;
        s_re[2 * threadIdx.x + 1] = ne;
      }
      if (threadIdx.x == 0) s_numRanges = 2 * m;
      __syncthreads();
    }
    for (int k = threadIdx.x; k < n; k += blockDim.x) sortOrder[off + k] = s_ord[k];
    __syncthreads();
  }
}

__global__ void computePositionsKernel(int numPatches, const nbk_local_record* __restrict__ rec,
                                       const double3* __restrict__ centre, const Lattice12 L,
                                       const int* __restrict__ sortOrder, double qscale,
                                       const double* __restrict__ px, const double* __restrict__ py,
                                       const double* __restrict__ pz,
                                       const float* __restrict__ charge, float4* __restrict__ xyzq) {
  for (int p = blockIdx.x; p < numPatches; p += gridDim.x) {
    const int n = rec[p].numAtoms, off = rec[p].bufferOffset, offNB = rec[p].bufferOffsetNBPad;
    const int npad = rec[p].numAtomsNBPad;
    if (n <= 0) continue;
    const double3 s = centre[p];
    // Lattice::unscale: o + a sx + b sy + c sz
    const double ux = L.ox + L.ax * s.x + L.bx * s.y + L.cx * s.z;
    const double uy = L.oy + L.ay * s.x + L.by * s.y + L.cy * s.z;
    const double uz = L.oz + L.az * s.x + L.bz * s.y + L.cz * s.z;
    for (int i = threadIdx.x; i < npad; i += blockDim.x) {
      const int a = off + min(max(sortOrder[off + min(i, n - 1)], 0), n - 1);
      float4 q;
      q.x = (float)(px[a] - ux);
      q.y = (float)(py[a] - uy);
      q.z = (float)(pz[a] - uz);
      q.w = (float)((double)charge[a] * qscale);
      xyzq[offNB + i] = q;
    }
  }
}

__global__ void updateVdwTypesExclDeviceKernel(int numPatches, const nbk_local_record* __restrict__ rec,
                                               const int* __restrict__ vdw, const int* __restrict__ gid,
                                               const int* __restrict__ sortOrder,
                                               const int2* __restrict__ exclByAtom, int numExclAtoms,
                                               int ljDim, int storage, int* __restrict__ vdwTypes,
                                               int* __restrict__ atomIndex, int2* __restrict__ excl,
                                               int* __restrict__ status) {
  for (int p = blockIdx.x; p < numPatches; p += gridDim.x) {
    const int n = rec[p].numAtoms, off = rec[p].bufferOffset, offNB = rec[p].bufferOffsetNBPad;
    const int npad = rec[p].numAtomsNBPad;
    if (n <= 0) continue;
    for (int i = threadIdx.x; i < npad; i += blockDim.x) {
      if (offNB + i >= storage) break;
      const int a = off + min(max(sortOrder[off + min(i, n - 1)], 0), n - 1);
      int t = vdw[a];
      const int id = gid[a];
      int2 e = make_int2(0, 0);
      bool bad = false;
      if (t < 0 || t >= ljDim) {
        t = 0;
        bad = true;
      }
      if (id >= 0 && id < numExclAtoms) {
        const int2 m = exclByAtom[id];  // (maxdiff, base)
        e = make_int2(m.y, m.x);
      } else {
        bad = true;
      }
      vdwTypes[offNB + i] = t;
      atomIndex[offNB + i] = id;
      excl[offNB + i] = e;
      if (bad && status && i < n) atomicAdd(status, 1);
    }
  }
}

__global__ void accumulateForcesKernel(const __grid_constant__ AccumulateArgs a) {
  for (int p = blockIdx.x; p < a.numPatches; p += gridDim.x) {
    const int n = a.rec[p].numAtoms, off = a.rec[p].bufferOffset, offNB = a.rec[p].bufferOffsetNBPad;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int b = off + min(max(a.sortOrder[off + k], 0), n - 1);  // buffer index of slot k
      const size_t slot = (size_t)offNB + k;
      double fn[3], fb[3], fs[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        fn[c] = a.fBond ? a.fBond[b + (size_t)c * a.forceStride] : 0.0;
        fb[c] = (double)a.fixed[slot + (size_t)c * a.stride] * kForceScaleInv;
        if (a.fBondNbond) fb[c] += a.fBondNbond[b + (size_t)c * a.forceStride];
        fs[c] = a.fPme ? (double)(&a.fPme[b].x)[c] : 0.0;
        fs[c] += (double)a.fixed[slot + (size_t)(3 + c) * a.stride] * kForceScaleInv;
        if (a.fBondSlow) fs[c] += a.fBondSlow[b + (size_t)c * a.forceStride];
      }
      a.fNormal[0][b] = fn[0];
      a.fNormal[1][b] = fn[1];
      a.fNormal[2][b] = fn[2];
      if (a.maxForceNumber >= 1) {
        a.fNbond[0][b] = fb[0];
        a.fNbond[1][b] = fb[1];
        a.fNbond[2][b] = fb[2];
      }
      if (a.maxForceNumber >= 2) {
        a.fSlow[0][b] = fs[0];
        a.fSlow[1][b] = fs[1];
        a.fSlow[2][b] = fs[2];
      }
    }
  }
}

}  // namespace

cudaError_t launchAccumulateForces(const AccumulateArgs& a, cudaStream_t st) {
  if (a.numPatches <= 0) return cudaSuccess;
  accumulateForcesKernel<<<min(a.numPatches, 65535), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launchUpdateVdwTypesExclDevice(int numPatches, const nbk_local_record* rec,
                                           const int* vdw, const int* gid, const int* sortOrder,
                                           const int2* exclByAtom, int numExclAtoms, int ljDim,
                                           int storage, int* vdwTypes, int* atomIndex, int2* excl,
                                           int* status, cudaStream_t st) {
  if (numPatches <= 0) return cudaSuccess;
  updateVdwTypesExclDeviceKernel<<<min(numPatches, 65535), 256, 0, st>>>(
      numPatches, rec, vdw, gid, sortOrder, exclByAtom, numExclAtoms, ljDim, storage, vdwTypes,
      atomIndex, excl, status);
  return cudaGetLastError();
}

}  // namespace nbk

using namespace nbk;

extern "C" NBK_API int nbk_sort_patch_atoms(int numPatches, const nbk_local_record* d_rec,
                                            int maxPatchAtoms, const double* d_x, const double* d_y,
                                            const double* d_z, const int* d_id, int* d_sortOrder,
                                            int* d_status, void* stream) {
  if (numPatches < 0 || (numPatches && (!d_rec || !d_x || !d_y || !d_z || !d_id || !d_sortOrder)))
    return setLastError(NBK_ERR_ARG, "nbk_sort_patch_atoms: NULL argument");
  if (maxPatchAtoms < 1 || maxPatchAtoms > NBK_MAX_PATCH_ATOMS)
    return setLastError(NBK_ERR_ARG, "nbk_sort_patch_atoms: maxPatchAtoms must be in 1.." +
                                         std::to_string(NBK_MAX_PATCH_ATOMS));
  if (numPatches == 0) return NBK_OK;
  const size_t smem = (size_t)maxPatchAtoms * (4 * sizeof(double) + 4 * sizeof(int));
  cudaError_t e = cudaFuncSetAttribute(sortPatchAtomsKernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    sortPatchAtomsKernel<<<min(numPatches, 65535), kSortThreads, smem, (cudaStream_t)stream>>>(
        numPatches, d_rec, maxPatchAtoms, d_x, d_y, d_z, d_id, d_sortOrder, d_status);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess)
    return setLastError(NBK_ERR_CUDA, std::string("nbk_sort_patch_atoms: ") + cudaGetErrorString(e));
  return NBK_OK;
}

extern "C" NBK_API int nbk_set_compute_positions(int numPatches, const nbk_local_record* d_rec,
                                                 const nbk_double3* d_centre, const double* lattice,
                                                 const int* d_sortOrder, double chargeScaling,
                                                 const double* d_x, const double* d_y,
                                                 const double* d_z, const float* d_charge,
                                                 nbk_float4* d_xyzq, void* stream) {
  if (numPatches < 0 || !lattice ||
      (numPatches && (!d_rec || !d_centre || !d_sortOrder || !d_x || !d_y || !d_z || !d_charge ||
                      !d_xyzq)))
    return setLastError(NBK_ERR_ARG, "nbk_set_compute_positions: NULL argument");
  if (numPatches == 0) return NBK_OK;
  Lattice12 L;
  double* l = &L.ax;
  for (int k = 0; k < 12; ++k) l[k] = lattice[k];
  computePositionsKernel<<<min(numPatches, 65535), 128, 0, (cudaStream_t)stream>>>(
      numPatches, d_rec, reinterpret_cast<const double3*>(d_centre), L, d_sortOrder, chargeScaling,
      d_x, d_y, d_z, d_charge, reinterpret_cast<float4*>(d_xyzq));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return setLastError(NBK_ERR_CUDA,
                        std::string("nbk_set_compute_positions: ") + cudaGetErrorString(e));
  return NBK_OK;
}
