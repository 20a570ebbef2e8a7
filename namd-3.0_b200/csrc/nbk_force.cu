// Nonbonded force kernel of the B200 path.
//
// One warp owns one tile list (32 i atoms of one patch against the j tiles of
// a compute's partner patch), as CudaComputeNonbondedKernel's
// nonbondedForceKernel does (src/CudaComputeNonbondedKernel.cu:629-1644), but:
//   - j forces ride in registers and rotate one lane per step with a shuffle
//     (lane l works on j = (l+t) & 31 at step t), so the inner loop touches
//     shared memory only for the broadcast-free j coordinate load;
//   - in steady state, steps whose bit is clear in every lane's mask are
//     skipped warp-uniformly (the rotation jumps by the step distance);
//   - per-tile FP32 partial forces are folded into 64-bit fixed point with
//     integer atomics, so the summed forces do not depend on the order in
//     which lists run; energies and virials are folded into fixed point per
//     list for the same reason.
#include "nbk_internal.cuh"
#include "nbk_launch.h"

namespace nbk {

constexpr int kForceWarps = 4;
constexpr int kForceThreads = kForceWarps * kWarp;

template <bool doEnergy, bool doVirial, bool doSlow, bool doPairlist>
__global__ void __launch_bounds__(kForceThreads)
    forceKernel(const __grid_constant__ ForceArgs a) {
  extern __shared__ float2 s_lj[];  // [ljDim*ljDim]
  __shared__ float4 s_xyzq[kForceWarps][kWarp];
  __shared__ int s_type[kForceWarps][kWarp];
  __shared__ int s_jidx[kForceWarps][kWarp];
  __shared__ long long s_red[kForceWarps][kAccCount];

  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const NbkConst& c = a.c;
  const int dim = c.ljDim;
  for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) s_lj[k] = a.ljTable[k];
  __syncthreads();

  const int numLists = a.numListsDev ? *a.numListsDev : a.numListsHost;

  // per-warp fixed-point accumulators: lane k < 9 owns virial[k], 9 <= k < 18
  // owns virialSlow[k-9]; lane 0 also owns the three energies.
  long long accE0 = 0, accE1 = 0, accE2 = 0, accVir = 0;
  int nexcl = 0;
  int npair = 0;  // interacting pairs seen by this lane (energy evaluations)

  for (int L = blockIdx.x * kForceWarps + wib; L < numLists; L += gridDim.x * kForceWarps) {
    const nbk_tile_list tl = a.lists[L];
    if (tl.jtileEnd < tl.jtileStart) continue;  // empty (warp-uniform)
    const float3 off = make_float3(tl.offsetXYZ.x, tl.offsetXYZ.y, tl.offsetXYZ.z);
    const float3 sh = shiftOf(off, a.lata, a.latb, a.latc);
    const bool zeroShift = !(dist2(sh.x, sh.y, sh.z) > 0.0f);
    const bool selfCompute = (tl.patchInd.x == tl.patchInd.y) && zeroShift;

    const int iatom = tl.iatomStart + lane;
    float4 xi = a.xyzq[iatom];
    xi.x = __fadd_rn(xi.x, sh.x);
    xi.y = __fadd_rn(xi.y, sh.y);
    xi.z = __fadd_rn(xi.z, sh.z);
    const int ti = a.vdwTypes[iatom] * dim;

    int nfreei = 32, jatomSize = 0, jatomFreeSize = 0, iIndex = 0, exBase = 0, exMax = -1;
    if (doPairlist) {
      const PatchPair pp = a.patchPairs[L];
      const int nloopi = min(pp.iatomSize - tl.iatomStart, 32);
      nfreei = max(pp.iatomFreeSize - tl.iatomStart, 0);
      jatomSize = pp.jatomSize;
      jatomFreeSize = pp.jatomFreeSize;
      if (lane >= nloopi) xi.x = xi.y = xi.z = -1.0e10f;
      iIndex = a.atomIndex[iatom];
      const int2 em = a.exclIndexMaxDiff[iatom];
      exBase = em.x;
      exMax = em.y;
    }

    float fix = 0.f, fiy = 0.f, fiz = 0.f, fisx = 0.f, fisy = 0.f, fisz = 0.f;
    double eV = 0.0, eE = 0.0, eS = 0.0;
    int activeTiles = 0;

    for (int jt = tl.jtileStart; jt <= tl.jtileEnd; ++jt) {
      const int jstart = a.tileJatomStart[jt];
      unsigned mask = 0;
      unsigned stepMask;
      if (!doPairlist) {
        mask = a.tileExcls[jt].excl[lane];
        stepMask = __reduce_or_sync(0xffffffffu, mask);
        if (stepMask == 0) continue;
      } else {
        stepMask = 0xffffffffu;
      }
      const bool diag = selfCompute && (jstart == tl.iatomStart);
      float4 xj = a.xyzq[jstart + lane];
      int nfreej = 32;
      if (doPairlist) {
        const int nloopj = min(jatomSize - jstart, 32);
        nfreej = max(jatomFreeSize - jstart, 0);
        if (lane >= nloopj) xj.x = xj.y = xj.z = 1.0e10f;
        s_jidx[wib][lane] = a.atomIndex[jstart + lane];
      }
      s_xyzq[wib][lane] = xj;
      s_type[wib][lane] = a.vdwTypes[jstart + lane];
      __syncwarp();

      float fjx = 0.f, fjy = 0.f, fjz = 0.f, fjsx = 0.f, fjsy = 0.f, fjsz = 0.f;
      float eVt = 0.f, eEt = 0.f, eSt = 0.f;
      unsigned newMask = 0;
      int tPrev = 0;
      while (stepMask) {
        const int t = __ffs(stepMask) - 1;
        stepMask &= stepMask - 1;
        // rotate the j accumulators so this lane holds those of j = (lane+t)&31
        const int delta = t - tPrev;
        if (delta) {
          const int src = (lane + delta) & 31;
          fjx = __shfl_sync(0xffffffffu, fjx, src);
          fjy = __shfl_sync(0xffffffffu, fjy, src);
          fjz = __shfl_sync(0xffffffffu, fjz, src);
          if (doSlow) {
            fjsx = __shfl_sync(0xffffffffu, fjsx, src);
            fjsy = __shfl_sync(0xffffffffu, fjsy, src);
            fjsz = __shfl_sync(0xffffffffu, fjsz, src);
          }
        }
        tPrev = t;
        const int j = (lane + t) & 31;
        const float4 xjj = s_xyzq[wib][j];
        const float dx = __fsub_rn(xjj.x, xi.x);
        const float dy = __fsub_rn(xjj.y, xi.y);
        const float dz = __fsub_rn(xjj.z, xi.z);
        const float r2 = dist2(dx, dy, dz);
        bool active;
        if (doPairlist) {
          bool cand = diag ? (t > 0 && lane + t < 32) : true;
          cand = cand && (r2 < c.plcutoff2) && (j < nfreej || lane < nfreei);
          bool excluded = false;
          if (cand) {
            int diff = s_jidx[wib][j] - iIndex;
            if (abs(diff) <= exMax) {
              const unsigned bit = (unsigned)(diff + exBase);
              const unsigned w = ((int)(bit >> 5) < a.numExclWords) ? __ldg(&a.exclBits[bit >> 5]) : 0u;
              excluded = (w >> (bit & 31)) & 1u;
            }
            if (excluded) ++nexcl;
            else newMask |= 1u << t;
          }
          active = cand && !excluded && (r2 < c.cutoff2);
        } else {
          active = ((mask >> t) & 1u) && (r2 < c.cutoff2);
        }
        if (active) {
          if (doEnergy) ++npair;
          const float2 ab = s_lj[ti + s_type[wib][j]];
          float f, fs;
          pairForce<doEnergy, doSlow>(r2, xi.w * xjj.w, ab, c, f, fs, eVt, eEt, eSt);
          const float fx = dx * f, fy = dy * f, fz = dz * f;
          fix += fx;
          fiy += fy;
          fiz += fz;
          fjx -= fx;
          fjy -= fy;
          fjz -= fz;
          if (doSlow) {
            const float sx = dx * fs, sy = dy * fs, sz = dz * fs;
            fisx += sx;
            fisy += sy;
            fisz += sz;
            fjsx -= sx;
            fjsy -= sy;
            fjsz -= sz;
          }
        }
      }
      // final rotation: lane l holds the accumulators of j = l again
      {
        const int src = (lane + (32 - tPrev)) & 31;
        fjx = __shfl_sync(0xffffffffu, fjx, src);
        fjy = __shfl_sync(0xffffffffu, fjy, src);
        fjz = __shfl_sync(0xffffffffu, fjz, src);
        if (doSlow) {
          fjsx = __shfl_sync(0xffffffffu, fjsx, src);
          fjsy = __shfl_sync(0xffffffffu, fjsy, src);
          fjsz = __shfl_sync(0xffffffffu, fjsz, src);
        }
      }
      const int jatom = jstart + lane;
      if (fjx != 0.f || fjy != 0.f || fjz != 0.f) {
        atomicAddFixed(&a.force[0 * (size_t)a.stride + jatom], toFixedForce(fjx));
        atomicAddFixed(&a.force[1 * (size_t)a.stride + jatom], toFixedForce(fjy));
        atomicAddFixed(&a.force[2 * (size_t)a.stride + jatom], toFixedForce(fjz));
      }
      if (doSlow && (fjsx != 0.f || fjsy != 0.f || fjsz != 0.f)) {
        atomicAddFixed(&a.force[3 * (size_t)a.stride + jatom], toFixedForce(fjsx));
        atomicAddFixed(&a.force[4 * (size_t)a.stride + jatom], toFixedForce(fjsy));
        atomicAddFixed(&a.force[5 * (size_t)a.stride + jatom], toFixedForce(fjsz));
      }
      if (doEnergy) {
        eV += (double)eVt;
        eE += (double)eEt;
        if (doSlow) eS += (double)eSt;
      }
      if (doPairlist) {
        a.tileExcls[jt].excl[lane] = newMask;
        const bool any = __any_sync(0xffffffffu, newMask != 0);
        if (lane == 0) a.jtileActive[jt] = any ? 1 : 0;
        activeTiles += any ? 1 : 0;
      }
      __syncwarp();
    }  // jt

    // i forces (fixed point) and the list's shift part of the virial
    const unsigned long long qx = toFixedForce(fix), qy = toFixedForce(fiy), qz = toFixedForce(fiz);
    if (fix != 0.f || fiy != 0.f || fiz != 0.f) {
      atomicAddFixed(&a.force[0 * (size_t)a.stride + iatom], qx);
      atomicAddFixed(&a.force[1 * (size_t)a.stride + iatom], qy);
      atomicAddFixed(&a.force[2 * (size_t)a.stride + iatom], qz);
    }
    unsigned long long sx = 0, sy = 0, sz = 0;
    if (doSlow) {
      sx = toFixedForce(fisx);
      sy = toFixedForce(fisy);
      sz = toFixedForce(fisz);
      if (fisx != 0.f || fisy != 0.f || fisz != 0.f) {
        atomicAddFixed(&a.force[3 * (size_t)a.stride + iatom], sx);
        atomicAddFixed(&a.force[4 * (size_t)a.stride + iatom], sy);
        atomicAddFixed(&a.force[5 * (size_t)a.stride + iatom], sz);
      }
    }
    if (doVirial && !zeroShift) {
      // W[a][b] += (sum_i F_i)[a] * shift[b] for this list
      const long long Fx = warpSumLL((long long)qx), Fy = warpSumLL((long long)qy),
                      Fz = warpSumLL((long long)qz);
      long long Gx = 0, Gy = 0, Gz = 0;
      if (doSlow) {
        Gx = warpSumLL((long long)sx);
        Gy = warpSumLL((long long)sy);
        Gz = warpSumLL((long long)sz);
      }
      if (lane < 18) {
        const int comp = lane % 9;
        const int ca = comp / 3, cb = comp % 3;
        long long Fa;
        if (lane < 9) Fa = (ca == 0) ? Fx : (ca == 1) ? Fy : Fz;
        else Fa = (ca == 0) ? Gx : (ca == 1) ? Gy : Gz;
        const float s_b = (cb == 0) ? sh.x : (cb == 1) ? sh.y : sh.z;
        if (lane < 9 || doSlow)
          accVir += toFixedEnergy((double)Fa * kForceScaleInv * (double)s_b);
      }
    }
    if (doEnergy) {
      const double sV = warpSumD(eV), sE = warpSumD(eE), sS = doSlow ? warpSumD(eS) : 0.0;
      if (lane == 0) {
        accE0 += toFixedEnergy(sV);
        accE1 += toFixedEnergy(sE);
        accE2 += toFixedEnergy(sS);
      }
    }
    if (doPairlist && lane == 0) a.listActive[L] = activeTiles;
  }  // lists

  // block reduction of the fixed-point accumulators, then one atomic each
  if (doEnergy || doVirial || doPairlist) {
    long long* r = s_red[wib];
    if (lane < kAccCount) r[lane] = 0;
    __syncwarp();
    if (doVirial && lane < 18) r[kAccVir + lane] = accVir;
    if (doEnergy && lane == 0) {
      r[kAccEVdw] = accE0;
      r[kAccEElec] = accE1;
      r[kAccESlow] = accE2;
    }
    if (doPairlist) {
      int s = nexcl;
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) r[kAccNumExcl] = s;
    }
    if (doEnergy) {
      int s = npair;
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) r[kAccNumPairs] = s;
    }
    __syncthreads();
    if (threadIdx.x < kAccCount) {
      long long tot = 0;
      for (int w = 0; w < kForceWarps; ++w) tot += s_red[w][threadIdx.x];
      if (tot != 0) atomicAddFixed(&a.acc[threadIdx.x], (unsigned long long)tot);
    }
  }
}

template <bool E, bool V, bool S, bool P>
static cudaError_t launchT(const ForceArgs& a, int grid, cudaStream_t st) {
  const size_t shmem = sizeof(float2) * (size_t)a.c.ljDim * a.c.ljDim;
  auto k = forceKernel<E, V, S, P>;
  if (shmem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
    if (e != cudaSuccess) return e;
  }
  k<<<grid, kForceThreads, shmem, st>>>(a);
  return cudaGetLastError();
}

template <bool E, bool V, bool S, bool P>
static int occupancyT(int ljDim) {
  int nb = 0;
  const size_t shmem = sizeof(float2) * (size_t)ljDim * ljDim;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, forceKernel<E, V, S, P>, kForceThreads, shmem);
  return nb;
}

cudaError_t launchForce(const ForceArgs& a, unsigned flags, int numSM, cudaStream_t st) {
  const bool E = flags & NBK_ENERGY, V = flags & NBK_VIRIAL, S = flags & NBK_SLOW,
             P = flags & NBK_PAIRLIST;
  const int idx = (E ? 8 : 0) | (V ? 4 : 0) | (S ? 2 : 0) | (P ? 1 : 0);
  static int occ[16] = {0};
  static int occDim[16] = {0};
  int nb = (occDim[idx] == a.c.ljDim) ? occ[idx] : 0;
  if (nb == 0) {
#define NBK_OCC(i, e, v, s, p) \
  case i:                      \
    nb = occupancyT<e, v, s, p>(a.c.ljDim); \
    break;
    switch (idx) {
      NBK_OCC(0, false, false, false, false)
      NBK_OCC(1, false, false, false, true)
      NBK_OCC(2, false, false, true, false)
      NBK_OCC(3, false, false, true, true)
      NBK_OCC(4, false, true, false, false)
      NBK_OCC(5, false, true, false, true)
      NBK_OCC(6, false, true, true, false)
      NBK_OCC(7, false, true, true, true)
      NBK_OCC(8, true, false, false, false)
      NBK_OCC(9, true, false, false, true)
      NBK_OCC(10, true, false, true, false)
      NBK_OCC(11, true, false, true, true)
      NBK_OCC(12, true, true, false, false)
      NBK_OCC(13, true, true, false, true)
      NBK_OCC(14, true, true, true, false)
      NBK_OCC(15, true, true, true, true)
    }
#undef NBK_OCC
    if (nb <= 0) nb = 1;
    occ[idx] = nb;
    occDim[idx] = a.c.ljDim;
  }
  const int grid = numSM * nb;
#define NBK_LAUNCH(i, e, v, s, p) \
  case i:                         \
    return launchT<e, v, s, p>(a, grid, st);
  switch (idx) {
    NBK_LAUNCH(0, false, false, false, false)
    NBK_LAUNCH(1, false, false, false, true)
    NBK_LAUNCH(2, false, false, true, false)
    NBK_LAUNCH(3, false, false, true, true)
    NBK_LAUNCH(4, false, true, false, false)
    NBK_LAUNCH(5, false, true, false, true)
    NBK_LAUNCH(6, false, true, true, false)
    NBK_LAUNCH(7, false, true, true, true)
    NBK_LAUNCH(8, true, false, false, false)
    NBK_LAUNCH(9, true, false, false, true)
    NBK_LAUNCH(10, true, false, true, false)
    NBK_LAUNCH(11, true, false, true, true)
    NBK_LAUNCH(12, true, true, false, false)
    NBK_LAUNCH(13, true, true, false, true)
    NBK_LAUNCH(14, true, true, true, false)
    NBK_LAUNCH(15, true, true, true, true)
  }
#undef NBK_LAUNCH
  return cudaErrorInvalidValue;
}

}  // namespace nbk
