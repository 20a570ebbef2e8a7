// Excluded / modified pair corrections, the fixed-point -> float4 force
// output with the per-atom part of the virial, and the energy/virial read-out.
#include "nbk_internal.cuh"
#include "nbk_launch.h"

namespace nbk {

// One thread per correction tuple (ComputeBondedCUDAKernel modifiedExclusionForce,
// src/ComputeBondedCUDAKernel.cu:315-626, and exclusionForce, :632-778),
// with r_ij = x_i + shift - x_j and analytic pair math in place of the tables.
//   modified (1-4): LJ with (A14 - A, B14 - B); remove (1 - scale14) of the
//     fast Coulomb and of the smooth (3 - r^2/rc^2)/(2 rc) part of the slow one
//   excluded: slow -qq erf(beta r)/r
// Both only within the cutoff, as the reference.
// Adds a thread's energy/virial accumulators (slots 0..20) to one replica's
// block: warp-reduced when the whole warp holds the same replica, else per thread.
__device__ __forceinline__ void flushThreadAcc(long long* accBase, int rep, long long* acc) {
  const int lane = threadIdx.x & 31;
  const int rep0 = __shfl_sync(0xffffffffu, rep, 0);
  const bool uniform = __all_sync(0xffffffffu, rep == rep0);
#pragma unroll
  for (int p = 0; p < kAccCount - 3; ++p) {
    if (uniform) {
      const long long v = warpSumLL(acc[p]);
      if (lane == 0 && v != 0) atomicAddFixed(&accBase[(size_t)rep0 * kAccCount + p], (unsigned long long)v);
    } else if (acc[p] != 0) {
      atomicAddFixed(&accBase[(size_t)rep * kAccCount + p], (unsigned long long)acc[p]);
    }
    acc[p] = 0;
  }
}

// Forces are FP32 (fixed-point accumulated, like the nonbonded kernel's);
// energies and the slow virial are formed per tuple in FP64 from FP64
// geometry (the shift formed in FP64 from the FP32 offsets and lattice), the
// same precision as the force kernel's precise pass; the fast virial comes
// from the forces: the per-atom part in the finalize pass, the shift part
// F_i (x) shift here.
template <bool doEnergy, bool doVirial, bool doSlow>
__global__ void correctionsKernel(const CorrArgs a) {
  const NbkConst& c = a.c;
  const int total = a.numModified + (doSlow ? a.numExcluded : 0);
  long long acc[kAccCount - 3] = {};  // energies + virials, thread-local
  // each warp owns a contiguous range of tuples (lanes interleaved), so its
  // tuples belong to one replica except at replica boundaries
  const int lane = threadIdx.x & 31;
  const int warpsTotal = (gridDim.x * blockDim.x) >> 5;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int per = ((total + warpsTotal - 1) / warpsTotal + 31) & ~31;
  const int kEnd = min(total, (gw + 1) * per);
  int curRep = 0;
  for (int k0 = gw * per; k0 < kEnd; k0 += 32) {
    const int k = k0 + lane;
    const bool valid = k < kEnd;
    const bool modified = k < a.numModified;
    nbk_exclusion e{};
    if (valid) e = modified ? a.modified[k] : a.excluded[k - a.numModified];
    int rep = 0;
    float3 la = a.lata, lb = a.latb, lc = a.latc;
    const float2* ljx = a.ljExclTable;
    if (a.slotRep && valid) {
      rep = a.slotRep[e.i];
      la = a.repLat[3 * rep];
      lb = a.repLat[3 * rep + 1];
      lc = a.repLat[3 * rep + 2];
      ljx = a.repLJExcl + (size_t)rep * c.ljDim * c.ljDim;
    }
    if ((doEnergy || doVirial) && a.slotRep) {
      // a warp-wide replica change flushes the accumulators first
      const bool change = valid && rep != curRep;
      if (__any_sync(0xffffffffu, change)) {
        flushThreadAcc(a.acc, curRep, acc);
        curRep = valid ? rep : curRep;
      }
    }
    if (!valid) continue;
    const float3 sh = shiftOf(make_float3(e.ioffsetXYZ.x, e.ioffsetXYZ.y, e.ioffsetXYZ.z), la, lb, lc);
    const float4 xi = a.xyzq[e.i];
    const float4 xj = a.xyzq[e.j];
    // d = x_j - (x_i + shift): the nonbonded kernel's sign convention
    const float dx = __fsub_rn(xj.x, __fadd_rn(xi.x, sh.x));
    const float dy = __fsub_rn(xj.y, __fadd_rn(xi.y, sh.y));
    const float dz = __fsub_rn(xj.z, __fadd_rn(xi.z, sh.z));
    const float r2 = dist2(dx, dy, dz);
    if (!(r2 < c.cutoff2)) continue;
    const float rinv = rsqrtf(r2);
    const float rinv2 = rinv * rinv;
    const float rinv3 = rinv * rinv2;
    const float qq = xi.w * xj.w;
    float g = 0.f, gs = 0.f;
    float2 ab = make_float2(0.f, 0.f);
    if (modified) {
      ab = ljx[e.vdwtypei * c.ljDim + e.vdwtypej];
      const float rinv6 = rinv2 * rinv2 * rinv2;
      const float ab6 = fmaf(ab.x, rinv6, -ab.y);
      const float w = ab6 * rinv6;
      const float dw = fmaf(ab.x, rinv6, ab6) * (-6.0f * rinv2 * rinv6);
      float s = 1.0f, ds = 0.0f;
      if (c.switching) {
        const float t2 = fmaxf(r2, c.rs2);
        const float d = c.rc2 - t2;
        s = d * d * fmaf(c.lj1, t2, c.lj0);
        ds = d * fmaf(c.lj2, t2, c.lj3);
      }
      const float q14 = c.one14 * qq;
      g = fmaf(w, ds, dw * s) - q14 * (c.rc3inv - rinv3);
      if (doSlow) gs = q14 * c.rc3inv;
    } else {
      const float r = r2 * rinv;
      const float x = c.beta * r;
      // (dE/dr)/r of -qq erf(x)/r is qq (erf(x) - 2/sqrt(pi) x e^{-x^2}) / r^3. The
      // bracket is O(x^3) and cancels badly at excluded-pair distances (O-H:
      // x = 0.25), so below x = 0.5 it is taken from its Taylor series in x^2:
      // 2/sqrt(pi) x sum_{n>=1} (-1)^{n+1} 2n x^{2n} / ((2n+1) n!).
      float bracket;
      if (x < 0.5f) {
        const float y = x * x;
        float q = 1.0f / 5400.0f;
        q = fmaf(q, y, -1.0f / 780.0f);
        q = fmaf(q, y, 1.0f / 132.0f);
        q = fmaf(q, y, -1.0f / 27.0f);
        q = fmaf(q, y, 1.0f / 7.0f);
        q = fmaf(q, y, -2.0f / 5.0f);
        q = fmaf(q, y, 2.0f / 3.0f);
        bracket = 1.1283791671f * x * y * q;
      } else {
        bracket = erff(x) - c.beta2Pi * r * __expf(-x * x);
      }
      gs = qq * bracket * rinv3;
    }
    // F_i += g d, F_j -= g d
    const float fx = g * dx, fy = g * dy, fz = g * dz;
    const unsigned long long qx = toFixedForce(fx), qy = toFixedForce(fy), qz = toFixedForce(fz);
    if (modified) {
      atomicAddFixed(&a.force[0 * (size_t)a.stride + e.i], qx);
      atomicAddFixed(&a.force[1 * (size_t)a.stride + e.i], qy);
      atomicAddFixed(&a.force[2 * (size_t)a.stride + e.i], qz);
      atomicAddFixed(&a.force[0 * (size_t)a.stride + e.j], (unsigned long long)(-(long long)qx));
      atomicAddFixed(&a.force[1 * (size_t)a.stride + e.j], (unsigned long long)(-(long long)qy));
      atomicAddFixed(&a.force[2 * (size_t)a.stride + e.j], (unsigned long long)(-(long long)qz));
    }
    if (doSlow) {
      const unsigned long long sx = toFixedForce(gs * dx), sy = toFixedForce(gs * dy),
                               sz = toFixedForce(gs * dz);
      atomicAddFixed(&a.force[3 * (size_t)a.stride + e.i], sx);
      atomicAddFixed(&a.force[4 * (size_t)a.stride + e.i], sy);
      atomicAddFixed(&a.force[5 * (size_t)a.stride + e.i], sz);
      atomicAddFixed(&a.force[3 * (size_t)a.stride + e.j], (unsigned long long)(-(long long)sx));
      atomicAddFixed(&a.force[4 * (size_t)a.stride + e.j], (unsigned long long)(-(long long)sy));
      atomicAddFixed(&a.force[5 * (size_t)a.stride + e.j], (unsigned long long)(-(long long)sz));
    }
    if (doEnergy || (doVirial && doSlow)) {
      const double S0 = (double)e.ioffsetXYZ.x, S1 = (double)e.ioffsetXYZ.y,
                   S2 = (double)e.ioffsetXYZ.z;
      const double d[3] = {
          (double)xj.x - ((double)xi.x + (S0 * la.x + S1 * lb.x + S2 * lc.x)),
          (double)xj.y - ((double)xi.y + (S0 * la.y + S1 * lb.y + S2 * lc.y)),
          (double)xj.z - ((double)xi.z + (S0 * la.z + S1 * lb.z + S2 * lc.z))};
      const double r2d = fma(d[2], d[2], fma(d[1], d[1], d[0] * d[0]));
      const double ri = rsqrt(r2d), ri2 = ri * ri;
      const double qqd = (double)xi.w * (double)xj.w;
      const NbkConst64& k = a.c64;
      double gsd = 0.0, eVd = 0.0, eEd = 0.0, eSd = 0.0;
      if (modified) {
        const double q14 = k.one14 * qqd, h = fma(k.hB, r2d, k.hA);
        if (doEnergy) {
          const double ri6 = ri2 * ri2 * ri2;
          const double w = fma((double)ab.x, ri6, -(double)ab.y) * ri6;
          double sw = 1.0;
          if (k.switching) {
            const double t2 = fmax(r2d, k.rs2), dd = k.rc2 - t2;
            sw = dd * dd * fma(k.lj1, t2, k.lj0);
          }
          eVd = w * sw;
          eEd = -q14 * (ri - h);
          if (doSlow) eSd = -q14 * h;
        }
        if (doSlow) gsd = q14 * k.rc3inv;
      } else {
        const double r = r2d * ri, x = k.beta * r, erfx = erf(x);
        gsd = qqd * (erfx * ri2 * ri - k.beta2Pi * exp(-x * x) * ri2);
        eSd = -qqd * erfx * ri;
      }
      if (doEnergy) {
        acc[kAccEVdw] += toFixedEnergy(eVd);
        acc[kAccEElec] += toFixedEnergy(eEd);
        acc[kAccESlow] += toFixedEnergy(eSd);
      }
      if (doVirial && doSlow) {
#pragma unroll
        for (int p = 0; p < 9; ++p) acc[kAccVirSlow + p] += toFixedEnergy(-gsd * (d[p / 3] * d[p % 3]));
      }
    }
    if (doVirial && modified) {
      // shift part of the fast virial: F_i (x) shift; the per-atom part comes
      // from the finalize pass
      const double S[3] = {(double)sh.x, (double)sh.y, (double)sh.z};
      const double Fi[3] = {(double)(long long)qx * kForceScaleInv,
                            (double)(long long)qy * kForceScaleInv,
                            (double)(long long)qz * kForceScaleInv};
#pragma unroll
      for (int p = 0; p < 9; ++p) acc[kAccVir + p] += toFixedEnergy(Fi[p / 3] * S[p % 3]);
    }
  }
  if (doEnergy || doVirial) flushThreadAcc(a.acc, a.slotRep ? curRep : 0, acc);
}

cudaError_t launchCorrections(const CorrArgs& a, unsigned flags, cudaStream_t st) {
  const bool E = flags & NBK_ENERGY, V = flags & NBK_VIRIAL, S = flags & NBK_SLOW;
  const int total = a.numModified + (S ? a.numExcluded : 0);
  if (total <= 0) return cudaSuccess;
  const int threads = 256;
  const int blocks = min((total + threads - 1) / threads, 2048);
  const int idx = (E ? 4 : 0) | (V ? 2 : 0) | (S ? 1 : 0);
  switch (idx) {
#define NBK_CASE(i, e, v, s) \
  case i:                    \
    correctionsKernel<e, v, s><<<blocks, threads, 0, st>>>(a); \
    break;
    NBK_CASE(0, false, false, false)
    NBK_CASE(1, false, false, true)
    NBK_CASE(2, false, true, false)
    NBK_CASE(3, false, true, true)
    NBK_CASE(4, true, false, false)
    NBK_CASE(5, true, false, true)
    NBK_CASE(6, true, true, false)
    NBK_CASE(7, true, true, true)
#undef NBK_CASE
  }
  return cudaGetLastError();
}

// Fixed point -> float4 forces (transposeForcesKernel's role,
// src/CudaComputeNonbondedKernel.cu:2057-2072) and the per-atom part of the
// fast virial, sum_i F_i (x) x_i over patch-centred positions
// (reduceNonbondedVirialKernel, :1649-1763), folded into fixed point per atom.
// (The slow virial is summed over pairs in FP64 by the force and correction
// kernels.) Each warp owns a contiguous slot range so that, with batched
// replicas, its slots belong to one replica except at boundaries.
constexpr int kFinalizeThreads = 256;

__global__ void __launch_bounds__(kFinalizeThreads)
    finalizeKernel(int n, const long long* __restrict__ F, int stride,
                   const float4* __restrict__ xyzq, float4* __restrict__ outF,
                   float4* __restrict__ outS, float4* __restrict__ outFH,
                   float4* __restrict__ outSH, int doSlow, int doVirial,
                   long long* __restrict__ accBase, const int* __restrict__ slotRep,
                   const ShiftVirialArgs shift) {
  long long v[9] = {};
  const int lane = threadIdx.x & 31;
  const int warpsTotal = (gridDim.x * blockDim.x) >> 5;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int per = ((n + warpsTotal - 1) / warpsTotal + 31) & ~31;
  const int iEnd = min(n, (gw + 1) * per);
  int curRep = 0;
  for (int i0 = gw * per; i0 < iEnd; i0 += 32) {
    const int i = i0 + lane;
    const bool valid = i < iEnd;
    if (doVirial && slotRep) {
      const int rep = valid ? slotRep[i] : curRep;
      if (__any_sync(0xffffffffu, rep != curRep)) {
        // flush per thread into the replica it accumulated for
#pragma unroll
        for (int p = 0; p < 9; ++p) {
          if (v[p] != 0) atomicAddFixed(&accBase[(size_t)curRep * kAccCount + kAccVir + p], (unsigned long long)v[p]);
          v[p] = 0;
        }
        curRep = rep;
      }
    }
    if (!valid) continue;
    const long long fx = F[i], fy = F[stride + i], fz = F[2 * (size_t)stride + i];
    long long gx = 0, gy = 0, gz = 0;
    if (doSlow) {
      gx = F[3 * (size_t)stride + i];
      gy = F[4 * (size_t)stride + i];
      gz = F[5 * (size_t)stride + i];
    }
    const float4 f4 = make_float4((float)(fx * kForceScaleInv), (float)(fy * kForceScaleInv),
                                  (float)(fz * kForceScaleInv), 0.0f);
    const float4 g4 = make_float4((float)(gx * kForceScaleInv), (float)(gy * kForceScaleInv),
                                  (float)(gz * kForceScaleInv), 0.0f);
    if (outF) outF[i] = f4;
    if (outS) outS[i] = g4;
    // page-locked host outputs: the stores cross PCIe while the kernel runs
    if (outFH) outFH[i] = f4;
    if (outSH) outSH[i] = g4;
    if (doVirial) {
      const float4 x = xyzq[i];
      const double X[3] = {(double)x.x, (double)x.y, (double)x.z};
      const double Fd[3] = {fx * kForceScaleInv, fy * kForceScaleInv, fz * kForceScaleInv};
#pragma unroll
      for (int p = 0; p < 9; ++p) v[p] += toFixedEnergy(Fd[p / 3] * X[p % 3]);
    }
  }
  if (!doVirial) return;
  // The lattice-shift part, (sum_i F_i) (x) shift for each compute, from the
  // exact integer i-force sums of the compute (the split of
  // reduceNonbondedVirialKernel / reduceVirialEnergyKernel,
  // src/CudaComputeNonbondedKernel.cu:1649-1920). Each compute's product is
  // rounded once, so the result does not depend on how lists were scheduled.
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < shift.numComputes;
       c += gridDim.x * blockDim.x) {
    const int rep = shift.compRep ? shift.compRep[c] : 0;
    if (rep != curRep) {
#pragma unroll
      for (int p = 0; p < 9; ++p) {
        if (v[p] != 0) atomicAddFixed(&accBase[(size_t)curRep * kAccCount + kAccVir + p], (unsigned long long)v[p]);
        v[p] = 0;
      }
      curRep = rep;
    }
    const long long* Fc = shift.compF + 6 * (size_t)c;
    const nbk_compute_record cr = shift.computes[c];
    float3 la = shift.lata, lb = shift.latb, lc = shift.latc;
    if (shift.compRep) {
      la = shift.repLat[3 * rep];
      lb = shift.repLat[3 * rep + 1];
      lc = shift.repLat[3 * rep + 2];
    }
    const float3 sh = shiftOf(make_float3(cr.offsetXYZ.x, cr.offsetXYZ.y, cr.offsetXYZ.z), la, lb, lc);
    const double S[3] = {(double)sh.x, (double)sh.y, (double)sh.z};
#pragma unroll
    for (int p = 0; p < 9; ++p) v[p] += toFixedEnergy((double)Fc[p / 3] * kForceScaleInv * S[p % 3]);
  }
  // Reduce the warp, then the block, before touching the 9 accumulator
  // words: every block adds each word once (per-warp adds only where a block
  // spans two replicas), which keeps same-address atomics off the critical path.
  __shared__ long long s_v[kFinalizeThreads / 32][9];
  __shared__ int s_rep[kFinalizeThreads / 32];
  const int wib = threadIdx.x >> 5;
  const int rep0 = __shfl_sync(0xffffffffu, curRep, 0);
  const bool uniform = __all_sync(0xffffffffu, curRep == rep0);
#pragma unroll
  for (int p = 0; p < 9; ++p) {
    if (uniform) {
      const long long sw = warpSumLL(v[p]);
      if (lane == 0) s_v[wib][p] = sw;
    } else {
      if (v[p] != 0) atomicAddFixed(&accBase[(size_t)curRep * kAccCount + kAccVir + p], (unsigned long long)v[p]);
      if (lane == 0) s_v[wib][p] = 0;
    }
  }
  if (lane == 0) s_rep[wib] = uniform ? rep0 : -1;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (threadIdx.x < 9) {
    const int p = threadIdx.x;
    bool same = true;
    for (int w = 1; w < nw; ++w) same = same && (s_rep[w] == s_rep[0] || s_rep[w] < 0);
    if (same && s_rep[0] >= 0) {
      long long sb = 0;
      for (int w = 0; w < nw; ++w) sb += s_v[w][p];
      if (sb != 0) atomicAddFixed(&accBase[(size_t)s_rep[0] * kAccCount + kAccVir + p], (unsigned long long)sb);
    } else {
      for (int w = 0; w < nw; ++w)
        if (s_rep[w] >= 0 && s_v[w][p] != 0)
          atomicAddFixed(&accBase[(size_t)s_rep[w] * kAccCount + kAccVir + p], (unsigned long long)s_v[w][p]);
    }
  }
}

cudaError_t launchFinalizeForces(int n, const long long* force, int stride, const float4* xyzq,
                                 float4* outF, float4* outS, unsigned flags, long long* acc,
                                 int numSM, cudaStream_t st, const int* slotRep,
                                 const ShiftVirialArgs* shift, float4* outFHost,
                                 float4* outSHost) {
  if (n <= 0) return cudaSuccess;
  const bool V = flags & NBK_VIRIAL;
  if (!V && !outF && !outS && !outFHost && !outSHost) return cudaSuccess;
  const int threads = kFinalizeThreads;
  // two blocks per SM keep enough loads in flight (one per SM left the
  // kernel latency-bound: 11 -> 9 us at 97k slots)
  const int blocks = min((n + threads - 1) / threads, 2 * numSM);
  ShiftVirialArgs sv{};
  if (shift && V) sv = *shift;
  finalizeKernel<<<blocks, threads, 0, st>>>(n, force, stride, xyzq, outF, outS, outFHost,
                                             outSHost, (flags & NBK_SLOW) ? 1 : 0, V ? 1 : 0, acc,
                                             slotRep, sv);
  return cudaGetLastError();
}

void* mappedHostPointer(void* p) {
  if (!p) return nullptr;
  cudaPointerAttributes at{};
  int dev = -1;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  // page-locked memory of the current device's context only (memory pinned
  // in another context without the portable flag gets the copy instead)
  return (at.type == cudaMemoryTypeHost && at.device == dev) ? at.devicePointer : nullptr;
}

__global__ void energyVirialKernel(const long long* __restrict__ accBase, nbk_virial_energy* outBase) {
  const int t = threadIdx.x;
  const long long* acc = accBase + (size_t)blockIdx.x * kAccCount;
  double* o = reinterpret_cast<double*>(outBase + blockIdx.x);
  const int nd = (int)(sizeof(nbk_virial_energy) / sizeof(double));
  // one store per word: virial[9], virialSlow[9], the three energies, then
  // the FEP / TI / GBIS words (zero); the record may be page-locked host memory
  if (t < nd) {
    long long q = 0;
    if (t < 9) q = acc[kAccVir + t];
    else if (t < 18) q = acc[kAccVirSlow + t - 9];
    else if (t == 18) q = acc[kAccEVdw];
    else if (t == 19) q = acc[kAccEElec];
    else if (t == 20) q = acc[kAccESlow];
    o[t] = (double)q * kEnergyScaleInv;
  }
}

cudaError_t launchEnergyVirial(const long long* acc, nbk_virial_energy* out, cudaStream_t st,
                               int numReplicas) {
  energyVirialKernel<<<numReplicas, 32, 0, st>>>(acc, out);
  return cudaGetLastError();
}

}  // namespace nbk
