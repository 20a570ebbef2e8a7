// Adjoint of the nonbonded evaluation: for cotangents wF, wS on the fast and
// slow forces and cV, cE, cS on the three energies, the gradient of
//   L = sum_i wF_i . F_i + sum_i wS_i . Fslow_i + cV E_vdw + cE E_elec + cS E_slow
// with respect to the positions (a Hessian-vector product), the scaled charges
// and the scaled LJ table entries. Pair terms are recomputed from the refined
// tile lists; nothing from the forward pass is stored.
//
// Per pair, with s = r^2, d = x_j - x_i, uF = wF_i - wF_j, pF = uF . d (same
// for S), and g = (dE/dr)/r of each term (2 dE/ds = g):
//   dL/dd = g uF + gs uS + d [2 (pF g' + pS gs') + cV g_lj + cE qq g_f + cS qq g_s]
//   dL/dx_j = dL/dd, dL/dx_i = -dL/dd
//   dL/dqq = pF g_f + pS g_s + cE phi_f + cS phi_s
//   dL/dA = pF gA + cV EA, dL/dB = pF gB + cV EB   (LJ is linear in A and B)
// where ' = d/ds. The slow-term derivatives cancel to O(x) at small
// x = beta r and are taken from their Taylor series there.
#include "nbk_internal.cuh"
#include "nbk_launch.h"

namespace nbk {

constexpr int kAdjWarps = 4;
constexpr int kAdjThreads = kAdjWarps * kWarp;

// Slow (PME real-space) electrostatics per unit qq, as functions of s = r^2:
//   g_s  = -1/rc^3 + beta^3 J(x),  J = (erf x - 2/sqrt(pi) x e^{-x^2}) / x^3
//   g_s' = beta^5 K(x),            K = e^{-x^2}(2/x^2 + 3/x^4)/sqrt(pi) - 1.5 erf(x)/x^5
//   phi_s = h(s) - erf(x)/r
__device__ __forceinline__ void slowTerms(float r, float rinv, float x, float beta, float rc3inv,
                                          float h, float& gs, float& dgs, float& phis) {
  const float y = x * x;
  const float ex = __expf(-y);
  const float erfc_ = erfcShared(x, ex);
  const float erfx = 1.0f - erfc_;
  const float b2 = beta * beta, b3 = b2 * beta, b5 = b3 * b2;
  float J, K;
  if (x < 0.7f) {
    // J = 2/sqrt(pi) sum_{n>=1} (-1)^{n+1} 2n y^{n-1} / ((2n+1) n!)
    float q = 14.0f / (15.0f * 5040.0f);  // n = 7
    q = fmaf(q, -y, 12.0f / (13.0f * 720.0f));
    q = fmaf(q, -y, 10.0f / (11.0f * 120.0f));
    q = fmaf(q, -y, 8.0f / (9.0f * 24.0f));
    q = fmaf(q, -y, 6.0f / (7.0f * 6.0f));
    q = fmaf(q, -y, 4.0f / (5.0f * 2.0f));
    q = fmaf(q, -y, 2.0f / 3.0f);
    J = 1.1283791671f * q;
    // K = 1/sqrt(pi) sum_{m>=2} (-1)^m 4m(1-m) / (m! (2m+1)) y^{m-2}
    float k = -4.0f * 10.0f * 9.0f / (3628800.0f * 21.0f);           // m = 10
    k = fmaf(k, y, 4.0f * 9.0f * 8.0f / (362880.0f * 19.0f));        // m = 9
    k = fmaf(k, y, -4.0f * 8.0f * 7.0f / (40320.0f * 17.0f));        // m = 8
    k = fmaf(k, y, 4.0f * 7.0f * 6.0f / (5040.0f * 15.0f));          // m = 7
    k = fmaf(k, y, -4.0f * 6.0f * 5.0f / (720.0f * 13.0f));          // m = 6
    k = fmaf(k, y, 4.0f * 5.0f * 4.0f / (120.0f * 11.0f));           // m = 5
    k = fmaf(k, y, -4.0f * 4.0f * 3.0f / (24.0f * 9.0f));            // m = 4
    k = fmaf(k, y, 4.0f * 3.0f * 2.0f / (6.0f * 7.0f));              // m = 3
    k = fmaf(k, y, -4.0f * 2.0f * 1.0f / (2.0f * 5.0f));             // m = 2
    K = 0.5641895835f * k;
  } else {
    const float xi = 1.0f / x, xi2 = xi * xi, xi3 = xi2 * xi;
    J = (erfx - 1.1283791671f * x * ex) * xi3;
    K = 0.5641895835f * ex * (2.0f + 3.0f * xi2) * xi2 - 1.5f * erfx * xi3 * xi2;
  }
  gs = fmaf(b3, J, -rc3inv);
  dgs = b5 * K;
  phis = h - erfx * rinv;
  (void)r;
}



template <bool doSlow>
__global__ void __launch_bounds__(kAdjThreads, 6) adjointKernel(const __grid_constant__ AdjArgs a) {
  extern __shared__ float s_dyn[];  // s_lj (float2[dim^2]) then s_gAB (float[2 dim^2])
  __shared__ float4 s_x[kAdjWarps][kWarp];
  __shared__ float4 s_wf[kAdjWarps][kWarp];
  __shared__ float4 s_ws[kAdjWarps][kWarp];
  __shared__ int s_t[kAdjWarps][kWarp];
  const NbkConst& c = a.c;
  const int dim = c.ljDim, d2 = dim * dim;
  float2* s_lj = reinterpret_cast<float2*>(s_dyn);
  float* s_gA = s_dyn + 2 * d2;
  float* s_gB = s_gA + d2;
  for (int k = threadIdx.x; k < d2; k += blockDim.x) {
    s_lj[k] = a.ljTable[k];
    s_gA[k] = 0.0f;
    s_gB[k] = 0.0f;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int numLists = *a.numListsDev;
  for (;;) {
    int L = 0;
    if (lane == 0) L = atomicAdd(a.workCounter, 1);
    L = __shfl_sync(0xffffffffu, L, 0);
    if (L >= numLists) break;
    const nbk_tile_list tl = a.lists[L];
    if (tl.jtileEnd < tl.jtileStart) continue;
    const float3 sh = shiftOf(make_float3(tl.offsetXYZ.x, tl.offsetXYZ.y, tl.offsetXYZ.z), a.lata,
                              a.latb, a.latc);
    const int iatom = tl.iatomStart + lane;
    float4 xi = a.xyzq[iatom];
    xi.x = __fadd_rn(xi.x, sh.x);
    xi.y = __fadd_rn(xi.y, sh.y);
    xi.z = __fadd_rn(xi.z, sh.z);
    const int tiRaw = a.vdwTypes[iatom];
    const int ti = tiRaw * dim;
    const bool mi = a.typeMask[tiRaw] != 0;
    const float4 wfi = a.wF[iatom];
    const float4 wsi = doSlow ? a.wS[iatom] : make_float4(0.f, 0.f, 0.f, 0.f);
    float gix = 0.f, giy = 0.f, giz = 0.f, giq = 0.f;
    for (int jt = tl.jtileStart; jt <= tl.jtileEnd; ++jt) {
      const unsigned mask = a.tileExcls[jt].excl[lane];
      unsigned stepMask = __reduce_or_sync(0xffffffffu, mask);
      if (!stepMask) continue;
      const int jstart = a.tileJatomStart[jt];
      s_x[wib][lane] = a.xyzq[jstart + lane];
      s_wf[wib][lane] = a.wF[jstart + lane];
      if (doSlow) s_ws[wib][lane] = a.wS[jstart + lane];
      s_t[wib][lane] = a.vdwTypes[jstart + lane];
      __syncwarp();
      float gjx = 0.f, gjy = 0.f, gjz = 0.f, gjq = 0.f;
      int tPrev = 0;
      while (stepMask) {
        const int t = __ffs(stepMask) - 1;
        stepMask &= stepMask - 1;
        const int delta = t - tPrev;
        if (delta) {
          const int src = (lane + delta) & 31;
          gjx = __shfl_sync(0xffffffffu, gjx, src);
          gjy = __shfl_sync(0xffffffffu, gjy, src);
          gjz = __shfl_sync(0xffffffffu, gjz, src);
          gjq = __shfl_sync(0xffffffffu, gjq, src);
        }
        tPrev = t;
        const int j = (lane + t) & 31;
        const float4 xj = s_x[wib][j];
        const float dx = __fsub_rn(xj.x, xi.x), dy = __fsub_rn(xj.y, xi.y), dz = __fsub_rn(xj.z, xi.z);
        const float r2 = dist2(dx, dy, dz);
        if (((mask >> t) & 1u) && r2 < c.cutoff2) {
          const float4 wfj = s_wf[wib][j];
          const float ufx = wfi.x - wfj.x, ufy = wfi.y - wfj.y, ufz = wfi.z - wfj.z;
          const float pF = fmaf(ufz, dz, fmaf(ufy, dy, ufx * dx));
          float usx = 0.f, usy = 0.f, usz = 0.f, pS = 0.f;
          if (doSlow) {
            const float4 wsj = s_ws[wib][j];
            usx = wsi.x - wsj.x;
            usy = wsi.y - wsj.y;
            usz = wsi.z - wsj.z;
            pS = fmaf(usz, dz, fmaf(usy, dy, usx * dx));
          }
          const int tj = s_t[wib][j];
          const float2 ab = s_lj[ti + tj];
          const float rinv = rsqrtf(r2);
          const float si = rinv * rinv;               // 1/s
          const float s3 = si * si * si, s6 = s3 * s3;
          // LJ: W = A s^-6 - B s^-3 and its s-derivatives; switch S(s)
          const float WA1 = -6.0f * s6 * si, WB1 = 3.0f * s3 * si;
          const float WA2 = 42.0f * s6 * si * si, WB2 = -12.0f * s3 * si * si;
          float S = 1.0f, S1 = 0.0f, S2 = 0.0f;
          if (c.switching) {
            const float t2 = fmaxf(r2, c.rs2);
            const float dd = c.rc2 - t2;
            // lj0..lj3 carry c1 = 1/(rc2-rs2)^3
            S = dd * dd * fmaf(c.lj1, t2, c.lj0);
            S1 = 0.5f * dd * fmaf(c.lj2, t2, c.lj3);  // 6 c1 (rc2-s)(rs2-s)
            // S'' = 6 c1 (2s - rs2 - rc2) above rs, 0 below (lj1 = 2 c1)
            S2 = (r2 > c.rs2) ? c.lj1 * (6.0f * t2 - 3.0f * c.rs2 - 3.0f * c.rc2) : 0.0f;
          }
          const float gA = 2.0f * fmaf(WA1, S, s6 * S1);
          const float gB = 2.0f * fmaf(WB1, S, -s3 * S1);
          const float glj = fmaf(ab.x, gA, ab.y * gB);
          const float dglj = 2.0f * (ab.x * fmaf(WA2, S, fmaf(2.0f * WA1, S1, s6 * S2)) +
                                     ab.y * fmaf(WB2, S, fmaf(2.0f * WB1, S1, -s3 * S2)));
          const float qi = xi.w, qj = xj.w, qq = qi * qj;
          const float rinv3 = rinv * si;
          const float gf = c.rc3inv - rinv3;
          const float dgf = 1.5f * rinv3 * si;
          const float h = fmaf(c.hB, r2, c.hA);
          const float phif = rinv - h;
          float gs = 0.f, dgs = 0.f, phis = 0.f;
          if (doSlow) slowTerms(r2 * rinv, rinv, c.beta * r2 * rinv, c.beta, c.rc3inv, h, gs, dgs, phis);
          const float g = fmaf(qq, gf, glj);
          const float radial = 2.0f * fmaf(pF, fmaf(qq, dgf, dglj), pS * qq * dgs) +
                               fmaf(a.cV, glj, qq * fmaf(a.cE, gf, a.cS * gs));
          const float gsq = qq * gs;
          const float vx = fmaf(radial, dx, fmaf(g, ufx, gsq * usx));
          const float vy = fmaf(radial, dy, fmaf(g, ufy, gsq * usy));
          const float vz = fmaf(radial, dz, fmaf(g, ufz, gsq * usz));
          gjx += vx;
          gjy += vy;
          gjz += vz;
          gix -= vx;
          giy -= vy;
          giz -= vz;
          const float dqq = fmaf(pF, gf, fmaf(pS, gs, fmaf(a.cE, phif, a.cS * phis)));
          giq = fmaf(qj, dqq, giq);
          gjq = fmaf(qi, dqq, gjq);
          if (mi || a.typeMask[tj]) {
            const float EA = s6 * S, EB = -s3 * S;
            atomicAdd(&s_gA[ti + tj], fmaf(pF, gA, a.cV * EA));
            atomicAdd(&s_gB[ti + tj], fmaf(pF, gB, a.cV * EB));
          }
        }
      }
      {
        const int src = (lane + (32 - tPrev)) & 31;
        gjx = __shfl_sync(0xffffffffu, gjx, src);
        gjy = __shfl_sync(0xffffffffu, gjy, src);
        gjz = __shfl_sync(0xffffffffu, gjz, src);
        gjq = __shfl_sync(0xffffffffu, gjq, src);
      }
      const int jatom = jstart + lane;
      if (gjx != 0.f || gjy != 0.f || gjz != 0.f || gjq != 0.f) {
        atomicAddFixed(&a.grad[0 * (size_t)a.stride + jatom], toFixedForce(gjx));
        atomicAddFixed(&a.grad[1 * (size_t)a.stride + jatom], toFixedForce(gjy));
        atomicAddFixed(&a.grad[2 * (size_t)a.stride + jatom], toFixedForce(gjz));
        atomicAddFixed(&a.grad[3 * (size_t)a.stride + jatom], toFixedForce(gjq));
      }
      __syncwarp();
    }
    if (gix != 0.f || giy != 0.f || giz != 0.f || giq != 0.f) {
      atomicAddFixed(&a.grad[0 * (size_t)a.stride + iatom], toFixedForce(gix));
      atomicAddFixed(&a.grad[1 * (size_t)a.stride + iatom], toFixedForce(giy));
      atomicAddFixed(&a.grad[2 * (size_t)a.stride + iatom], toFixedForce(giz));
      atomicAddFixed(&a.grad[3 * (size_t)a.stride + iatom], toFixedForce(giq));
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < d2; k += blockDim.x) {
    if (s_gA[k] != 0.0f) atomicAdd(&a.gradAB[k], (double)s_gA[k]);
    if (s_gB[k] != 0.0f) atomicAdd(&a.gradAB[d2 + k], (double)s_gB[k]);
  }
}

// Fixed-point gradients -> float4 (gx, gy, gz, gq) per slot.
__global__ void adjointOutKernel(int n, const long long* __restrict__ g, int stride,
                                 float4* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = make_float4((float)(g[i] * kForceScaleInv), (float)(g[stride + i] * kForceScaleInv),
                         (float)(g[2 * (size_t)stride + i] * kForceScaleInv),
                         (float)(g[3 * (size_t)stride + i] * kForceScaleInv));
}

cudaError_t launchAdjoint(const AdjArgs& a, bool doSlow, int numSM, int n, float4* out,
                          cudaStream_t st) {
  const size_t shmem = (size_t)a.c.ljDim * a.c.ljDim * (sizeof(float2) + 2 * sizeof(float));
  auto k = doSlow ? adjointKernel<true> : adjointKernel<false>;
  if (shmem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
    if (e != cudaSuccess) return e;
  }
  int nb = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kAdjThreads, shmem);
  if (e != cudaSuccess) return e;
  k<<<numSM * (nb > 0 ? nb : 1), kAdjThreads, shmem, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess || !out) return e;
  adjointOutKernel<<<min((n + 255) / 256, numSM * 4), 256, 0, st>>>(n, a.grad, a.stride, out);
  return cudaGetLastError();
}

}  // namespace nbk
