// Device-side types and the FP32 pair math of the B200 nonbonded path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "nbk.h"

namespace nbk {

constexpr int kWarp = 32;
// Forces are accumulated as 64-bit fixed point with 2^32 units per kcal/mol/A.
constexpr float kForceScale = 4294967296.0f;
constexpr double kForceScaleInv = 1.0 / 4294967296.0;
// Energies and virials are accumulated as 64-bit fixed point with 2^30 units.
constexpr double kEnergyScale = 1073741824.0;
constexpr double kEnergyScaleInv = 1.0 / 1073741824.0;

// Slots of the 64-bit accumulator block (energies, virials, counters).
enum AccSlot {
  kAccEVdw = 0,
  kAccEElec = 1,
  kAccESlow = 2,
  kAccVir = 3,       // 9 entries, virial[3*a+b]
  kAccVirSlow = 12,  // 9 entries
  kAccNumExcl = 21,  // number of excluded pairs within the pairlist cutoff
  kAccNumPairs = 22, // pairs evaluated within the cutoff (energy evaluations only)
  kAccCount = 24
};

// Constants of the energy-switched LJ and C1-split PME real-space pair math.
// The switching constants follow CudaComputeNonbonded::getNonbondedCoef
// (src/CudaComputeNonbonded.C:2318-2349): lj0 = c1(rc^2 - 3 rs^2), lj1 = 2 c1,
// lj2 = -12 c1, lj3 = 12 c1 rs^2 with c1 = 1/(rc^2 - rs^2)^3.
struct NbkConst {
  float cutoff2;
  float plcutoff2;
  float rc2;          // == cutoff2, switching upper end
  float rs2;          // switch distance^2
  float lj0, lj1, lj2, lj3;
  float rc3inv;       // 1/rc^3
  float hA, hB;       // (3 - r^2/rc^2)/(2 rc) = hA + hB r^2
  float beta;         // Ewald coefficient
  float beta2Pi;      // 2 beta / sqrt(pi)
  float one14;        // 1 - scale14
  float pBeta;        // erfcShared's p times beta (packed steady-state math)
  float gaussK;       // -beta^2 log2(e): exp(-beta^2 r^2) = 2^(gaussK r^2)
  float s0;           // 0 with switching, 1 without (packed math: S = d^2 P + s0)
  int ljDim;          // LJ table row length
  int switching;      // 0 when switchdist >= cutoff (plain truncated LJ)
  double hAd, hBd;    // hA, hB in FP64 (precise kernel)
  double betad;       // Ewald coefficient in FP64
};

// FP64 copies of the pair-math constants (the corrections kernel's energies and slow virial).
struct NbkConst64 {
  double rc2, rs2, lj0, lj1, lj2, lj3, rc3inv, hA, hB, beta, beta2Pi, one14;
  int switching;
};

// Bounding box of one 32-atom tile: centre and half-widths.
struct BBox {
  float x, y, z, wx, wy, wz;
};

// Per-list patch-pair record (PatchPairRecord, src/CudaTileListKernel.h:24-29).
struct PatchPair {
  int iatomSize, iatomFreeSize, jatomSize, jatomFreeSize;
};

// Sparse-list descriptor built on the host for every (compute, i-tile).
struct ListSeed {
  int icompute;
  int itile;       // i-tile index inside patch 1
  int jcapStart;   // first j-tile slot reserved for this list
  int pad;
};

// Shift of the i atoms, offset . lattice, as the reference's expression
// o.x a + o.y b + o.z c (src/CudaComputeNonbondedKernel.cu:720-722) rounds
// once contracted: the first product fused into the first sum, fma(o.x, a,
// o.y b), then fma(o.z, c, that). Written out as FMAs so that host and device
// agree bit for bit. (With an orthorhombic lattice only one term of each
// component is not 0, and every order gives the same bits.)
__device__ __forceinline__ float3 shiftOf(const float3 o, const float3 a, const float3 b,
                                          const float3 c) {
  float3 s;
  s.x = __fmaf_rn(o.z, c.x, __fmaf_rn(o.x, a.x, __fmul_rn(o.y, b.x)));
  s.y = __fmaf_rn(o.z, c.y, __fmaf_rn(o.x, a.y, __fmul_rn(o.y, b.y)));
  s.z = __fmaf_rn(o.z, c.z, __fmaf_rn(o.x, a.z, __fmul_rn(o.y, b.z)));
  return s;
}

// r^2 of d = xj - xi as the reference's dx*dx + dy*dy + dz*dz
// (src/CudaComputeNonbondedKernel.cu:1225-1230) rounds once contracted the same
// way: fma(dz, dz, fma(dx, dx, dy dy)). Its kernels list a pair whose r^2 is
// 182.249985 in this order and exactly plcutoff^2 = 182.25 in the order
// fma(dz, dz, fma(dy, dy, dx dx)) (a triclinic test cell).
__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
  return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// erfc(x) = t P(t) exp(-x^2), t = 1/(1 + p x): Hastings' rational form (the
// form of Abramowitz & Stegun 7.1.26) with a degree-7 P whose coefficients
// were fitted by least squares on [0, 4] (oracle/fit_erfc.py; max relative error
// 1.6e-8). `ex` is exp(-x^2), shared with the force's Gaussian term.
constexpr float kErfcP = 4.067848869e-01f;
constexpr float kErfcC0 = 8.043135869e-02f, kErfcC1 = -4.030445941e-01f,
                kErfcC2 = 6.621032108e-01f, kErfcC3 = -3.509793830e-01f,
                kErfcC4 = 3.971568035e-01f, kErfcC5 = 1.455091497e-01f,
                kErfcC6 = 2.400594718e-01f, kErfcC7 = 2.287639988e-01f;
__device__ __forceinline__ float erfcShared(const float x, const float ex) {
  const float t = __fdividef(1.0f, fmaf(kErfcP, x, 1.0f));
  float q = kErfcC0;
  q = fmaf(q, t, kErfcC1);
  q = fmaf(q, t, kErfcC2);
  q = fmaf(q, t, kErfcC3);
  q = fmaf(q, t, kErfcC4);
  q = fmaf(q, t, kErfcC5);
  q = fmaf(q, t, kErfcC6);
  q = fmaf(q, t, kErfcC7);
  return t * q * ex;
}

// ---- two pairs at once with sm_100's packed FP32 instructions --------------
// fma/mul/add .f32x2 issue two IEEE-rounded FP32 operations per instruction,
// so every element below is rounded exactly as the scalar form would be;
// only the number of issued instructions halves.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// PTX approximate reciprocal, base-2 exponential and reciprocal square root
// (rcp/ex2/rsqrt.approx.ftz.f32). The inputs here are normal numbers (r^2 is
// at least the square of the shortest pair distance, 2^(gaussK r^2) lies in
// (2^-15, 1], 1 + p beta r lies in [1, 3]), where the ftz forms equal the
// non-ftz ones.
__device__ __forceinline__ float rcpApprox(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2Approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrtApprox(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// PTX rsqrt.approx.ftz.f64: relative error below 2^-20 for normal inputs
// (measured 2^-20.1 over [0.5, 200] on B200); callers refine it.
__device__ __forceinline__ double rsqrtApprox64(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}

// FP32 pair math for two pairs (x and y elements); nB = -B. F, FS = (dE/dr)/r
// of LJ + fast electrostatics and of the slow (PME real-space remainder)
// electrostatics; the caller applies F_i += F (x_j - x_i), F_j -= F (x_j - x_i).
//   LJ      E = (A r^-12 - B r^-6) S(r^2), S = 1 below rs, Hermite switch above
//   fast    E = qq (1/r - (3 - r^2/rc^2)/(2 rc))
//   slow    E = qq ((3 - r^2/rc^2)/(2 rc) + (erfc(beta r) - 1)/r)
// (src/CudaComputeNonbondedInteractions.h:37-159 states the same forms.) Only
// the LJ energy is summed here (doVdwEnergy): the electrostatic energies and
// the slow virial are formed in FP64 by the precise kernel (nbk_force.cu).
// An element with qq = A = nB = 0 and r2 = cutoff^2 contributes exactly zero
// to F, FS and the energy, which is how callers switch a pair off without a
// branch. The slow term regroups the same quantities: with x = beta r,
// t = 1/(1 + p x) and e = exp(-x^2) = 2^(gaussK r^2), erfc = t P(t) e and the
// force factor erfc + (2 beta/sqrt(pi)) r e = (t P(t) + (2 beta/sqrt(pi)) r) e.
template <bool doVdwEnergy, bool doSlow>
__device__ __forceinline__ void pairForce2(const float2 r2, const float2 qq, const float2 A,
                                           const float2 nB, const NbkConst& c, float2& f,
                                           float2& fs, float2& eVdw) {
  const float2 rinv = make_float2(rsqrtApprox(r2.x), rsqrtApprox(r2.y));
  const float2 rinv2 = mul2(rinv, rinv);
  const float2 rinv6 = mul2(mul2(rinv2, rinv2), rinv2);
  const float2 rinv3 = mul2(rinv, rinv2);
  const float2 ab6 = fma2(A, rinv6, nB);
  const float2 w = mul2(ab6, rinv6);
  const float2 dw = mul2(fma2(A, rinv6, ab6), mul2(mul2(f2(-6.0f), rinv2), rinv6));
  // switch without a branch: without switching rs2 = rc2 and lj0..lj3 = 0,
  // so d = 0 for every pair inside the cutoff and S = s0 = 1, dS = 0
  const float2 t2 = make_float2(fmaxf(r2.x, c.rs2), fmaxf(r2.y, c.rs2));
  const float2 d = add2(f2(c.rc2), neg2(t2));
  const float2 s = fma2(mul2(d, d), fma2(f2(c.lj1), t2, f2(c.lj0)), f2(c.s0));
  const float2 ds = mul2(d, fma2(f2(c.lj2), t2, f2(c.lj3)));
  f = fma2(w, ds, mul2(dw, s));
  f = fma2(qq, add2(f2(c.rc3inv), neg2(rinv3)), f);
  if (doVdwEnergy) eVdw = fma2(w, s, eVdw);
  if (doSlow) {
    const float2 r = mul2(r2, rinv);
    const float2 den = fma2(f2(c.pBeta), r, f2(1.0f));
    const float2 t = make_float2(rcpApprox(den.x), rcpApprox(den.y));
    const float2 g = mul2(r2, f2(c.gaussK));
    const float2 ex = make_float2(ex2Approx(g.x), ex2Approx(g.y));
    float2 q = f2(kErfcC0);
    q = fma2(q, t, f2(kErfcC1));
    q = fma2(q, t, f2(kErfcC2));
    q = fma2(q, t, f2(kErfcC3));
    q = fma2(q, t, f2(kErfcC4));
    q = fma2(q, t, f2(kErfcC5));
    q = fma2(q, t, f2(kErfcC6));
    q = fma2(q, t, f2(kErfcC7));
    const float2 corr = mul2(fma2(f2(c.beta2Pi), r, mul2(t, q)), ex);
    fs = mul2(qq, fma2(add2(f2(1.0f), neg2(corr)), rinv3, f2(-c.rc3inv)));
  } else {
    fs = f2(0.0f);
  }
}

// ---- the FP64 slow-term table ------------------------------------------------
// The slow electrostatic energy per unit qq, phi_s(s) = h(s) - erf(beta sqrt(s))/sqrt(s)
// with s = r^2 and h(s) = (3 - s/rc^2)/(2 rc), is an entire function of s (the
// 1/r singularities of erfc(beta r)/r and of the fast part cancel), so a
// piecewise polynomial in s represents it closely: with a step D (a power of
// two, at most 32 A^2), row k holds the degree-5 Chebyshev interpolant on s in
// [k D - D/2, k D + D/2] in the monomial basis of w = s - k D (6 coefficients,
// 48 bytes: three 16-byte loads per pair). Its derivative gives the slow force
// factor, (dE/dr)/r = 2 qq phi_s'(s), without the rc^-3 - r^-3 cancellation of
// the FP32 form. Built on the host at handle creation (buildSlowTable) from
// FP64 erf, with D chosen so that the fit is within 1e-12 of the function's
// scale and its derivative within ~1e-9 (94 rows at the benchmark's
// parameters): a systematic error that, even summed over every pair with the
// same sign, stays below 1e-7 of the slow energy.
constexpr double kSlowTableStepMax = 32.0;  // A^2
constexpr int kSlowTableDeg = 5;
constexpr int kSlowTableDeg1 = kSlowTableDeg + 1;  // coefficients per row
constexpr int kSlowTableRow = 6;  // doubles per row of the global copy
constexpr double kSlowTableTol = 1e-12;  // fit error, relative to max |phi_s| + 1/rc

// Component k (0..8, row-major 3x3) of a symmetric tensor stored as
// xx, xy, xz, yy, yz, zz.
__device__ __forceinline__ int symIndex(int k) {
  const int a = k / 3, b = k % 3;
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}

__device__ __forceinline__ unsigned long long toFixedForce(float v) {
  return (unsigned long long)__float2ll_rn(v * kForceScale);
}

__device__ __forceinline__ long long toFixedEnergy(double v) {
  return __double2ll_rn(v * kEnergyScale);
}

// The same conversion from FP32: v * 2^30 is exact, so the result equals
// toFixedEnergy((double)v).
__device__ __forceinline__ long long toFixedEnergyF(float v) {
  return __float2ll_rn(v * 1073741824.0f);
}

__device__ __forceinline__ void atomicAddFixed(long long* p, unsigned long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), v);
}

__device__ __forceinline__ long long warpSumLL(long long v) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warpSumD(double v) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---- kernel argument blocks ---------------------------------------------------
struct ForceArgs {
  const nbk_tile_list* lists;
  const int* numListsDev;      // device count (compacted lists) or NULL
  int numListsHost;            // used when numListsDev == NULL
  const int* tileJatomStart;
  nbk_tile_excl* tileExcls;    // read by the force kernel, written by refineKernel
  int* jtileActive;            // refineKernel: written
  int* listActive;             // refineKernel: number of active j-tiles per list
  const PatchPair* patchPairs; // refineKernel
  const float4* xyzq;
  const int* vdwTypes;
  const int* atomIndex;
  const int2* exclIndexMaxDiff;
  const unsigned* exclBits;
  int numExclWords;
  const float2* ljTable;       // [ljDim*ljDim] (A, B) * scaling
  float3 lata, latb, latc;
  NbkConst c;
  long long* force;            // SoA [6][stride] fixed point
  int stride;
  long long* acc;              // [kAccCount]
  int* workCounter;            // next work item to hand out (zeroed before the launch)
  int splitLog2;               // force kernel: 2^splitLog2 work items per list
  long long* compF;            // virial: [numComputes][6] i-force sums per compute (0..2 used)
  const double2* slowTable;    // [slowTableRows * kSlowTableRow / 2] phi_s rows (FP64)
  int slowTableRows;
  double slowStep, slowInvStep;  // table step D (a power of two) and 1/D
  unsigned* liveOut;           // [numJtiles][32] interacting-pair words (force kernel writes,
                               // precise kernel reads)
  // replicas (batched evaluation; all NULL for a single system)
  const int* compRep;          // [numComputes] replica of each compute
  const float3* repLat;        // [3*numReplicas] lattice vectors a, b, c
  const float2* repLJ;         // [numReplicas][ljDim*ljDim] (A, B) * scaling
};

}  // namespace nbk
