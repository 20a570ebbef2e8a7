// Host-side harness around the reference's own pair-math device functions
// (src/CudaComputeNonbondedInteractions.h, compiled unmodified from the
// reference tree by oracle/ref_pin/Makefile with g++, where __device__ and
// __forceinline__ expand to host code). TEST INFRASTRUCTURE ONLY: it produces
// the golden vectors that pin the FP64 oracle's pair formulas to the
// reference's code; nothing in the product links it.
#include <math.h>

#include "CudaComputeNonbondedInteractions.h"

namespace {
// The constants of CudaComputeNonbonded::getNonbondedCoef
// (src/CudaComputeNonbonded.C:2318-2349), formed from the same inputs.
CudaNBConstants makeConstants(double cutoff, double switchdist, double ewaldcof, double slowScale) {
  const float cutoffF = (float)cutoff;
  const float cutoff2 = (float)(cutoff * cutoff);
  const float cutoffInv = 1.0f / cutoffF;
  const float cutoff2Inv = 1.0f / cutoff2;
  const double sw2 = switchdist * switchdist, rc2 = cutoff * cutoff;
  const double c0 = 1.0 / (rc2 - sw2);
  const float denom = (float)(c0 * c0 * c0);
  const float scutoff2 = (float)sw2;
  CudaNBConstants c;
  c.lj_0 = denom * cutoff2 - 3.0f * scutoff2 * denom;
  c.lj_1 = denom * 2.0f;
  c.lj_2 = denom * -12.0f;
  c.lj_3 = 12.0f * denom * scutoff2;
  c.lj_4 = cutoff2;
  c.lj_5 = scutoff2;
  c.e_0 = cutoff2Inv * cutoffInv;
  c.e_0_slow = cutoff2Inv * cutoffInv * (1.0f - (float)slowScale);
  c.e_1 = cutoff2Inv;
  c.e_2 = cutoffInv;
  c.ewald_0 = (float)ewaldcof;
  c.ewald_1 = (float)(1.12837916709551 * ewaldcof);
  c.ewald_2 = (float)(ewaldcof * ewaldcof);
  c.ewald_3_slow = (float)(ewaldcof * ewaldcof * ewaldcof * slowScale);
  c.slowScale = (float)slowScale;
  return c;
}
}  // namespace

extern "C" {
// Nonbonded pair: out = {f, fSlow, eVdw, eElec, eSlow} with the reference's
// sign convention F_i += f * (x_j - x_i).
void ref_nonbonded_pair(int n, const float* r2, const float* qq, const float* A, const float* B,
                        double cutoff, double switchdist, double ewaldcof, float* out) {
  const CudaNBConstants c = makeConstants(cutoff, switchdist, ewaldcof, 1.0);
  for (int k = 0; k < n; ++k) {
    float f = 0, fs = 0, ev = 0, ee = 0, es = 0;
    const float rinv = 1.0f / sqrtf(r2[k]);
    cudaNBForceMagCalc_VdwEnergySwitch_PMEC1<true, true>(r2[k], rinv, qq[k], make_float2(A[k], B[k]),
                                                         c, f, fs, ev, ee, es);
    out[5 * k + 0] = f;
    out[5 * k + 1] = fs;
    out[5 * k + 2] = ev;
    out[5 * k + 3] = ee;
    out[5 * k + 4] = es;
  }
}

// Modified (1-4) exclusion correction with qq already scaled by (1 - scale14)
// and (A, B) = (A14 - A, B14 - B): out = {f, fSlow, eVdw, eElec, eSlow} with
// the bonded kernel's convention F_i += f * (x_i - x_j).
void ref_modified_pair(int n, const float* r2, const float* qq, const float* A, const float* B,
                       double cutoff, double switchdist, double ewaldcof, float* out) {
  const CudaNBConstants c = makeConstants(cutoff, switchdist, ewaldcof, 1.0);
  for (int k = 0; k < n; ++k) {
    float f = 0, fs = 0, ev = 0, ee = 0, es = 0;
    const float rinv = 1.0f / sqrtf(r2[k]);
    cudaModExclForceMagCalc_VdwEnergySwitch_PMEC1<true>(1, 1, r2[k], rinv, qq[k],
                                                        make_float2(A[k], B[k]), c, f, fs, ev, ee, es);
    out[5 * k + 0] = f;
    out[5 * k + 1] = fs;
    out[5 * k + 2] = ev;
    out[5 * k + 3] = ee;
    out[5 * k + 4] = es;
  }
}
}
