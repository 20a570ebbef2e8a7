// Host-side launchers of the B200 nonbonded kernels (internal to libnbk).
#pragma once

#include <cuda_runtime.h>

#include "nbk_internal.cuh"

namespace nbk {

cudaError_t launchForce(const ForceArgs& a, unsigned flags, int numSM, cudaStream_t st);

cudaError_t launchBBoxes(int numTiles, const float4* xyzq, BBox* bb, cudaStream_t st);

cudaError_t launchBuildLists(int numLists, const ListSeed* seeds,
                             const nbk_compute_record* computes, const nbk_patch_record* patches,
                             const BBox* bb, float3 lata, float3 latb, float3 latc,
                             float plcutoff2Culling, nbk_tile_list* lists, PatchPair* pp,
                             int* tileJatomStart, cudaStream_t st);

cudaError_t launchCompact(int numLists, const nbk_tile_list* src, const int* listActive,
                          const int* jtileActive, const int* jatomSrc, const nbk_tile_excl* exclSrc,
                          nbk_tile_list* dst, int* jatomDst, nbk_tile_excl* exclDst, int* counters,
                          int numSM, cudaStream_t st);

struct CorrArgs {
  const nbk_exclusion* modified;
  int numModified;
  const nbk_exclusion* excluded;
  int numExcluded;
  const float4* xyzq;
  const float2* ljExclTable;  // (A14 - A, B14 - B) * scaling
  float3 lata, latb, latc;
  NbkConst c;
  long long* force;
  int stride;
  long long* acc;
  NbkConst64 c64;
};
cudaError_t launchCorrections(const CorrArgs& a, unsigned flags, cudaStream_t st);

cudaError_t launchFinalizeForces(int n, const long long* force, int stride, const float4* xyzq,
                                 float4* outF, float4* outS, unsigned flags, long long* acc,
                                 int numSM, cudaStream_t st);

cudaError_t launchEnergyVirial(const long long* acc, nbk_virial_energy* out, cudaStream_t st);

}  // namespace nbk
