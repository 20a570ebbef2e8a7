// Host-side launchers of the B200 nonbonded kernels (internal to libnbk).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "nbk_internal.cuh"

namespace nbk {

// Pair-math constants from the caller's parameters (nbk_consts.cu); shared by
// the handle and by the allocation-free entry point.
void makeConstants(const nbk_params& p, int ljDim, NbkConst& c, NbkConst64& k);
// The FP64 slow-term table of the force kernel's precise pass; returns rows.
int buildSlowTable(double beta, double cutoff, double pairlistdist, std::vector<double>& out,
                   double* step);

// minBlocks: 4, 5 or 6 CTAs per SM (the register cap); a.splitLog2 set by the caller.
cudaError_t launchForce(const ForceArgs& a, unsigned flags, int minBlocks, int numSM,
                        cudaStream_t st);
// The precise energy / virial kernel after the force kernel (same lists, the
// force kernel's live words, its own work counter a.workCounter); no-op when
// flags need neither energies nor the slow virial.
bool needsPrecise(unsigned flags);
cudaError_t launchPrecise(const ForceArgs& a, unsigned flags, int numSM, cudaStream_t st);
// Pairlist refinement of the culled lists a.lists[0, a.numListsHost): writes
// a.tileExcls, a.jtileActive, a.listActive and the excluded-pair counts.
cudaError_t launchRefine(const ForceArgs& a, int numSM, cudaStream_t st);

// The compacted lists [0, *numListsDev) of src copied to dst in order of
// decreasing j-tile count (lengths clamped to maxLen); hist: maxLen + 1 ints.
cudaError_t launchSortLists(int numListsMax, const nbk_tile_list* src, const int* numListsDev,
                            int maxLen, int* hist, nbk_tile_list* dst, int numSM, cudaStream_t st);

cudaError_t launchBBoxes(int numTiles, const float4* xyzq, BBox* bb, cudaStream_t st);

cudaError_t launchBuildLists(int numLists, const ListSeed* seeds,
                             const nbk_compute_record* computes, const nbk_patch_record* patches,
                             const BBox* bb, float3 lata, float3 latb, float3 latc,
                             const int* compRep, const float3* repLat, float plcutoff2Culling,
                             nbk_tile_list* lists, PatchPair* pp, int* tileJatomStart,
                             cudaStream_t st);

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
  // replicas (batched evaluation; NULL for a single system)
  const int* slotRep;          // [atomStorageSize] replica of each atom slot
  const float3* repLat;        // [3*numReplicas]
  const float2* repLJExcl;     // [numReplicas][ljDim*ljDim] (A14 - A, B14 - B) * scaling
};
cudaError_t launchCorrections(const CorrArgs& a, unsigned flags, cudaStream_t st);

// The lattice-shift part of the virial, (sum_i F_i) (x) shift per compute,
// from the exact integer i-force sums the force kernel leaves per compute.
struct ShiftVirialArgs {
  int numComputes;
  const long long* compF;                // [numComputes][6] (0..2: fast i-force sums)
  const nbk_compute_record* computes;
  float3 lata, latb, latc;
  const int* compRep;                    // batched replicas, else NULL
  const float3* repLat;
};

// With NBK_VIRIAL: the per-atom part of the fast virial, and with shift also
// its lattice-shift part, into the accumulators.
cudaError_t launchFinalizeForces(int n, const long long* force, int stride, const float4* xyzq,
                                 float4* outF, float4* outS, unsigned flags, long long* acc,
                                 int numSM, cudaStream_t st, const int* slotRep = nullptr,
                                 const ShiftVirialArgs* shift = nullptr,
                                 float4* outFHost = nullptr, float4* outSHost = nullptr);

// Device-visible address of host memory page-locked in the current device's
// context (the same pointer under unified addressing), or nullptr for any
// other pointer.
void* mappedHostPointer(void* p);

// Converts numReplicas accumulator blocks into numReplicas nbk_virial_energy records.
cudaError_t launchEnergyVirial(const long long* acc, nbk_virial_energy* out, cudaStream_t st,
                               int numReplicas = 1);

struct AdjArgs {
  const nbk_tile_list* lists;
  const int* numListsDev;
  const int* tileJatomStart;
  const nbk_tile_excl* tileExcls;
  const float4* xyzq;
  const int* vdwTypes;
  const float2* ljTable;
  const int* typeMask;   // [ljDim] 1: accumulate LJ gradients of pairs touching this type
  const float4* wF;      // fast-force cotangent per slot (w ignored)
  const float4* wS;      // slow-force cotangent per slot (NULL: zero)
  float cV, cE, cS;
  float3 lata, latb, latc;
  NbkConst c;
  long long* grad;       // SoA [4][stride]: gx, gy, gz, gq (fixed point, force scale)
  int stride;
  double* gradAB;        // [2][ljDim*ljDim] (FP64 atomics)
  int* workCounter;
};
cudaError_t launchAdjoint(const AdjArgs& a, bool doSlow, int numSM, int n, float4* out,
                          cudaStream_t st);

// Integrator force arrays from the fixed-point sums (nbk_accumulate_forces_to_soa).
struct AccumulateArgs {
  int numPatches, maxForceNumber, stride, forceStride;
  const nbk_local_record* rec;
  const int* sortOrder;
  const long long* fixed;     // [6][stride]: fast x y z, slow x y z
  const double* fBond;        // [3][forceStride] or NULL
  const double* fBondNbond;
  const double* fBondSlow;
  const float3* fPme;         // per buffer atom or NULL
  double* fNormal[3];
  double* fNbond[3];
  double* fSlow[3];
};
cudaError_t launchAccumulateForces(const AccumulateArgs& a, cudaStream_t st);

// Sets the message nbk_last_error returns on this thread; returns code.
int setLastError(int code, const std::string& msg);

// Per-slot vdW types, atom indices and exclusion indices from per-atom arrays
// in buffer order (GPU-resident marshaling, nbk_resident.cu).
cudaError_t launchUpdateVdwTypesExclDevice(int numPatches, const nbk_local_record* rec,
                                           const int* vdw, const int* gid, const int* sortOrder,
                                           const int2* exclByAtom, int numExclAtoms, int ljDim,
                                           int storage, int* vdwTypes, int* atomIndex, int2* excl,
                                           int* status, cudaStream_t st);

}  // namespace nbk
