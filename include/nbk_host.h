/*
 * nbk_host.h — host-side C-ABI that prepares the inputs of the nonbonded
 * path the way NAMD's host code does before it calls the GPU kernels:
 *
 *   - LJ combining into the A/B/A14/B14 table      (LJTable::compute_vdw_params,
 *                                                   src/LJTable.C:51-140)
 *   - patch decomposition, per-patch recursive-bisection atom order,
 *     patch-centred FP32 xyzq with charge scaling, padding of each patch to a
 *     multiple of 32 with copies of its last atom   (HomePatch::positionsReady,
 *                                                   src/HomePatch.C:1010-1131;
 *                                                   sortAtomsForCUDA, src/SortAtoms.C:45-133;
 *                                                   CudaComputeNonbonded::updatePatches /
 *                                                   copyAtomsSubset,
 *                                                   src/CudaComputeNonbonded.C:691-758,903-930)
 *   - self + half-shell compute records with offsetXYZ
 *                                                  (registerComputeSelf/Pair,
 *                                                   src/CudaComputeNonbonded.C:170-195)
 *   - exclusion bit array and per-slot (base, maxdiff)
 *                                                  (buildExclusions,
 *                                                   src/CudaComputeNonbonded.C:2191-2316;
 *                                                   updateVdwTypesExclSubset, :836-851)
 *   - excluded / modified (1-4) pair tuples for the corrections
 *                                                  (CudaExclusion, src/TupleTypesCUDA.h:76-81)
 *
 * plus the seeded synthetic system generator used by the tests and the
 * benchmark (water boxes and water + random-walk chain mixtures).
 *
 * All arrays live in host memory owned by the returned objects; the *_view
 * structs expose them as plain pointers (valid until the object is freed or
 * re-packed).
 */
#ifndef NBK_HOST_H
#define NBK_HOST_H

#include "nbk.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- synthetic systems ---------------------------------------------------- */
#define NBK_SYS_WATER 0   /* rigid TIP3P-like waters on a jittered lattice */
#define NBK_SYS_MIXED 1   /* random-walk chains (solute) + water */

typedef struct nbk_system_s* nbk_system;

typedef struct {
  int natoms;
  int ntypes;
  int numFullExclPairs;  /* 1-2 and 1-3 pairs (i < j) */
  int numModPairs;       /* 1-4 pairs (i < j) */
  int numWaters;
  int numSolute;
  double box[3];         /* orthorhombic box lengths (A) */
  double* pos;           /* [3*natoms] wrapped into [0, box) */
  double* charge;        /* [natoms] (e) */
  int* type;             /* [natoms] LJ type index */
  double* sigma;         /* [ntypes] (A) */
  double* epsilon;       /* [ntypes] (kcal/mol) */
  int* fullExcl;         /* [2*numFullExclPairs] */
  int* modPairs;         /* [2*numModPairs] */
} nbk_system_view;

/* kind: NBK_SYS_WATER or NBK_SYS_MIXED. natoms: total atoms (water: multiple
 * of 3). box: lengths; box[0] <= 0 sizes a cube to 0.1 atoms/A^3.
 * solute_frac: fraction of atoms in chains (MIXED only). */
NBK_API int nbk_system_generate(int kind, uint64_t seed, int natoms, double solute_frac,
                                const double* box, nbk_system* out);
NBK_API int nbk_system_view_get(nbk_system s, nbk_system_view* v);
/* Adds N(0, sigma) noise to every coordinate (seeded) and re-wraps. */
NBK_API int nbk_system_perturb(nbk_system s, uint64_t seed, double sigma);
NBK_API int nbk_system_free(nbk_system s);

/* LJ table of LJTable::compute_vdw_params for types with (sigma, epsilon);
 * 1-4 parameters equal the normal ones. geometric != 0 uses sqrt(si*sj). */
NBK_API int nbk_lj_table(int ntypes, const double* sigma, const double* epsilon,
                         int geometric, double* A, double* B, double* A14, double* B14);

/* Chain rule of the adjoint's LJ output: gradients w.r.t. the scaled table
 * entries (gA, gB at ordered type pair [i*ntypes + j]) to per-type sigma and
 * epsilon under the combining rule of nbk_lj_table. Types with epsilon 0
 * receive no epsilon gradient (the combining rule is not differentiable there). */
NBK_API int nbk_lj_param_grad(int ntypes, const double* sigma, const double* epsilon, int geometric,
                              double scaling, const double* gA, const double* gB, double* gSigma,
                              double* gEps);

/* ---- packing (host mirror of CudaComputeNonbonded's input preparation) ---- */
typedef struct nbk_packed_s* nbk_packed;

typedef struct {
  int natoms;
  int numPatches;
  int patchGrid[3];
  int atomStorageSize;
  int maxTileListLen;
  int numComputes;
  int numExclusionWords;
  int numModified;
  int numExcluded;
  nbk_float3 lata, latb, latc;
  nbk_patch_record* patches;        /* [numPatches] */
  nbk_compute_record* computes;     /* [numComputes] */
  nbk_float4* xyzq;                 /* [atomStorageSize] patch-centred, q scaled */
  int* vdwTypes;                    /* [atomStorageSize] */
  int* atomIndex;                   /* [atomStorageSize] global atom id */
  nbk_int2* exclIndexMaxDiff;       /* [atomStorageSize] (base, maxdiff) */
  unsigned int* exclusionBits;      /* [numExclusionWords] */
  nbk_exclusion* modified;          /* [numModified] 1-4 tuples */
  nbk_exclusion* excluded;          /* [numExcluded] full-exclusion tuples */
  int* slotOfAtom;                  /* [natoms] global atom -> slot */
  double* patchCenter;              /* [3*numPatches] unscaled centres (A) */
  /* replicas (nbk_pack_many; a single packing is one replica) */
  int numReplicas;
  int* replicaOfCompute;            /* [numComputes] */
  int* replicaSlotStart;            /* [numReplicas+1] slot range of each replica */
  int* replicaAtomStart;            /* [numReplicas+1] atom range (global ids) */
  nbk_float3* replicaLattice;       /* [3*numReplicas] a, b, c of each replica */
} nbk_packed_view;

/* patchDim: patch side lower bound (NAMD: pairlistdist, src/SimParameters.C:3481).
 * coulombScaling = scaling / dielectric; q = charge*sqrt(332.0636*coulombScaling). */
NBK_API int nbk_pack(nbk_system s, double patchDim, double coulombScaling, nbk_packed* out);
NBK_API int nbk_packed_view_get(nbk_packed p, nbk_packed_view* v);
/* Packs n independent systems (replicas) into one concatenated layout: patch,
 * compute, slot and atom indices and exclusion-bit bases are offset per replica
 * so that one handle evaluates all of them (nbk_set_replicas). */
NBK_API int nbk_pack_many(const nbk_system* systems, int n, double patchDim,
                          double coulombScaling, nbk_packed* out);
/* Re-pack xyzq from the system's current positions, keeping the patch
 * assignment and slot order (steps between pairlist rebuilds). */
NBK_API int nbk_pack_update_positions(nbk_packed p, nbk_system s);
NBK_API int nbk_packed_free(nbk_packed p);

/* Message of the last failure of an nbk_host call on this thread. */
NBK_API const char* nbk_host_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* NBK_HOST_H */
