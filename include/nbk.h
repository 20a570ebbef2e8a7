/*
 * nbk.h — C-ABI of the B200 short-range nonbonded path (tile-list build +
 * force kernel) that replaces NAMD 3.0's CudaTileListKernel /
 * CudaComputeNonbondedKernel pair for one GPU.
 *
 * Every entry point:
 *   - returns 0 on success or a negative NBK_ERR_* code; the message of the
 *     last failure on the calling thread is returned by nbk_last_error().
 *     Nothing here aborts the process (the reference calls NAMD_die /
 *     cudaDie, src/CudaUtils.C:9-28, src/CudaUtils.h:214-221);
 *   - takes the caller's CUDA stream (cudaStream_t passed as void*; NULL =
 *     legacy default stream) and only enqueues work on it, except where a
 *     comment says "synchronises";
 *   - is NOT thread-safe per handle (the reference is called from masterPe
 *     only, src/CudaComputeNonbonded.C:1090,1154,1607). Separate handles are
 *     independent.
 *
 * Record layouts mirror the reference's structs field for field so a NAMD
 * caller can hand its arrays over unchanged (see each struct's citation).
 * Types are plain C: no CUDA or torch types appear in the signatures.
 */
#ifndef NBK_H
#define NBK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NBK_API __attribute__((visibility("default")))

/* ---- status codes --------------------------------------------------- */
#define NBK_OK 0
#define NBK_ERR_ARG (-1)       /* bad argument (null pointer, size, flag) */
#define NBK_ERR_CUDA (-2)      /* a CUDA runtime call failed               */
#define NBK_ERR_STATE (-3)     /* call out of order (e.g. force before build) */
#define NBK_ERR_NOMEM (-4)     /* device or host allocation failed          */
#define NBK_ERR_OVERFLOW (-5)  /* a size limit of the tile lists was exceeded */
#define NBK_ERR_DEVICE (-6)    /* no usable sm_100 device                     */

/* ---- flags for nbk_nonbonded_force / nbk_reduce_virial_energy -------- */
#define NBK_ENERGY 1u      /* doEnergy   (src/CudaComputeNonbondedKernel.cu:2076) */
#define NBK_VIRIAL 2u      /* doVirial */
#define NBK_SLOW 4u        /* doSlow: PME real-space correction into the slow buffers */
#define NBK_PAIRLIST 8u    /* doPairlist: refine tile lists to exclusion masks */
#define NBK_CORRECTIONS 16u /* also apply excluded / modified (1-4) pair corrections
                              (reference: ComputeBondedCUDAKernel exclusionForce /
                              modifiedExclusionForce) in the same evaluation */
#define NBK_ENERGY_FP64 32u /* accepted for compatibility, no effect: electrostatic energies
                              and the slow virial are always formed in FP64 (see
                              nbk_nonbonded_force) */

/* ---- POD types -------------------------------------------------------- */
typedef struct { float x, y, z; } nbk_float3;
typedef struct { float x, y, z, w; } nbk_float4;     /* CudaAtom {x,y,z,q}: src/CudaRecord.h:58-60 */
typedef struct { int x, y; } nbk_int2;

/* CudaComputeRecord, src/CudaTileListKernel.h:47-50 (24 bytes: CUDA's int2
 * is 8-byte aligned, so the reference record ends in 4 bytes of padding and an
 * array of them has a 24-byte stride). */
typedef struct {
  nbk_int2 patchInd;      /* (i-patch, j-patch) indices into the patch array */
  nbk_float3 offsetXYZ;   /* i-shift in lattice units: center(pi)-center(pj)+image */
  int pad;                /* tail padding of the reference layout; ignored */
} nbk_compute_record;

/* CudaPatchRecord with NODEGROUP_FORCE_REGISTER, src/CudaTileListKernel.h:55-63. */
typedef struct {
  int numAtoms;
  int numFreeAtoms;
  int atomStart;          /* multiple of 32; padded slots repeat the last atom */
  int patchID;
} nbk_patch_record;

/* TileList, src/CudaTileListKernel.h:10-22 (48 bytes: 44 bytes of fields
 * and, as int2 is 8-byte aligned in CUDA, 4 bytes of tail padding). */
typedef struct {
  int iatomStart;
  int jtileStart;
  int jtileEnd;           /* inclusive */
  nbk_float3 offsetXYZ;
  nbk_int2 patchInd;
  nbk_int2 patchNumList;
  int icompute;
  int pad;                /* tail padding of the reference layout */
} nbk_tile_list;

/* TileExcl, src/CudaTileListKernel.h:5-8: bit t of excl[lane] = 1 iff the pair
 * (i = iatomStart+lane, j = jatomStart+((lane+t)&31)) is within the pairlist
 * cutoff and not excluded. */
typedef struct { unsigned int excl[32]; } nbk_tile_excl;

/* TileListStat, src/CudaTileListKernel.h:65-73 (bool widened to int). */
typedef struct {
  int numTileLists;
  int numTileListsGBIS;
  int numJtiles;
  int numExcluded;
  int patchReadyQueueCount;
  int outputOrderIndex;
  int tilesSizeExceeded;
} nbk_tile_list_stat;

/* VirialEnergy, src/CudaTileListKernel.h:98-117. virial[3*a+b] = sum F_a * x_b. */
typedef struct {
  double virial[9];
  double virialSlow[9];
  double energyVdw;
  double energyElec;
  double energySlow;
  double energyVdw_s, energyElec_s, energySlow_s;          /* FEP: always 0 here */
  double energyVdw_ti_1, energyVdw_ti_2;                   /* TI: always 0 here  */
  double energyElec_ti_1, energyElec_ti_2;
  double energySlow_ti_1, energySlow_ti_2;
  double energyGBIS;                                       /* GBIS: always 0     */
} nbk_virial_energy;

/* CudaExclusion, src/TupleTypesCUDA.h:76-81. */
typedef struct {
  int i, j, vdwtypei, vdwtypej;
  nbk_float3 ioffsetXYZ;  /* i-shift in lattice units */
  int pswitch;            /* alchemical partition switch: must be 0 (no alchemy) */
} nbk_exclusion;

/* Nonbonded parameters: the ComputeNonbondedUtil statics the reference path
 * reads (src/ComputeNonbondedUtil.C:506-576, src/CudaComputeNonbonded.C:
 * 2318-2349) plus the LJ table that CudaNonbondedTables builds
 * (src/CudaNonbondedTables.C:110-148). Arrays are host memory, copied. */
typedef struct {
  double cutoff;          /* cutoff (A) */
  double switchdist;      /* switchdist (A); == cutoff disables switching */
  double pairlistdist;    /* pairlistdist (A) */
  double ewaldcof;        /* Ewald coefficient beta (1/A) */
  double scaling;         /* nonbondedScaling */
  double scale14;         /* 1-4scaling (1.0 unless exclude = scaled1-4) */
  double slowScale;       /* fullElectFrequency / nonbondedFrequency */
  int vdwTableDim;        /* number of LJ types */
  const double* ljA;      /* [dim*dim] LJTable A   (unscaled) */
  const double* ljB;      /* [dim*dim] LJTable B */
  const double* ljA14;    /* [dim*dim] LJTable A for 1-4 pairs */
  const double* ljB14;    /* [dim*dim] LJTable B for 1-4 pairs */
} nbk_params;

typedef struct nbk_context* nbk_handle;

/* ---- lifetime ---------------------------------------------------------- */
NBK_API const char* nbk_last_error(void);
NBK_API int nbk_version(void);

/* CudaComputeNonbondedKernel(deviceID, CudaNonbondedTables&, doStreaming)
 * (src/CudaComputeNonbondedKernel.h:86-135) + CudaTileListKernel(deviceID,
 * doStreaming) (src/CudaTileListKernel.h:302) + CudaNonbondedTables(deviceID)
 * (src/CudaNonbondedTables.C:10-34) in one handle. */
NBK_API int nbk_create(int deviceID, const nbk_params* params, nbk_handle* out);
NBK_API int nbk_destroy(nbk_handle h);

/* ---- set-up (mirror of the reference's set-up calls) ------------------- */

/* CudaTileListKernel::updateComputes, src/CudaTileListKernel.cu:893-902. */
NBK_API int nbk_update_computes(nbk_handle h, int numComputes,
                                const nbk_compute_record* h_computes, void* stream);

/* CudaComputeNonbondedKernel::bindExclusions, src/CudaComputeNonbondedKernel.cu:3633-3639.
 * bits: the exclusion bit array built by CudaComputeNonbonded::buildExclusions. */
NBK_API int nbk_bind_exclusions(nbk_handle h, int numExclusions, const unsigned int* h_bits);

/* CudaComputeNonbondedKernel::updateVdwTypesExcl, src/CudaComputeNonbondedKernel.cu:2038-2048.
 * exclIndexMaxDiff[k] = (bit base, maxdiff) for slot k, as the reference. */
NBK_API int nbk_update_vdw_types_excl(nbk_handle h, int atomStorageSize, const int* h_vdwTypes,
                                      const nbk_int2* h_exclIndexMaxDiff, const int* h_atomIndex,
                                      void* stream);

/* ---- per-step work -------------------------------------------------------- */

/* CudaTileListKernel::buildTileLists, src/CudaTileListKernel.cu:1022-1192.
 * Bounding boxes per 32-atom tile and bbox culling of every compute into tile
 * lists. xyzq is a host pointer (xyzqOnDevice = 0, copied on `stream`) or a
 * device pointer kept by reference (xyzqOnDevice = 1; it must stay valid
 * until the next build). No host synchronisation: capacities are exact upper
 * bounds computed from the patch records. A patch with more 32-atom tiles than
 * maxTileListLen, or maxTileListLen >= 65536, returns NBK_ERR_OVERFLOW and sets
 * tilesSizeExceeded in the TileListStat (the reference's tilesSizeExceeded,
 * src/CudaTileListKernel.cu:505-509; it reallocates and rebuilds, the caller
 * here rebuilds with a larger maxTileListLen). lata, latb, latc are the
 * general (triclinic) lattice vectors, as the reference takes them; a compute's
 * shift is offsetXYZ.x lata + offsetXYZ.y latb + offsetXYZ.z latc, rounded in
 * FP32 as the reference's kernels round it. */
NBK_API int nbk_build_tile_lists(nbk_handle h, int numPatches, int atomStorageSize,
                                 int maxTileListLen, nbk_float3 lata, nbk_float3 latb,
                                 nbk_float3 latc, const nbk_patch_record* h_patches,
                                 const nbk_float4* xyzq, int xyzqOnDevice, float plcutoff2,
                                 void* stream);

/* CudaComputeNonbondedKernel::nonbondedForce, src/CudaComputeNonbondedKernel.cu:2076-3590.
 * flags = NBK_ENERGY|NBK_VIRIAL|NBK_SLOW|NBK_PAIRLIST|NBK_CORRECTIONS.
 * xyzq as for nbk_build_tile_lists (NULL = reuse the build's positions).
 * Forces are accumulated deterministically as 64-bit fixed point (2^32 per
 * kcal/mol/A) and then written as float4 to any non-NULL output:
 *   d_forces / d_forcesSlow : device float4[atomStorageSize] (w = 0)
 *   h_forces / h_forcesSlow : host float4[atomStorageSize] (needs the matching
 *                             device buffer); page-locked memory is written by
 *                             the finalizing kernel itself, other host memory
 *                             by a copy on `stream` after it
 *   d_forcesFixed           : device int64[6*atomStorageSize] SoA
 *                             (fx, fy, fz, fslowx, fslowy, fslowz)
 * With NBK_PAIRLIST the tile lists are refined: masks of pairs within the
 * pairlist cutoff that are not excluded, empty tiles and lists compacted.
 * Precision: pair forces are FP32 (the reference's arithmetic), summed in
 * fixed point. With NBK_ENERGY the electrostatic (fast and slow) pair
 * energies, and with NBK_VIRIAL | NBK_SLOW the slow virial, are formed per
 * interacting pair in FP64 from FP64 geometry (1/r refined by a Newton step,
 * the slow term from an FP64 piecewise polynomial, nbk_slow_table) and summed
 * in fixed point: relative error ~1e-10 or better against an FP64 evaluation
 * of the same FP32 positions, where FP32 pair energies resolve totals that
 * cancel to 1e-4 of the sum of |pair energies| only to ~1e-5. The LJ energy
 * (FP32 per pair) and the fast virial (from the fixed-point forces) hold
 * ~3e-7. Cost, measured on a B200 at 92,224 atoms (34 M pairs): the FP64
 * energy kernel runs 0.195 ms after the 0.403 ms force kernel, so an
 * evaluation with NBK_ENERGY costs about 1.5x a forces-only one. */
NBK_API int nbk_nonbonded_force(nbk_handle h, int atomStorageSize, unsigned flags,
                                nbk_float3 lata, nbk_float3 latb, nbk_float3 latc,
                                const nbk_float4* xyzq, int xyzqOnDevice, float cutoff2,
                                nbk_float4* d_forces, nbk_float4* d_forcesSlow,
                                nbk_float4* h_forces, nbk_float4* h_forcesSlow,
                                long long* d_forcesFixed, void* stream);

/* CudaComputeNonbondedKernel::reduceVirialEnergy, src/CudaComputeNonbondedKernel.cu:3595-3631.
 * Writes the energies and virials of the last nbk_nonbonded_force into
 * ve (device pointer if veOnDevice, else host pointer: page-locked memory is
 * written by the read-out kernel, other memory by a copy on `stream`). */
NBK_API int nbk_reduce_virial_energy(nbk_handle h, unsigned flags, nbk_virial_energy* ve,
                                     int veOnDevice, void* stream);

/* Exclusion corrections of ComputeBondedCUDAKernel (modifiedExclusionForce,
 * src/ComputeBondedCUDAKernel.cu:315-626; exclusionForce, :632-778): uploads
 * the tuples; they are applied by every later nbk_nonbonded_force whose flags
 * contain NBK_CORRECTIONS. modified = 1-4 pairs, excluded = full exclusions. */
NBK_API int nbk_set_exclusion_tuples(nbk_handle h, int numModified, const nbk_exclusion* h_modified,
                                     int numExcluded, const nbk_exclusion* h_excluded,
                                     void* stream);

/* CudaTileListKernel::reSortTileLists, src/CudaTileListKernel.cu:1605-1665.
 * Compaction happens on the device inside nbk_nonbonded_force(NBK_PAIRLIST);
 * this call only reads back the TileListStat and therefore synchronises. */
NBK_API int nbk_get_tile_list_stat(nbk_handle h, nbk_tile_list_stat* out, void* stream);

/* Test/debug export of the active tile lists (synchronises). Pass NULL
 * arrays to query the counts first. */
NBK_API int nbk_export_tile_lists(nbk_handle h, int* numTileLists, int* numJtiles,
                                  nbk_tile_list* tileLists, int* tileJatomStart,
                                  nbk_tile_excl* tileExcls, void* stream);

/* ---- adjoint ------------------------------------------------------------------- */

/* No counterpart in the reference. Gradient of
 *   L = sum_i wF_i.F_i + sum_i wS_i.Fslow_i + cV E_vdw + cE E_elec + cS E_slow
 * for the last refined tile lists and the bound positions (call after an
 * nbk_nonbonded_force of the same positions): with respect to the positions
 * (a Hessian-vector product), the scaled charges xyzq.w, and the scaled LJ
 * table entries. Pair terms are recomputed from the tile lists; nothing of
 * the forward pass is stored. wS and cS are used with NBK_SLOW in flags.
 *   d_wF, d_wS   : device float4[atomStorageSize] cotangents (w ignored)
 *   h_typeMask   : host int[vdwTableDim]; LJ gradients are accumulated for
 *                  pairs that touch a type with a non-zero entry (NULL: all)
 *   d_gradXQ     : device float4[atomStorageSize] (dL/dx, dL/dy, dL/dz, dL/dq)
 *   d_gradFixed  : optional device int64[4*atomStorageSize] SoA, 2^32 units
 *   d_gradAB     : device double[2*dim*dim]: dL/dA then dL/dB at ordered type
 *                  pairs (i-type, j-type); fold with nbk_lj_param_grad */
NBK_API int nbk_adjoint(nbk_handle h, unsigned flags, const nbk_float4* d_wF,
                        const nbk_float4* d_wS, double cV, double cE, double cS,
                        const int* h_typeMask, nbk_float4* d_gradXQ, long long* d_gradFixed,
                        double* d_gradAB, void* stream);

/* ---- batched replicas -------------------------------------------------------- */

/* No counterpart in the reference (NAMD runs independent systems as separate
 * processes). Turns the handle into a batch of numReplicas independent
 * systems evaluated by the same launches: the computes, patches and atom slots
 * given to the other calls are the replicas' arrays concatenated (replica r
 * owns atom slots [replicaSlotStart[r], replicaSlotStart[r+1]) and the computes
 * with replicaOfCompute[c] == r), each replica with its own lattice (a, b, c)
 * and its own LJ tables ljA/ljB/ljA14/ljB14 [numReplicas][dim*dim] (dim =
 * params.vdwTableDim). Call after nbk_update_computes; the lattice arguments
 * of later calls are then ignored. Energies, virials and pair counts are kept
 * per replica (nbk_reduce_virial_energy_batch, nbk_get_pair_counts). */
NBK_API int nbk_set_replicas(nbk_handle h, int numReplicas, const int* h_replicaOfCompute,
                             const int* h_replicaSlotStart, const nbk_float3* h_lattices,
                             const double* ljA, const double* ljB, const double* ljA14,
                             const double* ljB14, void* stream);
/* Per-replica VirialEnergy records of the last evaluation: ve[numReplicas]. */
NBK_API int nbk_reduce_virial_energy_batch(nbk_handle h, unsigned flags, nbk_virial_energy* ve,
                                           int veOnDevice, void* stream);
/* Per-replica pair counts of the last NBK_ENERGY evaluation (synchronises). */
NBK_API int nbk_get_pair_counts(nbk_handle h, long long* counts, int maxCount, void* stream);

/* ---- allocation-free variant ------------------------------------------------ */

/* No counterpart in the reference. For callers that cannot call cudaMalloc
 * (a host framework that owns all device memory through its own pool, code
 * between captured regions that must not touch the allocator, runtimes with a
 * device heap fixed at start-up): the excluded / modified (1-4) pair
 * corrections of NBK_CORRECTIONS without a handle and without allocating.
 * Scratch (fixed-point accumulators and a tuple staging copy) is a static
 * device array of about 11 MB that every GPU loading the library holds until
 * exit; it limits atomStorageSize to 65,536 slots and numModified + numExcluded
 * to 262,144 tuples (larger sizes return NBK_ERR_ARG). Inputs: device xyzq,
 * device LJ delta table float2[ljDim*ljDim] = (A14 - A, B14 - B) * scaling,
 * host tuple arrays (validated, then copied into the scratch); scalar fields of
 * params (cutoff, switchdist, ewaldcof, scale14) are read, its LJ arrays are
 * not. flags: NBK_ENERGY | NBK_VIRIAL | NBK_SLOW (and NBK_ENERGY_FP64 is not
 * accepted). Outputs: device float4 forces (and slow forces with NBK_SLOW),
 * device nbk_virial_energy with NBK_ENERGY or NBK_VIRIAL. The first call on a
 * device looks up the scratch address for that device; make it before any
 * stream capture. All calls share the scratch: calls that overlap on the GPU
 * race, so the caller serialises them (same stream, one at a time). */
NBK_API int nbk_exclusion_force_noalloc(const nbk_params* params, const float* d_ljExclTable,
                                        int ljDim, int atomStorageSize, const nbk_float4* d_xyzq,
                                        int numModified, const nbk_exclusion* h_modified,
                                        int numExcluded, const nbk_exclusion* h_excluded,
                                        nbk_float3 lata, nbk_float3 latb, nbk_float3 latc,
                                        unsigned flags, nbk_float4* d_forces,
                                        nbk_float4* d_forcesSlow, nbk_virial_energy* d_ve,
                                        void* stream);
/* Message of the last failure of nbk_exclusion_force_noalloc on this thread. */
NBK_API const char* nbk_noalloc_last_error(void);

/* No counterpart in the reference (its slow term comes from interpolated
 * texture tables, src/CudaNonbondedTables.C:158-303). The FP64 slow-term table
 * the precise energy / virial kernel evaluates. With step D (*step; a power
 * of two, 32 A^2 or less, chosen so that the fit is within 1e-12 of
 * max |phi_s| + 1/rc), row k (6 doubles) holds the degree-5 Chebyshev
 * interpolant of phi_s(s) = (3 - s/rc^2)/(2 rc) - erf(ewaldcof sqrt(s))/sqrt(s),
 * s = r^2, on s in [k D - D/2, k D + D/2], as coefficients c0..c5 of powers of
 * (s - k D).
 * The slow pair energy is qq phi_s(s), the slow force factor
 * (dE/dr)/r = 2 qq phi_s'(s). Rows cover s up to pairlistdist^2 + 2.
 * Host-only (no GPU needed): returns the number of rows and, when out is not
 * NULL, writes them (maxRows must be at least that number); step may be NULL;
 * NBK_ERR_ARG for bad parameters. */
NBK_API int nbk_slow_table(double ewaldcof, double cutoff, double pairlistdist, double* out,
                           int maxRows, double* step);

/* ---- test hooks -------------------------------------------------------------- */

/* Allocation-failure injection for tests of the error paths: the
 * countdown-th device allocation made for any handle from now on (counting
 * the buffers that nbk_create, nbk_update_*, nbk_build_tile_lists,
 * nbk_nonbonded_force ... grow) fails as an out-of-memory cudaMalloc would,
 * and the call that made it returns NBK_ERR_NOMEM; later calls allocate
 * normally. 0 disarms. Process-wide. */
NBK_API int nbk_debug_fail_alloc(int countdown);

/* ---- measurement ----------------------------------------------------------- */

/* Enables (1) or disables (0) CUDA-event timing of every force-kernel launch
 * of this handle; enabling clears the recorded launches. */
NBK_API int nbk_set_kernel_timing(nbk_handle h, int enable);
/* Durations (ms) of the evaluations recorded since timing was enabled,
 * oldest first (synchronises): the force kernel, with the refinement,
 * compaction and sort before it on pairlist evaluations. *count receives the
 * number recorded (at most 4096 are kept); at most maxCount are written. */
NBK_API int nbk_get_kernel_times(nbk_handle h, float* ms, int maxCount, int* count);
/* The same evaluations' precise energy / virial kernel (the FP64 pass after
 * the force kernel on evaluations with NBK_ENERGY, or NBK_VIRIAL | NBK_SLOW;
 * about 0 otherwise). */
NBK_API int nbk_get_precise_times(nbk_handle h, float* ms, int maxCount, int* count);
/* Pairs evaluated within the cutoff by the last nbk_nonbonded_force, which
 * must have had NBK_ENERGY (the work unit of the pairs/s metric; synchronises). */
NBK_API int nbk_get_pair_count(nbk_handle h, long long* pairs, void* stream);
/* Number of kernels this handle has launched since it was created. */
NBK_API long long nbk_launch_count(nbk_handle h);
/* FP32 FMA throughput of the device (TFLOP/s, FMA = 2 flops), measured with a
 * register-resident FMA loop over all SMs (synchronises; ~50 ms). */
NBK_API int nbk_measure_fp32_peak(int deviceID, double* tflops);
/* FP64 FMA throughput of the device, measured the same way. */
NBK_API int nbk_measure_fp64_peak(int deviceID, double* tflops);

/* Autotuner of the force kernel's launch shape (no counterpart in the
 * reference, whose launch shape is fixed: NONBONDKERNEL_NUM_WARP warps per
 * block, src/CudaComputeNonbondedKernel.cu:32,2151-2152). Times every shape on
 * the handle's current refined lists, positions and lattice (those of the last
 * nbk_nonbonded_force call, which must still be valid) with `iterations`
 * launches each, and keeps the fastest for this flag combination (energy,
 * virial, slow; batched or not): CTAs per SM 4, 5 or 6 (the register cap:
 * 128, 96 or 80 registers) times 1, 2 or 4 warps per tile list (a list's j
 * tiles split into contiguous parts of whole groups of four tiles, handed out
 * separately). The choice changes no result: FP32 partials are folded into
 * integer fixed point at the end of every j tile (j forces) and of every
 * group of four tiles (i forces, LJ energy), and all further sums are integer.
 * Synchronises the stream; overwrites the handle's force and energy
 * accumulators, so call it before an evaluation, not between an evaluation
 * and its nbk_reduce_virial_energy. Untuned handles use 4 CTAs per SM and one
 * warp per list; the tuner keeps that default unless another shape is at
 * least 3% faster, since shapes are timed back to back on a warm L2. */
NBK_API int nbk_autotune(nbk_handle h, unsigned flags, int iterations, void* stream);

/* The launch shape in use for a flag combination and the time per force
 * launch measured by nbk_autotune (0 before tuning). */
NBK_API int nbk_get_tuning(nbk_handle h, unsigned flags, int* minBlocksPerSM, int* listSplit,
                           float* ms);

/* Pins the launch shape for a flag combination without timing (CTAs per SM 4,
 * 5 or 6; 1, 2 or 4 warps per tile list). */
NBK_API int nbk_set_tuning(nbk_handle h, unsigned flags, int minBlocksPerSM, int listSplit);

/* ---- GPU-resident input marshaling -------------------------------------------
 * For callers whose atoms stay on the device between steps (NAMD's
 * GPU-resident integrator, SequencerCUDA with device migration): the patch
 * atom order, the patch-centred xyzq and the per-slot vdW types / exclusion
 * indices are produced by kernels from the integrator's per-atom arrays
 * instead of host loops and copies. The per-atom arrays are in "buffer
 * order": patch p's atoms occupy [bufferOffset, bufferOffset + numAtoms) of
 * every per-atom array, in any order; its nonbonded slots are
 * [bufferOffsetNBPad, bufferOffsetNBPad + numAtomsNBPad). All pointers named
 * d_* are device pointers. */

/* CudaLocalRecord, src/CudaRecord.h:35-52 (128 bytes; the five CudaPeerRecords
 * are carried as opaque words). Only patchID..numAtomsNBPad are read. */
typedef struct {
  int patchID;
  int bufferOffset;        /* first atom of the patch in the per-atom arrays */
  int bufferOffsetNBPad;   /* first nonbonded slot of the patch (multiple of 32) */
  int numAtoms;
  int numAtomsNBPad;       /* numAtoms rounded up to a multiple of 32 */
  int isProxy;
  int numPeerRecord;
  int peerRecordStartIndex;
  int bufferOffsetOld;
  int numMigrationGroups;
  int numAtomsNew;
  int numAtomsLocal;
  int inlinePeers[20];     /* CudaPeerRecord[5]; not read */
} nbk_local_record;

typedef struct { double x, y, z; } nbk_double3;

/* Largest patch nbk_sort_patch_atoms orders (atoms per patch). */
#define NBK_MAX_PATCH_ATOMS 2048

/* Patch sort: the nonbonded order of every patch's atoms, recursive
 * bisection of the patch at multiples of 32, then 16, then 8 atoms along the
 * longest extent of each part, ties broken by global atom id (the atom order
 * of src/SortAtoms.C:45-133 that the reference's host caller produces; on the
 * GPU-resident path the reference sorts in src/MigrationCUDAKernel.cu:103-460).
 * The atom sets of every 8-atom block (hence of every 32-atom tile) are those
 * of the host order nbk_pack builds; within a block the atoms are in (coordinate,
 * id) order. Writes d_sortOrder[bufferOffset + i] = the index within the patch
 * (0..numAtoms-1) of the atom placed in the patch's nonbonded slot i.
 * maxPatchAtoms: an upper bound of numAtoms over the patches (at most
 * NBK_MAX_PATCH_ATOMS). d_status (may be NULL): a device int that is
 * incremented for every patch larger than the bound (such a patch keeps its
 * buffer order). */
NBK_API int nbk_sort_patch_atoms(int numPatches, const nbk_local_record* d_localRecords,
                                 int maxPatchAtoms, const double* d_pos_x, const double* d_pos_y,
                                 const double* d_pos_z, const int* d_id, int* d_sortOrder,
                                 int* d_status, void* stream);

/* The nonbonded part of setComputePositionsKernel, src/SequencerCUDAKernel.cu:
 * 1950-2041: xyzq[slot] = (x - centre, q * chargeScaling) with the patch centre
 * unscaled from fractional coordinates (o + a sx + b sy + c sz, FP64) and the
 * difference rounded once to FP32; the slots past numAtoms repeat the last
 * atom. lattice: a, b, c, origin as 12 doubles (host). d_charge: FP32 charges
 * (the product with chargeScaling is formed in FP64, as the reference does). */
NBK_API int nbk_set_compute_positions(int numPatches, const nbk_local_record* d_localRecords,
                                      const nbk_double3* d_patchCenter, const double* lattice,
                                      const int* d_sortOrder, double chargeScaling,
                                      const double* d_pos_x, const double* d_pos_y,
                                      const double* d_pos_z, const float* d_charge,
                                      nbk_float4* d_xyzq, void* stream);

/* SequencerCUDAKernel::accumulateForceToSOA, src/SequencerCUDAKernel.cu:179-297
 * (one device): the integrator's per-atom FP64 force arrays, in buffer order,
 * from the 64-bit fixed-point sums of the last nbk_nonbonded_force of this
 * handle (converted exactly, not through its float4 outputs), the PME forces
 * and the bonded force arrays:
 *   f_normal = f_bond
 *   f_nbond  = nonbonded fast + f_bond_nbond
 *   f_slow   = PME + nonbonded slow + f_bond_slow   (added in this order)
 * maxForceNumber 0 writes f_normal only, 1 also f_nbond, 2 also f_slow (the
 * reference's levels). d_sortOrder as nbk_sort_patch_atoms writes it (the
 * reference takes its inverse, patchUnsortOrder). d_f_bond, d_f_bond_nbond,
 * d_f_bond_slow: [3][forceStride] FP64 (x, y, z rows; NULL = zero). d_f_pme:
 * Cartesian float3 per atom in buffer order (NULL = zero), e.g. from
 * nbk_pme_gather_force on the same atoms. */
NBK_API int nbk_accumulate_forces_to_soa(nbk_handle h, int maxForceNumber, int numPatches,
                                         const nbk_local_record* d_localRecords,
                                         const int* d_sortOrder, const double* d_f_bond,
                                         const double* d_f_bond_nbond, const double* d_f_bond_slow,
                                         int forceStride, const nbk_float3* d_f_pme,
                                         double* d_f_normal_x, double* d_f_normal_y,
                                         double* d_f_normal_z, double* d_f_nbond_x,
                                         double* d_f_nbond_y, double* d_f_nbond_z,
                                         double* d_f_slow_x, double* d_f_slow_y,
                                         double* d_f_slow_z, void* stream);

/* ---- PME reciprocal space -------------------------------------------------------
 * The long-range half of the slow (PME) forces that the short-range kernel's
 * slow buffers hold the real-space half of: smooth particle-mesh Ewald on one
 * GPU, the single-device path of CudaPmeRealSpaceCompute /
 * CudaPmeKSpaceCompute / CudaFFTCompute (src/CudaPmeSolverUtil.h:60-160,
 * src/CudaPmeSolverUtilKernel.cu). Atoms are CudaAtom records holding
 * fractional coordinates in [0, 1) and scaled charges, as ComputePmeCUDA
 * sends them (src/ComputePmeCUDA.C:281-300). Charges are spread with the
 * reference's B-spline order and grid-offset convention into a 64-bit
 * fixed-point grid (deterministic: integer sums do not depend on the order of
 * the atomics), transformed with cuFFT (real-to-complex, x fastest), scaled by
 * the influence function with the reference's B-spline moduli, transformed
 * back and interpolated to forces. Not thread-safe per handle. */
typedef struct nbk_pme_s* nbk_pme;

/* PmeGrid (src/PmeBase.h): grid points per lattice vector and B-spline
 * order (4, 6 or 8). */
typedef struct {
  int K1, K2, K3;
  int order;
} nbk_pme_grid;

NBK_API int nbk_pme_create(int deviceID, const nbk_pme_grid* grid, double ewaldcof, nbk_pme* out);
NBK_API int nbk_pme_destroy(nbk_pme pme);

/* ComputePmeCUDA::sendAtoms' conversion (src/ComputePmeCUDA.C:281-300) on the
 * device: w = r . a_r shifted into [0, 1) by w - (floor(w + 1/2) - 1/2), in
 * FP64, rounded to FP32 (a value rounded up to 1 becomes 0); q = charge *
 * chargeScaling in FP64. lattice: a, b, c, origin (12 doubles, host). */
NBK_API int nbk_pme_atoms_from_positions(int numAtoms, const double* d_x, const double* d_y,
                                         const double* d_z, const float* d_charge,
                                         double chargeScaling, const double* lattice,
                                         nbk_float4* d_atoms, void* stream);

/* CudaPmeRealSpaceCompute::copyAtoms + spreadCharge (src/CudaPmeSolverUtil.C,
 * spread_charge_kernel src/CudaPmeSolverUtilKernel.cu:427-530). */
NBK_API int nbk_pme_spread_charge(nbk_pme pme, int numAtoms, const nbk_float4* d_atoms,
                                  void* stream);

/* CudaFFTCompute::forward, CudaPmeKSpaceCompute::solve (scalar_sum_kernel,
 * src/CudaPmeSolverUtilKernel.cu:74-325) and CudaFFTCompute::backward.
 * lattice: a, b, c (9 doubles, host). flags: NBK_ENERGY and/or NBK_VIRIAL.
 * Consumes the charge grid of the last nbk_pme_spread_charge: afterwards the
 * grid holds the potential that nbk_pme_gather_force interpolates, so every
 * solve needs a spread before it. */
NBK_API int nbk_pme_solve(nbk_pme pme, const double* lattice, unsigned flags, void* stream);

/* CudaPmeRealSpaceCompute::gatherForce (gather_force,
 * src/CudaPmeSolverUtilKernel.cu:708-945) followed by ComputePmeCUDA's
 * conversion to Cartesian forces (src/ComputePmeCUDA.C:640-652):
 * d_force[i] = f1 a_r + f2 b_r + f3 c_r. lattice: a, b, c (9 doubles, host). */
NBK_API int nbk_pme_gather_force(nbk_pme pme, int numAtoms, const nbk_float4* d_atoms,
                                 const double* lattice, nbk_float3* d_force, void* stream);

/* CudaPmeKSpaceCompute::getEnergy / getVirial of the last nbk_pme_solve
 * (synchronises). virial: 9 doubles, row-major, sum of r (x) F convention. */
NBK_API int nbk_pme_get_energy_virial(nbk_pme pme, double* energy, double* virial, void* stream);

/* The Ewald self energy -beta/sqrt(pi) sum q^2 (selfEnergyKernel,
 * src/CudaPmeSolverUtilKernel.cu:1192-1216; synchronises). */
NBK_API int nbk_pme_self_energy(nbk_pme pme, int numAtoms, const nbk_float4* d_atoms,
                                double* selfEnergy, void* stream);

/* CudaComputeNonbondedKernel::setExclusionsByAtom, src/CudaComputeNonbondedKernel.cu:
 * 3640-3645: per global atom id, (maxdiff, base) of its exclusion list in the
 * bit array bound by nbk_bind_exclusions (host array, copied; synchronises). */
NBK_API int nbk_set_exclusions_by_atom(nbk_handle h, int numAtoms,
                                       const nbk_int2* h_exclusionsByAtom);

/* CudaComputeNonbondedKernel::updateVdwTypesExclOnGPU, src/CudaComputeNonbondedKernel.cu:
 * 3648-3724: the handle's per-slot vdW types, global atom indices and
 * (base, maxdiff) exclusion indices from per-atom arrays in buffer order
 * through d_sortOrder, as nbk_update_vdw_types_excl does from host arrays.
 * Unlike the reference kernel, the padding slots repeat the patch's last atom.
 * A vdW type outside the LJ table or an id outside the nbk_set_exclusions_by_atom
 * range is written as type 0 / no exclusions and counted in d_status (a device
 * int, may be NULL). */
NBK_API int nbk_update_vdw_types_excl_device(nbk_handle h, int numPatches, int atomStorageSize,
                                             const nbk_local_record* d_localRecords,
                                             const int* d_vdwTypes, const int* d_id,
                                             const int* d_sortOrder, int* d_status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NBK_H */
