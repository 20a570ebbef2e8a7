// Tile-list build of the B200 nonbonded path: tile bounding boxes, bbox
// culling of every (compute, i-tile) into a j-tile list, and the compaction
// that follows the pairlist refinement.
//
// The reference (src/CudaTileListKernel.cu:1022-1192) culls with one thread
// per i-tile looping over the partner patch's tiles, allocates output with
// atomics and re-launches after a host synchronisation when its buffer
// overflows. Here one warp culls one i-tile (its lanes test 32 j-tiles at a
// time, ballot + popc place the survivors), and every list writes into a
// slot range reserved on the host from the patch sizes, so the build never
// overflows, never synchronises with the host and can be captured in a graph.
#include <atomic>
#include "nbk_internal.cuh"
#include "nbk_launch.h"

namespace nbk {

// One warp per 32-atom tile: min/max reduction over the tile's atoms
// (buildBoundingBoxesKernel, src/CudaTileListKernel.cu:242-281).
__global__ void bboxKernel(int numTiles, const float4* __restrict__ xyzq, BBox* __restrict__ bb) {
  const int lane = threadIdx.x & 31;
  const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < numTiles; t += warpsPerGrid) {
    const float4 x = xyzq[(size_t)t * 32 + lane];
    float lx = x.x, ly = x.y, lz = x.z, hx = x.x, hy = x.y, hz = x.z;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, o));
      ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, o));
      lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, o));
      hx = fmaxf(hx, __shfl_xor_sync(0xffffffffu, hx, o));
      hy = fmaxf(hy, __shfl_xor_sync(0xffffffffu, hy, o));
      hz = fmaxf(hz, __shfl_xor_sync(0xffffffffu, hz, o));
    }
    if (lane == 0) {
      BBox b;
      b.x = 0.5f * (lx + hx);
      b.y = 0.5f * (ly + hy);
      b.z = 0.5f * (lz + hz);
      b.wx = 0.5f * (hx - lx);
      b.wy = 0.5f * (hy - ly);
      b.wz = 0.5f * (hz - lz);
      bb[t] = b;
    }
  }
}

// Lower bound of the distance^2 between two boxes (src/CudaTileListKernel.cu:286-292).
__device__ __forceinline__ float bbDist2(const BBox& a, const BBox& b) {
  const float dx = fmaxf(0.0f, fabsf(a.x - b.x) - a.wx - b.wx);
  const float dy = fmaxf(0.0f, fabsf(a.y - b.y) - a.wy - b.wy);
  const float dz = fmaxf(0.0f, fabsf(a.z - b.z) - a.wz - b.wz);
  return dx * dx + dy * dy + dz * dz;
}

// One warp per (compute, i-tile): j tiles of the partner patch whose box is
// within the pairlist cutoff (self computes: j-tile >= i-tile).
__global__ void buildListsKernel(int numLists, const ListSeed* __restrict__ seeds,
                                 const nbk_compute_record* __restrict__ computes,
                                 const nbk_patch_record* __restrict__ patches,
                                 const BBox* __restrict__ bb, float3 lata, float3 latb, float3 latc,
                                 const int* __restrict__ compRep, const float3* __restrict__ repLat,
                                 float cull2, nbk_tile_list* __restrict__ lists,
                                 PatchPair* __restrict__ pp, int* __restrict__ tileJatomStart) {
  const int lane = threadIdx.x & 31;
  const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
  for (int L = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; L < numLists; L += warpsPerGrid) {
    const ListSeed sd = seeds[L];
    const nbk_compute_record cr = computes[sd.icompute];
    const nbk_patch_record p1 = patches[cr.patchInd.x];
    const nbk_patch_record p2 = patches[cr.patchInd.y];
    float3 la = lata, lb = latb, lc = latc;
    if (compRep) {  // batched replicas: this compute's replica lattice
      const int rep = compRep[sd.icompute];
      la = repLat[3 * rep];
      lb = repLat[3 * rep + 1];
      lc = repLat[3 * rep + 2];
    }
    const float3 sh = shiftOf(make_float3(cr.offsetXYZ.x, cr.offsetXYZ.y, cr.offsetXYZ.z), la, lb, lc);
    const bool zeroShift = !(dist2(sh.x, sh.y, sh.z) > 0.0f);
    const bool self = zeroShift && (p1.atomStart == p2.atomStart);
    BBox bi = bb[p1.atomStart / 32 + sd.itile];
    bi.x += sh.x;
    bi.y += sh.y;
    bi.z += sh.z;
    const int ntiles2 = (p2.numAtoms + 31) / 32;
    int count = 0;
    for (int k0 = 0; k0 < ntiles2; k0 += 32) {
      const int k = k0 + lane;
      bool pass = false;
      if (k < ntiles2 && (!self || k >= sd.itile)) pass = bbDist2(bi, bb[p2.atomStart / 32 + k]) < cull2;
      const unsigned ball = __ballot_sync(0xffffffffu, pass);
      if (pass) {
        const int rank = __popc(ball & ((1u << lane) - 1u));
        tileJatomStart[sd.jcapStart + count + rank] = p2.atomStart + k * 32;
      }
      count += __popc(ball);
    }
    if (lane == 0) {
      nbk_tile_list t;
      t.iatomStart = p1.atomStart + sd.itile * 32;
      t.jtileStart = sd.jcapStart;
      t.jtileEnd = sd.jcapStart + count - 1;
      t.offsetXYZ = cr.offsetXYZ;
      t.patchInd = cr.patchInd;
      t.patchNumList.x = 0;
      t.patchNumList.y = 0;
      t.icompute = sd.icompute;
      lists[L] = t;
      PatchPair q;
      q.iatomSize = p1.atomStart + p1.numAtoms;
      q.iatomFreeSize = p1.atomStart + p1.numFreeAtoms;
      q.jatomSize = p2.atomStart + p2.numAtoms;
      q.jatomFreeSize = p2.atomStart + p2.numFreeAtoms;
      pp[L] = q;
    }
  }
}

// After the pairlist refinement: drop j tiles without interacting pairs and
// lists left empty (reSortTileLists' compaction, src/CudaTileListKernel.cu:
// 1605-1665). counters[0] = lists kept, counters[1] = j tiles kept. A block
// of kCompactWarps warps takes as many lists at a time, one per warp; one
// thread reserves the output of all of them with one pair of atomics.
constexpr int kCompactWarps = 8;

__global__ void __launch_bounds__(kCompactWarps * 32)
    compactKernel(int numLists, const nbk_tile_list* __restrict__ src,
                  const int* __restrict__ listActive, const int* __restrict__ jtileActive,
                  const int* __restrict__ jatomSrc, const nbk_tile_excl* __restrict__ exclSrc,
                  nbk_tile_list* __restrict__ dst, int* __restrict__ jatomDst,
                  nbk_tile_excl* __restrict__ exclDst, int* __restrict__ counters) {
  __shared__ int s_n[kCompactWarps], s_pos[kCompactWarps], s_jpos[kCompactWarps];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  for (int Lb = blockIdx.x * kCompactWarps; Lb < numLists; Lb += gridDim.x * kCompactWarps) {
    const int L = Lb + wib;
    int n = 0;
    nbk_tile_list s;
    if (L < numLists) {
      s = src[L];
      // listActive is only written for lists with tiles (empty lists skip the refinement)
      if (s.jtileEnd >= s.jtileStart) n = listActive[L];
    }
    if (lane == 0) s_n[wib] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
      int kept = 0, tiles = 0;
      for (int w = 0; w < kCompactWarps; ++w) {
        s_pos[w] = kept;
        s_jpos[w] = tiles;
        kept += s_n[w] > 0 ? 1 : 0;
        tiles += s_n[w];
      }
      const int p0 = kept ? atomicAdd(&counters[0], kept) : 0;
      const int j0 = kept ? atomicAdd(&counters[1], tiles) : 0;
      for (int w = 0; w < kCompactWarps; ++w) {
        s_pos[w] += p0;
        s_jpos[w] += j0;
      }
    }
    __syncthreads();
    if (n > 0) {  // warp-uniform
      const int pos = s_pos[wib], jpos = s_jpos[wib];
      int w = 0;
      for (int j0 = s.jtileStart; j0 <= s.jtileEnd; j0 += 32) {
        const int jt = j0 + lane;
        const bool act = (jt <= s.jtileEnd) && jtileActive[jt];
        unsigned ball = __ballot_sync(0xffffffffu, act);
        if (act) jatomDst[jpos + w + __popc(ball & ((1u << lane) - 1u))] = jatomSrc[jt];
        while (ball) {
          const int b = __ffs(ball) - 1;
          ball &= ball - 1;
          exclDst[jpos + w].excl[lane] = exclSrc[j0 + b].excl[lane];
          ++w;
        }
      }
      if (lane == 0) {
        nbk_tile_list d = s;
        d.jtileStart = jpos;
        d.jtileEnd = jpos + n - 1;
        dst[pos] = d;
      }
    }
  }
}

// Pairlist refinement without force math: for every j tile of every culled
// list, bit t of TileExcl.excl[lane] is set when the pair (i = iatomStart +
// lane, j = jatomStart + ((lane + t) & 31)) lies within the pairlist cutoff
// (FP32 r^2 with the shift and operand order of shiftOf / dist2), is not a
// padding pair, is not the diagonal or lower triangle of a self tile and is
// not a full exclusion (the pairlist pass of nonbondedForceKernel,
// src/CudaComputeNonbondedKernel.cu:1202-1249,1424-1443). Writes the masks
// in place, jtileActive / listActive for the compaction and the per-replica
// count of excluded pairs within the pairlist cutoff. One warp per list,
// lists handed out from a.workCounter.
//
// Layout of the work: every lane tests its i atom against j = 0..31 in
// natural order, two j atoms (k, k + 16) per packed-FP32 step, with the j
// tile's coordinates and indices read as warp-wide broadcasts from shared
// memory. The sign bits of r^2 - plcutoff^2 (the same per-element rounding
// as dist2; the sign of a rounded difference is the sign of the exact one)
// are shifted into a word whose bit j marks pair (lane, j); one rotation by
// the lane number turns it into the TileExcl order (bit t <-> j = (lane + t)
// & 31). Exclusions are only looked up for candidates whose global indices
// lie within the i atom's maxdiff window: |jIndex - iIndex| <= maxdiff is
// tested as the sign of (jIndex - iIndex)^2 - (maxdiff^2 + 1/2) in FP32,
// exact while indices are below 2^24 and maxdiff <= kFpWindowMaxDiff (the
// difference and maxdiff^2 + 1/2 are then representable, and a fused
// multiply-add rounds once and keeps the sign). Outside those bounds every
// candidate is looked up.
constexpr int kFpWindowMaxDiff = 2896;  // 2896^2 + 1/2 < 2^23

__global__ void __launch_bounds__(128) refineKernel(const __grid_constant__ ForceArgs a) {
  // per warp: s_p0[k] = (x_k, x_k+16, y_k, y_k+16), s_p1[k] = (z_k, z_k+16, index_k, index_k+16)
  __shared__ float4 s_p0[4][16], s_p1[4][16];
  __shared__ int s_jidx[4][32];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const float2 nPlc2 = f2(-a.c.plcutoff2);
  float* const p0 = reinterpret_cast<float*>(&s_p0[wib][lane & 15]) + (lane >> 4);
  float* const p1 = reinterpret_cast<float*>(&s_p1[wib][lane & 15]) + (lane >> 4);
  int nexcl = 0, curRep = 0;
  for (;;) {
    int L = 0;
    if (lane == 0) L = atomicAdd(a.workCounter, 1);
    L = __shfl_sync(0xffffffffu, L, 0);
    if (L >= a.numListsHost) break;
    const nbk_tile_list tl = a.lists[L];
    if (tl.jtileEnd < tl.jtileStart) continue;  // warp-uniform
    float3 la = a.lata, lb = a.latb, lc = a.latc;
    if (a.compRep) {
      const int rep = __ldg(&a.compRep[tl.icompute]);
      if (rep != curRep) {
        const int s = __reduce_add_sync(0xffffffffu, nexcl);
        if (lane == 0 && s) atomicAddFixed(&a.acc[(size_t)curRep * kAccCount + kAccNumExcl], (unsigned long long)s);
        nexcl = 0;
        curRep = rep;
      }
      la = a.repLat[3 * rep];
      lb = a.repLat[3 * rep + 1];
      lc = a.repLat[3 * rep + 2];
    }
    const float3 sh = shiftOf(make_float3(tl.offsetXYZ.x, tl.offsetXYZ.y, tl.offsetXYZ.z), la, lb, lc);
    const bool zeroShift = !(dist2(sh.x, sh.y, sh.z) > 0.0f);
    const bool selfCompute = (tl.patchInd.x == tl.patchInd.y) && zeroShift;
    const int iatom = tl.iatomStart + lane;
    const PatchPair pp = a.patchPairs[L];
    const int nloopi = min(pp.iatomSize - tl.iatomStart, 32);
    const int nfreei = max(pp.iatomFreeSize - tl.iatomStart, 0);
    float4 xi = a.xyzq[iatom];
    xi.x = __fadd_rn(xi.x, sh.x);
    xi.y = __fadd_rn(xi.y, sh.y);
    xi.z = __fadd_rn(xi.z, sh.z);
    if (lane >= nloopi) xi.x = xi.y = xi.z = -1.0e10f;
    const int iIndex = a.atomIndex[iatom];
    const int2 em = a.exclIndexMaxDiff[iatom];
    const bool fpList = __all_sync(0xffffffffu, lane >= nloopi || ((unsigned)iIndex < (1u << 24) &&
                                                                    em.y <= kFpWindowMaxDiff));
    const float emy = (float)min(max(em.y, 0), kFpWindowMaxDiff);
    const float2 nXi = f2(-xi.x), nYi = f2(-xi.y), nZi = f2(-xi.z);
    const float2 nIi = f2(-(float)iIndex), nT = f2(-fmaf(emy, emy, 0.5f));
    int activeTiles = 0;
    for (int jt0 = tl.jtileStart; jt0 <= tl.jtileEnd; jt0 += 32) {
      const int nt = min(32, tl.jtileEnd - jt0 + 1);
      const int jsLane = lane < nt ? a.tileJatomStart[jt0 + lane] : 0;
      // software pipeline: the next tile's atoms are loaded before this tile's math
      int jsNext = __shfl_sync(0xffffffffu, jsLane, 0);
      float4 xjNext = a.xyzq[jsNext + lane];
      int idxNext = a.atomIndex[jsNext + lane];
      for (int u = 0; u < nt; ++u) {
        const int jt = jt0 + u;
        const int jstart = jsNext;
        float4 xj = xjNext;
        const int jIndex = idxNext;
        if (u + 1 < nt) {  // warp-uniform
          jsNext = __shfl_sync(0xffffffffu, jsLane, u + 1);
          xjNext = a.xyzq[jsNext + lane];
          idxNext = a.atomIndex[jsNext + lane];
        }
        const bool diag = selfCompute && (jstart == tl.iatomStart);
        const int nloopj = min(pp.jatomSize - jstart, 32);
        const int nfreej = max(pp.jatomFreeSize - jstart, 0);
        if (lane >= nloopj) xj.x = xj.y = xj.z = 1.0e10f;
        p0[0] = xj.x;
        p0[2] = xj.y;
        p1[0] = xj.z;
        p1[2] = (float)jIndex;
        s_jidx[wib][lane] = jIndex;
        const bool fpTile = fpList && __all_sync(0xffffffffu, lane >= nloopj || (unsigned)jIndex < (1u << 24));
        __syncwarp();
        unsigned cA = 0, cB = 0, wA = 0, wB = 0;
#pragma unroll
        for (int k = 15; k >= 0; --k) {
          const float4 P0 = s_p0[wib][k], P1 = s_p1[wib][k];
          const float2 DX = add2(make_float2(P0.x, P0.y), nXi);
          const float2 DY = add2(make_float2(P0.z, P0.w), nYi);
          const float2 DZ = add2(make_float2(P1.x, P1.y), nZi);
          const float2 R2 = fma2(DZ, DZ, fma2(DX, DX, mul2(DY, DY)));  // dist2's order
          const float2 C = add2(R2, nPlc2);  // negative: within the pairlist cutoff
          const float2 DI = add2(make_float2(P1.z, P1.w), nIi);
          const float2 W = fma2(DI, DI, nT);  // negative: within the maxdiff window
          cA = __funnelshift_l(__float_as_uint(C.x), cA, 1);
          cB = __funnelshift_l(__float_as_uint(C.y), cB, 1);
          wA = __funnelshift_l(__float_as_uint(W.x), wA, 1);
          wB = __funnelshift_l(__float_as_uint(W.y), wB, 1);
        }
        unsigned mw = cA | (cB << 16);  // bit j: pair (lane, j) within the pairlist cutoff
        if (diag) mw &= 0xFFFFFFFEu << lane;                          // self tile: j > lane only
        if (lane >= nfreei && nfreej < 32) mw &= (1u << nfreej) - 1u;  // fixed-fixed pairs
        unsigned need = fpTile ? (mw & (wA | (wB << 16))) : mw;
        while (need) {
          const int j = __ffs(need) - 1;
          need &= need - 1u;
          const int diff = s_jidx[wib][j] - iIndex;
          if (abs(diff) <= em.y) {
            const unsigned bit = (unsigned)(diff + em.x);
            const unsigned w = ((int)(bit >> 5) < a.numExclWords) ? __ldg(&a.exclBits[bit >> 5]) : 0u;
            if ((w >> (bit & 31)) & 1u) {
              mw &= ~(1u << j);
              ++nexcl;
            }
          }
        }
        const unsigned m = __funnelshift_r(mw, mw, lane);  // bit t <-> j = (lane + t) & 31
        a.tileExcls[jt].excl[lane] = m;
        const bool any = __any_sync(0xffffffffu, m != 0);
        if (lane == 0) a.jtileActive[jt] = any ? 1 : 0;
        activeTiles += any ? 1 : 0;
        __syncwarp();
      }
    }
    if (lane == 0) a.listActive[L] = activeTiles;
  }
  const int s = __reduce_add_sync(0xffffffffu, nexcl);
  if (lane == 0 && s) atomicAddFixed(&a.acc[(size_t)curRep * kAccCount + kAccNumExcl], (unsigned long long)s);
}

cudaError_t launchRefine(const ForceArgs& a, int numSM, cudaStream_t st) {
  if (a.numListsHost <= 0) return cudaSuccess;
  // blocks per SM of this kernel (no dynamic shared memory, so the same on
  // every device of one architecture); an atomic, as handles on several host
  // threads may launch it at once
  static std::atomic<int> cachedBlocks{0};
  int blocks = cachedBlocks.load(std::memory_order_relaxed);
  if (!blocks) {
    int nb = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, refineKernel, 128, 0);
    if (e != cudaSuccess) return e;
    blocks = nb > 0 ? nb : 1;
    cachedBlocks.store(blocks, std::memory_order_relaxed);
  }
  refineKernel<<<numSM * blocks, 128, 0, st>>>(a);
  return cudaGetLastError();
}

// The compacted lists in order of decreasing length (the order sortTileLists
// establishes, src/CudaTileListKernel.cu:1208-1600): with lists handed out
// longest first from the work counter, the last lists to start are the
// shortest, which trims the tail of the force launch (0.483 -> 0.448 ms at
// 92k atoms). A counting sort over the lengths: histogram, offsets in
// decreasing length, scatter. Lanes of a warp holding lists of the same
// length combine their atomics (__match_any_sync), so popular lengths do not
// serialise on one counter. Lists of equal length land in any order; nothing
// computed from them depends on list order.
__device__ __forceinline__ int listLength(const nbk_tile_list& t, int maxLen) {
  return min(max(t.jtileEnd - t.jtileStart + 1, 0), maxLen);
}

__global__ void listLengthHistKernel(const nbk_tile_list* __restrict__ lists,
                                     const int* __restrict__ numLists, int maxLen,
                                     int* __restrict__ hist) {
  const int n = *numLists;
  const int lane = threadIdx.x & 31;
  for (int L0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; L0 < n; L0 += gridDim.x * blockDim.x) {
    const int L = L0 + lane;
    const int len = L < n ? listLength(lists[L], maxLen) : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, len);
    if (len >= 0 && lane == __ffs(peers) - 1) atomicAdd(&hist[len], __popc(peers));
  }
}

__global__ void listLengthScanKernel(int maxLen, int* __restrict__ hist) {
  if (threadIdx.x != 0) return;
  int off = 0;
  for (int len = maxLen; len >= 0; --len) {
    const int c = hist[len];
    hist[len] = off;
    off += c;
  }
}

__global__ void listScatterKernel(const nbk_tile_list* __restrict__ src, const int* __restrict__ numLists,
                                  int maxLen, int* __restrict__ cursor, nbk_tile_list* __restrict__ dst) {
  const int n = *numLists;
  const int lane = threadIdx.x & 31;
  for (int L0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; L0 < n; L0 += gridDim.x * blockDim.x) {
    const int L = L0 + lane;
    nbk_tile_list t;
    int len = -1;
    if (L < n) {
      t = src[L];
      len = listLength(t, maxLen);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, len);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (len >= 0 && lane == leader) base = atomicAdd(&cursor[len], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (len >= 0) dst[base + __popc(peers & ((1u << lane) - 1u))] = t;
  }
}

cudaError_t launchSortLists(int numListsMax, const nbk_tile_list* src, const int* numListsDev,
                            int maxLen, int* hist, nbk_tile_list* dst, int numSM, cudaStream_t st) {
  if (numListsMax <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(int) * ((size_t)maxLen + 1), st);
  if (e != cudaSuccess) return e;
  const int blocks = min((numListsMax + 255) / 256, numSM * 4);
  listLengthHistKernel<<<blocks, 256, 0, st>>>(src, numListsDev, maxLen, hist);
  listLengthScanKernel<<<1, 32, 0, st>>>(maxLen, hist);
  listScatterKernel<<<blocks, 256, 0, st>>>(src, numListsDev, maxLen, hist, dst);
  return cudaGetLastError();
}

cudaError_t launchBBoxes(int numTiles, const float4* xyzq, BBox* bb, cudaStream_t st) {
  if (numTiles <= 0) return cudaSuccess;
  const int threads = 256;
  const int blocks = min((numTiles + 7) / 8, 4096);
  bboxKernel<<<blocks, threads, 0, st>>>(numTiles, xyzq, bb);
  return cudaGetLastError();
}

cudaError_t launchBuildLists(int numLists, const ListSeed* seeds,
                             const nbk_compute_record* computes, const nbk_patch_record* patches,
                             const BBox* bb, float3 lata, float3 latb, float3 latc,
                             const int* compRep, const float3* repLat, float cull2,
                             nbk_tile_list* lists, PatchPair* pp, int* tileJatomStart,
                             cudaStream_t st) {
  if (numLists <= 0) return cudaSuccess;
  const int threads = 256;
  const int blocks = min((numLists + 7) / 8, 8192);
  buildListsKernel<<<blocks, threads, 0, st>>>(numLists, seeds, computes, patches, bb, lata, latb,
                                               latc, compRep, repLat, cull2, lists, pp,
                                               tileJatomStart);
  return cudaGetLastError();
}

cudaError_t launchCompact(int numLists, const nbk_tile_list* src, const int* listActive,
                          const int* jtileActive, const int* jatomSrc, const nbk_tile_excl* exclSrc,
                          nbk_tile_list* dst, int* jatomDst, nbk_tile_excl* exclDst, int* counters,
                          int numSM, cudaStream_t st) {
  if (numLists <= 0) return cudaSuccess;
  const int blocks = min((numLists + kCompactWarps - 1) / kCompactWarps, numSM * 8);
  compactKernel<<<blocks, kCompactWarps * 32, 0, st>>>(numLists, src, listActive, jtileActive, jatomSrc,
                                            exclSrc, dst, jatomDst, exclDst, counters);
  return cudaGetLastError();
}

}  // namespace nbk
