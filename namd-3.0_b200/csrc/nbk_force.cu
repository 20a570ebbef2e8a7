// Nonbonded force kernel of the B200 path.
//
// One warp owns one tile list (32 i atoms of one patch against the j tiles of
// a compute's partner patch), as CudaComputeNonbondedKernel's
// nonbondedForceKernel does (src/CudaComputeNonbondedKernel.cu:629-1644), but:
//   - j forces ride in registers and rotate one lane per step with a shuffle
//     (lane l works on j = (l+t) & 31 at step t), so the inner loop touches
//     shared memory only for the broadcast-free j coordinate load;
//   - steps whose bit is clear in every lane's mask are skipped warp-uniformly
//     (the rotation jumps by the step distance);
//   - the lists it reads are already refined (TileExcl masks from
//     refineKernel); a pairlist step refines, compacts, then runs this kernel;
//   - per-tile FP32 partial forces are folded into 64-bit fixed point with
//     integer atomics, so the summed forces do not depend on the order in
//     which lists run; energies and virials are folded into fixed point per
//     list for the same reason.
#include "nbk_internal.cuh"
#include "nbk_launch.h"

namespace nbk {

constexpr int kForceWarps = 4;
// FP32 mode: i-force and energy partials are folded into fixed point once per
// group of kFoldTiles j tiles (groups counted from the start of the list; a
// list's parts hold whole groups), so every sum is independent of the split.
constexpr int kFoldTiles = 4;
constexpr int kForceThreads = kForceWarps * kWarp;


// Adds a warp's fixed-point accumulators to one replica's accumulator block.
template <bool doEnergy, bool doVirial>
__device__ __forceinline__ void flushWarp(long long* acc, int lane, long long& accE0,
                                          long long& accE1, long long& accE2, long long& accVir,
                                          int& npair) {
  if (doVirial && lane < 18 && accVir != 0)
    atomicAddFixed(&acc[kAccVir + lane], (unsigned long long)accVir);
  if (doEnergy && lane == 0) {
    if (accE0) atomicAddFixed(&acc[kAccEVdw], (unsigned long long)accE0);
    if (accE1) atomicAddFixed(&acc[kAccEElec], (unsigned long long)accE1);
    if (accE2) atomicAddFixed(&acc[kAccESlow], (unsigned long long)accE2);
  }
  if (doEnergy) {
    int s = npair;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0 && s) atomicAddFixed(&acc[kAccNumPairs], (unsigned long long)s);
  }
  accE0 = accE1 = accE2 = accVir = 0;
  npair = 0;
}

// MINB: CTAs per SM the register budget is cut for (4, 5 or 6 -> 128, 96 or
// 80 registers; the packed loop holds two pairs' state, and 5 is the untuned
// default); a.splitLog2: each list's j tiles are shared by 2^splitLog2
// work items (warps), contiguous parts of equal tile count. Both are launch
// choices of the autotuner; results do not depend on them (fixed-point sums).
template <bool doEnergy, bool doVirial, bool doSlow, bool doE64, bool doBatch, int MINB>
__global__ void __launch_bounds__(kForceThreads, MINB)
    forceKernel(const __grid_constant__ ForceArgs a) {
  extern __shared__ float2 s_lj[];  // [ljDim*ljDim]
  __shared__ float4 s_xyzq[kForceWarps][kWarp];
  // packed loop: the j tile as five rows (x, y, z, q, type bits) of 64
  // entries; entry m holds the values of atoms m & 31 and (m & 31) ^ 16, so
  // that the two packed elements of iteration k, j = (lane + k) & 31 and
  // j ^ 16, come from one 8-byte load at the fixed offset lane + k
  __shared__ float2 s_jt[kForceWarps][5][2 * kWarp];
  __shared__ int s_type[kForceWarps][kWarp];
  // FP32 mode: each lane's i force of the current list part in fixed point,
  // folded in at the end of every j tile, so that the sums do not depend on
  // how a list's tiles are split among warps
  __shared__ long long s_fi[kForceWarps][6][kWarp];
  // FP32 mode: each lane's energies of the current list part in fixed point
  // (s_eq) and of the current tile group in FP32 (s_eg), and the warp's
  // fixed-point energy totals (s_acc, lane 0), kept in shared memory rather
  // than in registers the pair loop needs
  __shared__ long long s_eq[kForceWarps][3][kWarp];
  __shared__ float s_eg[kForceWarps][3][kWarp];
  __shared__ long long s_acc[kForceWarps][3];

  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const NbkConst& c = a.c;
  const int dim = c.ljDim;
  if (!doBatch) {
    for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) s_lj[k] = a.ljTable[k];
    __syncthreads();
  }

  const int numLists = a.numListsDev ? *a.numListsDev : a.numListsHost;

  // per-warp fixed-point accumulators: lane k < 9 owns virial[k], 9 <= k < 18
  // owns virialSlow[k-9]; lane 0 also owns the three energies.
  long long accE0 = 0, accE1 = 0, accE2 = 0, accVir = 0;
  int npair = 0;
  if (!doE64) {
#pragma unroll
    for (int q = 0; q < 6; ++q) s_fi[wib][q][lane] = 0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      s_eq[wib][q][lane] = 0;
      s_eg[wib][q][lane] = 0.f;
    }
    if (lane < 3) s_acc[wib][lane] = 0;
  }  // interacting pairs seen by this lane (energy evaluations)
  int curRep = 0;  // replica whose accumulators the warp is holding

  // lists are handed out one at a time from a global counter, so warps that
  // draw short lists keep working instead of idling at the end
  const int split = 1 << a.splitLog2;
  for (;;) {
    int W = 0;
    if (lane == 0) W = atomicAdd(a.workCounter, 1);
    W = __shfl_sync(0xffffffffu, W, 0);
    if (W >= numLists * split) break;
    const int L = W >> a.splitLog2, part = W & (split - 1);
    const nbk_tile_list tl = a.lists[L];
    if (tl.jtileEnd < tl.jtileStart) continue;  // empty (warp-uniform)
    const int chunk = ((((tl.jtileEnd - tl.jtileStart + split) >> a.splitLog2) + kFoldTiles - 1) /
                       kFoldTiles) * kFoldTiles;
    const int jtFirst = tl.jtileStart + part * chunk;
    const int jtLast = min(tl.jtileEnd, jtFirst + chunk - 1);
    if (jtLast < jtFirst) continue;  // this part has no tiles
    float3 la = a.lata, lb = a.latb, lc = a.latc;
    const float2* ljRow = nullptr;  // batched: this replica's LJ table (global)
    if (doBatch) {
      const int rep = __ldg(&a.compRep[tl.icompute]);
      if (rep != curRep) {
        if (!doE64 && lane == 0) {
          accE0 = s_acc[wib][0];
          accE1 = s_acc[wib][1];
          accE2 = s_acc[wib][2];
          s_acc[wib][0] = s_acc[wib][1] = s_acc[wib][2] = 0;
        }
        flushWarp<doEnergy, doVirial>(a.acc + (size_t)curRep * kAccCount, lane, accE0, accE1,
                                      accE2, accVir, npair);
        curRep = rep;
      }
      la = a.repLat[3 * rep];
      lb = a.repLat[3 * rep + 1];
      lc = a.repLat[3 * rep + 2];
      ljRow = a.repLJ + (size_t)rep * dim * dim;
    }
    const float3 off = make_float3(tl.offsetXYZ.x, tl.offsetXYZ.y, tl.offsetXYZ.z);
    const float3 sh = shiftOf(off, la, lb, lc);
    const bool zeroShift = !(dist2(sh.x, sh.y, sh.z) > 0.0f);

    const int iatom = tl.iatomStart + lane;
    float4 xi = a.xyzq[iatom];
    // FP64 shifted i position (FP64 energy mode): the shift is formed in FP64
    // from the FP32 offsets and lattice, without the FP32 rounding of sh
    double xid = 0.0, yid = 0.0, zid = 0.0;
    if (doE64) {
      xid = (double)xi.x + ((double)off.x * la.x + (double)off.y * lb.x + (double)off.z * lc.x);
      yid = (double)xi.y + ((double)off.x * la.y + (double)off.y * lb.y + (double)off.z * lc.y);
      zid = (double)xi.z + ((double)off.x * la.z + (double)off.y * lb.z + (double)off.z * lc.z);
    }
    xi.x = __fadd_rn(xi.x, sh.x);
    xi.y = __fadd_rn(xi.y, sh.y);
    xi.z = __fadd_rn(xi.z, sh.z);
    const int ti = a.vdwTypes[iatom] * dim;

    float fix = 0.f, fiy = 0.f, fiz = 0.f, fisx = 0.f, fisy = 0.f, fisz = 0.f;
    // packed loop: this tile's two partial i sums per component
    float2 fix2 = f2(0.f), fiy2 = f2(0.f), fiz2 = f2(0.f);
    float2 fisx2 = f2(0.f), fisy2 = f2(0.f), fisz2 = f2(0.f);
    double eV = 0.0, eE = 0.0, eS = 0.0;         // FP64 energy mode, per list
    double wv[6] = {0, 0, 0, 0, 0, 0}, ws[6] = {0, 0, 0, 0, 0, 0};  // FP64 pair virials

    for (int jt = jtFirst; jt <= jtLast; ++jt) {
      const int jstart = a.tileJatomStart[jt];
      const unsigned mask = a.tileExcls[jt].excl[lane];
      unsigned stepMask = __reduce_or_sync(0xffffffffu, mask);
      if (stepMask == 0) continue;
      const float4 xj = a.xyzq[jstart + lane];
      if constexpr (!doE64) {
        const float tyj = __int_as_float(a.vdwTypes[jstart + lane]);
        // entry m holds (atom m & 31, atom (m & 31) ^ 16): one 8-byte load
        // gives both packed elements of an iteration
        const float2 ex = make_float2(xj.x, __shfl_xor_sync(0xffffffffu, xj.x, 16));
        const float2 ey = make_float2(xj.y, __shfl_xor_sync(0xffffffffu, xj.y, 16));
        const float2 ez = make_float2(xj.z, __shfl_xor_sync(0xffffffffu, xj.z, 16));
        const float2 eq = make_float2(xj.w, __shfl_xor_sync(0xffffffffu, xj.w, 16));
        const float2 et = make_float2(tyj, __shfl_xor_sync(0xffffffffu, tyj, 16));
        s_jt[wib][0][lane] = s_jt[wib][0][lane + kWarp] = ex;
        s_jt[wib][1][lane] = s_jt[wib][1][lane + kWarp] = ey;
        s_jt[wib][2][lane] = s_jt[wib][2][lane + kWarp] = ez;
        s_jt[wib][3][lane] = s_jt[wib][3][lane + kWarp] = eq;
        s_jt[wib][4][lane] = s_jt[wib][4][lane + kWarp] = et;
      } else {
        s_xyzq[wib][lane] = xj;
      }
      s_type[wib][lane] = a.vdwTypes[jstart + lane];
      __syncwarp();

      float fjx = 0.f, fjy = 0.f, fjz = 0.f, fjsx = 0.f, fjsy = 0.f, fjsz = 0.f;
      float eVt = 0.f, eEt = 0.f, eSt = 0.f;
      if constexpr (!doE64) {
        // Iteration k takes steps k and k+16 together through
        // the packed FP32 math (element x = step k, element y = step k+16);
        // iterations whose two steps are clear in every lane are skipped.
        // i forces keep two partial sums (x, y), folded at the end of the
        // list. j forces keep two accumulator sets: P follows step k, Q step
        // k+16, so both rotate by the same amount; they are folded at the
        // end of the tile.
        float2 PQx = f2(0.f), PQy = f2(0.f), PQz = f2(0.f);     // (P, Q) fast
        float2 PQsx = f2(0.f), PQsy = f2(0.f), PQsz = f2(0.f);  // (P, Q) slow
        float2 eV2 = f2(0.f), eE2 = f2(0.f), eS2 = f2(0.f);
        const float2 nXi = f2(-xi.x), nYi = f2(-xi.y), nZi = f2(-xi.z);
        int kLast = 0;
        unsigned mk = mask;  // bit k of the mask moved to bit 0 (and k+16 to 16)
#pragma unroll 2
        for (int k = 0; k < 16; ++k, mk >>= 1) {
          if (!((stepMask >> k) & 0x10001u)) continue;  // warp-uniform
          // element x: j = (lane + k) & 31, element y: j ^ 16
          const float2* pA = &s_jt[wib][0][lane + k];
          const float2 X = pA[0];
          const float2 Y = pA[64];
          const float2 Z = pA[128];
          const float2 DX = add2(X, nXi), DY = add2(Y, nYi), DZ = add2(Z, nZi);
          const float2 R2 = fma2(DZ, DZ, fma2(DY, DY, mul2(DX, DX)));
          const bool aA = (mk & 1u) && (R2.x < c.cutoff2);
          const bool aB = (mk & 0x10000u) && (R2.y < c.cutoff2);
          if (!__any_sync(0xffffffffu, aA || aB)) continue;
          if (doEnergy) npair += (int)aA + (int)aB;
          const float2 TY = pA[256];
          const int tyA = __float_as_int(TY.x), tyB = __float_as_int(TY.y);
          const float2 abA = doBatch ? __ldg(&ljRow[ti + tyA]) : s_lj[ti + tyA];
          const float2 abB = doBatch ? __ldg(&ljRow[ti + tyB]) : s_lj[ti + tyB];
          const float2 QQ = mul2(f2(xi.w), pA[192]);
          const float2 r2s = make_float2(aA ? R2.x : c.cutoff2, aB ? R2.y : c.cutoff2);
          const float2 qqs = make_float2(aA ? QQ.x : 0.f, aB ? QQ.y : 0.f);
          const float2 As = make_float2(aA ? abA.x : 0.f, aB ? abB.x : 0.f);
          const float2 nBs = make_float2(aA ? -abA.y : 0.f, aB ? -abB.y : 0.f);
          float2 F, FS;
          pairForce2<doEnergy, doSlow>(r2s, qqs, As, nBs, c, F, FS, eV2, eE2, eS2);
          // i: two partial sums; inactive elements add exact zeros
          fix2 = fma2(DX, F, fix2);
          fiy2 = fma2(DY, F, fiy2);
          fiz2 = fma2(DZ, F, fiz2);
          if (doSlow) {
            fisx2 = fma2(DX, FS, fisx2);
            fisy2 = fma2(DY, FS, fisy2);
            fisz2 = fma2(DZ, FS, fisz2);
          }
          // j: bring P to step k and Q to step k+16 (one shift for both), subtract
          const int src = (lane + (k - kLast)) & 31;
          kLast = k;
          PQx = make_float2(__shfl_sync(0xffffffffu, PQx.x, src), __shfl_sync(0xffffffffu, PQx.y, src));
          PQy = make_float2(__shfl_sync(0xffffffffu, PQy.x, src), __shfl_sync(0xffffffffu, PQy.y, src));
          PQz = make_float2(__shfl_sync(0xffffffffu, PQz.x, src), __shfl_sync(0xffffffffu, PQz.y, src));
          PQx = fma2(neg2(DX), F, PQx);
          PQy = fma2(neg2(DY), F, PQy);
          PQz = fma2(neg2(DZ), F, PQz);
          if (doSlow) {
            PQsx = make_float2(__shfl_sync(0xffffffffu, PQsx.x, src),
                               __shfl_sync(0xffffffffu, PQsx.y, src));
            PQsy = make_float2(__shfl_sync(0xffffffffu, PQsy.x, src),
                               __shfl_sync(0xffffffffu, PQsy.y, src));
            PQsz = make_float2(__shfl_sync(0xffffffffu, PQsz.x, src),
                               __shfl_sync(0xffffffffu, PQsz.y, src));
            PQsx = fma2(neg2(DX), FS, PQsx);
            PQsy = fma2(neg2(DY), FS, PQsy);
            PQsz = fma2(neg2(DZ), FS, PQsz);
          }
        }
        // rotate P (at step kLast) and Q (at step kLast+16) back to j = lane
        {
          const int srcP = (lane + 32 - kLast) & 31, srcQ = (lane + 16 - kLast) & 31;
          fjx = __shfl_sync(0xffffffffu, PQx.x, srcP) + __shfl_sync(0xffffffffu, PQx.y, srcQ);
          fjy = __shfl_sync(0xffffffffu, PQy.x, srcP) + __shfl_sync(0xffffffffu, PQy.y, srcQ);
          fjz = __shfl_sync(0xffffffffu, PQz.x, srcP) + __shfl_sync(0xffffffffu, PQz.y, srcQ);
          if (doSlow) {
            fjsx = __shfl_sync(0xffffffffu, PQsx.x, srcP) + __shfl_sync(0xffffffffu, PQsx.y, srcQ);
            fjsy = __shfl_sync(0xffffffffu, PQsy.x, srcP) + __shfl_sync(0xffffffffu, PQsy.y, srcQ);
            fjsz = __shfl_sync(0xffffffffu, PQsz.x, srcP) + __shfl_sync(0xffffffffu, PQsz.y, srcQ);
          }
        }
        eVt = eV2.x + eV2.y;
        eEt = eE2.x + eE2.y;
        eSt = eS2.x + eS2.y;
      } else {
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
          if (((mask >> t) & 1u) && (r2 < c.cutoff2)) {
            if (doEnergy) ++npair;
            const float2 ab = doBatch ? __ldg(&ljRow[ti + s_type[wib][j]]) : s_lj[ti + s_type[wib][j]];
            float f, fs;
            pairForce<doEnergy, doSlow>(r2, xi.w * xjj.w, ab, c, f, fs, eVt, eEt, eSt);
            if (doE64) {
              // electrostatic energies and the pair virials again in FP64 from
              // FP64 geometry; the FP32 eEt/eSt are discarded in this mode
              const double ex = (double)xjj.x - xid, ey = (double)xjj.y - yid,
                           ez = (double)xjj.z - zid;
              const double r2d = fma(ez, ez, fma(ey, ey, ex * ex));
              double g, gs;
              pairFP64<doSlow>(r2d, (double)xi.w * (double)xjj.w, (double)ab.x, (double)ab.y,
                               a.c64, g, gs, eE, eS);
              if (doVirial) {
                const double d[3] = {ex, ey, ez};
  #pragma unroll
                for (int u = 0, q = 0; u < 3; ++u)
  #pragma unroll
                  for (int v = u; v < 3; ++v, ++q) {
                    const double dd = d[u] * d[v];
                    wv[q] = fma(-g, dd, wv[q]);
                    if (doSlow) ws[q] = fma(-gs, dd, ws[q]);
                  }
              }
            }
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
        if (doE64) {
          eV += (double)eVt;
        } else {
          s_eg[wib][0][lane] += eVt;
          s_eg[wib][1][lane] += eEt;
          if (doSlow) s_eg[wib][2][lane] += eSt;
        }
      }
      if (!doE64 && ((((jt - tl.jtileStart + 1) & (kFoldTiles - 1)) == 0) || jt == jtLast)) {
        // end of a tile group: its energies and i forces into fixed point
        if (doEnergy) {
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            if (q == 2 && !doSlow) break;
            s_eq[wib][q][lane] += toFixedEnergyF(s_eg[wib][q][lane]);
            s_eg[wib][q][lane] = 0.f;
          }
        }
        s_fi[wib][0][lane] += (long long)toFixedForce(fix2.x + fix2.y);
        s_fi[wib][1][lane] += (long long)toFixedForce(fiy2.x + fiy2.y);
        s_fi[wib][2][lane] += (long long)toFixedForce(fiz2.x + fiz2.y);
        fix2 = fiy2 = fiz2 = f2(0.f);
        if (doSlow) {
          s_fi[wib][3][lane] += (long long)toFixedForce(fisx2.x + fisx2.y);
          s_fi[wib][4][lane] += (long long)toFixedForce(fisy2.x + fisy2.y);
          s_fi[wib][5][lane] += (long long)toFixedForce(fisz2.x + fisz2.y);
          fisx2 = fisy2 = fisz2 = f2(0.f);
        }
      }
      __syncwarp();
    }  // jt

    // i forces (fixed point)
    unsigned long long qx, qy, qz, sx = 0, sy = 0, sz = 0;
    if (!doE64) {
      qx = (unsigned long long)s_fi[wib][0][lane];
      qy = (unsigned long long)s_fi[wib][1][lane];
      qz = (unsigned long long)s_fi[wib][2][lane];
      s_fi[wib][0][lane] = s_fi[wib][1][lane] = s_fi[wib][2][lane] = 0;
      if (doSlow) {
        sx = (unsigned long long)s_fi[wib][3][lane];
        sy = (unsigned long long)s_fi[wib][4][lane];
        sz = (unsigned long long)s_fi[wib][5][lane];
        s_fi[wib][3][lane] = s_fi[wib][4][lane] = s_fi[wib][5][lane] = 0;
      }
    } else {
      qx = toFixedForce(fix);
      qy = toFixedForce(fiy);
      qz = toFixedForce(fiz);
      if (doSlow) {
        sx = toFixedForce(fisx);
        sy = toFixedForce(fisy);
        sz = toFixedForce(fisz);
      }
    }
    if (qx | qy | qz) {
      atomicAddFixed(&a.force[0 * (size_t)a.stride + iatom], qx);
      atomicAddFixed(&a.force[1 * (size_t)a.stride + iatom], qy);
      atomicAddFixed(&a.force[2 * (size_t)a.stride + iatom], qz);
    }
    if (doSlow && (sx | sy | sz)) {
      atomicAddFixed(&a.force[3 * (size_t)a.stride + iatom], sx);
      atomicAddFixed(&a.force[4 * (size_t)a.stride + iatom], sy);
      atomicAddFixed(&a.force[5 * (size_t)a.stride + iatom], sz);
    }
    if (doVirial && doE64) {
      // FP64 mode: the complete pair virial of this list, W = -sum g d (x) d
      double tv[6], ts[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        tv[q] = warpSumD(wv[q]);
        ts[q] = doSlow ? warpSumD(ws[q]) : 0.0;
      }
      if (lane < 18) {
        const int q = symIndex(lane % 9);
        double v = tv[0];
#pragma unroll
        for (int k = 1; k < 6; ++k)
          if (k == q) v = (lane < 9) ? tv[k] : ts[k];
        if (q == 0) v = (lane < 9) ? tv[0] : ts[0];
        if (lane < 9 || doSlow) accVir += toFixedEnergy(v);
      }
    } else if (doVirial && !zeroShift) {
      // the lattice-shift part of the virial, (sum_i F_i) (x) shift, is formed
      // per compute by shiftVirialKernel from these exact integer sums
      const long long Fx = warpSumLL((long long)qx), Fy = warpSumLL((long long)qy),
                      Fz = warpSumLL((long long)qz);
      long long Gx = 0, Gy = 0, Gz = 0;
      if (doSlow) {
        Gx = warpSumLL((long long)sx);
        Gy = warpSumLL((long long)sy);
        Gz = warpSumLL((long long)sz);
      }
      long long* cf = a.compF + 6 * (size_t)tl.icompute;
      if (lane == 0) {
        if (Fx) atomicAddFixed(&cf[0], (unsigned long long)Fx);
        if (Fy) atomicAddFixed(&cf[1], (unsigned long long)Fy);
        if (Fz) atomicAddFixed(&cf[2], (unsigned long long)Fz);
        if (doSlow) {
          if (Gx) atomicAddFixed(&cf[3], (unsigned long long)Gx);
          if (Gy) atomicAddFixed(&cf[4], (unsigned long long)Gy);
          if (Gz) atomicAddFixed(&cf[5], (unsigned long long)Gz);
        }
      }
    }
    if (doEnergy) {
      long long sV, sE, sS = 0;
      if (doE64) {
        sV = toFixedEnergy(warpSumD(eV));
        sE = toFixedEnergy(warpSumD(eE));
        if (doSlow) sS = toFixedEnergy(warpSumD(eS));
      } else {
        sV = warpSumLL(s_eq[wib][0][lane]);
        sE = warpSumLL(s_eq[wib][1][lane]);
        if (doSlow) sS = warpSumLL(s_eq[wib][2][lane]);
        s_eq[wib][0][lane] = s_eq[wib][1][lane] = s_eq[wib][2][lane] = 0;
      }
      if (lane == 0) {
        if (doE64) {
          accE0 += sV;
          accE1 += sE;
          accE2 += sS;
        } else {
          s_acc[wib][0] += sV;
          s_acc[wib][1] += sE;
          s_acc[wib][2] += sS;
        }
      }
    }
  }  // lists

  // per-warp flush of the fixed-point accumulators (no block barrier, so a
  // warp that runs out of lists retires at once)
  if (!doE64 && lane == 0) {
    accE0 = s_acc[wib][0];
    accE1 = s_acc[wib][1];
    accE2 = s_acc[wib][2];
  }
  flushWarp<doEnergy, doVirial>(a.acc + (size_t)curRep * kAccCount, lane, accE0, accE1, accE2,
                                accVir, npair);
}

template <bool E, bool V, bool S, bool D, bool B, int MINB>
static cudaError_t launchT(const ForceArgs& a, int numSM, cudaStream_t st) {
  const size_t shmem = B ? 0 : sizeof(float2) * (size_t)a.c.ljDim * a.c.ljDim;
  auto k = forceKernel<E, V, S, D, B, MINB>;
  static int cachedDim = -1, cachedBlocks = 0;
  if (cachedDim != a.c.ljDim) {
    if (shmem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
      if (e != cudaSuccess) return e;
    }
    int nb = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kForceThreads, shmem);
    if (e != cudaSuccess) return e;
    cachedBlocks = nb > 0 ? nb : 1;
    cachedDim = a.c.ljDim;
  }
  k<<<numSM * cachedBlocks, kForceThreads, shmem, st>>>(a);
  return cudaGetLastError();
}

template <bool E, bool V, bool S, bool D, bool B>
static cudaError_t launchShape(const ForceArgs& a, int minBlocks, int numSM, cudaStream_t st) {
  switch (minBlocks) {
    case 4: return launchT<E, V, S, D, B, 4>(a, numSM, st);
    case 5: return launchT<E, V, S, D, B, 5>(a, numSM, st);
    case 6: return launchT<E, V, S, D, B, 6>(a, numSM, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launchForce(const ForceArgs& a, unsigned flags, int minBlocks, int numSM,
                        cudaStream_t st) {
  const bool E = flags & NBK_ENERGY;
  const bool B = a.compRep != nullptr;
  const int idx = (B ? 16 : 0) | (E ? 8 : 0) | ((flags & NBK_VIRIAL) ? 4 : 0) |
                  ((flags & NBK_SLOW) ? 2 : 0) | ((E && (flags & NBK_ENERGY_FP64)) ? 1 : 0);
  switch (idx) {
#define NBK_CASE(i, e, v, s, d, b) \
  case i:                          \
    return launchShape<e, v, s, d, b>(a, minBlocks, numSM, st);
    NBK_CASE(0, false, false, false, false, false)
    NBK_CASE(2, false, false, true, false, false)
    NBK_CASE(4, false, true, false, false, false)
    NBK_CASE(6, false, true, true, false, false)
    NBK_CASE(8, true, false, false, false, false)
    NBK_CASE(9, true, false, false, true, false)
    NBK_CASE(10, true, false, true, false, false)
    NBK_CASE(11, true, false, true, true, false)
    NBK_CASE(12, true, true, false, false, false)
    NBK_CASE(13, true, true, false, true, false)
    NBK_CASE(14, true, true, true, false, false)
    NBK_CASE(15, true, true, true, true, false)
    // batched replicas (FP32 energy mode)
    NBK_CASE(16, false, false, false, false, true)
    NBK_CASE(18, false, false, true, false, true)
    NBK_CASE(20, false, true, false, false, true)
    NBK_CASE(22, false, true, true, false, true)
    NBK_CASE(24, true, false, false, false, true)
    NBK_CASE(26, true, false, true, false, true)
    NBK_CASE(28, true, true, false, false, true)
    NBK_CASE(30, true, true, true, false, true)
#undef NBK_CASE
  }
  return cudaErrorInvalidValue;
}

}  // namespace nbk
