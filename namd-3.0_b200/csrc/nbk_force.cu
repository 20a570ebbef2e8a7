// Nonbonded force kernel of the B200 path.
//
// One warp owns one tile list (32 i atoms of one patch against the j tiles of
// a compute's partner patch), as CudaComputeNonbondedKernel's
// nonbondedForceKernel does (src/CudaComputeNonbondedKernel.cu:629-1644), but:
//   - two pair steps per iteration run through sm_100's packed FP32
//     instructions; j forces ride in registers and rotate with a shuffle, so
//     the inner loop touches shared memory only for the j-tile loads;
//   - steps whose bit is clear in every lane's mask are skipped warp-uniformly;
//   - the lists it reads are already refined (TileExcl masks from
//     refineKernel); a pairlist step refines, compacts, then runs this kernel;
//   - per-tile FP32 partial forces are folded into 64-bit fixed point with
//     integer atomics, so the summed forces do not depend on the order in
//     which lists run;
//   - on energy and virial evaluations the electrostatic energies and the
//     slow virial are formed in FP64 by a precise pass over the tile's
//     interacting pairs, compacted into a queue (see precisePass), and folded
//     into fixed point per tile; the LJ energy is summed in FP32 per group of
//     tiles and the fast virial comes from the fixed-point forces.
#include "nbk_internal.cuh"
#include "nbk_launch.h"

#include <mutex>

namespace nbk {

constexpr int kForceWarps = 4;
// Forces and the LJ energy are folded into fixed point once per group of
// kFoldTiles j tiles (groups counted from the start of the list; a list's
// parts hold whole groups), so every sum is independent of the split.
constexpr int kFoldTiles = 4;
constexpr int kForceThreads = kForceWarps * kWarp;

// FP64 quantities of the precise pass; after a tile's pass lane q < kNumQ
// holds quantity q: the fast and slow electrostatic energies, then the six
// independent components of the slow virial (xx, xy, xz, yy, yz, zz).
constexpr int kQElec = 0, kQSlow = 1, kQVir = 2, kNumQ = 8;

// An atom in FP64 (position, scaled charge); 32 bytes, two 16-byte loads.
struct alignas(16) Atom64 {
  double x, y, z, q;
};

// virialSlow[3a+b] slots of symmetric component m (xx, xy, xz, yy, yz, zz);
// s1 < 0 for the diagonal.
__device__ __forceinline__ void symSlots(int m, int& s0, int& s1) {
  s0 = m == 0 ? 0 : m == 1 ? 1 : m == 2 ? 2 : m == 3 ? 4 : m == 4 ? 5 : 8;
  s1 = m == 1 ? 3 : m == 2 ? 6 : m == 4 ? 7 : -1;
}

// Adds a warp's fixed-point accumulators to one replica's accumulator block:
// lane 0 the LJ energy (accVdw) and, with the other lanes, the pair count;
// lane q < kNumQ its precise-pass quantity (accQ).
template <bool doEnergy>
__device__ __forceinline__ void flushWarp(long long* acc, int lane, long long& accVdw,
                                          long long& accQ, int& npair) {
  if (lane < kNumQ && accQ != 0) {
    if (lane == kQElec) {
      atomicAddFixed(&acc[kAccEElec], (unsigned long long)accQ);
    } else if (lane == kQSlow) {
      atomicAddFixed(&acc[kAccESlow], (unsigned long long)accQ);
    } else {
      int s0, s1;
      symSlots(lane - kQVir, s0, s1);
      atomicAddFixed(&acc[kAccVirSlow + s0], (unsigned long long)accQ);
      if (s1 >= 0) atomicAddFixed(&acc[kAccVirSlow + s1], (unsigned long long)accQ);
    }
  }
  if (doEnergy) {
    if (lane == 0 && accVdw != 0) atomicAddFixed(&acc[kAccEVdw], (unsigned long long)accVdw);
    int s = npair;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0 && s) atomicAddFixed(&acc[kAccNumPairs], (unsigned long long)s);
  }
  accVdw = accQ = 0;
  npair = 0;
}

// FP64 geometry of one queued pair: d = x_j - x_i and the charge product.
struct PairTerms {
  double dx, dy, dz, qq;
};

// One lane's precise-pass sums over the current tile group.
struct LaneSums {
  double eE, eS, w0, w1, w2, w3, w4, w5;
};

// The slow-term table as the precise pass reads it: in shared memory,
// coefficient n of row k at sh[n * rows + k] (a warp's lanes read one
// coefficient of up to 32 rows per load, few bank conflicts), or else the
// global row-major copy (8 doubles per row).
struct SlowTable {
  const double* sh;
  const double2* gl;
  int rows;
  unsigned last;
  double step, invStep;
};

// The FP64 terms of one interacting pair (qq = 0 contributes exact zeros):
// the fast energy qq (1/r - h(s)) with 1/r from the FP32 approximation
// refined by one Newton step, and from the slow-term table the slow energy
// qq phi_s(s) and the slow virial -2 qq phi_s'(s) d (x) d.
template <bool doEnergy, bool doVirial, bool doSlow>
__device__ __forceinline__ void precisePair(const PairTerms& u, const SlowTable& T,
                                            const NbkConst& c, LaneSums& L) {
  const double s = fma(u.dz, u.dz, fma(u.dy, u.dy, u.dx * u.dx));
  double p = 0.0, dp = 0.0;
  if (doSlow) {
    // row k = nearest integer to s/D: adding 1.5 * 2^52 rounds s/D (exact, D
    // a power of two) into the low word; the sum is clamped to the last row
    // in FP64, so k and w = s - k D come without an integer conversion
    const double magic = 6755399441055744.0;
    const double t = fmin(fma(s, T.invStep, magic), magic + (double)T.last);
    const unsigned k = (unsigned)__double2loint(t);
    const double wq = fma(-T.step, t - magic, s);
    double c0, c1, c2, c3, c4, c5, c6;
    if (T.sh) {
      const double* col = T.sh + k;
      c0 = col[0];
      c1 = col[T.rows];
      c2 = col[2 * T.rows];
      c3 = col[3 * T.rows];
      c4 = col[4 * T.rows];
      c5 = col[5 * T.rows];
      c6 = col[6 * T.rows];
    } else {
      const double2* row = T.gl + (size_t)k * (kSlowTableRow / 2);
      const double2 c01 = __ldg(row), c23 = __ldg(row + 1), c45 = __ldg(row + 2),
                    c67 = __ldg(row + 3);
      c0 = c01.x, c1 = c01.y, c2 = c23.x, c3 = c23.y, c4 = c45.x, c5 = c45.y, c6 = c67.x;
    }
    // Horner for p(w) and p'(w) together
    p = c6;
    dp = p;
    p = fma(p, wq, c5);
    dp = fma(dp, wq, p);
    p = fma(p, wq, c4);
    dp = fma(dp, wq, p);
    p = fma(p, wq, c3);
    dp = fma(dp, wq, p);
    p = fma(p, wq, c2);
    dp = fma(dp, wq, p);
    p = fma(p, wq, c1);
    dp = fma(dp, wq, p);
    p = fma(p, wq, c0);
  }
  if (doEnergy) {
    // y0 has relative error below 2^-22; after the step, below 2^-43
    const double y0 = (double)rsqrtApprox((float)s);
    const double hs = 0.5 * s;
    const double y = fma(y0, fma(-hs * y0, y0, 0.5), y0);
    L.eE = fma(u.qq, y - fma(c.hBd, s, c.hAd), L.eE);
    if (doSlow) L.eS = fma(u.qq, p, L.eS);
  }
  if (doVirial && doSlow) {
    const double g = (u.qq + u.qq) * dp;  // (dE/dr)/r
    const double gx = -g * u.dx, gy = -g * u.dy, gz = -g * u.dz;
    L.w0 = fma(gx, u.dx, L.w0);
    L.w1 = fma(gx, u.dy, L.w1);
    L.w2 = fma(gx, u.dz, L.w2);
    L.w3 = fma(gy, u.dy, L.w3);
    L.w4 = fma(gy, u.dz, L.w4);
    L.w5 = fma(gz, u.dz, L.w5);
  }
}

// The precise pass of one tile. live (per lane): bit t set when the pair
// (i = lane, j = (lane + t) & 31) is an interacting pair (mask bit set and
// FP32 r^2 below the cutoff, the classification the FP32 math used). The
// warp compacts the tile's interacting pairs into a queue in shared memory
// (entry = i | t << 5, lane-major order; at most 32 * 32 two-byte entries,
// the 2 KB of pq) and processes them in FP64, two per lane per iteration
// (entries e and e + 32: independent dependency chains; an entry past the
// end gets d = (1, 0, 0) and qq = 0, which contributes exact zeros -- its
// atoms may be one and the same atom, so their own distance, 0, would turn
// the zero into a NaN), adding to the lane's group sums L. Every step is
// warp-synchronous and the sums depend only on the tile group.
template <bool doEnergy, bool doVirial, bool doSlow>
__device__ __forceinline__ void precisePass(const unsigned live, const int lane,
                                            const Atom64* __restrict__ ai,
                                            const Atom64* __restrict__ aj, double* pq,
                                            const SlowTable& T, const NbkConst& c, LaneSums& L,
                                            int& npair) {
  const int n = __popc(live);
  if (doEnergy) npair += n;
  int incl = n;
#pragma unroll
  for (int o = 1; o < kWarp; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int total = __shfl_sync(0xffffffffu, incl, kWarp - 1);
  if (total == 0) return;  // warp-uniform
  unsigned short* q = reinterpret_cast<unsigned short*>(pq);
  int pos = incl - n;
  for (unsigned w = live; w; w &= w - 1) q[pos++] = (unsigned short)(lane | ((__ffs(w) - 1) << 5));
  __syncwarp();
  for (int base = 0; base < total; base += 2 * kWarp) {  // warp-uniform
    PairTerms u[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int e = base + h * kWarp + lane;
      if (e < total) {
        const unsigned ent = q[e];
        const int i = ent & 31, j = (i + (ent >> 5)) & 31;
        const Atom64 A = ai[i], B = aj[j];
        u[h].dx = B.x - A.x;
        u[h].dy = B.y - A.y;
        u[h].dz = B.z - A.z;
        u[h].qq = A.q * B.q;
      } else {
        u[h].dx = 1.0;
        u[h].dy = u[h].dz = u[h].qq = 0.0;
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) precisePair<doEnergy, doVirial, doSlow>(u[h], T, c, L);
  }
  __syncwarp();  // the queue is consumed before pq is written again
}

// End of a tile group: each lane's sums are written to shared memory (pq,
// [kNumQ][32]) and reduced per quantity in a fixed order (lane L sums
// quantity L & 7 over lanes 8 (L >> 3) .. 8 (L >> 3) + 7, then two butterfly
// steps combine the four groups), and lane q < kNumQ adds quantity q, in
// fixed point, to accQ; the sums restart at zero.
__device__ __forceinline__ void reduceGroup(const int lane, double* pq, LaneSums& L,
                                            long long& accQ) {
  pq[kQElec * kWarp + lane] = L.eE;
  pq[kQSlow * kWarp + lane] = L.eS;
  pq[(kQVir + 0) * kWarp + lane] = L.w0;
  pq[(kQVir + 1) * kWarp + lane] = L.w1;
  pq[(kQVir + 2) * kWarp + lane] = L.w2;
  pq[(kQVir + 3) * kWarp + lane] = L.w3;
  pq[(kQVir + 4) * kWarp + lane] = L.w4;
  pq[(kQVir + 5) * kWarp + lane] = L.w5;
  __syncwarp();
  const double* src = pq + (lane & 7) * kWarp + (lane >> 3) * 8;
  double v = src[0];
#pragma unroll
  for (int m = 1; m < 8; ++m) v += src[m];
  v += __shfl_xor_sync(0xffffffffu, v, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 16);
  if (lane < kNumQ) accQ += toFixedEnergy(v);
  L = LaneSums{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  __syncwarp();  // pq is free for the next tile's queue
}

// MINB: CTAs per SM the register budget is cut for (4, 5 or 6 -> 128, 96 or
// 80 registers; the packed loop holds two pairs' state, and 5 is the untuned
// default); a.splitLog2: each list's j tiles are shared by 2^splitLog2
// work items (warps), contiguous parts of equal tile count. Both are launch
// choices of the autotuner; results do not depend on them (fixed-point sums
// per tile group, precise-pass sums per tile).
template <bool doEnergy, bool doVirial, bool doSlow, bool doBatch, int MINB>
__global__ void __launch_bounds__(kForceThreads, MINB)
    forceKernel(const __grid_constant__ ForceArgs a) {
  // the precise pass runs on energy evaluations and on virial evaluations
  // with slow forces (it forms the slow virial)
  constexpr bool kPrecise = doEnergy || (doVirial && doSlow);
  constexpr int kPW = kPrecise ? kForceWarps : 1;
  // dynamic: the LJ table [ljDim*ljDim] (single system), then, when it fits,
  // the slow-term table in its transposed layout [7][rows] (precise pass)
  extern __shared__ float2 s_lj[];
  // the j tile as five rows (x, y, z, q, type bits) of 64 entries; entry m
  // holds the values of atoms m & 31 and (m & 31) ^ 16, so that the two
  // packed elements of iteration k, j = (lane + k) & 31 and j ^ 16, come from
  // one 8-byte load at the fixed offset lane + k
  __shared__ float2 s_jt[kForceWarps][5][2 * kWarp];
  // each lane's i force of the current list part in fixed point, folded in
  // at the end of every tile group, so that the sums do not depend on how a
  // list's tiles are split among warps
  __shared__ long long s_fi[kForceWarps][6][kWarp];
  // each lane's LJ energy of the list part in fixed point (s_ev) and of the
  // current tile group in FP32 (s_evg), and the warp's fixed-point LJ total
  // (s_evw, lane 0), kept in shared memory rather than in registers the pair
  // loop needs
  __shared__ long long s_ev[kForceWarps][kWarp];
  __shared__ float s_evg[kForceWarps][kWarp];
  __shared__ long long s_evw[kForceWarps];
  // precise pass: FP64 shifted i atoms of the list, FP64 j atoms of the tile,
  // and the pair queue / lane partials (2 KB per warp)
  __shared__ Atom64 s_ai[kPW][kWarp];
  __shared__ Atom64 s_aj[kPW][kWarp];
  __shared__ double s_pq[kPW][kNumQ * kWarp];

  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const NbkConst& c = a.c;
  const int dim = c.ljDim;
  const int ljWords = doBatch ? 0 : dim * dim;
  SlowTable T;
  T.rows = a.slowTableRows;
  T.last = (unsigned)(a.slowTableRows - 1);
  T.step = a.slowStep;
  T.invStep = a.slowInvStep;
  T.gl = a.slowTable;
  T.sh = nullptr;
  if (!doBatch)
    for (int k = threadIdx.x; k < ljWords; k += blockDim.x) s_lj[k] = a.ljTable[k];
  if (kPrecise && doSlow && a.slowTableShared) {
    double* st = reinterpret_cast<double*>(s_lj + ljWords);
    const double* g = reinterpret_cast<const double*>(a.slowTable);
    for (int k = threadIdx.x; k < kSlowTableDeg1 * T.rows; k += blockDim.x) {
      const int n = k / T.rows, r = k - n * T.rows;
      st[k] = g[(size_t)r * kSlowTableRow + n];
    }
    T.sh = st;
  }
  if (!doBatch || (kPrecise && doSlow && a.slowTableShared)) __syncthreads();

  const int numLists = a.numListsDev ? *a.numListsDev : a.numListsHost;

  long long accVdw = 0;  // lane 0: LJ energy to flush (batched replica change)
  long long accQ = 0;    // lane q < kNumQ: precise-pass quantity q
  LaneSums lsum{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // this lane's precise-pass group sums
  int npair = 0;         // interacting pairs counted by this lane (energy evaluations)
#pragma unroll
  for (int q = 0; q < 6; ++q) s_fi[wib][q][lane] = 0;
  s_ev[wib][lane] = 0;
  s_evg[wib][lane] = 0.f;
  if (lane == 0) s_evw[wib] = 0;
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
        if (lane == 0) {
          accVdw = s_evw[wib];
          s_evw[wib] = 0;
        }
        flushWarp<doEnergy>(a.acc + (size_t)curRep * kAccCount, lane, accVdw, accQ, npair);
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
    if (kPrecise) {
      // FP64 shifted i atom: the shift formed in FP64 from the FP32 offsets
      // and lattice (the exact lattice translation), without the FP32
      // rounding of sh
      const double sx = (double)off.x * la.x + (double)off.y * lb.x + (double)off.z * lc.x;
      const double sy = (double)off.x * la.y + (double)off.y * lb.y + (double)off.z * lc.y;
      const double sz = (double)off.x * la.z + (double)off.y * lb.z + (double)off.z * lc.z;
      Atom64 ai;
      ai.x = (double)xi.x + sx;
      ai.y = (double)xi.y + sy;
      ai.z = (double)xi.z + sz;
      ai.q = (double)xi.w;
      s_ai[wib][lane] = ai;
    }
    xi.x = __fadd_rn(xi.x, sh.x);
    xi.y = __fadd_rn(xi.y, sh.y);
    xi.z = __fadd_rn(xi.z, sh.z);
    const int ti = a.vdwTypes[iatom] * dim;

    // this tile group's two partial i sums per component
    float2 fix2 = f2(0.f), fiy2 = f2(0.f), fiz2 = f2(0.f);
    float2 fisx2 = f2(0.f), fisy2 = f2(0.f), fisz2 = f2(0.f);

    for (int jt = jtFirst; jt <= jtLast; ++jt) {
      const int jstart = a.tileJatomStart[jt];
      const unsigned mask = a.tileExcls[jt].excl[lane];
      const unsigned stepMask = __reduce_or_sync(0xffffffffu, mask);
      if (stepMask != 0) {
        const float4 xj = a.xyzq[jstart + lane];
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
        if (kPrecise) {
          Atom64 aj;
          aj.x = (double)xj.x;
          aj.y = (double)xj.y;
          aj.z = (double)xj.z;
          aj.q = (double)xj.w;
          s_aj[wib][lane] = aj;
        }
        __syncwarp();

        // Iteration k takes steps k and k+16 together through the packed
        // FP32 math (element x = step k, element y = step k+16); iterations
        // whose two steps are clear in every lane are skipped. j forces keep
        // two accumulator sets: P follows step k, Q step k+16, so both rotate
        // by the same amount; they are folded at the end of the tile.
        float2 PQx = f2(0.f), PQy = f2(0.f), PQz = f2(0.f);     // (P, Q) fast
        float2 PQsx = f2(0.f), PQsy = f2(0.f), PQsz = f2(0.f);  // (P, Q) slow
        float2 eV2 = f2(0.f);
        const float2 nXi = f2(-xi.x), nYi = f2(-xi.y), nZi = f2(-xi.z);
        int kLast = 0;
        unsigned live = 0;   // precise pass: interacting pairs, TileExcl bit order
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
          if (kPrecise) live |= ((aA ? 1u : 0u) | (aB ? 0x10000u : 0u)) << k;
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
          pairForce2<doEnergy, doSlow>(r2s, qqs, As, nBs, c, F, FS, eV2);
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
        float fjx, fjy, fjz, fjsx = 0.f, fjsy = 0.f, fjsz = 0.f;
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
        if (doEnergy) s_evg[wib][lane] += eV2.x + eV2.y;
        if (kPrecise)
          precisePass<doEnergy, doVirial, doSlow>(live, lane, s_ai[wib], s_aj[wib], s_pq[wib], T,
                                                  c, lsum, npair);
      }
      if (((((jt - tl.jtileStart + 1) & (kFoldTiles - 1)) == 0) || jt == jtLast)) {
        // end of a tile group: its LJ energy, i forces and precise-pass sums
        // into fixed point
        if (kPrecise) reduceGroup(lane, s_pq[wib], lsum, accQ);
        if (doEnergy) {
          s_ev[wib][lane] += toFixedEnergyF(s_evg[wib][lane]);
          s_evg[wib][lane] = 0.f;
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
    if (doVirial && !zeroShift) {
      // the lattice-shift part of the fast virial, (sum_i F_i) (x) shift, is
      // formed per compute by the finalize kernel from these exact integer sums
      const long long Fx = warpSumLL((long long)qx), Fy = warpSumLL((long long)qy),
                      Fz = warpSumLL((long long)qz);
      long long* cf = a.compF + 6 * (size_t)tl.icompute;
      if (lane == 0) {
        if (Fx) atomicAddFixed(&cf[0], (unsigned long long)Fx);
        if (Fy) atomicAddFixed(&cf[1], (unsigned long long)Fy);
        if (Fz) atomicAddFixed(&cf[2], (unsigned long long)Fz);
      }
    }
    if (doEnergy) {
      const long long sV = warpSumLL(s_ev[wib][lane]);
      s_ev[wib][lane] = 0;
      if (lane == 0) s_evw[wib] += sV;
    }
  }  // lists

  // per-warp flush of the fixed-point accumulators (no block barrier, so a
  // warp that runs out of lists retires at once)
  if (lane == 0) accVdw = s_evw[wib];
  flushWarp<doEnergy>(a.acc + (size_t)curRep * kAccCount, lane, accVdw, accQ, npair);
}

// Blocks per SM of one kernel instance on one device for one dynamic
// shared-memory size, with the opt-in set on that device; looked up once per
// (device, size) and kept per instance, under a lock, so handles on different
// devices or threads neither share a stale entry nor race.
constexpr int kMaxDevicesCached = 64;
struct OccCache {
  std::mutex mu;
  size_t shmem[kMaxDevicesCached];
  int blocks[kMaxDevicesCached];
  OccCache() {
    for (int d = 0; d < kMaxDevicesCached; ++d) shmem[d] = (size_t)-1, blocks[d] = 0;
  }
};

// Dynamic shared memory of a force-kernel launch: the LJ table (single
// system) and the transposed slow-term table when the precise pass reads it
// from shared memory.
size_t forceShmem(const ForceArgs& a, bool E, bool V, bool S, bool B) {
  size_t bytes = B ? 0 : sizeof(float2) * (size_t)a.c.ljDim * a.c.ljDim;
  if ((E || (V && S)) && S && a.slowTableShared)
    bytes += sizeof(double) * kSlowTableDeg1 * (size_t)a.slowTableRows;
  return bytes;
}

template <bool E, bool V, bool S, bool B, int MINB>
static cudaError_t launchT(const ForceArgs& a, int numSM, cudaStream_t st) {
  const size_t shmem = forceShmem(a, E, V, S, B);
  auto k = forceKernel<E, V, S, B, MINB>;
  static OccCache cache;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevicesCached) return cudaErrorInvalidDevice;
  int blocks = 0;
  {
    std::lock_guard<std::mutex> lock(cache.mu);
    if (cache.shmem[dev] != shmem) {
      e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
      if (e != cudaSuccess) return e;
      int nb = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kForceThreads, shmem);
      if (e != cudaSuccess) return e;
      cache.blocks[dev] = nb > 0 ? nb : 1;
      cache.shmem[dev] = shmem;
    }
    blocks = cache.blocks[dev];
  }
  k<<<numSM * blocks, kForceThreads, shmem, st>>>(a);
  return cudaGetLastError();
}

template <bool E, bool V, bool S, bool B>
static cudaError_t launchShape(const ForceArgs& a, int minBlocks, int numSM, cudaStream_t st) {
  switch (minBlocks) {
    case 4: return launchT<E, V, S, B, 4>(a, numSM, st);
    case 5: return launchT<E, V, S, B, 5>(a, numSM, st);
    case 6: return launchT<E, V, S, B, 6>(a, numSM, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launchForce(const ForceArgs& a, unsigned flags, int minBlocks, int numSM,
                        cudaStream_t st) {
  const bool B = a.compRep != nullptr;
  const int idx = (B ? 8 : 0) | ((flags & NBK_ENERGY) ? 4 : 0) | ((flags & NBK_VIRIAL) ? 2 : 0) |
                  ((flags & NBK_SLOW) ? 1 : 0);
  switch (idx) {
#define NBK_CASE(i, e, v, s, b) \
  case i:                       \
    return launchShape<e, v, s, b>(a, minBlocks, numSM, st);
    NBK_CASE(0, false, false, false, false)
    NBK_CASE(1, false, false, true, false)
    NBK_CASE(2, false, true, false, false)
    NBK_CASE(3, false, true, true, false)
    NBK_CASE(4, true, false, false, false)
    NBK_CASE(5, true, false, true, false)
    NBK_CASE(6, true, true, false, false)
    NBK_CASE(7, true, true, true, false)
    NBK_CASE(8, false, false, false, true)
    NBK_CASE(9, false, false, true, true)
    NBK_CASE(10, false, true, false, true)
    NBK_CASE(11, false, true, true, true)
    NBK_CASE(12, true, false, false, true)
    NBK_CASE(13, true, false, true, true)
    NBK_CASE(14, true, true, false, true)
    NBK_CASE(15, true, true, true, true)
#undef NBK_CASE
  }
  return cudaErrorInvalidValue;
}

}  // namespace nbk
