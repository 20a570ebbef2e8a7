// Nonbonded force kernel of the B200 path, and the precise energy / virial
// kernel that follows it on energy and virial evaluations.
//
// forceKernel: one warp owns one tile list (32 i atoms of one patch against
// the j tiles of a compute's partner patch), as CudaComputeNonbondedKernel's
// nonbondedForceKernel does (src/CudaComputeNonbondedKernel.cu:629-1644), but:
//   - two pair steps per iteration run through sm_100's packed FP32
//     instructions; j forces ride in registers and rotate with a shuffle, so
//     the inner loop touches shared memory only for the j-tile loads;
//   - steps whose bit is clear in every lane's mask are skipped warp-uniformly;
//   - the lists it reads are already refined (TileExcl masks from
//     refineKernel); a pairlist step refines, compacts, then runs this kernel;
//   - per-tile FP32 partial forces are folded into 64-bit fixed point with
//     integer atomics, so the summed forces do not depend on the order in
//     which lists run; the LJ energy is summed in FP32 per group of tiles and
//     folded the same way; the fast virial comes from the fixed-point forces;
//   - on energy and virial evaluations it stores, per tile and lane, which of
//     the lane's pairs interact (the live words).
// preciseKernel: the electrostatic energies and the slow virial in FP64, from
// the live words: per tile, each lane walks a contiguous range of the tile's
// interacting pairs straight from the live words and evaluates them from
// FP64 geometry (see precisePass); its own
// launch runs at higher occupancy than the register- and shared-memory-heavy
// FP32 loop, which hides the FP64 dependency chains.
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

// virialSlow[3a+b] slots of symmetric component m (xx, xy, xz, yy, yz, zz);
// s1 < 0 for the diagonal.
__device__ __forceinline__ void symSlots(int m, int& s0, int& s1) {
  s0 = m == 0 ? 0 : m == 1 ? 1 : m == 2 ? 2 : m == 3 ? 4 : m == 4 ? 5 : 8;
  s1 = m == 1 ? 3 : m == 2 ? 6 : m == 4 ? 7 : -1;
}

// Adds the force kernel's LJ energy (lane 0) to one replica's accumulators.
template <bool doEnergy>
__device__ __forceinline__ void flushVdw(long long* acc, int lane, long long& accVdw) {
  if (doEnergy && lane == 0 && accVdw != 0) atomicAddFixed(&acc[kAccEVdw], (unsigned long long)accVdw);
  accVdw = 0;
}

// Adds the precise kernel's accumulators to one replica's block: lane
// q < kNumQ its quantity q (accQ), and the warp's pair count.
template <bool doEnergy>
__device__ __forceinline__ void flushPrecise(long long* acc, int lane, long long& accQ, int& npair) {
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
    int s = npair;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0 && s) atomicAddFixed(&acc[kAccNumPairs], (unsigned long long)s);
  }
  accQ = 0;
  npair = 0;
}

// FP64 geometry of one interacting pair: d = x_j - x_i and the charge product.
struct PairTerms {
  double dx, dy, dz, qq;
};

// The warp's atoms as the precise pass reads them: the list's i atoms in FP64
// (shifted by the exact lattice translation) as two rows of 32 (x, y) and
// (z, q) pairs, and the current j tile as it is stored (FP32 x, y, z, q, exact
// in FP64). A pair reads two 16-byte entries of its i atom and one of its j
// atom: the j reads span the 512 bytes of the row, half of what FP64 rows
// would, and the four conversions to FP64 cost less than the second load.
struct Atoms64 {
  double2 ixy[kWarp], izq[kWarp];
  float4 j[kWarp];
};

// One lane's precise-pass sums over the current tile group.
struct LaneSums {
  double eE, eS, w0, w1, w2, w3, w4, w5;
};

// The slow-term table as the precise pass reads it. kCopies > 0: kCopies
// interleaved copies in shared memory (s_slowTab), 16-byte pair n of row k of
// copy c at s_slowTab[(k * P + n) * kCopies + c] with P = kSlowTableDeg1 / 2;
// lane l reads copy l % kCopies, so with 8 copies the 8 lanes of a quarter
// warp (one 16-byte bank group each) never conflict, whatever rows they read.
// kCopies == 0: the global copy (kSlowTableRow doubles per row).
extern __shared__ __align__(16) double2 s_slowTab[];

struct SlowTable {
  const double2* gl;
  unsigned last;
  double step, invStep;
};

template <int kCopies>
__device__ __forceinline__ double2 slowPair(const SlowTable& T, const unsigned k, const int n,
                                            const int lane) {
  if (kCopies > 0) {
    return s_slowTab[(k * (kSlowTableDeg1 / 2) + n) * kCopies + (lane & (kCopies - 1))];
  } else {
    return __ldg(T.gl + (size_t)k * (kSlowTableRow / 2) + n);
  }
}

// The FP64 terms of one interacting pair (qq = 0 contributes exact zeros):
// the fast energy qq (1/r - h(s)) with 1/r from the FP64 approximation
// refined by one Newton step, and from the slow-term table the slow energy
// qq phi_s(s) and the slow virial -2 qq phi_s'(s) d (x) d. The geometry is
// FP64 throughout: the electrostatic totals are small differences of large
// sums (for 9,000 water atoms the fast energy is 4e-5 of the sum of its pair
// terms' magnitudes), so even the unbiased FP32 rounding of r^2 would move
// them by ~3e-6.
template <bool doEnergy, bool doVirial, bool doSlow, int kCopies>
__device__ __forceinline__ void precisePair(const PairTerms& u, const SlowTable& T,
                                            const NbkConst& c, const int lane, LaneSums& L) {
  const double s = fma(u.dz, u.dz, fma(u.dy, u.dy, u.dx * u.dx));
  double p = 0.0, dp = 0.0;
  if (doSlow) {
    // row k = nearest integer to s/D: adding 1.5 * 2^52 rounds s/D (exact, D
    // a power of two) into the low word; k is clamped to the last row (any
    // bit pattern stays in the table) and w = s - k D
    const double magic = 6755399441055744.0;
    const double t = fma(s, T.invStep, magic);
    const unsigned k = min((unsigned)__double2loint(t), T.last);
    const double wq = fma(-T.step, (double)k, s);
    double cf[kSlowTableDeg1];
#pragma unroll
    for (int n = 0; n < kSlowTableDeg1; n += 2) {
      const double2 v = slowPair<kCopies>(T, k, n / 2, lane);
      cf[n] = v.x;
      cf[n + 1] = v.y;
    }
    // Horner for p(w) and p'(w) together
    p = cf[kSlowTableDeg];
    dp = 0.0;
#pragma unroll
    for (int n = kSlowTableDeg - 1; n >= 0; --n) {
      dp = fma(dp, wq, p);
      p = fma(p, wq, cf[n]);
    }
  }
  if (doEnergy) {
    // y0 (rsqrt.approx.ftz.f64) has relative error below 2^-20; after one
    // Newton step, below 2^-39
    const double y0 = rsqrtApprox64(s);
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

// The FP64 pair terms of the pair (i, j = (i + t) & 31) from the warp's atoms
// in shared memory; qq = 0 (exact zeros) when the lane has no pair left and
// repeats its last one, a real interacting pair (so its distance is not 0).
__device__ __forceinline__ void pairTerms(const Atoms64& A, const int i, const int t,
                                          const bool valid, PairTerms& u) {
  const double2 ia = A.ixy[i], ib = A.izq[i];
  const float4 jb = A.j[(i + t) & 31];
  u.dx = (double)jb.x - ia.x;
  u.dy = (double)jb.y - ia.y;
  u.dz = (double)jb.z - ib.x;
  u.qq = valid ? ib.y * (double)jb.w : 0.0;
}

// w without its r lowest set bits (r < popc(w)): the bits from the position p
// of its (r + 1)-th set bit up, p being the largest position with at most r
// set bits below it (a binary search over popc of w's low bits; p + step
// stays below 32).
__device__ __forceinline__ unsigned dropLowBits(const unsigned w, const int r) {
  int p = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1)
    if (__popc(w & ((1u << (p + step)) - 1u)) <= r) p += step;
  return w & (0xffffffffu << p);
}

// One lane's walk over the tile's interacting pairs in lane-major order: the
// owner lane i whose live bits w are not taken yet, and the last pair taken
// (pi, pt).
struct PairWalk {
  int i, pi, pt;
  unsigned w;
};

// Takes the lane's next pair when valid (the lowest bit of w; w is not 0 while
// the lane has pairs left), then, once w is spent, moves on to the next lane
// with live bits (nonEmpty: the lanes whose live word is not 0). Every lane
// runs the shuffle; the source lane is in [0, 31].
__device__ __forceinline__ void walkNext(PairWalk& s, const bool valid, const unsigned live,
                                         const unsigned nonEmpty) {
  if (valid) {
    s.pt = __ffs(s.w) - 1;
    s.pi = s.i;
    s.w &= s.w - 1;
  }
  const int inext = __ffs(nonEmpty & (0xfffffffeu << s.i)) - 1;  // -1: none after i
  const unsigned wn = __shfl_sync(0xffffffffu, live, inext & 31);
  if (valid && s.w == 0u && inext >= 0) {
    s.i = inext;
    s.w = wn;
  }
}

// The precise pass of one tile. live (per lane): bit t set when the pair
// (i = lane, j = (lane + t) & 31) is an interacting pair (mask bit set and
// FP32 r^2 below the cutoff, the classification the FP32 math used). The
// tile's `total` interacting pairs, in lane-major order (by i, then t), are
// split into 32 contiguous ranges of m = ceil(total / 32): lane k takes pairs
// k m .. k m + m - 1 (the last lanes fewer or none). A lane finds the owner
// of its first pair by a binary search over the lanes' inclusive counts
// (shuffles), skips the owner's lower bits, and then walks the live words bit
// by bit (walkNext), two pairs per iteration (independent dependency
// chains). No queue is written. Each lane's sums take its pairs in a fixed
// order, so they depend only on the tile's live words. A lane without pairs
// repeats the tile's first pair with qq = 0.
template <bool doEnergy, bool doVirial, bool doSlow, int kCopies>
__device__ __forceinline__ void precisePass(const unsigned live, const int lane, const Atoms64& A,
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
  const int m = (total + kWarp - 1) / kWarp;
  const unsigned nonEmpty = __ballot_sync(0xffffffffu, live != 0u);
  int e0 = lane * m;
  const int cnt = min(m, max(0, total - e0));
  if (e0 >= total) e0 = 0;
  // owner of pair e0: the number of lanes whose inclusive count is <= e0
  int owner = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const int v = __shfl_sync(0xffffffffu, incl, owner + step - 1);
    if (v <= e0) owner += step;
  }
  const int ownerExcl = __shfl_sync(0xffffffffu, incl - n, owner);
  const unsigned ownerLive = __shfl_sync(0xffffffffu, live, owner);
  PairWalk s;
  s.i = owner;
  s.w = dropLowBits(ownerLive, e0 - ownerExcl);
  s.pi = owner;
  s.pt = __ffs(s.w) - 1;
  __syncwarp();  // the i rows and this j tile, written by the lanes, are visible
  int k = 0;
  for (; k + 1 < m; k += 2) {  // warp-uniform
    PairTerms u[2];
    walkNext(s, k < cnt, live, nonEmpty);
    pairTerms(A, s.pi, s.pt, k < cnt, u[0]);
    walkNext(s, k + 1 < cnt, live, nonEmpty);
    pairTerms(A, s.pi, s.pt, k + 1 < cnt, u[1]);
#pragma unroll
    for (int h = 0; h < 2; ++h) precisePair<doEnergy, doVirial, doSlow, kCopies>(u[h], T, c, lane, L);
  }
  if (k < m) {  // warp-uniform
    PairTerms u;
    walkNext(s, k < cnt, live, nonEmpty);
    pairTerms(A, s.pi, s.pt, k < cnt, u);
    precisePair<doEnergy, doVirial, doSlow, kCopies>(u, T, c, lane, L);
  }
  __syncwarp();  // the j rows are consumed before they are written again
}

// End of a tile group: the lanes' sums are reduced per quantity by a fixed
// butterfly that halves the quantities a lane holds at each step (lanes l and
// l ^ 16 exchange four of their eight, then l ^ 8 two, l ^ 4 one; two more
// steps add within groups of four lanes), so that lane 4q holds the warp's
// total of quantity q; lane q < kNumQ then adds quantity q, in fixed point,
// to accQ, and the sums restart at zero. No shared memory: a transposition
// through it costs more than these 20 shuffles (its reads conflict 16-way).
__device__ __forceinline__ void reduceGroup(const int lane, LaneSums& L, long long& accQ) {
  double v[kNumQ] = {L.eE, L.eS, L.w0, L.w1, L.w2, L.w3, L.w4, L.w5};
  static_assert(kQElec == 0 && kQSlow == 1 && kQVir == 2 && kNumQ == 8, "quantity order");
  // lanes with bit 4 set keep quantities 4..7, the others 0..3
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double send = b4 ? v[k] : v[k + 4];
    const double keep = b4 ? v[k + 4] : v[k];
    v[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double send = b3 ? v[k] : v[k + 2];
    const double keep = b3 ? v[k + 2] : v[k];
    v[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  {
    const double send = b2 ? v[0] : v[1];
    const double keep = b2 ? v[1] : v[0];
    v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  // lane l now holds quantity (l >> 2) summed over the lanes l' with
  // l' & 3 == l & 3; complete the sums within each group of four lanes
  v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
  v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
  const double tot = __shfl_sync(0xffffffffu, v[0], 4 * (lane & 7));
  if (lane < kNumQ) accQ += toFixedEnergy(tot);
  L = LaneSums{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
}

// MINB: CTAs per SM the register budget is cut for (4, 5 or 6 -> 128, 96 or
// 80 registers; the packed loop holds two pairs' state, and 5 is the untuned
// default); a.splitLog2: each list's j tiles are shared by 2^splitLog2
// work items (warps), contiguous parts of equal tile count. Both are launch
// choices of the autotuner; results do not depend on them (fixed-point sums
// per tile group).
template <bool doEnergy, bool doVirial, bool doSlow, bool doBatch, int MINB>
__global__ void __launch_bounds__(kForceThreads, MINB)
    forceKernel(const __grid_constant__ ForceArgs a) {
  // the live words feed the precise kernel, which runs on energy evaluations
  // and on virial evaluations with slow forces (it forms the slow virial)
  constexpr bool kLive = doEnergy || (doVirial && doSlow);
  extern __shared__ __align__(16) float2 s_lj[];  // [ljDim*ljDim] (single system)
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

  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const NbkConst& c = a.c;
  const int dim = c.ljDim;
  if (!doBatch) {
    for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) s_lj[k] = a.ljTable[k];
    __syncthreads();
  }

  const int numLists = a.numListsDev ? *a.numListsDev : a.numListsHost;

  long long accVdw = 0;  // lane 0: LJ energy to flush (batched replica change)
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
        flushVdw<doEnergy>(a.acc + (size_t)curRep * kAccCount, lane, accVdw);
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
    xi.x = __fadd_rn(xi.x, sh.x);
    xi.y = __fadd_rn(xi.y, sh.y);
    xi.z = __fadd_rn(xi.z, sh.z);
    const int ti = a.vdwTypes[iatom] * dim;

    // this tile group's two partial i sums per component
    float2 fix2 = f2(0.f), fiy2 = f2(0.f), fiz2 = f2(0.f);
    float2 fisx2 = f2(0.f), fisy2 = f2(0.f), fisz2 = f2(0.f);

    // the next tile's mask word and j atom are loaded while the current tile
    // is computed; the j-tile starts come 32 at a time (lane t holds tile
    // jtFirst + 32 b + t) and are handed out by a shuffle
    int jsBlock = 0;
    unsigned maskNext = 0;
    float4 xjNext = make_float4(0.f, 0.f, 0.f, 0.f);
    int tyNext = 0;
    for (int jt = jtFirst; jt <= jtLast; ++jt) {
      const int tb = (jt - jtFirst) & 31;
      if (tb == 0) {
        const int jtl = jt + lane;
        jsBlock = jtl <= jtLast ? a.tileJatomStart[jtl] : 0;
        const int js0 = __shfl_sync(0xffffffffu, jsBlock, 0);
        maskNext = a.tileExcls[jt].excl[lane];
        xjNext = a.xyzq[js0 + lane];
        tyNext = a.vdwTypes[js0 + lane];
      }
      const int jstart = __shfl_sync(0xffffffffu, jsBlock, tb);
      const unsigned mask = maskNext;
      const float4 xj = xjNext;
      const float tyj = __int_as_float(tyNext);
      if (jt < jtLast && tb < 31) {
        const int js1 = __shfl_sync(0xffffffffu, jsBlock, tb + 1);
        maskNext = a.tileExcls[jt + 1].excl[lane];
        xjNext = a.xyzq[js1 + lane];
        tyNext = a.vdwTypes[js1 + lane];
      }
      const unsigned stepMask = __reduce_or_sync(0xffffffffu, mask);
      unsigned live = 0;  // interacting pairs of this lane, TileExcl bit order
      if (stepMask != 0) {
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
          const float2 R2 = fma2(DZ, DZ, fma2(DX, DX, mul2(DY, DY)));  // dist2's order
          const bool aA = (mk & 1u) && (R2.x < c.cutoff2);
          const bool aB = (mk & 0x10000u) && (R2.y < c.cutoff2);
          if (!__any_sync(0xffffffffu, aA || aB)) continue;
          if (kLive) live |= ((aA ? 1u : 0u) | (aB ? 0x10000u : 0u)) << k;
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
      }
      if (kLive) a.liveOut[(size_t)jt * kWarp + lane] = live;
      if (((((jt - tl.jtileStart + 1) & (kFoldTiles - 1)) == 0) || jt == jtLast)) {
        // end of a tile group: its LJ energy and i forces into fixed point
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

  // per-warp flush of the LJ energy (no block barrier, so a warp that runs
  // out of lists retires at once)
  if (lane == 0) accVdw = s_evw[wib];
  flushVdw<doEnergy>(a.acc + (size_t)curRep * kAccCount, lane, accVdw);
}

// The precise kernel: one warp per refined tile list (handed out by a global
// counter in the force kernel's order, longest first). Per list the i atoms,
// shifted in FP64 by the shift formed in FP64 from the FP32 offsets and
// lattice (the exact lattice translation, without the FP32 rounding of the
// force kernel's shift), go to the warp's FP64 rows; per tile with interacting
// pairs the j atoms and the precise pass; per group of kFoldTiles tiles
// (counted from the list start, as the force kernel's) the lanes' sums go into
// fixed point. Results do not depend on the order in which lists run.
constexpr int kPreciseWarps = 8;
constexpr int kPreciseThreads = kPreciseWarps * kWarp;
constexpr int kPreciseMinBlocks = 3;

template <bool doEnergy, bool doVirial, bool doSlow, bool doBatch, int kCopies>
__global__ void __launch_bounds__(kPreciseThreads, kPreciseMinBlocks)
    preciseKernel(const __grid_constant__ ForceArgs a) {
  __shared__ Atoms64 s_atoms[kPreciseWarps];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  Atoms64& A = s_atoms[wib];
  SlowTable T;
  T.last = (unsigned)(a.slowTableRows - 1);
  T.step = a.slowStep;
  T.invStep = a.slowInvStep;
  T.gl = a.slowTable;
  if (doSlow && kCopies > 0) {
    constexpr int P = kSlowTableDeg1 / 2;
    for (int k = threadIdx.x; k < P * a.slowTableRows * kCopies; k += blockDim.x) {
      const int pair = k / (kCopies > 0 ? kCopies : 1);  // row * P + n
      s_slowTab[k] = a.slowTable[(size_t)(pair / P) * (kSlowTableRow / 2) + pair % P];
    }
    __syncthreads();
  }
  const int numLists = a.numListsDev ? *a.numListsDev : a.numListsHost;
  long long accQ = 0;  // lane q < kNumQ: quantity q
  int npair = 0;       // interacting pairs counted by this lane (energy evaluations)
  LaneSums lsum{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int curRep = 0;
  for (;;) {
    int L = 0;
    if (lane == 0) L = atomicAdd(a.workCounter, 1);
    L = __shfl_sync(0xffffffffu, L, 0);
    if (L >= numLists) break;
    const nbk_tile_list tl = a.lists[L];
    if (tl.jtileEnd < tl.jtileStart) continue;  // empty (warp-uniform)
    float3 la = a.lata, lb = a.latb, lc = a.latc;
    if (doBatch) {
      const int rep = __ldg(&a.compRep[tl.icompute]);
      if (rep != curRep) {
        flushPrecise<doEnergy>(a.acc + (size_t)curRep * kAccCount, lane, accQ, npair);
        curRep = rep;
      }
      la = a.repLat[3 * rep];
      lb = a.repLat[3 * rep + 1];
      lc = a.repLat[3 * rep + 2];
    }
    {
      const float3 off = make_float3(tl.offsetXYZ.x, tl.offsetXYZ.y, tl.offsetXYZ.z);
      const float4 xi = a.xyzq[tl.iatomStart + lane];
      A.ixy[lane] = make_double2(
          (double)xi.x + ((double)off.x * la.x + (double)off.y * lb.x + (double)off.z * lc.x),
          (double)xi.y + ((double)off.x * la.y + (double)off.y * lb.y + (double)off.z * lc.y));
      A.izq[lane] = make_double2(
          (double)xi.z + ((double)off.x * la.z + (double)off.y * lb.z + (double)off.z * lc.z),
          (double)xi.w);
    }
    // the next tile's live word and j atom are loaded while the current tile
    // is processed; the j-tile starts come 32 at a time (lane t holds tile
    // jt0 + t) and are handed out by a shuffle
    int jsBlock = 0;
    unsigned liveNext = 0;
    float4 xjNext = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int jt = tl.jtileStart; jt <= tl.jtileEnd; ++jt) {
      const int t = (jt - tl.jtileStart) & 31;
      if (t == 0) {
        const int jtl = jt + lane;
        jsBlock = jtl <= tl.jtileEnd ? a.tileJatomStart[jtl] : 0;
        liveNext = a.liveOut[(size_t)jt * kWarp + lane];
        xjNext = a.xyzq[__shfl_sync(0xffffffffu, jsBlock, 0) + lane];
      }
      const unsigned live = liveNext;
      const float4 xj = xjNext;
      if (jt < tl.jtileEnd && t < 31) {
        liveNext = a.liveOut[(size_t)(jt + 1) * kWarp + lane];
        xjNext = a.xyzq[__shfl_sync(0xffffffffu, jsBlock, t + 1) + lane];
      }
      if (__any_sync(0xffffffffu, live != 0u)) {
        // the i rows and this j tile are visible after the pass's first __syncwarp
        A.j[lane] = xj;
        precisePass<doEnergy, doVirial, doSlow, kCopies>(live, lane, A, T, a.c,
                                                         lsum, npair);
      }
      if (((jt - tl.jtileStart + 1) & (kFoldTiles - 1)) == 0 || jt == tl.jtileEnd)
        reduceGroup(lane, lsum, accQ);
    }
  }
  flushPrecise<doEnergy>(a.acc + (size_t)curRep * kAccCount, lane, accQ, npair);
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

template <typename K>
static cudaError_t launchPersistent(K kernel, OccCache& cache, int threads, size_t shmem,
                                    int numSM, cudaStream_t st, const ForceArgs& a) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevicesCached) return cudaErrorInvalidDevice;
  int blocks = 0;
  {
    std::lock_guard<std::mutex> lock(cache.mu);
    if (cache.shmem[dev] != shmem) {
      e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
      if (e != cudaSuccess) return e;
      int nb = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, shmem);
      if (e != cudaSuccess) return e;
      cache.blocks[dev] = nb > 0 ? nb : 1;
      cache.shmem[dev] = shmem;
    }
    blocks = cache.blocks[dev];
  }
  kernel<<<numSM * blocks, threads, shmem, st>>>(a);
  return cudaGetLastError();
}

template <bool E, bool V, bool S, bool B, int MINB>
static cudaError_t launchT(const ForceArgs& a, int numSM, cudaStream_t st) {
  static OccCache cache;
  const size_t shmem = B ? 0 : sizeof(float2) * (size_t)a.c.ljDim * a.c.ljDim;
  return launchPersistent(forceKernel<E, V, S, B, MINB>, cache, kForceThreads, shmem, numSM, st,
                          a);
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

bool needsPrecise(unsigned flags) {
  return (flags & NBK_ENERGY) || ((flags & NBK_VIRIAL) && (flags & NBK_SLOW));
}

template <bool E, bool V, bool S, bool B, int C>
static cudaError_t launchPC(const ForceArgs& a, int numSM, cudaStream_t st) {
  static OccCache cache;
  const size_t shmem = (S && C > 0) ? sizeof(double) * kSlowTableDeg1 * (size_t)a.slowTableRows * C
                                    : 0;
  return launchPersistent(preciseKernel<E, V, S, B, C>, cache, kPreciseThreads, shmem, numSM, st,
                          a);
}

// the table in shared memory with 8 interleaved copies when they fit in 40 KB
// (106 rows), else read from global memory
template <bool E, bool V, bool S, bool B>
static cudaError_t launchP(const ForceArgs& a, int numSM, cudaStream_t st) {
  if (sizeof(double) * kSlowTableDeg1 * (size_t)a.slowTableRows * 8 <= 40 * 1024)
    return launchPC<E, V, S, B, 8>(a, numSM, st);
  return launchPC<E, V, S, B, 0>(a, numSM, st);
}

cudaError_t launchPrecise(const ForceArgs& a, unsigned flags, int numSM, cudaStream_t st) {
  if (!needsPrecise(flags)) return cudaSuccess;
  const bool B = a.compRep != nullptr;
  const int idx = (B ? 8 : 0) | ((flags & NBK_ENERGY) ? 4 : 0) | ((flags & NBK_VIRIAL) ? 2 : 0) |
                  ((flags & NBK_SLOW) ? 1 : 0);
  switch (idx) {
#define NBK_CASE(i, e, v, s, b) \
  case i:                       \
    return launchP<e, v, s, b>(a, numSM, st);
    NBK_CASE(3, false, true, true, false)
    NBK_CASE(4, true, false, false, false)
    NBK_CASE(5, true, false, true, false)
    NBK_CASE(6, true, true, false, false)
    NBK_CASE(7, true, true, true, false)
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
