/*
 * nbk_oracle.c — FP64 CPU oracle of NAMD 3.0's short-range nonbonded path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that the GPU path is
 * compared against; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it. The product path never calls it.
 *
 * It restates, in plain C and double precision:
 *   - the pair-set rule of the tile-list refinement: a pair (i,j) of a compute
 *     (i in patch1, j in patch2; j after i in slot order for a self compute)
 *     is listed iff its FP32 distance^2, formed with the reference's operand
 *     order (shift = offset . lattice; dx = xj - (xi + shift);
 *     r2 = dx*dx + dy*dy + dz*dz, each sum contracted as the reference's
 *     compiled kernels round it: the first product fused into the first sum,
 *     fma(dz, dz, fma(dx, dx, dy*dy)), and likewise the shift), is below
 *     the FP32 pairlist cutoff^2, the pair is not a full exclusion, and at
 *     least one atom is free            (src/CudaComputeNonbondedKernel.cu:720-750,
 *                                        1225-1249; src/CudaTileListKernel.cu:405-548)
 *   - the exclusion test through the per-atom (base, maxdiff) bit array
 *                                       (src/CudaComputeNonbondedKernel.cu:1234-1247;
 *                                        src/CudaComputeNonbonded.C:2191-2316)
 *   - the pair energies and forces of energy-switched LJ and C1-split PME
 *     real-space electrostatics, analytically in FP64
 *                                       (src/CudaComputeNonbondedInteractions.h:37-159;
 *                                        src/ComputeNonbondedUtil.C:852-975)
 *   - the excluded-pair (-qq erf(br)/r) and modified 1-4 pair corrections
 *                                       (src/ComputeBondedCUDAKernel.cu:315-778;
 *                                        src/ComputeNonbondedCUDAExcl.C:186-299)
 *   - virial W[a][b] = sum over pairs of F_a * r_b (src/CudaComputeNonbondedKernel.cu:
 *     1649-1920 reduce to this pair sum).
 * Pairs are classified against the cutoffs in FP32 exactly as the GPU does, so
 * that borderline pairs fall on the same side; their values are FP64.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  int atomStorageSize;
  int numPatches;
  int numComputes;
  int vdwDim;
  const float* xyzq;          /* [4*storage] */
  const int* patches;         /* [4*numPatches] numAtoms, numFreeAtoms, atomStart, id */
  const int* computePatch;    /* [2*numComputes] */
  const float* computeOffset; /* [3*numComputes] lattice units */
  const float* lattice;       /* [9] lata, latb, latc */
  const int* vdwTypes;        /* [storage] */
  const int* atomIndex;       /* [storage] */
  const int* exclIndexMaxDiff;/* [2*storage] base, maxdiff */
  const unsigned* exclBits;
  long long numExclWords;
  const double* ljA;          /* [dim*dim], unscaled */
  const double* ljB;
  const double* ljA14;
  const double* ljB14;
  double cutoff, switchdist, ewaldcof, scaling, scale14;
  float cutoff2f, plcutoff2f;
} oracle_system;

/* 32-byte correction tuple, layout of CudaExclusion */
typedef struct {
  int i, j, ti, tj;
  float ox, oy, oz;
  int pswitch;
} oracle_tuple;

/* ---- FP32 pair-set geometry (exact operand order) -------------------- */
static inline void shift_f32(const oracle_system* s, int c, float* sh) {
  const float ox = s->computeOffset[3 * c], oy = s->computeOffset[3 * c + 1],
              oz = s->computeOffset[3 * c + 2];
  const float* L = s->lattice;
  for (int d = 0; d < 3; ++d) sh[d] = fmaf(oz, L[6 + d], fmaf(ox, L[d], oy * L[3 + d]));
}

static inline float r2_f32(const float* xi_shifted, const float* xj) {
  const float dx = xj[0] - xi_shifted[0];
  const float dy = xj[1] - xi_shifted[1];
  const float dz = xj[2] - xi_shifted[2];
  return fmaf(dz, dz, fmaf(dx, dx, dy * dy));
}

static inline int excluded(const oracle_system* s, int i, int j) {
  int diff = s->atomIndex[j] - s->atomIndex[i];
  const int base = s->exclIndexMaxDiff[2 * i], maxdiff = s->exclIndexMaxDiff[2 * i + 1];
  if (abs(diff) > maxdiff) return 0;
  const unsigned idx = (unsigned)(diff + base);
  if ((long long)(idx >> 5) >= s->numExclWords) return 0;
  return (s->exclBits[idx >> 5] >> (idx & 31)) & 1u;
}

/* Enumerates the listed pairs of compute c. keys (if non-NULL) receive
 * i_slot * storage + j_slot. Returns the number of listed pairs; adds the
 * excluded pairs within the pairlist cutoff to *nexcl. */
static long long compute_pairs(const oracle_system* s, int c, unsigned long long* keys,
                               long long* nexcl) {
  const int p1 = s->computePatch[2 * c], p2 = s->computePatch[2 * c + 1];
  const int* P1 = s->patches + 4 * p1;
  const int* P2 = s->patches + 4 * p2;
  float sh[3];
  shift_f32(s, c, sh);
  const int zeroShift = !(fmaf(sh[2], sh[2], fmaf(sh[0], sh[0], sh[1] * sh[1])) > 0.0f);
  const int self = (p1 == p2) && zeroShift;
  long long n = 0, ne = 0;
  for (int a = 0; a < P1[0]; ++a) {
    const int i = P1[2] + a;
    const float* xi = s->xyzq + 4 * (size_t)i;
    float xs[3] = {xi[0] + sh[0], xi[1] + sh[1], xi[2] + sh[2]};
    for (int b = self ? a + 1 : 0; b < P2[0]; ++b) {
      const int j = P2[2] + b;
      const float r2 = r2_f32(xs, s->xyzq + 4 * (size_t)j);
      if (!(r2 < s->plcutoff2f)) continue;
      if (!(b < P2[1] || a < P1[1])) continue; /* both fixed */
      if (excluded(s, i, j)) {
        ++ne;
        continue;
      }
      if (keys) keys[n] = (unsigned long long)i * (unsigned long long)s->atomStorageSize + j;
      ++n;
    }
  }
  if (nexcl) *nexcl += ne;
  return n;
}

/* Pair set of the refined tile lists. keys == NULL: count only. */
long long oracle_pairs(const oracle_system* s, unsigned long long* keys, long long* numExcluded) {
  long long* cnt = (long long*)calloc((size_t)s->numComputes + 1, sizeof(long long));
  long long* exc = (long long*)calloc((size_t)s->numComputes, sizeof(long long));
  if (!cnt || !exc) return -1;
#pragma omp parallel for schedule(dynamic, 4)
  for (int c = 0; c < s->numComputes; ++c) cnt[c + 1] = compute_pairs(s, c, NULL, &exc[c]);
  for (int c = 0; c < s->numComputes; ++c) cnt[c + 1] += cnt[c];
  const long long total = cnt[s->numComputes];
  if (keys) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int c = 0; c < s->numComputes; ++c) compute_pairs(s, c, keys + cnt[c], NULL);
  }
  if (numExcluded) {
    long long e = 0;
    for (int c = 0; c < s->numComputes; ++c) e += exc[c];
    *numExcluded = e;
  }
  free(cnt);
  free(exc);
  return total;
}

/* ---- FP64 pair math ---------------------------------------------------- */
typedef struct {
  double rc2, rs2, rcinv, rc3inv, beta, twoBetaOverSqrtPi, swDenomInv;
  int switching;
} pair_consts;

static pair_consts make_consts(const oracle_system* s) {
  pair_consts k;
  k.rc2 = s->cutoff * s->cutoff;
  k.switching = s->switchdist < s->cutoff;
  k.rs2 = k.switching ? s->switchdist * s->switchdist : k.rc2;
  k.rcinv = 1.0 / s->cutoff;
  k.rc3inv = k.rcinv * k.rcinv * k.rcinv;
  k.beta = s->ewaldcof;
  k.twoBetaOverSqrtPi = 2.0 * s->ewaldcof / sqrt(M_PI);
  k.swDenomInv = k.switching ? 1.0 / ((k.rc2 - k.rs2) * (k.rc2 - k.rs2) * (k.rc2 - k.rs2)) : 0.0;
  return k;
}

/* Energy-switched LJ: energy and g = (dE/dr)/r. */
static inline void lj_switched(const pair_consts* k, double r2, double A, double B, double* E,
                               double* g) {
  const double r2inv = 1.0 / r2;
  const double r6 = r2inv * r2inv * r2inv;
  const double w = (A * r6 - B) * r6;
  const double dw = (-12.0 * A * r6 + 6.0 * B) * r6 * r2inv; /* (dw/dr)/r */
  if (k->switching && r2 > k->rs2) {
    const double d = k->rc2 - r2;
    const double S = d * d * (k->rc2 + 2.0 * r2 - 3.0 * k->rs2) * k->swDenomInv;
    const double dS = 12.0 * d * (k->rs2 - r2) * k->swDenomInv; /* (dS/dr)/r */
    *E = w * S;
    *g = w * dS + dw * S;
  } else {
    *E = w;
    *g = dw;
  }
}

/* C1-split electrostatics for unit qq: fast = shifted Coulomb, slow = PME
 * real-space remainder; E and g = (dE/dr)/r for each. */
static inline void elec_split(const pair_consts* k, double r2, double* Ef, double* gf, double* Es,
                              double* gs) {
  const double r = sqrt(r2);
  const double rinv = 1.0 / r;
  const double rinv3 = rinv * rinv * rinv;
  const double h = 0.5 * k->rcinv * (3.0 - r2 * k->rcinv * k->rcinv); /* (3 - r2/rc2)/(2 rc) */
  const double x = k->beta * r;
  const double ec = erfc(x);
  const double ex = exp(-x * x);
  *Ef = rinv - h;
  *gf = -rinv3 + k->rc3inv;
  *Es = h + (ec - 1.0) * rinv;
  *gs = -k->rc3inv - (ec - 1.0) * rinv3 - k->twoBetaOverSqrtPi * ex * rinv * rinv;
}

static inline void add_pair(double* F, double* Fs, int i, int j, const double* d, double g,
                            double gs, double* W, double* Ws) {
  /* d = xj - xi; F_i += g*d, F_j -= g*d; W -= g d (x) d */
  for (int a = 0; a < 3; ++a) {
    F[3 * (size_t)i + a] += g * d[a];
    F[3 * (size_t)j + a] -= g * d[a];
    Fs[3 * (size_t)i + a] += gs * d[a];
    Fs[3 * (size_t)j + a] -= gs * d[a];
    for (int b = 0; b < 3; ++b) {
      W[3 * a + b] -= g * d[a] * d[b];
      Ws[3 * a + b] -= gs * d[a] * d[b];
    }
  }
}

/* out[0..2] = E_vdw, E_elec, E_slow; out[3..11] virial; out[12..20] virialSlow;
 * out[21] = pairs within the cutoff (the work unit); out[22..24] = sums of
 * |pair energy| of each term (the scale against which a sum of FP32 pair
 * energies can be resolved). */
#define ORACLE_NOUT 25

static void nonbonded_compute(const oracle_system* s, const pair_consts* k, int c, double* F,
                              double* Fs, double* out) {
  const int p1 = s->computePatch[2 * c], p2 = s->computePatch[2 * c + 1];
  const int* P1 = s->patches + 4 * p1;
  const int* P2 = s->patches + 4 * p2;
  float sh[3];
  shift_f32(s, c, sh);
  const int zeroShift = !(fmaf(sh[2], sh[2], fmaf(sh[0], sh[0], sh[1] * sh[1])) > 0.0f);
  const int self = (p1 == p2) && zeroShift;
  /* FP64 shift from the FP32 offsets (the exact lattice translation) */
  double shd[3];
  for (int a = 0; a < 3; ++a)
    shd[a] = (double)s->computeOffset[3 * c] * s->lattice[a] +
             (double)s->computeOffset[3 * c + 1] * s->lattice[3 + a] +
             (double)s->computeOffset[3 * c + 2] * s->lattice[6 + a];
  const int dim = s->vdwDim;
  for (int a = 0; a < P1[0]; ++a) {
    const int i = P1[2] + a;
    const float* xi = s->xyzq + 4 * (size_t)i;
    float xs[3] = {xi[0] + sh[0], xi[1] + sh[1], xi[2] + sh[2]};
    for (int b = self ? a + 1 : 0; b < P2[0]; ++b) {
      const int j = P2[2] + b;
      const float* xj = s->xyzq + 4 * (size_t)j;
      const float r2f = r2_f32(xs, xj);
      if (!(r2f < s->cutoff2f)) continue;
      if (!(r2f < s->plcutoff2f)) continue;
      if (!(b < P2[1] || a < P1[1])) continue;
      if (excluded(s, i, j)) continue;
      double d[3];
      for (int q = 0; q < 3; ++q) d[q] = (double)xj[q] - ((double)xi[q] + shd[q]);
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const int ti = s->vdwTypes[i], tj = s->vdwTypes[j];
      const double A = s->ljA[ti * dim + tj] * s->scaling, B = s->ljB[ti * dim + tj] * s->scaling;
      const double qq = (double)xi[3] * (double)xj[3];
      double Elj, glj, Ef, gf, Es, gs;
      lj_switched(k, r2, A, B, &Elj, &glj);
      elec_split(k, r2, &Ef, &gf, &Es, &gs);
      out[0] += Elj;
      out[1] += qq * Ef;
      out[2] += qq * Es;
      out[21] += 1.0;
      out[22] += fabs(Elj);
      out[23] += fabs(qq * Ef);
      out[24] += fabs(qq * Es);
      add_pair(F, Fs, i, j, d, glj + qq * gf, qq * gs, out + 3, out + 12);
    }
  }
}

/* Corrections: modified (1-4) and excluded pairs within the cutoff, with the
 * tuple's own shift: r_ij = x_i + shift - x_j (bonded-kernel convention). */
static void correction_tuple(const oracle_system* s, const pair_consts* k, const oracle_tuple* t,
                             int modified, double* F, double* Fs, double* out) {
  const float* xi = s->xyzq + 4 * (size_t)t->i;
  const float* xj = s->xyzq + 4 * (size_t)t->j;
  const float* L = s->lattice;
  float shf[3];
  for (int d = 0; d < 3; ++d) shf[d] = fmaf(t->oz, L[6 + d], fmaf(t->ox, L[d], t->oy * L[3 + d]));
  const float xf = xi[0] + shf[0] - xj[0], yf = xi[1] + shf[1] - xj[1], zf = xi[2] + shf[2] - xj[2];
  const float r2f = fmaf(zf, zf, fmaf(xf, xf, yf * yf));
  if (!(r2f < s->cutoff2f)) return;
  double shd[3], dij[3];
  for (int a = 0; a < 3; ++a) {
    shd[a] = (double)t->ox * L[a] + (double)t->oy * L[3 + a] + (double)t->oz * L[6 + a];
    dij[a] = ((double)xi[a] + shd[a]) - (double)xj[a]; /* x_i - x_j */
  }
  const double r2 = dij[0] * dij[0] + dij[1] * dij[1] + dij[2] * dij[2];
  const double qq = (double)xi[3] * (double)xj[3];
  double E_vdw = 0, g = 0, E_el = 0, E_sl = 0, gs = 0;
  if (modified) {
    const int dim = s->vdwDim;
    const double dA = (s->ljA14[t->ti * dim + t->tj] - s->ljA[t->ti * dim + t->tj]) * s->scaling;
    const double dB = (s->ljB14[t->ti * dim + t->tj] - s->ljB[t->ti * dim + t->tj]) * s->scaling;
    double Elj, glj, Ef, gf, Es, gsl;
    lj_switched(k, r2, dA, dB, &Elj, &glj);
    elec_split(k, r2, &Ef, &gf, &Es, &gsl);
    const double one14 = 1.0 - s->scale14;
    /* remove (1-scale14) of the full 1/r Coulomb: fast part and the smooth
     * part (3 - r2/rc2)/(2rc) of the slow buffer */
    const double h = 0.5 * k->rcinv * (3.0 - r2 * k->rcinv * k->rcinv);
    E_vdw = Elj;
    E_el = -one14 * qq * Ef;
    E_sl = -one14 * qq * h;
    g = glj - one14 * qq * gf;
    /* E = -c qq (3 - r2/rc2)/(2rc): dE/dr = c qq r/rc^3, so g = c qq / rc^3 */
    gs = one14 * qq * k->rc3inv;
  } else {
    const double r = sqrt(r2);
    const double x = k->beta * r;
    const double erfx = erf(x);
    E_sl = -qq * erfx / r;
    /* d/dr(-erf(br)/r) = erf/r^2 - (2b/sqrt(pi)) exp(-b^2 r^2)/r */
    gs = qq * (erfx / (r2 * r) - k->twoBetaOverSqrtPi * exp(-x * x) / r2);
  }
  /* d for add_pair is x_j - x_i = -dij */
  double d[3] = {-dij[0], -dij[1], -dij[2]};
  out[0] += E_vdw;
  out[1] += E_el;
  out[2] += E_sl;
  out[22] += fabs(E_vdw);
  out[23] += fabs(E_el);
  out[24] += fabs(E_sl);
  add_pair(F, Fs, t->i, t->j, d, g, gs, out + 3, out + 12);
}

/* Evaluates computes [c0, c1) (mode bit 0) and/or the correction tuples
 * (mode bit 1) on all OpenMP threads. F/Fs: [3*storage] (overwritten);
 * out: [ORACLE_NOUT]. */
int oracle_nonbonded_sub(const oracle_system* s, int mode, int c0, int c1, int numModified,
                         const oracle_tuple* mod, int numExcluded, const oracle_tuple* exc,
                         double* F, double* Fs, double* out) {
  const pair_consts k = make_consts(s);
  const size_t n3 = 3 * (size_t)s->atomStorageSize;
  if (c0 < 0) c0 = 0;
  if (c1 < 0 || c1 > s->numComputes) c1 = s->numComputes;
  memset(F, 0, n3 * sizeof(double));
  memset(Fs, 0, n3 * sizeof(double));
  memset(out, 0, ORACLE_NOUT * sizeof(double));
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  double* bufF = (double*)calloc(n3 * nthreads, sizeof(double));
  double* bufS = (double*)calloc(n3 * nthreads, sizeof(double));
  double* bufO = (double*)calloc((size_t)ORACLE_NOUT * nthreads, sizeof(double));
  if (!bufF || !bufS || !bufO) {
    free(bufF);
    free(bufS);
    free(bufO);
    return -1;
  }
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* myF = bufF + n3 * tid;
    double* myS = bufS + n3 * tid;
    double* myO = bufO + (size_t)ORACLE_NOUT * tid;
    if (mode & 1) {
#pragma omp for schedule(dynamic, 4)
      for (int c = c0; c < c1; ++c) nonbonded_compute(s, &k, c, myF, myS, myO);
    }
    if (mode & 2) {
#pragma omp for schedule(static)
      for (int t = 0; t < numModified; ++t) correction_tuple(s, &k, &mod[t], 1, myF, myS, myO);
#pragma omp for schedule(static)
      for (int t = 0; t < numExcluded; ++t) correction_tuple(s, &k, &exc[t], 0, myF, myS, myO);
    }
  }
  for (int t = 0; t < nthreads; ++t) {
    const double* a = bufF + n3 * t;
    const double* b = bufS + n3 * t;
    for (size_t q = 0; q < n3; ++q) {
      F[q] += a[q];
      Fs[q] += b[q];
    }
    for (int q = 0; q < ORACLE_NOUT; ++q) out[q] += bufO[(size_t)ORACLE_NOUT * t + q];
  }
  free(bufF);
  free(bufS);
  free(bufO);
  return 0;
}

/* mode bit 0: nonbonded kernel part (normal + modified pairs at full strength);
 * bit 1: corrections. F/Fs: [3*storage] (overwritten). out: [ORACLE_NOUT]. */
int oracle_nonbonded(const oracle_system* s, int mode, int numModified, const oracle_tuple* mod,
                     int numExcluded, const oracle_tuple* exc, double* F, double* Fs,
                     double* out) {
  return oracle_nonbonded_sub(s, mode, 0, -1, numModified, mod, numExcluded, exc, F, Fs, out);
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Single-pair FP64 evaluations (pinned against the reference's own pair-math
 * functions by tests/golden): out[5k..5k+4] = {g, gs, E_vdw, E_elec, E_slow}
 * with g = (dE/dr)/r, i.e. the nonbonded kernel's F_i += g (x_j - x_i). */
void oracle_pair_nonbonded(int n, const double* r2, const double* qq, const double* A,
                           const double* B, double cutoff, double switchdist, double ewaldcof,
                           double* out) {
  oracle_system s;
  memset(&s, 0, sizeof(s));
  s.cutoff = cutoff;
  s.switchdist = switchdist;
  s.ewaldcof = ewaldcof;
  const pair_consts k = make_consts(&s);
  for (int q = 0; q < n; ++q) {
    double Elj, glj, Ef, gf, Es, gs;
    lj_switched(&k, r2[q], A[q], B[q], &Elj, &glj);
    elec_split(&k, r2[q], &Ef, &gf, &Es, &gs);
    out[5 * q + 0] = glj + qq[q] * gf;
    out[5 * q + 1] = qq[q] * gs;
    out[5 * q + 2] = Elj;
    out[5 * q + 3] = qq[q] * Ef;
    out[5 * q + 4] = qq[q] * Es;
  }
}

/* Modified (1-4) correction of one pair, qq already times (1 - scale14) and
 * (A, B) = (A14 - A, B14 - B); same output layout and sign convention. */
void oracle_pair_modified(int n, const double* r2, const double* qq, const double* A,
                          const double* B, double cutoff, double switchdist, double ewaldcof,
                          double* out) {
  oracle_system s;
  memset(&s, 0, sizeof(s));
  s.cutoff = cutoff;
  s.switchdist = switchdist;
  s.ewaldcof = ewaldcof;
  const pair_consts k = make_consts(&s);
  for (int q = 0; q < n; ++q) {
    double Elj, glj, Ef, gf, Es, gs;
    lj_switched(&k, r2[q], A[q], B[q], &Elj, &glj);
    elec_split(&k, r2[q], &Ef, &gf, &Es, &gs);
    const double h = 0.5 * k.rcinv * (3.0 - r2[q] * k.rcinv * k.rcinv);
    out[5 * q + 0] = glj - qq[q] * gf;
    out[5 * q + 1] = qq[q] * k.rc3inv;
    out[5 * q + 2] = Elj;
    out[5 * q + 3] = -qq[q] * Ef;
    out[5 * q + 4] = -qq[q] * h;
  }
}

/* ---- adjoint (config: L = sum wF.F_fast + sum wS.F_slow + cV E_vdw + cE E_elec + cS E_slow) ----
 * Restated from the pair math above: with s = r^2, each pair contributes
 *   l = pF g(s) + pS gs(s) + cV E_lj(s) + cE qq phi_f(s) + cS qq phi_s(s),
 *   pF = (wF_i - wF_j).d, pS = (wS_i - wS_j).d, d = x_j - x_i,
 * so dl/dd = g uF + gs uS + d [2 (pF g' + pS gs') + cV g_lj + cE qq g_f + cS qq g_s]
 * (' = d/ds; 2 dE/ds = g for every term). */

/* Second derivatives d/ds of the (dE/dr)/r functions, FP64. */
static inline void pair_second(const pair_consts* k, double s, double A, double B, double* glj,
                               double* dglj, double* gA, double* gB, double* EA, double* EB,
                               double* gf, double* dgf, double* gsl, double* dgsl, double* phf,
                               double* phs) {
  const double si = 1.0 / s, s3 = si * si * si, s6 = s3 * s3;
  /* W(s) = A s^-6 - B s^-3 */
  const double WA = s6, WB = -s3;
  const double WA1 = -6.0 * s6 * si, WB1 = 3.0 * s3 * si;
  const double WA2 = 42.0 * s6 * si * si, WB2 = -12.0 * s3 * si * si;
  double S = 1.0, S1 = 0.0, S2 = 0.0;
  if (k->switching && s > k->rs2) {
    const double d = k->rc2 - s;
    S = d * d * (k->rc2 + 2.0 * s - 3.0 * k->rs2) * k->swDenomInv;
    S1 = 6.0 * d * (k->rs2 - s) * k->swDenomInv;
    S2 = 6.0 * (2.0 * s - k->rs2 - k->rc2) * k->swDenomInv;
  }
  *gA = 2.0 * (WA1 * S + WA * S1);
  *gB = 2.0 * (WB1 * S + WB * S1);
  *EA = WA * S;
  *EB = WB * S;
  *glj = A * (*gA) + B * (*gB);
  *dglj = 2.0 * (A * (WA2 * S + 2.0 * WA1 * S1 + WA * S2) + B * (WB2 * S + 2.0 * WB1 * S1 + WB * S2));
  const double r = sqrt(s), ri = 1.0 / r;
  const double ri2 = ri * ri, ri3 = ri2 * ri, ri5 = ri3 * ri2;
  const double h = 0.5 * k->rcinv * (3.0 - s * k->rcinv * k->rcinv);
  const double x = k->beta * r, ex = exp(-x * x), ec = erfc(x);
  *phf = ri - h;
  *phs = h + (ec - 1.0) * ri;
  *gf = -ri3 + k->rc3inv;
  *dgf = 1.5 * ri5;
  *gsl = -k->rc3inv - (ec - 1.0) * ri3 - k->twoBetaOverSqrtPi * ex * ri2;
  /* d/ds of gs: (beta/sqrt(pi)) e^{-x^2} (2 beta^2 / r^2 + 3 / r^4) + 1.5 (erfc - 1) / r^5 */
  const double b = k->beta;
  *dgsl = 0.5 * k->twoBetaOverSqrtPi * ex * (2.0 * b * b * ri2 + 3.0 * ri2 * ri2) + 1.5 * (ec - 1.0) * ri5;
}

/* Loss of one pair (FP64). */
static inline double pair_loss(const pair_consts* k, double s, double qq, double A, double B,
                               double pF, double pS, double cV, double cE, double cS) {
  double glj, dglj, gA, gB, EA, EB, gf, dgf, gsl, dgsl, phf, phs;
  pair_second(k, s, A, B, &glj, &dglj, &gA, &gB, &EA, &EB, &gf, &dgf, &gsl, &dgsl, &phf, &phs);
  const double Elj = A * EA + B * EB;
  return pF * (glj + qq * gf) + pS * qq * gsl + cV * Elj + cE * qq * phf + cS * qq * phs;
}

typedef struct {
  const double* wF; /* [3*storage] */
  const double* wS; /* [3*storage] */
  double cV, cE, cS;
} oracle_cot;

/* Walks the nonbonded pairs of compute c (kernel semantics: excluded pairs
 * skipped, 1-4 pairs at full strength). onlySlot >= 0 restricts to pairs
 * that involve that slot. Accumulates the loss and (if non-NULL) the gradients. */
static double adjoint_compute(const oracle_system* s, const pair_consts* k, int c,
                              const oracle_cot* cot, int onlySlot, double* gX, double* gQ,
                              double* gA_, double* gB_) {
  const int p1 = s->computePatch[2 * c], p2 = s->computePatch[2 * c + 1];
  const int* P1 = s->patches + 4 * p1;
  const int* P2 = s->patches + 4 * p2;
  float sh[3];
  shift_f32(s, c, sh);
  const int zeroShift = !(fmaf(sh[2], sh[2], fmaf(sh[0], sh[0], sh[1] * sh[1])) > 0.0f);
  const int self = (p1 == p2) && zeroShift;
  double shd[3];
  for (int a = 0; a < 3; ++a)
    shd[a] = (double)s->computeOffset[3 * c] * s->lattice[a] +
             (double)s->computeOffset[3 * c + 1] * s->lattice[3 + a] +
             (double)s->computeOffset[3 * c + 2] * s->lattice[6 + a];
  const int dim = s->vdwDim;
  double L = 0.0;
  for (int a = 0; a < P1[0]; ++a) {
    const int i = P1[2] + a;
    const float* xi = s->xyzq + 4 * (size_t)i;
    float xs[3] = {xi[0] + sh[0], xi[1] + sh[1], xi[2] + sh[2]};
    for (int b = self ? a + 1 : 0; b < P2[0]; ++b) {
      const int j = P2[2] + b;
      if (onlySlot >= 0 && i != onlySlot && j != onlySlot) continue;
      const float* xj = s->xyzq + 4 * (size_t)j;
      const float r2f = r2_f32(xs, xj);
      if (!(r2f < s->cutoff2f) || !(r2f < s->plcutoff2f)) continue;
      if (!(b < P2[1] || a < P1[1])) continue;
      if (excluded(s, i, j)) continue;
      double d[3], uF[3], uS[3], pF = 0, pS = 0;
      for (int q = 0; q < 3; ++q) {
        d[q] = (double)xj[q] - ((double)xi[q] + shd[q]);
        uF[q] = cot->wF[3 * (size_t)i + q] - cot->wF[3 * (size_t)j + q];
        uS[q] = cot->wS[3 * (size_t)i + q] - cot->wS[3 * (size_t)j + q];
        pF += uF[q] * d[q];
        pS += uS[q] * d[q];
      }
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const int ti = s->vdwTypes[i], tj = s->vdwTypes[j];
      const double A = s->ljA[ti * dim + tj] * s->scaling, B = s->ljB[ti * dim + tj] * s->scaling;
      const double qi = xi[3], qj = xj[3], qq = qi * qj;
      double glj, dglj, gA, gB, EA, EB, gf, dgf, gsl, dgsl, phf, phs;
      pair_second(k, r2, A, B, &glj, &dglj, &gA, &gB, &EA, &EB, &gf, &dgf, &gsl, &dgsl, &phf, &phs);
      const double g = glj + qq * gf, gs = qq * gsl;
      L += pF * g + pS * gs + cot->cV * (A * EA + B * EB) + cot->cE * qq * phf + cot->cS * qq * phs;
      if (gX) {
        const double dg = dglj + qq * dgf, dgs = qq * dgsl;
        const double radial = 2.0 * (pF * dg + pS * dgs) + cot->cV * glj + cot->cE * qq * gf +
                              cot->cS * qq * gsl;
        for (int q = 0; q < 3; ++q) {
          const double v = g * uF[q] + gs * uS[q] + radial * d[q];
          gX[3 * (size_t)j + q] += v;
          gX[3 * (size_t)i + q] -= v;
        }
      }
      if (gQ) {
        const double dqq = pF * gf + pS * gsl + cot->cE * phf + cot->cS * phs;
        gQ[i] += qj * dqq;
        gQ[j] += qi * dqq;
      }
      if (gA_) {
        /* d/dA and d/dB of the scaled table entries (ti, tj) */
        gA_[ti * dim + tj] += pF * gA + cot->cV * EA;
        gB_[ti * dim + tj] += pF * gB + cot->cV * EB;
      }
    }
  }
  return L;
}

/* Whole loss and (optionally) its FP64 gradient: gX [3*storage], gQ [storage]
 * (w.r.t. the scaled charges in xyzq.w), gA/gB [dim*dim] (w.r.t. the scaled
 * LJ table entries, ordered type pair (ti, tj) of i before j). */
double oracle_adjoint(const oracle_system* s, const double* wF, const double* wS, double cV,
                      double cE, double cS, double* gX, double* gQ, double* gA, double* gB) {
  const pair_consts k = make_consts(s);
  const oracle_cot cot = {wF, wS, cV, cE, cS};
  const size_t n = (size_t)s->atomStorageSize, d2 = (size_t)s->vdwDim * s->vdwDim;
  if (gX) memset(gX, 0, 3 * n * sizeof(double));
  if (gQ) memset(gQ, 0, n * sizeof(double));
  if (gA) memset(gA, 0, d2 * sizeof(double));
  if (gB) memset(gB, 0, d2 * sizeof(double));
  double L = 0.0;
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  double* bX = gX ? (double*)calloc(3 * n * nthreads, sizeof(double)) : NULL;
  double* bQ = gQ ? (double*)calloc(n * nthreads, sizeof(double)) : NULL;
  double* bA = gA ? (double*)calloc(d2 * nthreads, sizeof(double)) : NULL;
  double* bB = gB ? (double*)calloc(d2 * nthreads, sizeof(double)) : NULL;
#pragma omp parallel reduction(+ : L)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
#pragma omp for schedule(dynamic, 4)
    for (int c = 0; c < s->numComputes; ++c)
      L += adjoint_compute(s, &k, c, &cot, -1, bX ? bX + 3 * n * tid : NULL, bQ ? bQ + n * tid : NULL,
                           bA ? bA + d2 * tid : NULL, bB ? bB + d2 * tid : NULL);
  }
  for (int t = 0; t < nthreads; ++t) {
    if (gX) for (size_t q = 0; q < 3 * n; ++q) gX[q] += bX[3 * n * t + q];
    if (gQ) for (size_t q = 0; q < n; ++q) gQ[q] += bQ[n * t + q];
    if (gA) for (size_t q = 0; q < d2; ++q) gA[q] += bA[d2 * t + q];
    if (gB) for (size_t q = 0; q < d2; ++q) gB[q] += bB[d2 * t + q];
  }
  free(bX);
  free(bQ);
  free(bA);
  free(bB);
  return L;
}

/* The part of the loss from pairs that involve slot `slot` (for central
 * differences in that atom's position or charge). */
double oracle_loss_local(const oracle_system* s, int slot, const double* wF, const double* wS,
                         double cV, double cE, double cS) {
  const pair_consts k = make_consts(s);
  const oracle_cot cot = {wF, wS, cV, cE, cS};
  double L = 0.0;
  for (int c = 0; c < s->numComputes; ++c) {
    const int p1 = s->computePatch[2 * c], p2 = s->computePatch[2 * c + 1];
    const int* P1 = s->patches + 4 * p1;
    const int* P2 = s->patches + 4 * p2;
    const int in1 = slot >= P1[2] && slot < P1[2] + P1[0];
    const int in2 = slot >= P2[2] && slot < P2[2] + P2[0];
    if (in1 || in2) L += adjoint_compute(s, &k, c, &cot, slot, NULL, NULL, NULL, NULL);
  }
  return L;
}

/* Number of pairs of slot `slot` whose FP32 r^2 lies within `tol` of the
 * cutoff^2 (central differences across such pairs are not meaningful). */
int oracle_near_cutoff(const oracle_system* s, int slot, float tol) {
  int n = 0;
  for (int c = 0; c < s->numComputes; ++c) {
    const int p1 = s->computePatch[2 * c], p2 = s->computePatch[2 * c + 1];
    const int* P1 = s->patches + 4 * p1;
    const int* P2 = s->patches + 4 * p2;
    float sh[3];
    shift_f32(s, c, sh);
    const int zeroShift = !(fmaf(sh[2], sh[2], fmaf(sh[0], sh[0], sh[1] * sh[1])) > 0.0f);
    const int self = (p1 == p2) && zeroShift;
    for (int a = 0; a < P1[0]; ++a) {
      const int i = P1[2] + a;
      const float* xi = s->xyzq + 4 * (size_t)i;
      float xs[3] = {xi[0] + sh[0], xi[1] + sh[1], xi[2] + sh[2]};
      for (int b = self ? a + 1 : 0; b < P2[0]; ++b) {
        const int j = P2[2] + b;
        if (i != slot && j != slot) continue;
        const float r2 = r2_f32(xs, s->xyzq + 4 * (size_t)j);
        if (fabsf(r2 - s->cutoff2f) < tol) ++n;
      }
    }
  }
  return n;
}
