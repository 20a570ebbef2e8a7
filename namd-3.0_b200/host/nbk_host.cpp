// Host-side preparation of the nonbonded path's inputs (see include/nbk_host.h
// for the reference functions each part mirrors) and the seeded synthetic
// system generator used by the tests and the benchmark.
#include "nbk_host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

namespace {

thread_local std::string g_host_err;

int fail(int code, const std::string& msg) {
  g_host_err = msg;
  return code;
}

// ---- random numbers: splitmix64 seeding + xoshiro256** stream ----------------
struct Rng {
  uint64_t s[4];
  bool haveSpare = false;
  double spare = 0.0;
  explicit Rng(uint64_t seed) {
    uint64_t z = seed;
    for (int i = 0; i < 4; ++i) {
      z += 0x9E3779B97F4A7C15ull;
      uint64_t x = z;
      x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
      x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
      s[i] = x ^ (x >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  int below(int n) { return (int)(uniform() * n); }
  double normal() {  // Marsaglia polar method
    if (haveSpare) {
      haveSpare = false;
      return spare;
    }
    double u, v, q;
    do {
      u = 2.0 * uniform() - 1.0;
      v = 2.0 * uniform() - 1.0;
      q = u * u + v * v;
    } while (q >= 1.0 || q == 0.0);
    const double m = std::sqrt(-2.0 * std::log(q) / q);
    spare = v * m;
    haveSpare = true;
    return u * m;
  }
};

double wrap1(double x, double L) {
  double y = std::fmod(x, L);
  if (y < 0) y += L;
  if (y >= L) y -= L;
  return y;
}

// Uniform-random cell grid over a periodic box for minimum-distance queries.
struct CellGrid {
  double L[3];
  int n[3];
  double cs[3];
  std::vector<std::vector<int>> cells;
  const std::vector<double>* pos;
  CellGrid(const double box[3], double cutoff, const std::vector<double>* p) : pos(p) {
    for (int d = 0; d < 3; ++d) {
      L[d] = box[d];
      n[d] = std::max(1, (int)std::floor(box[d] / cutoff));
      cs[d] = box[d] / n[d];
    }
    cells.resize((size_t)n[0] * n[1] * n[2]);
  }
  int cellOf(const double* x, int c[3]) const {
    for (int d = 0; d < 3; ++d) {
      int k = (int)std::floor(x[d] / cs[d]);
      k %= n[d];
      if (k < 0) k += n[d];
      c[d] = k;
    }
    return c[0] + n[0] * (c[1] + n[1] * c[2]);
  }
  void insert(int idx) {
    int c[3];
    cells[cellOf(&(*pos)[3 * idx], c)].push_back(idx);
  }
  void erase(int idx) {
    int c[3];
    auto& v = cells[cellOf(&(*pos)[3 * idx], c)];
    for (size_t k = 0; k < v.size(); ++k)
      if (v[k] == idx) {
        v[k] = v.back();
        v.pop_back();
        return;
      }
  }
  // true if any stored point other than `skip` lies closer than r to x
  bool anyWithin(const double* x, double r, int skip) const {
    int c[3];
    cellOf(x, c);
    const double r2 = r * r;
    // distinct neighbour cells (a dimension with < 3 cells wraps onto itself)
    int ids[27], nid = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int cx = (c[0] + dx + n[0]) % n[0];
          const int cy = (c[1] + dy + n[1]) % n[1];
          const int cz = (c[2] + dz + n[2]) % n[2];
          const int id = cx + n[0] * (cy + n[1] * cz);
          bool seen = false;
          for (int k = 0; k < nid; ++k) seen |= (ids[k] == id);
          if (!seen) ids[nid++] = id;
        }
    for (int k = 0; k < nid; ++k) {
      for (int j : cells[ids[k]]) {
        if (j == skip) continue;
        double d2 = 0;
        for (int d = 0; d < 3; ++d) {
          double dd = (*pos)[3 * j + d] - x[d];
          dd -= L[d] * std::nearbyint(dd / L[d]);
          d2 += dd * dd;
        }
        if (d2 < r2) return true;
      }
    }
    return false;
  }
};

constexpr double kOH = 0.9572;
constexpr double kHOH = 104.52 * M_PI / 180.0;
constexpr double kQO = -0.834, kQH = 0.417;
constexpr double kSigmaO = 3.1507, kEpsO = 0.1521;

// Places one water: O at site, random orientation (uniform quaternion).
void placeWater(Rng& rng, const double site[3], double out[9]) {
  const double u1 = rng.uniform(), u2 = rng.uniform(), u3 = rng.uniform();
  const double a = std::sqrt(1 - u1), b = std::sqrt(u1);
  const double qx = a * std::sin(2 * M_PI * u2), qy = a * std::cos(2 * M_PI * u2);
  const double qz = b * std::sin(2 * M_PI * u3), qw = b * std::cos(2 * M_PI * u3);
  const double R[3][3] = {
      {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw)},
      {2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw)},
      {2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)}};
  const double hs = kOH * std::sin(0.5 * kHOH), hc = kOH * std::cos(0.5 * kHOH);
  const double body[3][3] = {{0, 0, 0}, {hs, hc, 0}, {-hs, hc, 0}};
  for (int k = 0; k < 3; ++k)
    for (int d = 0; d < 3; ++d)
      out[3 * k + d] = site[d] + R[d][0] * body[k][0] + R[d][1] * body[k][1] + R[d][2] * body[k][2];
}

}  // namespace

struct nbk_system_s {
  int natoms = 0, ntypes = 0, nwater = 0, nsolute = 0;
  double box[3] = {0, 0, 0};
  std::vector<double> pos, charge, sigma, epsilon;
  std::vector<int> type, fullExcl, modPairs;
};

struct nbk_packed_s {
  nbk_packed_view v{};
  int grid[3] = {0, 0, 0};
  double box[3] = {0, 0, 0};
  double qscale = 0;
  std::vector<nbk_patch_record> patches;
  std::vector<nbk_compute_record> computes;
  std::vector<nbk_float4> xyzq;
  std::vector<int> vdwTypes, atomIndex, slotOfAtom, patchOfAtom;
  std::vector<nbk_int2> exclIndexMaxDiff;
  std::vector<unsigned int> bits;
  std::vector<nbk_exclusion> modified, excluded;
  std::vector<double> centers;
  std::vector<std::vector<int>> patchAtoms;  // slot order of each patch
  std::vector<std::pair<int, int>> modPairsGlobal, exclPairsGlobal;
  // replicas: a single packing is replica 0
  std::vector<int> replicaOfCompute, replicaSlotStart, replicaAtomStart;
  std::vector<nbk_float3> replicaLattice;
  bool many = false;
};

extern "C" {

// ---------------------------------------------------------------------------
// Synthetic systems
// ---------------------------------------------------------------------------
NBK_API int nbk_system_generate(int kind, uint64_t seed, int natoms, double solute_frac,
                                const double* boxIn, nbk_system* out) {
  if (!out) return fail(NBK_ERR_ARG, "nbk_system_generate: out is NULL");
  if (natoms < 3) return fail(NBK_ERR_ARG, "nbk_system_generate: natoms < 3");
  if (kind != NBK_SYS_WATER && kind != NBK_SYS_MIXED)
    return fail(NBK_ERR_ARG, "nbk_system_generate: unknown kind");
  nbk_system_s* S = new (std::nothrow) nbk_system_s;
  if (!S) return fail(NBK_ERR_NOMEM, "nbk_system_generate: out of memory");
  Rng rng(seed);
  double box[3];
  if (!boxIn || boxIn[0] <= 0) {
    const double side = std::cbrt(natoms / 0.1);
    box[0] = box[1] = box[2] = side;
  } else {
    for (int d = 0; d < 3; ++d) box[d] = boxIn[d];
  }
  for (int d = 0; d < 3; ++d) S->box[d] = box[d];

  int nwater, nsolute;
  if (kind == NBK_SYS_WATER) {
    if (natoms % 3) {
      delete S;
      return fail(NBK_ERR_ARG, "nbk_system_generate: water system needs natoms % 3 == 0");
    }
    nwater = natoms / 3;
    nsolute = 0;
  } else {
    if (solute_frac < 0 || solute_frac > 1) {
      delete S;
      return fail(NBK_ERR_ARG, "nbk_system_generate: solute_frac outside [0,1]");
    }
    nwater = (int)std::lround((1.0 - solute_frac) * natoms / 3.0);
    nsolute = natoms - 3 * nwater;
    if (nsolute < 0) {
      nwater = natoms / 3;
      nsolute = natoms - 3 * nwater;
    }
  }
  S->natoms = natoms;
  S->nwater = nwater;
  S->nsolute = nsolute;
  S->pos.assign(3 * (size_t)natoms, 0.0);
  S->charge.assign(natoms, 0.0);
  S->type.assign(natoms, 0);

  // LJ types: 32 solute types (MIXED), then water O, then water H (no LJ).
  const int nsolTypes = (kind == NBK_SYS_MIXED) ? 32 : 0;
  S->ntypes = nsolTypes + 2;
  S->sigma.assign(S->ntypes, 0.0);
  S->epsilon.assign(S->ntypes, 0.0);
  for (int t = 0; t < nsolTypes; ++t) {
    S->sigma[t] = rng.uniform(2.0, 4.0);
    S->epsilon[t] = rng.uniform(0.02, 0.2);
  }
  const int typeO = nsolTypes, typeH = nsolTypes + 1;
  S->sigma[typeO] = kSigmaO;
  S->epsilon[typeO] = kEpsO;

  // ---- solute: self-avoiding random-walk chains of 200 atoms ----------------
  std::vector<double> solPos;  // 3*nsolute
  if (nsolute > 0) {
    solPos.assign(3 * (size_t)nsolute, 0.0);
    CellGrid grid(box, 2.5, &solPos);
    double minDist = 2.5;
    const double step = 1.5;
    int placed = 0;
    int chainStart = 0;
    int failures = 0;
    while (placed < nsolute) {
      const int len = std::min(200, nsolute - chainStart);
      bool ok = true;
      for (int k = 0; k < len; ++k) {
        const int idx = chainStart + k;
        double x[3];
        bool found = false;
        for (int attempt = 0; attempt < 400 && !found; ++attempt) {
          if (k == 0) {
            for (int d = 0; d < 3; ++d) x[d] = rng.uniform(0.0, box[d]);
          } else {
            double u[3], n2;
            do {
              for (int d = 0; d < 3; ++d) u[d] = rng.uniform(-1.0, 1.0);
              n2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
            } while (n2 > 1.0 || n2 < 1e-6);
            const double s = step / std::sqrt(n2);
            for (int d = 0; d < 3; ++d) x[d] = wrap1(solPos[3 * (idx - 1) + d] + s * u[d], box[d]);
          }
          for (int d = 0; d < 3; ++d) solPos[3 * idx + d] = x[d];
          // only the bonded predecessor may be closer than minDist
          found = !grid.anyWithin(x, minDist, k > 0 ? idx - 1 : -1);
        }
        if (!found) {
          ok = false;
          break;
        }
        grid.insert(idx);
        placed = idx + 1;
      }
      if (!ok) {
        // remove the partial chain and retry; relax the spacing if the box jams
        for (int idx = chainStart; idx < placed; ++idx) grid.erase(idx);
        placed = chainStart;
        if (++failures % 20 == 0) minDist *= 0.97;
        continue;
      }
      chainStart += len;
    }
    for (int i = 0; i < nsolute; ++i) {
      for (int d = 0; d < 3; ++d) S->pos[3 * i + d] = solPos[3 * i + d];
      S->type[i] = rng.below(nsolTypes);
    }
    // charges N(0, 0.3) shifted to a neutral total
    double sum = 0;
    for (int i = 0; i < nsolute; ++i) {
      S->charge[i] = 0.3 * rng.normal();
      sum += S->charge[i];
    }
    for (int i = 0; i < nsolute; ++i) S->charge[i] -= sum / nsolute;
    // exclusions 1-2, 1-3 and modified 1-4 along each chain
    for (int c0 = 0; c0 < nsolute; c0 += 200) {
      const int len = std::min(200, nsolute - c0);
      for (int k = 0; k < len; ++k) {
        const int i = c0 + k;
        if (k + 1 < len) S->fullExcl.insert(S->fullExcl.end(), {i, i + 1});
        if (k + 2 < len) S->fullExcl.insert(S->fullExcl.end(), {i, i + 2});
        if (k + 3 < len) S->modPairs.insert(S->modPairs.end(), {i, i + 3});
      }
    }
  }

  // ---- waters on a jittered lattice, uniform random orientations -------------
  if (nwater > 0) {
    std::vector<double> sites;
    const double vol = box[0] * box[1] * box[2];
    if (nsolute == 0) {
      // grid n_x * n_y * n_z with cells near the mean volume per water; the
      // first nwater sites (x fastest) are used.
      const double a = std::cbrt(vol / nwater);
      const int nx = std::max(1, (int)std::ceil(box[0] / a - 1e-9));
      const int ny = std::max(1, (int)std::ceil(box[1] / a - 1e-9));
      const int nz = std::max(1, (nwater + nx * ny - 1) / (nx * ny));
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            if ((int)(sites.size() / 3) >= nwater) break;
            sites.push_back((i + 0.5) * box[0] / nx);
            sites.push_back((j + 0.5) * box[1] / ny);
            sites.push_back((k + 0.5) * box[2] / nz);
          }
      for (size_t s = 0; s < sites.size(); ++s) sites[s] += rng.uniform(-0.2, 0.2);
    } else {
      // candidate sites on a finer jittered lattice, rejecting overlaps with
      // the solute; nwater of the survivors are drawn at random.
      CellGrid grid(box, 2.5, &solPos);
      for (int i = 0; i < nsolute; ++i) grid.insert(i);
      double ncand = 1.5 * nwater;
      for (int round = 0; round < 40; ++round) {
        sites.clear();
        const double a = std::cbrt(vol / ncand);
        int n[3];
        for (int d = 0; d < 3; ++d) n[d] = std::max(1, (int)std::floor(box[d] / a));
        for (int k = 0; k < n[2]; ++k)
          for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
              double x[3] = {(i + 0.5) * box[0] / n[0] + rng.uniform(-0.2, 0.2),
                             (j + 0.5) * box[1] / n[1] + rng.uniform(-0.2, 0.2),
                             (k + 0.5) * box[2] / n[2] + rng.uniform(-0.2, 0.2)};
              for (int d = 0; d < 3; ++d) x[d] = wrap1(x[d], box[d]);
              if (grid.anyWithin(x, 2.0, -1)) continue;
              sites.insert(sites.end(), {x[0], x[1], x[2]});
            }
        if ((int)(sites.size() / 3) >= nwater) break;
        ncand *= 1.25;
      }
      const int nsites = (int)(sites.size() / 3);
      if (nsites < nwater) {
        delete S;
        return fail(NBK_ERR_ARG, "nbk_system_generate: could not place the waters");
      }
      // partial Fisher-Yates draw of nwater sites
      std::vector<int> idx(nsites);
      for (int i = 0; i < nsites; ++i) idx[i] = i;
      std::vector<double> chosen(3 * (size_t)nwater);
      for (int w = 0; w < nwater; ++w) {
        const int r = w + rng.below(nsites - w);
        std::swap(idx[w], idx[r]);
        for (int d = 0; d < 3; ++d) chosen[3 * w + d] = sites[3 * idx[w] + d];
      }
      sites.swap(chosen);
    }
    for (int w = 0; w < nwater; ++w) {
      double xyz[9];
      placeWater(rng, &sites[3 * w], xyz);
      const int o = nsolute + 3 * w;
      for (int k = 0; k < 3; ++k)
        for (int d = 0; d < 3; ++d) S->pos[3 * (o + k) + d] = wrap1(xyz[3 * k + d], box[d]);
      S->charge[o] = kQO;
      S->charge[o + 1] = kQH;
      S->charge[o + 2] = kQH;
      S->type[o] = typeO;
      S->type[o + 1] = typeH;
      S->type[o + 2] = typeH;
      S->fullExcl.insert(S->fullExcl.end(), {o, o + 1, o, o + 2, o + 1, o + 2});
    }
  }
  *out = S;
  return NBK_OK;
}

NBK_API int nbk_system_view_get(nbk_system S, nbk_system_view* v) {
  if (!S || !v) return fail(NBK_ERR_ARG, "nbk_system_view_get: NULL argument");
  v->natoms = S->natoms;
  v->ntypes = S->ntypes;
  v->numFullExclPairs = (int)(S->fullExcl.size() / 2);
  v->numModPairs = (int)(S->modPairs.size() / 2);
  v->numWaters = S->nwater;
  v->numSolute = S->nsolute;
  for (int d = 0; d < 3; ++d) v->box[d] = S->box[d];
  v->pos = S->pos.data();
  v->charge = S->charge.data();
  v->type = S->type.data();
  v->sigma = S->sigma.data();
  v->epsilon = S->epsilon.data();
  v->fullExcl = S->fullExcl.empty() ? nullptr : S->fullExcl.data();
  v->modPairs = S->modPairs.empty() ? nullptr : S->modPairs.data();
  return NBK_OK;
}

NBK_API int nbk_system_perturb(nbk_system S, uint64_t seed, double sigma) {
  if (!S) return fail(NBK_ERR_ARG, "nbk_system_perturb: NULL system");
  Rng rng(seed);
  for (int i = 0; i < S->natoms; ++i)
    for (int d = 0; d < 3; ++d)
      S->pos[3 * i + d] = wrap1(S->pos[3 * i + d] + sigma * rng.normal(), S->box[d]);
  return NBK_OK;
}

NBK_API int nbk_system_free(nbk_system S) {
  delete S;
  return NBK_OK;
}

// LJTable::compute_vdw_params (src/LJTable.C:115-133): Lorentz-Berthelot or
// geometric sigma, eps_ij = sqrt(eps_i eps_j), B = 4 eps sigma^6, A = B sigma^6.
NBK_API int nbk_lj_table(int ntypes, const double* sigma, const double* epsilon, int geometric,
                         double* A, double* B, double* A14, double* B14) {
  if (ntypes <= 0 || !sigma || !epsilon || !A || !B)
    return fail(NBK_ERR_ARG, "nbk_lj_table: bad argument");
  for (int i = 0; i < ntypes; ++i)
    for (int j = 0; j < ntypes; ++j) {
      double s = geometric ? std::sqrt(sigma[i] * sigma[j]) : 0.5 * (sigma[i] + sigma[j]);
      const double e = std::sqrt(epsilon[i] * epsilon[j]);
      const double s6 = s * s * s * s * s * s;
      const double b = 4.0 * s6 * e;
      A[i * ntypes + j] = b * s6;
      B[i * ntypes + j] = b;
      if (A14) A14[i * ntypes + j] = b * s6;
      if (B14) B14[i * ntypes + j] = b;
    }
  return NBK_OK;
}

// Chain rule from gradients w.r.t. the scaled LJ table entries (A*scaling,
// B*scaling at ordered type pair (i, j)) to per-type sigma and epsilon, for the
// combining rule of nbk_lj_table (LJTable::compute_vdw_params).
NBK_API int nbk_lj_param_grad(int ntypes, const double* sigma, const double* epsilon, int geometric,
                              double scaling, const double* gA, const double* gB, double* gSigma,
                              double* gEps) {
  if (ntypes <= 0 || !sigma || !epsilon || !gA || !gB || !gSigma || !gEps)
    return fail(NBK_ERR_ARG, "nbk_lj_param_grad: bad argument");
  for (int t = 0; t < ntypes; ++t) gSigma[t] = gEps[t] = 0.0;
  for (int i = 0; i < ntypes; ++i)
    for (int j = 0; j < ntypes; ++j) {
      const double ga = gA[i * ntypes + j] * scaling, gb = gB[i * ntypes + j] * scaling;
      if (ga == 0.0 && gb == 0.0) continue;
      const double s = geometric ? std::sqrt(sigma[i] * sigma[j]) : 0.5 * (sigma[i] + sigma[j]);
      const double e = std::sqrt(epsilon[i] * epsilon[j]);
      const double s5 = s * s * s * s * s, s6 = s5 * s, s11 = s6 * s5, s12 = s6 * s6;
      // A = 4 e s^12, B = 4 e s^6
      const double dLds = ga * 48.0 * e * s11 + gb * 24.0 * e * s5;
      const double dLde = ga * 4.0 * s12 + gb * 4.0 * s6;
      // d s / d sigma_i (and _j), d e / d eps_i (and _j)
      const double dsi = geometric ? (sigma[i] > 0 ? 0.5 * s / sigma[i] : 0.0) : 0.5;
      const double dsj = geometric ? (sigma[j] > 0 ? 0.5 * s / sigma[j] : 0.0) : 0.5;
      const double dei = epsilon[i] > 0 ? 0.5 * e / epsilon[i] : 0.0;
      const double dej = epsilon[j] > 0 ? 0.5 * e / epsilon[j] : 0.0;
      gSigma[i] += dLds * dsi;
      gSigma[j] += dLds * dsj;
      gEps[i] += dLde * dei;
      gEps[j] += dLde * dej;
    }
  return NBK_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Packing
// ---------------------------------------------------------------------------
namespace {

// Orthogonal recursive bisection of one patch's atoms into compact tiles:
// splits only at multiples of 32 (then 16, then 8) nearest the median, along
// the longest extent of the current range. Compact 32-atom tiles make the
// tile bounding boxes tight; the finer 16/8 splits keep the quarter tiles
// compact too.
void orbPartition(std::vector<int>& ord, const double* pos, int begin, int end) {
  int W = 0;
  for (int w : {32, 16, 8})
    if (begin / w < (end - 1) / w) {
      W = w;
      break;
    }
  if (W == 0) return;
  int split = ((begin + end + W) / (2 * W)) * W;
  if (split <= begin) split += W;
  if (split >= end) split -= W;
  if (split <= begin || split >= end) return;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int k = begin; k < end; ++k)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], pos[3 * ord[k] + d]);
      hi[d] = std::max(hi[d], pos[3 * ord[k] + d]);
    }
  int axis = 0;
  for (int d = 1; d < 3; ++d)
    if (hi[d] - lo[d] > hi[axis] - lo[axis]) axis = d;
  std::nth_element(ord.begin() + begin, ord.begin() + split, ord.begin() + end, [&](int a, int b) {
    const double xa = pos[3 * a + axis], xb = pos[3 * b + axis];
    return xa < xb || (xa == xb && a < b);
  });
  orbPartition(ord, pos, begin, split);
  orbPartition(ord, pos, split, end);
}

void fillXyzq(nbk_packed_s* P, const nbk_system_s* S) {
  for (int p = 0; p < (int)P->patchAtoms.size(); ++p) {
    const auto& atoms = P->patchAtoms[p];
    const int start = P->patches[p].atomStart;
    const int n = (int)atoms.size();
    if (n == 0) continue;
    const int padded = ((n + 31) / 32) * 32;
    for (int k = 0; k < padded; ++k) {
      const int a = atoms[std::min(k, n - 1)];
      nbk_float4 q;
      float* f = &q.x;
      for (int d = 0; d < 3; ++d) {
        // minimum-image offset from the patch centre (atoms may have drifted
        // across the periodic boundary since the patches were assigned)
        double x = S->pos[3 * a + d] - P->centers[3 * p + d];
        x -= P->box[d] * std::nearbyint(x / P->box[d]);
        f[d] = (float)x;
      }
      q.w = (float)(P->qscale * S->charge[a]);
      P->xyzq[start + k] = q;
    }
  }
}

// Per-tuple i-shift so that xyzq[i] + shift - xyzq[j] is the minimum image of
// x_i - x_j (CudaExclusion::ioffsetXYZ semantics, lattice units).
nbk_exclusion makeTuple(const nbk_packed_s* P, const nbk_system_s* S, int a, int b) {
  nbk_exclusion e;
  e.i = P->slotOfAtom[a];
  e.j = P->slotOfAtom[b];
  e.vdwtypei = S->type[a];
  e.vdwtypej = S->type[b];
  e.pswitch = 0;
  const int pa = P->patchOfAtom[a], pb = P->patchOfAtom[b];
  float* o = &e.ioffsetXYZ.x;
  for (int d = 0; d < 3; ++d) {
    const double L = P->box[d];
    double dx = S->pos[3 * a + d] - S->pos[3 * b + d];
    const double image = std::nearbyint(dx / L);
    o[d] = (float)((P->centers[3 * pa + d] - P->centers[3 * pb + d]) / L - image);
  }
  return e;
}

}  // namespace

extern "C" {

NBK_API int nbk_pack(nbk_system S, double patchDim, double coulombScaling, nbk_packed* out) {
  if (!S || !out || patchDim <= 0) return fail(NBK_ERR_ARG, "nbk_pack: bad argument");
  nbk_packed_s* P = new (std::nothrow) nbk_packed_s;
  if (!P) return fail(NBK_ERR_NOMEM, "nbk_pack: out of memory");
  for (int d = 0; d < 3; ++d) {
    P->box[d] = S->box[d];
    P->grid[d] = (int)std::floor(S->box[d] / patchDim);
    if (P->grid[d] < 2) {
      delete P;
      return fail(NBK_ERR_ARG,
                  "nbk_pack: box must be at least 2 patch dimensions wide in every direction");
    }
  }
  P->qscale = std::sqrt(332.0636 * coulombScaling);
  const int nx = P->grid[0], ny = P->grid[1], nz = P->grid[2];
  const int np = nx * ny * nz;
  P->patchAtoms.assign(np, {});
  P->centers.assign(3 * (size_t)np, 0.0);
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) {
        const int p = ix + nx * (iy + ny * iz);
        P->centers[3 * p + 0] = (ix + 0.5) * S->box[0] / nx;
        P->centers[3 * p + 1] = (iy + 0.5) * S->box[1] / ny;
        P->centers[3 * p + 2] = (iz + 0.5) * S->box[2] / nz;
      }
  P->patchOfAtom.assign(S->natoms, 0);
  for (int a = 0; a < S->natoms; ++a) {
    int c[3];
    for (int d = 0; d < 3; ++d) {
      int k = (int)std::floor(S->pos[3 * a + d] / (S->box[d] / P->grid[d]));
      c[d] = std::min(std::max(k, 0), P->grid[d] - 1);
    }
    const int p = c[0] + nx * (c[1] + ny * c[2]);
    P->patchOfAtom[a] = p;
    P->patchAtoms[p].push_back(a);
  }
  // per-patch spatial order, layout and padding
  P->patches.resize(np);
  int atomStart = 0, maxTiles = 0;
  for (int p = 0; p < np; ++p) {
    auto& atoms = P->patchAtoms[p];
    orbPartition(atoms, S->pos.data(), 0, (int)atoms.size());
    const int n = (int)atoms.size();
    const int ntiles = (n + 31) / 32;
    maxTiles = std::max(maxTiles, ntiles);
    P->patches[p].numAtoms = n;
    P->patches[p].numFreeAtoms = n;
    P->patches[p].atomStart = atomStart;
    P->patches[p].patchID = p;
    atomStart += ntiles * 32;
  }
  const int storage = atomStart;
  P->xyzq.assign(storage, nbk_float4{0, 0, 0, 0});
  P->vdwTypes.assign(storage, 0);
  P->atomIndex.assign(storage, 0);
  P->exclIndexMaxDiff.assign(storage, nbk_int2{0, 0});
  P->slotOfAtom.assign(S->natoms, -1);
  for (int p = 0; p < np; ++p)
    for (int k = 0; k < (int)P->patchAtoms[p].size(); ++k)
      P->slotOfAtom[P->patchAtoms[p][k]] = P->patches[p].atomStart + k;
  fillXyzq(P, S);

  // ---- exclusion bit array (buildExclusions restated) ---------------------
  // per-atom sorted offset list {0} U {partner - self}; unique lists in order
  // of first appearance, stable-sorted by maxdiff; list k owns 2*maxdiff+1 bits
  // centred at base_k.
  std::vector<std::vector<int>> partners(S->natoms);
  for (size_t k = 0; k + 1 < S->fullExcl.size(); k += 2) {
    const int a = S->fullExcl[k], b = S->fullExcl[k + 1];
    partners[a].push_back(b);
    partners[b].push_back(a);
  }
  std::map<std::vector<int>, int> listId;
  std::vector<std::vector<int>> uniq;
  std::vector<int> atomList(S->natoms);
  for (int a = 0; a < S->natoms; ++a) {
    std::vector<int> cur{0};
    for (int b : partners[a]) cur.push_back(b - a);
    std::sort(cur.begin(), cur.end());
    cur.erase(std::unique(cur.begin(), cur.end()), cur.end());
    auto it = listId.find(cur);
    if (it == listId.end()) {
      it = listId.emplace(cur, (int)uniq.size()).first;
      uniq.push_back(cur);
    }
    atomList[a] = it->second;
  }
  std::vector<int> maxdiff(uniq.size()), order(uniq.size());
  for (size_t k = 0; k < uniq.size(); ++k) {
    maxdiff[k] = std::max(-uniq[k].front(), uniq[k].back());
    order[k] = (int)k;
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return maxdiff[a] < maxdiff[b]; });
  std::vector<long long> base(uniq.size());
  long long totalbits = 0;
  for (int k : order) {
    base[k] = totalbits + maxdiff[k];
    totalbits += 2LL * maxdiff[k] + 1;
  }
  if (totalbits & 31) totalbits += 32 - (totalbits & 31);
  if (totalbits / 32 > (1LL << 27)) {
    delete P;
    return fail(NBK_ERR_OVERFLOW, "nbk_pack: exclusion bit array exceeds 2^27 words");
  }
  P->bits.assign((size_t)(totalbits / 32), 0u);
  for (size_t k = 0; k < uniq.size(); ++k)
    for (int off : uniq[k]) {
      const long long bit = base[k] + off;
      P->bits[bit >> 5] |= 1u << (bit & 31);
    }
  for (int p = 0; p < np; ++p) {
    const auto& atoms = P->patchAtoms[p];
    const int n = (int)atoms.size();
    if (!n) continue;
    const int padded = ((n + 31) / 32) * 32;
    for (int k = 0; k < padded; ++k) {
      const int a = atoms[std::min(k, n - 1)];
      const int slot = P->patches[p].atomStart + k;
      P->vdwTypes[slot] = S->type[a];
      P->atomIndex[slot] = a;
      P->exclIndexMaxDiff[slot] = nbk_int2{(int)base[atomList[a]], maxdiff[atomList[a]]};
    }
  }

  // ---- computes: self + 13 half-shell neighbours ---------------------------
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) {
        const int p = ix + nx * (iy + ny * iz);
        for (int dz = -1; dz <= 1; ++dz)
          for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
              // upper half: (dz, dy, dx) lexicographically >= 0
              if (dz < 0 || (dz == 0 && (dy < 0 || (dy == 0 && dx < 0)))) continue;
              const int qx = (ix + dx + nx) % nx, qy = (iy + dy + ny) % ny, qz = (iz + dz + nz) % nz;
              nbk_compute_record c;
              c.pad = 0;
              c.patchInd.x = p;
              c.patchInd.y = qx + nx * (qy + ny * qz);
              // center(p) - center(q) + image, in lattice units == -d / n
              c.offsetXYZ.x = (float)(-(double)dx / nx);
              c.offsetXYZ.y = (float)(-(double)dy / ny);
              c.offsetXYZ.z = (float)(-(double)dz / nz);
              P->computes.push_back(c);
            }
      }

  // ---- correction tuples --------------------------------------------------
  for (size_t k = 0; k + 1 < S->fullExcl.size(); k += 2) {
    P->exclPairsGlobal.emplace_back(S->fullExcl[k], S->fullExcl[k + 1]);
    P->excluded.push_back(makeTuple(P, S, S->fullExcl[k], S->fullExcl[k + 1]));
  }
  for (size_t k = 0; k + 1 < S->modPairs.size(); k += 2) {
    P->modPairsGlobal.emplace_back(S->modPairs[k], S->modPairs[k + 1]);
    P->modified.push_back(makeTuple(P, S, S->modPairs[k], S->modPairs[k + 1]));
  }

  P->replicaOfCompute.assign(P->computes.size(), 0);
  P->replicaSlotStart = {0, storage};
  P->replicaAtomStart = {0, S->natoms};
  P->replicaLattice = {nbk_float3{(float)S->box[0], 0.f, 0.f}, nbk_float3{0.f, (float)S->box[1], 0.f},
                       nbk_float3{0.f, 0.f, (float)S->box[2]}};
  nbk_packed_view& v = P->v;
  v.natoms = S->natoms;
  v.numPatches = np;
  for (int d = 0; d < 3; ++d) v.patchGrid[d] = P->grid[d];
  v.atomStorageSize = storage;
  v.maxTileListLen = maxTiles;
  v.numComputes = (int)P->computes.size();
  v.numExclusionWords = (int)P->bits.size();
  v.numModified = (int)P->modified.size();
  v.numExcluded = (int)P->excluded.size();
  v.lata = nbk_float3{(float)S->box[0], 0.f, 0.f};
  v.latb = nbk_float3{0.f, (float)S->box[1], 0.f};
  v.latc = nbk_float3{0.f, 0.f, (float)S->box[2]};
  v.patches = P->patches.data();
  v.computes = P->computes.data();
  v.xyzq = P->xyzq.data();
  v.vdwTypes = P->vdwTypes.data();
  v.atomIndex = P->atomIndex.data();
  v.exclIndexMaxDiff = P->exclIndexMaxDiff.data();
  v.exclusionBits = P->bits.data();
  v.modified = P->modified.empty() ? nullptr : P->modified.data();
  v.excluded = P->excluded.empty() ? nullptr : P->excluded.data();
  v.slotOfAtom = P->slotOfAtom.data();
  v.patchCenter = P->centers.data();
  v.numReplicas = 1;
  v.replicaOfCompute = P->replicaOfCompute.data();
  v.replicaSlotStart = P->replicaSlotStart.data();
  v.replicaAtomStart = P->replicaAtomStart.data();
  v.replicaLattice = P->replicaLattice.data();
  *out = P;
  return NBK_OK;
}

NBK_API int nbk_pack_many(const nbk_system* systems, int n, double patchDim, double coulombScaling,
                          nbk_packed* out) {
  if (!systems || n <= 0 || !out) return fail(NBK_ERR_ARG, "nbk_pack_many: bad argument");
  nbk_packed_s* M = new (std::nothrow) nbk_packed_s;
  if (!M) return fail(NBK_ERR_NOMEM, "nbk_pack_many: out of memory");
  M->many = true;
  int slotOff = 0, patchOff = 0, atomOff = 0, maxTiles = 0;
  long long bitOff = 0;
  M->replicaSlotStart.push_back(0);
  M->replicaAtomStart.push_back(0);
  for (int r = 0; r < n; ++r) {
    nbk_packed one = nullptr;
    int rc = nbk_pack(systems[r], patchDim, coulombScaling, &one);
    if (rc) {
      delete M;
      return rc;
    }
    const nbk_packed_view& v = one->v;
    for (int p = 0; p < v.numPatches; ++p) {
      nbk_patch_record pr = one->patches[p];
      pr.atomStart += slotOff;
      pr.patchID += patchOff;
      M->patches.push_back(pr);
      for (int d = 0; d < 3; ++d) M->centers.push_back(one->centers[3 * p + d]);
    }
    for (const nbk_compute_record& c : one->computes) {
      nbk_compute_record cc = c;
      cc.patchInd.x += patchOff;
      cc.patchInd.y += patchOff;
      M->computes.push_back(cc);
      M->replicaOfCompute.push_back(r);
    }
    for (int k = 0; k < v.atomStorageSize; ++k) {
      M->xyzq.push_back(one->xyzq[k]);
      M->vdwTypes.push_back(one->vdwTypes[k]);
      M->atomIndex.push_back(one->atomIndex[k] + atomOff);
      nbk_int2 e = one->exclIndexMaxDiff[k];
      e.x += (int)bitOff;
      M->exclIndexMaxDiff.push_back(e);
    }
    for (unsigned w : one->bits) M->bits.push_back(w);
    for (int a = 0; a < v.natoms; ++a) M->slotOfAtom.push_back(one->slotOfAtom[a] + slotOff);
    for (nbk_exclusion e : one->modified) {
      e.i += slotOff;
      e.j += slotOff;
      M->modified.push_back(e);
    }
    for (nbk_exclusion e : one->excluded) {
      e.i += slotOff;
      e.j += slotOff;
      M->excluded.push_back(e);
    }
    M->replicaLattice.push_back(v.lata);
    M->replicaLattice.push_back(v.latb);
    M->replicaLattice.push_back(v.latc);
    maxTiles = std::max(maxTiles, v.maxTileListLen);
    slotOff += v.atomStorageSize;
    patchOff += v.numPatches;
    atomOff += v.natoms;
    bitOff += 32LL * (long long)one->bits.size();
    M->replicaSlotStart.push_back(slotOff);
    M->replicaAtomStart.push_back(atomOff);
    nbk_packed_free(one);
  }
  if (bitOff > (1LL << 31)) {
    delete M;
    return fail(NBK_ERR_OVERFLOW, "nbk_pack_many: exclusion bit array exceeds 2^31 bits");
  }
  nbk_packed_view& v = M->v;
  v.natoms = atomOff;
  v.numPatches = patchOff;
  v.patchGrid[0] = v.patchGrid[1] = v.patchGrid[2] = 0;
  v.atomStorageSize = slotOff;
  v.maxTileListLen = maxTiles;
  v.numComputes = (int)M->computes.size();
  v.numExclusionWords = (int)M->bits.size();
  v.numModified = (int)M->modified.size();
  v.numExcluded = (int)M->excluded.size();
  v.lata = M->replicaLattice[0];
  v.latb = M->replicaLattice[1];
  v.latc = M->replicaLattice[2];
  v.patches = M->patches.data();
  v.computes = M->computes.data();
  v.xyzq = M->xyzq.data();
  v.vdwTypes = M->vdwTypes.data();
  v.atomIndex = M->atomIndex.data();
  v.exclIndexMaxDiff = M->exclIndexMaxDiff.data();
  v.exclusionBits = M->bits.data();
  v.modified = M->modified.empty() ? nullptr : M->modified.data();
  v.excluded = M->excluded.empty() ? nullptr : M->excluded.data();
  v.slotOfAtom = M->slotOfAtom.data();
  v.patchCenter = M->centers.data();
  v.numReplicas = n;
  v.replicaOfCompute = M->replicaOfCompute.data();
  v.replicaSlotStart = M->replicaSlotStart.data();
  v.replicaAtomStart = M->replicaAtomStart.data();
  v.replicaLattice = M->replicaLattice.data();
  *out = M;
  return NBK_OK;
}

NBK_API int nbk_packed_view_get(nbk_packed P, nbk_packed_view* v) {
  if (!P || !v) return fail(NBK_ERR_ARG, "nbk_packed_view_get: NULL argument");
  *v = P->v;
  return NBK_OK;
}

NBK_API int nbk_pack_update_positions(nbk_packed P, nbk_system S) {
  if (P && P->many) return fail(NBK_ERR_ARG, "nbk_pack_update_positions: not for nbk_pack_many layouts");
  if (!P || !S || S->natoms != P->v.natoms)
    return fail(NBK_ERR_ARG, "nbk_pack_update_positions: system does not match the packing");
  fillXyzq(P, S);
  for (size_t k = 0; k < P->exclPairsGlobal.size(); ++k)
    P->excluded[k] = makeTuple(P, S, P->exclPairsGlobal[k].first, P->exclPairsGlobal[k].second);
  for (size_t k = 0; k < P->modPairsGlobal.size(); ++k)
    P->modified[k] = makeTuple(P, S, P->modPairsGlobal[k].first, P->modPairsGlobal[k].second);
  return NBK_OK;
}

NBK_API int nbk_packed_free(nbk_packed P) {
  delete P;
  return NBK_OK;
}

NBK_API const char* nbk_host_last_error(void) { return g_host_err.c_str(); }

}  // extern "C"
