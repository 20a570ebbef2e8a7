// PME reciprocal space on one B200: charge spreading, the forward and backward
// 3-D FFTs, the influence-function solve with energy and virial, and the force
// gather (the C-ABI of include/nbk.h, nbk_pme_*).
//
// Reference behaviour followed (the single-device path):
//   - B-spline weights and grid offsets: calc_one_theta / calc_theta_dtheta and
//     spread_charge_kernel / gather_force, src/CudaPmeSolverUtilKernel.cu:
//     329-530,708-945. An atom at fractional u spreads to grid points
//     floor(K u) + k, k = 0..order-1, with weight theta_k(K u - floor(K u)).
//   - B-spline moduli: compute_b_moduli, src/PmeKSpace.C:22-61.
//   - Influence function, energy and virial: scalar_sum_kernel,
//     src/CudaPmeSolverUtilKernel.cu:74-325.
//   - Self energy: selfEnergyKernel, src/CudaPmeSolverUtilKernel.cu:1192-1216.
//
// Design for the B200: the charge grid is accumulated in 64-bit fixed point
// (2^-32 units) with integer atomics, so the grid, and everything computed from
// it, is bit-for-bit independent of the order in which atoms land (the
// reference accumulates FP32 atomics). One pass converts it to the FP32 grid
// cuFFT transforms and clears it for the next step. Energies and virials are
// reduced per block in FP64 and the block partials summed in a fixed order.
// Each atom's force is one thread's sum in a fixed order.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <string>
#include <vector>

#include "nbk.h"
#include "nbk_internal.cuh"
#include "nbk_launch.h"

namespace nbk {
namespace {

constexpr float kGridScale = 4294967296.0f;  // 2^32 fixed-point units per charge unit
constexpr int kSolveThreads = 256;
constexpr int kMaxOrder = 8;

struct Recip {
  double r[9];  // a_r, b_r, c_r (rows)
};

// Reciprocal vectors of the lattice a, b, c (Lattice::a_r/b_r/c_r): a_r =
// b x c / (a . (b x c)) and cyclically; returns the volume.
double reciprocal(const double* L, Recip& R) {
  const double *a = L, *b = L + 3, *c = L + 6;
  const double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
  const double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
  const double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  const double vol = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
  for (int d = 0; d < 3; ++d) {
    R.r[d] = bc[d] / vol;
    R.r[3 + d] = ca[d] / vol;
    R.r[6 + d] = ab[d] / vol;
  }
  return vol;
}

// B-spline weights theta_k(w), k = 0..order-1, by the cardinal B-spline
// recursion of smooth PME (Essmann et al., J. Chem. Phys. 103, 8577 (1995),
// eq. 4.1; the reference's calc_one_theta, src/CudaPmeSolverUtilKernel.cu:
// 331-359, uses the same): order 2 from w, raised one order at a time.
template <typename T, int order>
__host__ __device__ __forceinline__ void bsplineTheta(const T w, T* theta) {
  theta[order - 1] = T(0);
  theta[1] = w;
  theta[0] = T(1) - w;
#pragma unroll
  for (int k = 3; k <= order; ++k) {
    const T div = T(1) / T(k - 1);
    theta[k - 1] = div * w * theta[k - 2];
#pragma unroll
    for (int j = 1; j <= k - 2; ++j)
      theta[k - j - 1] = div * ((w + T(j)) * theta[k - j - 2] + (T(k - j) - w) * theta[k - j - 1]);
    theta[0] = div * (T(1) - w) * theta[0];
  }
}

// theta and its derivative d theta / dw (from the order-1 weights).
template <int order>
__device__ __forceinline__ void bsplineThetaD(const float w, float* theta, float* dtheta) {
  float t1[order];
  bsplineTheta<float, order - 1>(w, t1);
  dtheta[0] = -t1[0];
#pragma unroll
  for (int j = 1; j < order - 1; ++j) dtheta[j] = t1[j - 1] - t1[j];
  dtheta[order - 1] = t1[order - 2];
  bsplineTheta<float, order>(w, theta);
}

__device__ __forceinline__ void gridCell(const float4 a, int K1, int K2, int K3, int& ix, int& iy,
                                         int& iz, float& wx, float& wy, float& wz) {
  const float fx = (float)K1 * a.x, fy = (float)K2 * a.y, fz = (float)K3 * a.z;
  ix = (int)fx;
  iy = (int)fy;
  iz = (int)fz;
  wx = fx - (float)ix;
  wy = fy - (float)iy;
  wz = fz - (float)iz;
}

// One warp spreads 32 atoms: each lane computes its atom's weights into
// shared memory, then the warp walks the atoms, its lanes covering the
// order^3 grid points of one atom (point p = lane + 32 h, x fastest, so
// neighbouring lanes add to neighbouring addresses).
template <int order>
__global__ void __launch_bounds__(128) spreadKernel(int n, const float4* __restrict__ atoms, int K1,
                                                    int K2, int K3,
                                                    unsigned long long* __restrict__ grid) {
  constexpr int kPts = order * order * order;
  __shared__ float s_th[4][3][order][32];
  __shared__ int s_i[4][3][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
  for (int a0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; a0 < n; a0 += warpsPerGrid * 32) {
    const int i = a0 + lane;
    if (i < n) {
      const float4 at = atoms[i];
      int ix, iy, iz;
      float wx, wy, wz, t[order];
      gridCell(at, K1, K2, K3, ix, iy, iz, wx, wy, wz);
      bsplineTheta<float, order>(wx, t);
#pragma unroll
      for (int k = 0; k < order; ++k) s_th[wib][0][k][lane] = at.w * t[k];
      bsplineTheta<float, order>(wy, t);
#pragma unroll
      for (int k = 0; k < order; ++k) s_th[wib][1][k][lane] = t[k];
      bsplineTheta<float, order>(wz, t);
#pragma unroll
      for (int k = 0; k < order; ++k) s_th[wib][2][k][lane] = t[k];
      s_i[wib][0][lane] = ix;
      s_i[wib][1][lane] = iy;
      s_i[wib][2][lane] = iz;
    }
    __syncwarp();
    const int na = min(32, n - a0);
    const int K12 = K1 * K2;  // grid indices below 2^31 (checked at creation)
    for (int m = 0; m < na; ++m) {
      const int bx = s_i[wib][0][m], by = s_i[wib][1][m], bz = s_i[wib][2][m];
#pragma unroll
      for (int h = 0; h < (kPts + 31) / 32; ++h) {
        const int p = lane + 32 * h;
        if (kPts % 32 == 0 || p < kPts) {
          const int x0 = p % order, y0 = (p / order) % order, z0 = p / (order * order);
          int x = bx + x0, y = by + y0, z = bz + z0;
          if (x >= K1) x -= K1;
          if (y >= K2) y -= K2;
          if (z >= K3) z -= K3;
          const float v = s_th[wib][0][x0][m] * s_th[wib][1][y0][m] * s_th[wib][2][z0][m];
          // v 2^32 is exact in FP32 (a power-of-two scaling), so this is the
          // same integer as the FP64 product rounded to the nearest
          const long long q = __float2ll_rn(v * kGridScale);
          atomicAdd(&grid[x + K1 * y + K12 * z], (unsigned long long)q);
        }
      }
    }
    __syncwarp();
  }
}

// Fixed point -> FP32 grid for the FFT; clears the fixed-point grid.
__global__ void gridToFloatKernel(size_t n, unsigned long long* __restrict__ g,
                                  float* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    // rounding the integer to FP32, then the exact scaling by 2^-32
    out[i] = __ll2float_rn((long long)g[i]) * (1.0f / kGridScale);
    g[i] = 0ull;
  }
}

struct SolveArgs {
  int K1, K2, K3, nh;   // nh = K1/2 + 1
  double r[9];          // reciprocal vectors a_r, b_r, c_r
  double piEwald;       // (pi / beta)^2
  double pivInv;        // 1 / (pi V)
  const float* bm1;     // B-spline moduli factors 1/|b(k)|^2
  const float* bm2;
  const float* bm3;
  float2* data;         // (K3, K2, nh), x fastest
  double* partial;      // [blocks][7]: energy, virial xx xy xz yy yz zz
  double* ev;           // energy, virial[9] (row-major)
  int* done;            // blocks finished (the last one sums the partials, resets it)
  int doEV;
};

// Influence function on the half-complex grid and, when asked, the block's
// energy and virial partial sums (scalar_sum_kernel's formulas).
__global__ void __launch_bounds__(kSolveThreads) solveKernel(const __grid_constant__ SolveArgs a) {
  const int total = a.nh * a.K2 * a.K3;  // below 2^31 (checked at creation)
  double e = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
  const int hx = (a.K1 & 1) ? -1 : a.K1 / 2;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int row = idx / a.nh;
    const int k1 = idx - row * a.nh;
    const int k3 = row / a.K2;
    const int k2 = row - k3 * a.K2;
    if (k1 == 0 && k2 == 0 && k3 == 0) {
      a.data[idx] = make_float2(0.f, 0.f);
      continue;
    }
    const int k2s = (k2 <= a.K2 / 2) ? k2 : k2 - a.K2;
    const int k3s = (k3 <= a.K3 / 2) ? k3 : k3 - a.K3;
    const double m1 = a.r[0] * k1 + a.r[3] * k2s + a.r[6] * k3s;
    const double m2 = a.r[1] * k1 + a.r[4] * k2s + a.r[7] * k3s;
    const double m3 = a.r[2] * k1 + a.r[5] * k2s + a.r[8] * k3s;
    const double msq = m1 * m1 + m2 * m2 + m3 * m3;
    const double msqInv = 1.0 / msq;
    const double theta3 = (double)a.bm1[k1] * (double)a.bm2[k2] * (double)a.bm3[k3];
    // the Gaussian in FP32 (expf, within 2 ulp): the grid it scales is FP32
    const double C = (double)expf((float)(-a.piEwald * msq)) * (a.pivInv * msqInv);
    float2 q = a.data[idx];
    if (a.doEV) {
      double q2 = 2.0 * ((double)q.x * q.x + (double)q.y * q.y) * theta3;
      if (k1 == 0 || k1 == hx) q2 *= 0.5;
      const double fac = q2 * C;
      const double vir = 2.0 * (a.piEwald + msqInv);
      e += fac;
      v0 += fac * (vir * m1 * m1 - 1.0);
      v1 += fac * vir * m1 * m2;
      v2 += fac * vir * m1 * m3;
      v3 += fac * (vir * m2 * m2 - 1.0);
      v4 += fac * vir * m2 * m3;
      v5 += fac * (vir * m3 * m3 - 1.0);
    }
    const float th = (float)(theta3 * C);
    q.x *= th;
    q.y *= th;
    a.data[idx] = q;
  }
  if (!a.doEV) return;
  // fixed-order block reduction (warp trees, then warp 0 over the warp sums)
  __shared__ double s_p[kSolveThreads / 32][7];
  double v[7] = {e, v0, v1, v2, v3, v4, v5};
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 7; ++q) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if (lane == 0) s_p[wib][q] = v[q];
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double s = 0;
    for (int w = 0; w < kSolveThreads / 32; ++w) s += s_p[w][threadIdx.x];
    a.partial[blockIdx.x * 7 + threadIdx.x] = s;
  }
  // the last block to finish sums the partials of all blocks in a fixed order
  // (warp q sums quantity q: lane l the blocks l, l + 32, ..., then a fixed
  // warp tree): energy = 0.5 sum, virial = -0.5 sum (scalar_sum_kernel's
  // final scaling), into ev[0] and ev[1..9]
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(a.done, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const int q = wib;
  if (q < 7) {
    double s = 0;
    for (int b = lane; b < (int)gridDim.x; b += 32) s += __ldcg(&a.partial[b * 7 + q]);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      if (q == 0) {
        a.ev[0] = 0.5 * s;
      } else {
        // xx xy xz yy yz zz -> row-major 3x3
        const int map[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
        const int r = map[q - 1][0], c = map[q - 1][1];
        a.ev[1 + 3 * r + c] = -0.5 * s;
        a.ev[1 + 3 * c + r] = -0.5 * s;
      }
    }
  }
  if (threadIdx.x == 0) *a.done = 0;  // ready for the next solve
}

struct GatherArgs {
  int n, K1, K2, K3;
  double r[9];
  const float4* atoms;
  const float* grid;  // potential, K3 x K2 x K1 (x fastest)
  float3* force;
};

// One thread per atom: the gradient of the interpolated potential, summed
// over the order^3 points in a fixed order (along x first, then row by row),
// then -q times the Cartesian gradient.
template <int order>
__global__ void gatherKernel(const __grid_constant__ GatherArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const float4 at = a.atoms[i];
    int ix, iy, iz;
    float wx, wy, wz;
    gridCell(at, a.K1, a.K2, a.K3, ix, iy, iz, wx, wy, wz);
    float tx[order], ty[order], tz[order], dx[order], dy[order], dz[order];
    bsplineThetaD<order>(wx, tx, dx);
    bsplineThetaD<order>(wy, ty, dy);
    bsplineThetaD<order>(wz, tz, dz);
    const int K12 = a.K1 * a.K2;  // grid indices below 2^31 (checked at creation)
    int xs[order];
#pragma unroll
    for (int x0 = 0; x0 < order; ++x0) xs[x0] = (ix + x0 >= a.K1) ? ix + x0 - a.K1 : ix + x0;
    // per grid row (y0, z0): the x sums of theta_x g and dtheta_x g, then the
    // row's y and z factors
    float f1 = 0.f, f2 = 0.f, f3 = 0.f;
#pragma unroll 2
    for (int z0 = 0; z0 < order; ++z0) {
      int z = iz + z0;
      if (z >= a.K3) z -= a.K3;
#pragma unroll
      for (int y0 = 0; y0 < order; ++y0) {
        int y = iy + y0;
        if (y >= a.K2) y -= a.K2;
        const float* row = a.grid + (a.K1 * y + K12 * z);
        float sx = 0.f, sdx = 0.f;
#pragma unroll
        for (int x0 = 0; x0 < order; ++x0) {
          const float g = __ldg(&row[xs[x0]]);
          sx = fmaf(tx[x0], g, sx);
          sdx = fmaf(dx[x0], g, sdx);
        }
        f1 = fmaf(sdx, ty[y0] * tz[z0], f1);
        f2 = fmaf(sx, dy[y0] * tz[z0], f2);
        f3 = fmaf(sx, ty[y0] * dz[z0], f3);
      }
    }
    const double q = -(double)at.w;
    const double g1 = q * f1 * a.K1, g2 = q * f2 * a.K2, g3 = q * f3 * a.K3;
    a.force[i] = make_float3((float)(g1 * a.r[0] + g2 * a.r[3] + g3 * a.r[6]),
                             (float)(g1 * a.r[1] + g2 * a.r[4] + g3 * a.r[7]),
                             (float)(g1 * a.r[2] + g2 * a.r[5] + g3 * a.r[8]));
  }
}

__global__ void atomsFromPositionsKernel(int n, const double* __restrict__ x,
                                         const double* __restrict__ y, const double* __restrict__ z,
                                         const float* __restrict__ charge, double qscale, Recip R,
                                         double ox, double oy, double oz, float4* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double px = x[i] - ox, py = y[i] - oy, pz = z[i] - oz;
    double w[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double s = px * R.r[3 * d] + py * R.r[3 * d + 1] + pz * R.r[3 * d + 2];
      w[d] = s - (floor(s + 0.5) - 0.5);
    }
    float4 a;
    a.x = (float)w[0];
    a.y = (float)w[1];
    a.z = (float)w[2];
    a.x -= (a.x >= 1.0f) ? 1.0f : 0.0f;
    a.y -= (a.y >= 1.0f) ? 1.0f : 0.0f;
    a.z -= (a.z >= 1.0f) ? 1.0f : 0.0f;
    a.w = (float)((double)charge[i] * qscale);
    out[i] = a;
  }
}

__global__ void selfEnergyKernel(int n, const float4* __restrict__ atoms, double* __restrict__ partial) {
  __shared__ double s_w[8];
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double q = atoms[i].w;
    s += q * q;
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_w[w];
    partial[blockIdx.x] = t;
  }
}

}  // namespace
}  // namespace nbk

using namespace nbk;

struct nbk_pme_s {
  int device = 0, numSM = 148;
  int K1 = 0, K2 = 0, K3 = 0, order = 4;
  double ewaldcof = 0;
  unsigned long long* gridFixed = nullptr;  // K1 K2 K3
  float* gridReal = nullptr;                // K1 K2 K3 (charges, then potential)
  float2* gridHat = nullptr;                // (K1/2+1) K2 K3
  float* bm = nullptr;                      // bm1 | bm2 | bm3
  double* partial = nullptr;                // solve partials, self-energy partials
  double* ev = nullptr;                     // energy, virial[9]
  int* done = nullptr;                      // solve blocks finished
  int solveBlocks = 0;
  cufftHandle fwd = 0, bwd = 0;
  bool plans = false;
};

namespace {

int pmeFail(int code, const std::string& msg) { return setLastError(code, msg); }

#define PME_CUDA(call, what)                                                              \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return pmeFail(NBK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define PME_FFT(call, what)                                                               \
  do {                                                                                    \
    cufftResult r_ = (call);                                                              \
    if (r_ != CUFFT_SUCCESS)                                                              \
      return pmeFail(NBK_ERR_CUDA, std::string(what) + ": cuFFT error " + std::to_string((int)r_)); \
  } while (0)

// compute_b_moduli: 1 / |DFT of the order-point B-spline weights at w = 0|^2.
void bModuli(int K, int order, std::vector<float>& out) {
  double th[kMaxOrder];
  switch (order) {
    case 4: bsplineTheta<double, 4>(0.0, th); break;
    case 6: bsplineTheta<double, 6>(0.0, th); break;
    default: bsplineTheta<double, 8>(0.0, th); break;
  }
  out.resize(K);
  for (int k = 0; k < K; ++k) {
    double s1 = 0, s2 = 0;
    for (int j = 0; j < order && j < K; ++j) {
      const double arg = 2.0 * M_PI * k * j / K;
      s1 += th[j] * std::cos(arg);
      s2 += th[j] * std::sin(arg);
    }
    out[k] = (float)(1.0 / (s1 * s1 + s2 * s2));
  }
}

int useDevice(nbk_pme p, const char* fn) {
  if (!p) return pmeFail(NBK_ERR_ARG, std::string(fn) + ": NULL handle");
  PME_CUDA(cudaSetDevice(p->device), fn);
  return NBK_OK;
}

}  // namespace

extern "C" NBK_API int nbk_pme_create(int deviceID, const nbk_pme_grid* g, double ewaldcof,
                                      nbk_pme* out) {
  if (!g || !out) return pmeFail(NBK_ERR_ARG, "nbk_pme_create: NULL argument");
  *out = nullptr;
  if (g->K1 < 8 || g->K2 < 8 || g->K3 < 8 || (g->order != 4 && g->order != 6 && g->order != 8) ||
      g->K1 < g->order || g->K2 < g->order || g->K3 < g->order || !(ewaldcof > 0) ||
      (double)g->K1 * g->K2 * g->K3 >= 2147483647.0)
    return pmeFail(NBK_ERR_ARG, "nbk_pme_create: grid sizes >= 8 and >= order, fewer than 2^31 "
                                "points, order 4, 6 or 8, ewaldcof > 0");
  PME_CUDA(cudaSetDevice(deviceID), "nbk_pme_create");
  nbk_pme p = new (std::nothrow) nbk_pme_s;
  if (!p) return pmeFail(NBK_ERR_NOMEM, "nbk_pme_create: out of memory");
  p->device = deviceID;
  p->K1 = g->K1;
  p->K2 = g->K2;
  p->K3 = g->K3;
  p->order = g->order;
  p->ewaldcof = ewaldcof;
  cudaDeviceGetAttribute(&p->numSM, cudaDevAttrMultiProcessorCount, deviceID);
  const size_t n = (size_t)p->K1 * p->K2 * p->K3;
  const size_t nh = (size_t)(p->K1 / 2 + 1) * p->K2 * p->K3;
  p->solveBlocks = (int)std::min<size_t>((nh + kSolveThreads - 1) / kSolveThreads, 4 * (size_t)p->numSM);
  cudaError_t e = cudaMalloc(&p->gridFixed, n * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&p->gridReal, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&p->gridHat, nh * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc(&p->bm, sizeof(float) * (p->K1 + p->K2 + p->K3));
  if (e == cudaSuccess)
    e = cudaMalloc(&p->partial, sizeof(double) * std::max<size_t>(7 * (size_t)p->solveBlocks, 1024));
  if (e == cudaSuccess) e = cudaMalloc(&p->ev, sizeof(double) * 10);
  if (e == cudaSuccess) e = cudaMalloc(&p->done, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(p->done, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(p->gridFixed, 0, n * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(p->ev, 0, sizeof(double) * 10);
  if (e == cudaSuccess) {
    std::vector<float> b1, b2, b3;
    bModuli(p->K1, p->order, b1);
    bModuli(p->K2, p->order, b2);
    bModuli(p->K3, p->order, b3);
    e = cudaMemcpy(p->bm, b1.data(), sizeof(float) * p->K1, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(p->bm + p->K1, b2.data(), sizeof(float) * p->K2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(p->bm + p->K1 + p->K2, b3.data(), sizeof(float) * p->K3, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    nbk_pme_destroy(p);
    return pmeFail(NBK_ERR_NOMEM, std::string("nbk_pme_create: ") + cudaGetErrorString(e));
  }
  // x fastest: cuFFT's last dimension is K1
  cufftResult r = cufftPlan3d(&p->fwd, p->K3, p->K2, p->K1, CUFFT_R2C);
  if (r == CUFFT_SUCCESS) r = cufftPlan3d(&p->bwd, p->K3, p->K2, p->K1, CUFFT_C2R);
  if (r != CUFFT_SUCCESS) {
    nbk_pme_destroy(p);
    return pmeFail(NBK_ERR_CUDA, "nbk_pme_create: cuFFT plan error " + std::to_string((int)r));
  }
  p->plans = true;
  *out = p;
  return NBK_OK;
}

extern "C" NBK_API int nbk_pme_destroy(nbk_pme p) {
  if (!p) return NBK_OK;
  cudaSetDevice(p->device);
  if (p->fwd) cufftDestroy(p->fwd);
  if (p->bwd) cufftDestroy(p->bwd);
  cudaFree(p->gridFixed);
  cudaFree(p->gridReal);
  cudaFree(p->gridHat);
  cudaFree(p->bm);
  cudaFree(p->partial);
  cudaFree(p->ev);
  cudaFree(p->done);
  delete p;
  return NBK_OK;
}

extern "C" NBK_API int nbk_pme_atoms_from_positions(int n, const double* x, const double* y,
                                                    const double* z, const float* charge,
                                                    double qscale, const double* lattice,
                                                    nbk_float4* atoms, void* stream) {
  if (n < 0 || !lattice || (n && (!x || !y || !z || !charge || !atoms)))
    return pmeFail(NBK_ERR_ARG, "nbk_pme_atoms_from_positions: NULL argument");
  if (!n) return NBK_OK;
  Recip R;
  const double vol = reciprocal(lattice, R);
  if (!(std::fabs(vol) > 0)) return pmeFail(NBK_ERR_ARG, "nbk_pme_atoms_from_positions: singular lattice");
  atomsFromPositionsKernel<<<std::min((n + 255) / 256, 4096), 256, 0, (cudaStream_t)stream>>>(
      n, x, y, z, charge, qscale, R, lattice[9], lattice[10], lattice[11],
      reinterpret_cast<float4*>(atoms));
  PME_CUDA(cudaGetLastError(), "nbk_pme_atoms_from_positions");
  return NBK_OK;
}

extern "C" NBK_API int nbk_pme_spread_charge(nbk_pme p, int n, const nbk_float4* atoms, void* stream) {
  int rc = useDevice(p, "nbk_pme_spread_charge");
  if (rc) return rc;
  if (n < 0 || (n && !atoms)) return pmeFail(NBK_ERR_ARG, "nbk_pme_spread_charge: bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t ng = (size_t)p->K1 * p->K2 * p->K3;
  if (n) {
    const int blocks = std::min((n + 127) / 128, p->numSM * 16);
    const float4* a = reinterpret_cast<const float4*>(atoms);
    switch (p->order) {
      case 4: spreadKernel<4><<<blocks, 128, 0, st>>>(n, a, p->K1, p->K2, p->K3, p->gridFixed); break;
      case 6: spreadKernel<6><<<blocks, 128, 0, st>>>(n, a, p->K1, p->K2, p->K3, p->gridFixed); break;
      default: spreadKernel<8><<<blocks, 128, 0, st>>>(n, a, p->K1, p->K2, p->K3, p->gridFixed); break;
    }
    PME_CUDA(cudaGetLastError(), "nbk_pme_spread_charge");
  }
  gridToFloatKernel<<<(int)std::min<size_t>((ng + 255) / 256, (size_t)p->numSM * 8), 256, 0, st>>>(
      ng, p->gridFixed, p->gridReal);
  PME_CUDA(cudaGetLastError(), "nbk_pme_spread_charge");
  return NBK_OK;
}

extern "C" NBK_API int nbk_pme_solve(nbk_pme p, const double* lattice, unsigned flags, void* stream) {
  int rc = useDevice(p, "nbk_pme_solve");
  if (rc) return rc;
  if (!lattice || (flags & ~(unsigned)(NBK_ENERGY | NBK_VIRIAL)))
    return pmeFail(NBK_ERR_ARG, "nbk_pme_solve: bad argument (flags: NBK_ENERGY, NBK_VIRIAL)");
  cudaStream_t st = (cudaStream_t)stream;
  SolveArgs a;
  const double vol = reciprocal(lattice, *reinterpret_cast<Recip*>(a.r));
  if (!(std::fabs(vol) > 0)) return pmeFail(NBK_ERR_ARG, "nbk_pme_solve: singular lattice");
  a.K1 = p->K1;
  a.K2 = p->K2;
  a.K3 = p->K3;
  a.nh = p->K1 / 2 + 1;
  a.piEwald = M_PI * M_PI / (p->ewaldcof * p->ewaldcof);
  a.pivInv = 1.0 / (M_PI * std::fabs(vol));
  a.bm1 = p->bm;
  a.bm2 = p->bm + p->K1;
  a.bm3 = p->bm + p->K1 + p->K2;
  a.data = p->gridHat;
  a.partial = p->partial;
  a.ev = p->ev;
  a.done = p->done;
  a.doEV = (flags & (NBK_ENERGY | NBK_VIRIAL)) ? 1 : 0;
  PME_FFT(cufftSetStream(p->fwd, st), "nbk_pme_solve");
  PME_FFT(cufftSetStream(p->bwd, st), "nbk_pme_solve");
  PME_FFT(cufftExecR2C(p->fwd, p->gridReal, reinterpret_cast<cufftComplex*>(p->gridHat)),
          "nbk_pme_solve: forward FFT");
  solveKernel<<<p->solveBlocks, kSolveThreads, 0, st>>>(a);
  PME_CUDA(cudaGetLastError(), "nbk_pme_solve");
  PME_FFT(cufftExecC2R(p->bwd, reinterpret_cast<cufftComplex*>(p->gridHat), p->gridReal),
          "nbk_pme_solve: backward FFT");
  return NBK_OK;
}

extern "C" NBK_API int nbk_pme_gather_force(nbk_pme p, int n, const nbk_float4* atoms,
                                            const double* lattice, nbk_float3* force, void* stream) {
  int rc = useDevice(p, "nbk_pme_gather_force");
  if (rc) return rc;
  if (n < 0 || !lattice || (n && (!atoms || !force)))
    return pmeFail(NBK_ERR_ARG, "nbk_pme_gather_force: bad argument");
  if (!n) return NBK_OK;
  GatherArgs a;
  const double vol = reciprocal(lattice, *reinterpret_cast<Recip*>(a.r));
  if (!(std::fabs(vol) > 0)) return pmeFail(NBK_ERR_ARG, "nbk_pme_gather_force: singular lattice");
  a.n = n;
  a.K1 = p->K1;
  a.K2 = p->K2;
  a.K3 = p->K3;
  a.atoms = reinterpret_cast<const float4*>(atoms);
  a.grid = p->gridReal;
  a.force = reinterpret_cast<float3*>(force);
  const int blocks = std::min((n + 127) / 128, p->numSM * 16);
  cudaStream_t st = (cudaStream_t)stream;
  switch (p->order) {
    case 4: gatherKernel<4><<<blocks, 128, 0, st>>>(a); break;
    case 6: gatherKernel<6><<<blocks, 128, 0, st>>>(a); break;
    default: gatherKernel<8><<<blocks, 128, 0, st>>>(a); break;
  }
  PME_CUDA(cudaGetLastError(), "nbk_pme_gather_force");
  return NBK_OK;
}

extern "C" NBK_API int nbk_pme_get_energy_virial(nbk_pme p, double* energy, double* virial,
                                                 void* stream) {
  int rc = useDevice(p, "nbk_pme_get_energy_virial");
  if (rc) return rc;
  double h[10];
  cudaStream_t st = (cudaStream_t)stream;
  PME_CUDA(cudaMemcpyAsync(h, p->ev, sizeof(h), cudaMemcpyDeviceToHost, st), "nbk_pme_get_energy_virial");
  PME_CUDA(cudaStreamSynchronize(st), "nbk_pme_get_energy_virial");
  if (energy) *energy = h[0];
  if (virial)
    for (int k = 0; k < 9; ++k) virial[k] = h[1 + k];
  return NBK_OK;
}

extern "C" NBK_API int nbk_pme_self_energy(nbk_pme p, int n, const nbk_float4* atoms, double* self,
                                           void* stream) {
  int rc = useDevice(p, "nbk_pme_self_energy");
  if (rc) return rc;
  if (n < 0 || !self || (n && !atoms)) return pmeFail(NBK_ERR_ARG, "nbk_pme_self_energy: bad argument");
  if (!n) {
    *self = 0;
    return NBK_OK;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int blocks = std::min((n + 255) / 256, 1024);
  selfEnergyKernel<<<blocks, 256, 0, st>>>(n, reinterpret_cast<const float4*>(atoms), p->partial);
  PME_CUDA(cudaGetLastError(), "nbk_pme_self_energy");
  std::vector<double> h(blocks);
  PME_CUDA(cudaMemcpyAsync(h.data(), p->partial, sizeof(double) * blocks, cudaMemcpyDeviceToHost, st),
           "nbk_pme_self_energy");
  PME_CUDA(cudaStreamSynchronize(st), "nbk_pme_self_energy");
  double s = 0;
  for (int b = 0; b < blocks; ++b) s += h[b];
  *self = -p->ewaldcof / std::sqrt(M_PI) * s;
  return NBK_OK;
}
