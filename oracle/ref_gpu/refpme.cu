// PME part of the test harness around the reference's own CUDA kernels.
//
// The Makefile beside this file compiles the reference's
// src/CudaPmeSolverUtilKernel.cu in place (never copied) into
// oracle/_ref/libref_nbgpu.so together with this file, which drives its
// spread_charge_v2 / scalar_sum / gather_force the way the reference's
// single-device PME does (CudaPmeOneDevice, src/CudaPmeSolverUtil.C):
//   - construction (src/CudaPmeSolverUtil.C:1364-1440): one real grid of
//     K1*K2*K3 floats (x fastest) and one half-complex grid of
//     (K1/2+1)*K2*K3, cufftPlan3d(K3, K2, K1) forward R2C and backward C2R on
//     the stream, a linear texture object over the real grid, and the
//     B-spline moduli as FP32 device arrays;
//   - one evaluation (src/CudaPmeSolverUtil.C:1540-1650): clear the grid and
//     the energy/virial record, spread_charge_v2 with the periodic full-grid
//     arguments, R2C, scalar_sum (orderXYZ, sizes K1/2+1, K2, K3), C2R,
//     gather_force into float3 forces.
// The moduli themselves come from the caller: the reference computes them
// with compute_b_moduli (src/PmeKSpace.C:42-61), outside the files compiled
// here. Forces come out as the reference leaves them, the gradient with
// respect to the fractional coordinates times -q (the caller scales them by
// the reciprocal vectors, Lattice::scale_force); energy and the six virial
// components (xx, xy, xz, yy, yz, zz) as scalar_sum accumulates them.
//
// Test infrastructure only: the product library never links this.
#include <cuda_runtime.h>
#include <cufft.h>

#include <stdexcept>
#include <string>

#include "CudaPmeSolverUtilKernel.h"

namespace {

thread_local std::string g_pmeErr;

void pck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
void fck(cufftResult r, const char* what) {
  if (r != CUFFT_SUCCESS) throw std::runtime_error(std::string(what) + ": cuFFT error " + std::to_string((int)r));
}

struct RefPme {
  int k1 = 0, k2 = 0, k3 = 0, order = 0;
  double kappa = 0;
  float* grid = nullptr;
  float2* trans = nullptr;
  float *bm1 = nullptr, *bm2 = nullptr, *bm3 = nullptr;
  double* ev = nullptr;  // energy, virial[6]
  cufftHandle fwd = 0, bwd = 0;
  bool plans = false;
  cudaTextureObject_t tex = 0;
};

template <class F>
int pguard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_pmeErr = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char* refpme_last_error() { return g_pmeErr.c_str(); }

int refpme_destroy(void* hp);

// bm1, bm2, bm3: host B-spline moduli of lengths K1, K2, K3.
int refpme_create(int k1, int k2, int k3, int order, double kappa, const float* bm1,
                  const float* bm2, const float* bm3, void** out) {
  RefPme* h = new RefPme();
  const int rc = pguard([&] {
    if (k1 < order || k2 < order || k3 < order || (order != 4 && order != 6 && order != 8))
      throw std::runtime_error("refpme_create: bad grid");
    h->k1 = k1;
    h->k2 = k2;
    h->k3 = k3;
    h->order = order;
    h->kappa = kappa;
    const size_t ng = (size_t)k1 * k2 * k3, nt = (size_t)(k1 / 2 + 1) * k2 * k3;
    pck(cudaMalloc(&h->grid, sizeof(float) * ng), "grid");
    pck(cudaMalloc(&h->trans, sizeof(float2) * nt), "trans");
    pck(cudaMalloc(&h->bm1, sizeof(float) * k1), "bm1");
    pck(cudaMalloc(&h->bm2, sizeof(float) * k2), "bm2");
    pck(cudaMalloc(&h->bm3, sizeof(float) * k3), "bm3");
    pck(cudaMalloc(&h->ev, sizeof(double) * 7), "ev");
    pck(cudaMemcpy(h->bm1, bm1, sizeof(float) * k1, cudaMemcpyHostToDevice), "bm1 copy");
    pck(cudaMemcpy(h->bm2, bm2, sizeof(float) * k2, cudaMemcpyHostToDevice), "bm2 copy");
    pck(cudaMemcpy(h->bm3, bm3, sizeof(float) * k3, cudaMemcpyHostToDevice), "bm3 copy");
    fck(cufftPlan3d(&h->fwd, k3, k2, k1, CUFFT_R2C), "forward plan");
    fck(cufftPlan3d(&h->bwd, k3, k2, k1, CUFFT_C2R), "backward plan");
    h->plans = true;
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeLinear;
    rd.res.linear.devPtr = h->grid;
    rd.res.linear.desc.f = cudaChannelFormatKindFloat;
    rd.res.linear.desc.x = sizeof(float) * 8;
    rd.res.linear.sizeInBytes = sizeof(float) * ng;
    cudaTextureDesc td = {};
    td.readMode = cudaReadModeElementType;
    pck(cudaCreateTextureObject(&h->tex, &rd, &td, nullptr), "grid texture");
  });
  if (rc) {
    refpme_destroy(h);
    return rc;
  }
  *out = h;
  return 0;
}

// atoms: device float4[n] fractional (x, y, z in [0, 1)) and scaled charge.
// recip9: reciprocal vectors a*, b*, c* (rows). forces: device float3[n].
int refpme_compute(void* hp, const void* atoms, int n, const double* recip9, double volume,
                   int doEnergyVirial, void* forces, void* stream) {
  RefPme* h = (RefPme*)hp;
  return pguard([&] {
    cudaStream_t st = (cudaStream_t)stream;
    const size_t ng = (size_t)h->k1 * h->k2 * h->k3;
    fck(cufftSetStream(h->fwd, st), "forward stream");
    fck(cufftSetStream(h->bwd, st), "backward stream");
    pck(cudaMemsetAsync(h->grid, 0, sizeof(float) * ng, st), "grid clear");
    pck(cudaMemsetAsync(h->ev, 0, sizeof(double) * 7, st), "ev clear");
    const int order3 = ((h->order * h->order * h->order - 1) / 32 + 1) * 32;
    if (n > 0)
      spread_charge_v2((const float4*)atoms, n, h->k1, h->k2, h->k3, (float)h->k1, (float)h->k2,
                       (float)h->k3, order3, h->k1, h->k2, h->k3, h->k1, 0, 0, true, true,
                       h->grid, h->order, st);
    pck(cudaGetLastError(), "spread_charge_v2");
    fck(cufftExecR2C(h->fwd, (cufftReal*)h->grid, (cufftComplex*)h->trans), "R2C");
    float r[9];
    for (int k = 0; k < 9; ++k) r[k] = (float)recip9[k];
    scalar_sum(true, h->k1, h->k2, h->k3, h->k1 / 2 + 1, h->k2, h->k3, h->kappa, r[0], r[1], r[2],
               r[3], r[4], r[5], r[6], r[7], r[8], volume, h->bm1, h->bm2, h->bm3, 0, 0,
               doEnergyVirial != 0, h->ev, h->ev + 1, h->trans, st);
    fck(cufftExecC2R(h->bwd, (cufftComplex*)h->trans, (cufftReal*)h->grid), "C2R");
    if (n > 0)
      gather_force((const float4*)atoms, n, h->k1, h->k2, h->k3, h->k1, h->k2, h->k3, h->k1, 0, 0,
                   true, true, h->grid, h->order, (float3*)forces, h->tex, st);
    pck(cudaGetLastError(), "gather_force");
  });
}

// out7: energy, virial xx, xy, xz, yy, yz, zz of the last evaluation. Synchronises.
int refpme_energy_virial(void* hp, double* out7) {
  RefPme* h = (RefPme*)hp;
  return pguard([&] {
    pck(cudaDeviceSynchronize(), "sync");
    pck(cudaMemcpy(out7, h->ev, sizeof(double) * 7, cudaMemcpyDeviceToHost), "ev copy");
  });
}

int refpme_destroy(void* hp) {
  RefPme* h = (RefPme*)hp;
  if (!h) return 0;
  const int rc = pguard([&] {
    cudaDeviceSynchronize();
    if (h->tex) cudaDestroyTextureObject(h->tex);
    if (h->plans) {
      cufftDestroy(h->fwd);
      cufftDestroy(h->bwd);
    }
    cudaFree(h->grid);
    cudaFree(h->trans);
    cudaFree(h->bm1);
    cudaFree(h->bm2);
    cudaFree(h->bm3);
    cudaFree(h->ev);
  });
  delete h;
  return rc;
}

}  // extern "C"
