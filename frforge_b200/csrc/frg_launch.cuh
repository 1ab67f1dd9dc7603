// Kernel launchers: build the constant-bank operator tables for one NP and
// dispatch on (flux, dissipation form).  Included once per NP by
// frg_launch_np<NP>.cu so the template instances compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "frg_stage1d.cuh"
#include "frg_stage2d.cuh"

namespace frg {

template <int NP>
OpsT<NP> make_ops(const HostOps& h) {
  OpsT<NP> o;
  for (int i = 0; i < NP; ++i) {
    for (int k = 0; k < NP; ++k) {
      o.Dt[i][k] = h.Dt[i][k];
      o.DtD[i][k] = h.DtD[i][k];
      o.DD[i][k] = h.DD[i][k];
      o.Vinv[i][k] = h.Vinv[i][k];
    }
    o.lL[i] = h.lL[i];
    o.lR[i] = h.lR[i];
    o.lLD[i] = h.lLD[i];
    o.lRD[i] = h.lRD[i];
    o.gL[i] = h.gLxi[i];
    o.gR[i] = h.gRxi[i];
    o.xi[i] = h.xi[i];
  }
  return o;
}

template <int NP, int FLUX, int AV>
int launch2d_inst(const Launch2D& L, const StageBufs& b, cudaStream_t st) {
  using T = Tile2D<NP>;
  using S = Smem2D<NP, T::TX, T::TY>;
  auto kern = stage2d_kernel<NP, FLUX, AV>;
  static bool configured = false;  // per instance; attribute is per function
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
    if (e != cudaSuccess) return (int)e;
    configured = true;
  }
  dim3 grid((L.mesh.nx + T::TX - 1) / T::TX, (L.mesh.ny + T::TY - 1) / T::TY);
  kern<<<grid, kStageThreads, S::bytes, st>>>(make_ops<NP>(*L.ops), L.mesh, L.phys, b);
  return (int)cudaGetLastError();
}

template <int NP, int FLUX, int AV>
int launch1d_inst(const Launch1D& L, const StageBufs& b, cudaStream_t st) {
  using S = Smem1D<NP>;
  auto kern = stage1d_kernel<NP, FLUX, AV>;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
    if (e != cudaSuccess) return (int)e;
    configured = true;
  }
  dim3 grid((L.mesh.nel + S::TX - 1) / S::TX);
  kern<<<grid, 256, S::bytes, st>>>(make_ops<NP>(*L.ops), L.mesh, L.phys, b);
  return (int)cudaGetLastError();
}

template <int NP>
int launch2d_np(const Launch2D& L, const StageBufs& b, cudaStream_t st) {
  const bool hllc = L.flux == FRG_FLUX_HLLC;
  switch (L.av) {
    case kAvBR0:
      return hllc ? launch2d_inst<NP, FRG_FLUX_HLLC, kAvBR0>(L, b, st)
                  : launch2d_inst<NP, FRG_FLUX_RUSANOV, kAvBR0>(L, b, st);
    case kAvDD:
      return hllc ? launch2d_inst<NP, FRG_FLUX_HLLC, kAvDD>(L, b, st)
                  : launch2d_inst<NP, FRG_FLUX_RUSANOV, kAvDD>(L, b, st);
    default:
      return hllc ? launch2d_inst<NP, FRG_FLUX_HLLC, kAvNone>(L, b, st)
                  : launch2d_inst<NP, FRG_FLUX_RUSANOV, kAvNone>(L, b, st);
  }
}

template <int NP>
int launch1d_np(const Launch1D& L, const StageBufs& b, cudaStream_t st) {
  const bool hllc = L.flux == FRG_FLUX_HLLC;
  switch (L.av) {
    case kAvBR0:
      return hllc ? launch1d_inst<NP, FRG_FLUX_HLLC, kAvBR0>(L, b, st)
                  : launch1d_inst<NP, FRG_FLUX_RUSANOV, kAvBR0>(L, b, st);
    case kAvDD:
      return hllc ? launch1d_inst<NP, FRG_FLUX_HLLC, kAvDD>(L, b, st)
                  : launch1d_inst<NP, FRG_FLUX_RUSANOV, kAvDD>(L, b, st);
    default:
      return hllc ? launch1d_inst<NP, FRG_FLUX_HLLC, kAvNone>(L, b, st)
                  : launch1d_inst<NP, FRG_FLUX_RUSANOV, kAvNone>(L, b, st);
  }
}

template <int NP>
size_t smem2d_bytes() {
  using T = Tile2D<NP>;
  return Smem2D<NP, T::TX, T::TY>::bytes;
}

}  // namespace frg

#define FRG_INSTANTIATE_NP(NPV)                                                              \
  namespace frg {                                                                            \
  int launch_stage2d_np##NPV(const Launch2D& L, const StageBufs& b, cudaStream_t st) {       \
    return launch2d_np<NPV>(L, b, st);                                                       \
  }                                                                                          \
  int launch_stage1d_np##NPV(const Launch1D& L, const StageBufs& b, cudaStream_t st) {       \
    return launch1d_np<NPV>(L, b, st);                                                       \
  }                                                                                          \
  size_t stage2d_smem_np##NPV() { return smem2d_bytes<NPV>(); }                              \
  }
