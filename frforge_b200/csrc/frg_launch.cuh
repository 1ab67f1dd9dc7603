// Kernel launchers: build the constant-bank operator tables for one NP and
// dispatch on (flux, dissipation form).  Included once per NP by
// frg_launch_np<NP>.cu so the template instances compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "frg_batch.cuh"
#include "frg_stage1d.cuh"
#include "frg_stage2d.cuh"

namespace frg {

// Kernel attributes (dynamic shared memory size, cluster size) belong to a
// function on one device.  KernelSetup records, per device, that a kernel's
// attributes were set, so a process whose contexts live on several GPUs sets
// them on each, and host threads that launch at the same time set them once.
constexpr int kMaxDevices = 64;
struct KernelSetup {
  std::mutex mu;
  std::atomic<bool> done[kMaxDevices] = {};
  // Runs set() once per device (again after a failure); returns 0 or a CUDA
  // error code.
  template <class F>
  int ensure(F&& set) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return (int)cudaErrorInvalidDevice;
    if (done[dev].load(std::memory_order_acquire)) return 0;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev].load(std::memory_order_relaxed)) return 0;
    const int rc = set();
    if (rc == 0) done[dev].store(true, std::memory_order_release);
    return rc;
  }
};

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
    o.w[i] = h.w[i];
  }
  return o;
}

// Tile variants per NP: (TX, TY, CTAs per SM, u0 staged in shared memory,
// and for FRG_VT the threads per CTA, a multiple of 32, else 256).
// Variant 0 is the default, the fastest measured on a B200 for large meshes
// (P<=3: 512^2, P=4/5: 384^2); the autotuner times all of them on the solve.
// The batched kernels use variant `batch`.
template <int NP>
struct Variants2D;
#define FRG_VT(NPv, idx, tx, ty, minb, u0s, nt)                                         \
  template <>                                                                             \
  struct Variants2D<NPv>::V_<idx> {                                                       \
    static constexpr int TX = tx, TY = ty, MINB = minb, NT = nt;                          \
    static constexpr bool U0S = u0s;                                                      \
  };
#define FRG_V(NPv, idx, tx, ty, minb, u0s) FRG_VT(NPv, idx, tx, ty, minb, u0s, kStageThreads)
template <>
struct Variants2D<2> {
  static constexpr int n = 4, batch = 3;
  template <int V> struct V_;
};
FRG_VT(2, 0, 16, 6, 2, false, 384)
FRG_VT(2, 1, 16, 8, 2, false, 512)
FRG_V(2, 2, 8, 8, 2, true)
FRG_V(2, 3, 8, 4, 3, false)
template <>
struct Variants2D<3> {
  static constexpr int n = 4, batch = 0;
  template <int V> struct V_;
};
FRG_VT(3, 0, 8, 8, 2, false, 512)
FRG_V(3, 1, 4, 4, 4, false)
FRG_V(3, 2, 8, 6, 2, true)
FRG_V(3, 3, 8, 3, 3, false)
template <>
struct Variants2D<4> {
  static constexpr int n = 5, batch = 0;
  template <int V> struct V_;
};
FRG_VT(4, 0, 8, 4, 2, false, 512)
FRG_V(4, 1, 8, 2, 4, false)
FRG_V(4, 2, 8, 3, 3, false)
FRG_V(4, 3, 8, 4, 2, true)
FRG_V(4, 4, 4, 4, 4, false)
template <>
struct Variants2D<5> {
  static constexpr int n = 3, batch = 0;
  template <int V> struct V_;
};
FRG_VT(5, 0, 8, 3, 2, false, 512)
FRG_V(5, 1, 4, 3, 3, false)
FRG_V(5, 2, 4, 4, 2, true)
template <>
struct Variants2D<6> {
  static constexpr int n = 3, batch = 0;
  template <int V> struct V_;
};
FRG_VT(6, 0, 6, 3, 2, false, 512)
FRG_V(6, 1, 3, 3, 3, false)
FRG_V(6, 2, 4, 3, 2, true)
#undef FRG_V
#undef FRG_VT

template <int NP, int FLUX, int AV, int V>
int launch2d_var(const Launch2D& L, const StageBufs& b, cudaStream_t st) {
  using VV = typename Variants2D<NP>::template V_<V>;
  using S = Smem2D<NP, VV::TX, VV::TY, VV::U0S, VV::MINB, VV::NT>;
  // affine and curved meshes have kernels of their own
  auto kaff = stage2d_kernel<NP, FLUX, AV, VV::TX, VV::TY, VV::MINB, VV::U0S, VV::NT, 0>;
  auto kcur = stage2d_kernel<NP, FLUX, AV, VV::TX, VV::TY, VV::MINB, VV::U0S, VV::NT, 1>;
  static KernelSetup setup;
  const int se = setup.ensure([&] {
    cudaError_t e = cudaFuncSetAttribute(kaff, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kcur, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
    return (int)e;
  });
  if (se) return se;
  auto kern = L.mesh.curved ? kcur : kaff;
  dim3 grid((L.mesh.nx + VV::TX - 1) / VV::TX, (L.mesh.ny + VV::TY - 1) / VV::TY);
  kern<<<grid, VV::NT, S::bytes, st>>>(make_ops<NP>(*L.ops), L.mesh, L.phys, b);
  return (int)cudaGetLastError();
}

// A stage with a preprocess_state hook (b.uw set): the default tile variant,
// staging the work state, with the mesh kind read from the descriptor.
template <int NP, int FLUX, int AV>
int launch2d_pre(const Launch2D& L, const StageBufs& b, cudaStream_t st) {
  using VV = typename Variants2D<NP>::template V_<0>;
  using S = Smem2D<NP, VV::TX, VV::TY, VV::U0S, VV::MINB, VV::NT>;
  auto kern = stage2d_kernel<NP, FLUX, AV, VV::TX, VV::TY, VV::MINB, VV::U0S, VV::NT, -1, true>;
  static KernelSetup setup;
  const int se = setup.ensure(
      [&] { return (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes); });
  if (se) return se;
  dim3 grid((L.mesh.nx + VV::TX - 1) / VV::TX, (L.mesh.ny + VV::TY - 1) / VV::TY);
  kern<<<grid, VV::NT, S::bytes, st>>>(make_ops<NP>(*L.ops), L.mesh, L.phys, b);
  return (int)cudaGetLastError();
}

template <int NP, int FLUX, int AV>
int launch2d_inst(const Launch2D& L, const StageBufs& b, cudaStream_t st) {
  if (b.uw) return launch2d_pre<NP, FLUX, AV>(L, b, st);
  const int v = (L.variant >= 0 && L.variant < Variants2D<NP>::n) ? L.variant : 0;
  switch (v) {
    case 1:
      if constexpr (Variants2D<NP>::n > 1) return launch2d_var<NP, FLUX, AV, 1>(L, b, st);
      break;
    case 2:
      if constexpr (Variants2D<NP>::n > 2) return launch2d_var<NP, FLUX, AV, 2>(L, b, st);
      break;
    case 3:
      if constexpr (Variants2D<NP>::n > 3) return launch2d_var<NP, FLUX, AV, 3>(L, b, st);
      break;
    case 4:
      if constexpr (Variants2D<NP>::n > 4) return launch2d_var<NP, FLUX, AV, 4>(L, b, st);
      break;
    case 5:
      if constexpr (Variants2D<NP>::n > 5) return launch2d_var<NP, FLUX, AV, 5>(L, b, st);
      break;
    default:
      break;
  }
  return launch2d_var<NP, FLUX, AV, 0>(L, b, st);
}

template <int NP, int FLUX, int AV>
int launch1d_inst(const Launch1D& L, const StageBufs& b, cudaStream_t st) {
  using S = Smem1D<NP>;
  auto kern = stage1d_kernel<NP, FLUX, AV>;
  static KernelSetup setup;
  const int se = setup.ensure(
      [&] { return (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes); });
  if (se) return se;
  dim3 grid((L.mesh.nel + S::TX - 1) / S::TX);
  kern<<<grid, 256, S::bytes, st>>>(make_ops<NP>(*L.ops), L.mesh, L.phys, b);
  return (int)cudaGetLastError();
}

// nsteps steps of a 1D solve of at most kLoop1DMaxTiles tiles by one cluster
// of LTX-element tiles
template <int NP, int FLUX, int AV, int LTX>
int loop1d_tx(const Launch1D& L, const Loop1DBufs& lb, DevScalars* sc, int nsteps, cudaStream_t st,
              int max_cluster = kLoop1DMaxTiles) {
  using S = Smem1D<NP, LTX>;
  auto kern = loop1d_kernel<NP, FLUX, AV, LTX>;
  // every instantiation launches with a single max_cluster value
  static KernelSetup setup;
  const int se = setup.ensure([&] {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
    if (e == cudaSuccess && max_cluster > kLoop1DMaxTiles)
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return (int)e;
  });
  if (se) return se;
  const int ntiles = (L.mesh.nel + S::TX - 1) / S::TX;
  if (ntiles < 1 || ntiles > max_cluster) return (int)cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ntiles);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = S::bytes;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = ntiles;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return (int)cudaLaunchKernelEx(&cfg, kern, make_ops<NP>(*L.ops), L.mesh, L.phys, lb, sc, nsteps);
}
// Whether a cluster of n CTAs of this loop kernel can be scheduled (n > 8
// is a non-portable size, allowed on this kernel first).
template <int NP, int FLUX, int AV, int LTX>
bool loop1d_cluster_fits(int n) {
  using S = Smem1D<NP, LTX>;
  auto kern = loop1d_kernel<NP, FLUX, AV, LTX>;
  // per device: 0 unknown, 1 fits, 2 does not (n is the same
  // kLoop1DMaxCluster every call)
  static std::atomic<int> fits[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return false;
  int f = fits[dev].load(std::memory_order_acquire);
  if (f == 0) {
    f = 2;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes) == cudaSuccess &&
        cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(n);
      cfg.blockDim = dim3(256);
      cfg.dynamicSmemBytes = S::bytes;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = n;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int nc = 0;
      if (cudaOccupancyMaxActiveClusters(&nc, kern, &cfg) == cudaSuccess && nc >= 1) f = 1;
    }
    cudaGetLastError();  // a refused query leaves no sticky error
    fits[dev].store(f, std::memory_order_release);
  }
  return f == 1;
}

// The narrowest tiles whose cluster holds the mesh: quarter-width tiles on up
// to kLoop1DMaxCluster CTAs where such a cluster can be scheduled, else
// half-width tiles on up to 8, else full tiles.  Narrower tiles mean more
// CTAs and fewer passes per thread in each phase.
template <int NP, int FLUX, int AV>
int loop1d_inst(const Launch1D& L, const Loop1DBufs& lb, DevScalars* sc, int nsteps, cudaStream_t st) {
  constexpr int TXQ = Tile1D<NP>::TX / 4, TXH = Tile1D<NP>::TX / 2;
  const int nq = (L.mesh.nel + TXQ - 1) / TXQ;
  if (nq <= kLoop1DMaxTiles ||
      (nq <= kLoop1DMaxCluster && loop1d_cluster_fits<NP, FLUX, AV, TXQ>(kLoop1DMaxCluster)))
    return loop1d_tx<NP, FLUX, AV, TXQ>(L, lb, sc, nsteps, st, kLoop1DMaxCluster);
  if (L.mesh.nel <= kLoop1DMaxTiles * TXH) return loop1d_tx<NP, FLUX, AV, TXH>(L, lb, sc, nsteps, st);
  return loop1d_tx<NP, FLUX, AV, Tile1D<NP>::TX>(L, lb, sc, nsteps, st);
}

template <int NP>
int loop1d_np(const Launch1D& L, const Loop1DBufs& lb, DevScalars* sc, int nsteps, cudaStream_t st) {
  const bool hllc = L.flux == FRG_FLUX_HLLC;
  switch (L.av) {
    case kAvBR0:
      return hllc ? loop1d_inst<NP, FRG_FLUX_HLLC, kAvBR0>(L, lb, sc, nsteps, st)
                  : loop1d_inst<NP, FRG_FLUX_RUSANOV, kAvBR0>(L, lb, sc, nsteps, st);
    case kAvDD:
      return hllc ? loop1d_inst<NP, FRG_FLUX_HLLC, kAvDD>(L, lb, sc, nsteps, st)
                  : loop1d_inst<NP, FRG_FLUX_RUSANOV, kAvDD>(L, lb, sc, nsteps, st);
    default:
      return hllc ? loop1d_inst<NP, FRG_FLUX_HLLC, kAvNone>(L, lb, sc, nsteps, st)
                  : loop1d_inst<NP, FRG_FLUX_RUSANOV, kAvNone>(L, lb, sc, nsteps, st);
  }
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

template <int NP, int FLUX, int AV, int V>
int batch2d_var(const HostOps& h, const BatchInst* insts, const BatchTile* tiles, int ntiles, int stage,
                int mode, cudaStream_t st) {
  using VV = typename Variants2D<NP>::template V_<V>;
  using S = Smem2D<NP, VV::TX, VV::TY, VV::U0S, VV::MINB, VV::NT>;
  auto kern = stage2d_batch_kernel<NP, FLUX, AV, VV::TX, VV::TY, VV::MINB, VV::U0S, VV::NT>;
  static KernelSetup setup;
  const int se = setup.ensure(
      [&] { return (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes); });
  if (se) return se;
  if (ntiles > 0) kern<<<ntiles, VV::NT, S::bytes, st>>>(make_ops<NP>(h), insts, tiles, stage, mode);
  return (int)cudaGetLastError();
}

// variant: a tile variant of the autotune table, or -1 for the default
// batched tile (Variants2D<NP>::batch)
template <int NP, int FLUX, int AV>
int batch2d_inst(const HostOps& h, int variant, const BatchInst* insts, const BatchTile* tiles, int ntiles,
                 int stage, int mode, cudaStream_t st) {
  switch (variant) {
    case 0:
      return batch2d_var<NP, FLUX, AV, 0>(h, insts, tiles, ntiles, stage, mode, st);
    case 1:
      if constexpr (Variants2D<NP>::n > 1) return batch2d_var<NP, FLUX, AV, 1>(h, insts, tiles, ntiles, stage, mode, st);
      break;
    case 2:
      if constexpr (Variants2D<NP>::n > 2) return batch2d_var<NP, FLUX, AV, 2>(h, insts, tiles, ntiles, stage, mode, st);
      break;
    case 3:
      if constexpr (Variants2D<NP>::n > 3) return batch2d_var<NP, FLUX, AV, 3>(h, insts, tiles, ntiles, stage, mode, st);
      break;
    case 4:
      if constexpr (Variants2D<NP>::n > 4) return batch2d_var<NP, FLUX, AV, 4>(h, insts, tiles, ntiles, stage, mode, st);
      break;
    default:
      break;
  }
  return batch2d_var<NP, FLUX, AV, Variants2D<NP>::batch>(h, insts, tiles, ntiles, stage, mode, st);
}

template <int NP>
int batch2d_np(const HostOps& h, int flux, int av, int variant, const BatchInst* insts, const BatchTile* tiles,
               int ntiles, int stage, int mode, cudaStream_t st) {
  const bool hllc = flux == FRG_FLUX_HLLC;
  switch (av) {
    case kAvBR0:
      return hllc ? batch2d_inst<NP, FRG_FLUX_HLLC, kAvBR0>(h, variant, insts, tiles, ntiles, stage, mode, st)
                  : batch2d_inst<NP, FRG_FLUX_RUSANOV, kAvBR0>(h, variant, insts, tiles, ntiles, stage, mode, st);
    case kAvDD:
      return hllc ? batch2d_inst<NP, FRG_FLUX_HLLC, kAvDD>(h, variant, insts, tiles, ntiles, stage, mode, st)
                  : batch2d_inst<NP, FRG_FLUX_RUSANOV, kAvDD>(h, variant, insts, tiles, ntiles, stage, mode, st);
    default:
      return hllc ? batch2d_inst<NP, FRG_FLUX_HLLC, kAvNone>(h, variant, insts, tiles, ntiles, stage, mode, st)
                  : batch2d_inst<NP, FRG_FLUX_RUSANOV, kAvNone>(h, variant, insts, tiles, ntiles, stage, mode, st);
  }
}

template <int NP, int FLUX, int AV>
int batch1d_inst(const HostOps& h, const BatchInst* insts, const BatchTile* tiles, int ntiles, int stage,
                 int mode, cudaStream_t st) {
  using S = Smem1D<NP>;
  auto kern = stage1d_batch_kernel<NP, FLUX, AV>;
  static KernelSetup setup;
  const int se = setup.ensure(
      [&] { return (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes); });
  if (se) return se;
  if (ntiles > 0) kern<<<ntiles, 256, S::bytes, st>>>(make_ops<NP>(h), insts, tiles, stage, mode);
  return (int)cudaGetLastError();
}

template <int NP>
int batch1d_np(const HostOps& h, int flux, int av, const BatchInst* insts, const BatchTile* tiles, int ntiles,
               int stage, int mode, cudaStream_t st) {
  const bool hllc = flux == FRG_FLUX_HLLC;
  switch (av) {
    case kAvBR0:
      return hllc ? batch1d_inst<NP, FRG_FLUX_HLLC, kAvBR0>(h, insts, tiles, ntiles, stage, mode, st)
                  : batch1d_inst<NP, FRG_FLUX_RUSANOV, kAvBR0>(h, insts, tiles, ntiles, stage, mode, st);
    case kAvDD:
      return hllc ? batch1d_inst<NP, FRG_FLUX_HLLC, kAvDD>(h, insts, tiles, ntiles, stage, mode, st)
                  : batch1d_inst<NP, FRG_FLUX_RUSANOV, kAvDD>(h, insts, tiles, ntiles, stage, mode, st);
    default:
      return hllc ? batch1d_inst<NP, FRG_FLUX_HLLC, kAvNone>(h, insts, tiles, ntiles, stage, mode, st)
                  : batch1d_inst<NP, FRG_FLUX_RUSANOV, kAvNone>(h, insts, tiles, ntiles, stage, mode, st);
  }
}

template <int NP, int V>
int tile_shape_v(int* tx, int* ty) {
  using VV = typename Variants2D<NP>::template V_<V>;
  *tx = VV::TX;
  *ty = VV::TY;
  return VV::MINB;
}

// Tile shape and CTAs per SM of the batched kernel for `variant` (-1 or out
// of range: the default batched tile).
template <int NP>
int tile_shape_np(int dim, int variant, int* tx, int* ty) {
  if (dim == 1) {
    *tx = Tile1D<NP>::TX;
    *ty = 1;
    return 1;
  }
  switch (variant) {
    case 0:
      return tile_shape_v<NP, 0>(tx, ty);
    case 1:
      if constexpr (Variants2D<NP>::n > 1) return tile_shape_v<NP, 1>(tx, ty);
      break;
    case 2:
      if constexpr (Variants2D<NP>::n > 2) return tile_shape_v<NP, 2>(tx, ty);
      break;
    case 3:
      if constexpr (Variants2D<NP>::n > 3) return tile_shape_v<NP, 3>(tx, ty);
      break;
    case 4:
      if constexpr (Variants2D<NP>::n > 4) return tile_shape_v<NP, 4>(tx, ty);
      break;
    default:
      break;
  }
  return tile_shape_v<NP, Variants2D<NP>::batch>(tx, ty);
}

template <int NP>
int variants2d() {
  return Variants2D<NP>::n;
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
  int launch_loop1d_np##NPV(const Launch1D& L, const Loop1DBufs& lb, DevScalars* sc, int n,  \
                            cudaStream_t st) {                                               \
    return loop1d_np<NPV>(L, lb, sc, n, st);                                                 \
  }                                                                                          \
  int stage2d_variants_np##NPV() { return variants2d<NPV>(); }                                \
  int launch_batch2d_np##NPV(const HostOps& h, int flux, int av, int variant, const BatchInst* insts, \
                             const BatchTile* tiles, int ntiles, int stage, int mode, cudaStream_t st) { \
    return batch2d_np<NPV>(h, flux, av, variant, insts, tiles, ntiles, stage, mode, st);     \
  }                                                                                          \
  int launch_batch1d_np##NPV(const HostOps& h, int flux, int av, const BatchInst* insts,     \
                             const BatchTile* tiles, int ntiles, int stage, int mode, cudaStream_t st) { \
    return batch1d_np<NPV>(h, flux, av, insts, tiles, ntiles, stage, mode, st);              \
  }                                                                                          \
  int tile_shape_np##NPV(int dim, int variant, int* tx, int* ty) {                           \
    return tile_shape_np<NPV>(dim, variant, tx, ty);                                         \
  }                                                                                          \
  }
