// Batched stage kernels: every CTA handles one tile of one instance of a
// batch.  The instance descriptor is copied to shared memory and the tile is
// processed by the same tile function as a single solve, so an instance's
// results do not depend on what else is in the batch.
#pragma once

#include "frg_stage1d.cuh"
#include "frg_stage2d.cuh"

namespace frg {

// Stage buffers of an instance for stage `stage` (or the prime pass, which
// the batched kernels run only as the post-step pass of a hooked group, on the
// instances whose step just completed).
FRG_DEV StageBufs batch_bufs(const BatchInst& I, int stage, int mode) {
  StageBufs b{};
  b.sc = I.sc;
  b.mode = mode;
  b.rk2 = I.rk2;
  if (mode == kModePrime) {
    b.us = I.U[0];
    b.eps_out = I.E[0];
    b.want_lambda = 1;
    return b;
  }
  b.use_sc = 1;
  b.stage = stage;
  b.u0 = I.U[0];
  if (stage == 1) {
    b.us = I.U[0];
    b.uout = I.U[1];
    b.eps_in = I.E[0];
    b.eps_out = I.E[1];
    b.a = 1.0;
    b.b = 0.0;
    b.c = 1.0;
  } else if (stage == 2 && I.rk2) {
    b.us = I.U[1];
    b.uout = I.U[0];
    b.eps_in = I.E[1];
    b.eps_out = I.E[0];
    b.a = 1.0 / 2.0;
    b.b = 1.0 / 2.0;
    b.c = 1.0 / 2.0;
    b.want_lambda = 1;
  } else if (stage == 2) {
    b.us = I.U[1];
    b.uout = I.U[2];
    b.eps_in = I.E[1];
    b.eps_out = I.E[2];
    b.a = 3.0 / 4.0;
    b.b = 1.0 / 4.0;
    b.c = 1.0 / 4.0;
  } else {
    b.us = I.U[2];
    b.uout = I.U[0];
    b.eps_in = I.E[2];
    b.eps_out = I.E[0];
    b.a = 1.0 / 3.0;
    b.b = 2.0 / 3.0;
    b.c = 2.0 / 3.0;
    b.want_lambda = 1;
  }
  return b;
}

// block-wide copy of a descriptor into shared memory (sizes are multiples of 8)
template <class T>
FRG_DEV void copy_to_smem(T* dst, const T* src) {
  static_assert(sizeof(T) % 8 == 0, "descriptor size");
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(T) / 8); i += blockDim.x) d[i] = s[i];
}

// The mesh, physics and stage descriptors of the CTA's instance live in
// static shared memory (at most kBatchStaticSmem bytes), read on demand by the
// tile function instead of occupying registers.
template <int NP, int FLUX, int AV, int TX, int TY, int MINB, bool U0S, int NTHR = kStageThreads>
__global__ void __launch_bounds__(NTHR, MINB)
    stage2d_batch_kernel(const OpsT<NP> ops, const BatchInst* __restrict__ insts,
                         const BatchTile* __restrict__ tiles, int stage, int mode) {
  __shared__ __align__(16) Mesh2Dev sM;
  __shared__ __align__(16) Phys sP;
  __shared__ __align__(16) StageBufs sB;
  static_assert(sizeof(Mesh2Dev) + sizeof(Phys) + sizeof(StageBufs) + 64 <= kBatchStaticSmem, "static smem");
  const BatchTile t = tiles[blockIdx.x];
  const BatchInst* I = &insts[t.inst];
  // the descriptor copies go out first; the instance's skip tests, whose
  // loads overlap them, come after (a skipped CTA has written nothing)
  copy_to_smem(&sM, &I->M2);
  copy_to_smem(&sP, &I->P);
  if ((mode == kModeStage && stage == 3 && I->rk2) ||     // SSP-RK2 has two stages
      (mode == kModePrime && !I->sc->stepped_ok))          // post-step pass: completed steps only
    return;
  if (threadIdx.x == 0) sB = batch_bufs(*I, stage, mode);
  __syncthreads();
  stage2d_tile<NP, FLUX, AV, TX, TY, MINB, U0S, NTHR>(ops, sM, sP, sB, t.x0, t.y0);
}

template <int NP, int FLUX, int AV>
__global__ void __launch_bounds__(256)
    stage1d_batch_kernel(const OpsT<NP> ops, const BatchInst* __restrict__ insts,
                         const BatchTile* __restrict__ tiles, int stage, int mode) {
  __shared__ __align__(16) Mesh1Dev sM;
  __shared__ __align__(16) Phys sP;
  __shared__ __align__(16) StageBufs sB;
  const BatchTile t = tiles[blockIdx.x];
  const BatchInst* I = &insts[t.inst];
  copy_to_smem(&sM, &I->M1);
  copy_to_smem(&sP, &I->P);
  if ((mode == kModeStage && stage == 3 && I->rk2) || (mode == kModePrime && !I->sc->stepped_ok)) return;
  if (threadIdx.x == 0) sB = batch_bufs(*I, stage, mode);
  __syncthreads();
  stage1d_tile<NP, FLUX, AV>(ops, sM, sP, sB, t.x0);
}

}  // namespace frg
