// Batched and served execution: many independent solves of different sizes,
// degrees and schemes advanced together on one GPU.
//
// Each instance is an ordinary frg_solve (its own state buffers, mesh arrays,
// tables and status word).  Instances are grouped by (dim, NP, flux,
// dissipation form, operator tables); a group advances as one chain of
// [begin, stage 1..3, end] kernels over its members, the stage kernels
// covering the ragged list of the members' tiles.  Groups are independent,
// so each is a parallel branch of a CUDA graph (fork / join through events)
// that holds several steps.  Instances keep their own dt, time, step count
// and status; finished instances become no-ops.  Adding or removing an
// instance rebuilds the lists and the graph at the next run (continuous
// batching).
//
// Lockstep mode (default): every group takes the same number of steps per
// run.  Multirate mode (frg_batch_set_multirate): a group whose step is
// cheaper takes proportionally more steps per round, so cheap solves that need
// many steps (long 1D meshes) are not held to the pace of heavy 2D ones.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "frg_control.cuh"
#include "frg_device.cuh"
#include "frg_runtime.h"

namespace frg {
int launch_batch2d_np2(const HostOps&, int, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int launch_batch2d_np3(const HostOps&, int, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int launch_batch2d_np4(const HostOps&, int, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int launch_batch2d_np5(const HostOps&, int, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int launch_batch2d_np6(const HostOps&, int, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int launch_batch1d_np2(const HostOps&, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int launch_batch1d_np3(const HostOps&, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int launch_batch1d_np4(const HostOps&, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int launch_batch1d_np5(const HostOps&, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int launch_batch1d_np6(const HostOps&, int, int, const BatchInst*, const BatchTile*, int, int, int, cudaStream_t);
int tile_shape_np2(int, int, int*, int*);
int tile_shape_np3(int, int, int*, int*);
int tile_shape_np4(int, int, int*, int*);
int tile_shape_np5(int, int, int*, int*);
int tile_shape_np6(int, int, int*, int*);

int launch_batch2d(const HostOps* ops, int flux, int av, int variant, const BatchInst* insts,
                   const BatchTile* tiles, int ntiles, int stage, int mode, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  switch (ops->np) {
    case 2: return launch_batch2d_np2(*ops, flux, av, variant, insts, tiles, ntiles, stage, mode, st);
    case 3: return launch_batch2d_np3(*ops, flux, av, variant, insts, tiles, ntiles, stage, mode, st);
    case 4: return launch_batch2d_np4(*ops, flux, av, variant, insts, tiles, ntiles, stage, mode, st);
    case 5: return launch_batch2d_np5(*ops, flux, av, variant, insts, tiles, ntiles, stage, mode, st);
    case 6: return launch_batch2d_np6(*ops, flux, av, variant, insts, tiles, ntiles, stage, mode, st);
  }
  return (int)cudaErrorInvalidValue;
}
int launch_batch1d(const HostOps* ops, int flux, int av, const BatchInst* insts, const BatchTile* tiles,
                   int ntiles, int stage, int mode, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  switch (ops->np) {
    case 2: return launch_batch1d_np2(*ops, flux, av, insts, tiles, ntiles, stage, mode, st);
    case 3: return launch_batch1d_np3(*ops, flux, av, insts, tiles, ntiles, stage, mode, st);
    case 4: return launch_batch1d_np4(*ops, flux, av, insts, tiles, ntiles, stage, mode, st);
    case 5: return launch_batch1d_np5(*ops, flux, av, insts, tiles, ntiles, stage, mode, st);
    case 6: return launch_batch1d_np6(*ops, flux, av, insts, tiles, ntiles, stage, mode, st);
  }
  return (int)cudaErrorInvalidValue;
}
int batch_tile_shape(int dim, int np, int variant, int* tx, int* ty) {
  switch (np) {
    case 2: return tile_shape_np2(dim, variant, tx, ty);
    case 3: return tile_shape_np3(dim, variant, tx, ty);
    case 4: return tile_shape_np4(dim, variant, tx, ty);
    case 5: return tile_shape_np5(dim, variant, tx, ty);
    case 6: return tile_shape_np6(dim, variant, tx, ty);
  }
  return -1;
}

// one thread per member of a group: the top / bottom of its loop body
__global__ void batch_begin_kernel(const BatchInst* insts, const int* members, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const BatchInst& I = insts[members[k]];
  if (I.sc) step_begin_device(I.sc);
}
__global__ void batch_end_kernel(const BatchInst* insts, const int* members, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const BatchInst& I = insts[members[k]];
  if (I.sc) step_end_device(I.sc, I.rk2 ? 2 : 3);
}
// gather every instance's status for one host copy; count running ones
__global__ void batch_status_kernel(const BatchInst* insts, int n, BatchStatus* out, int* nrun) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevScalars* sc = insts[i].sc;
  if (!sc) {
    out[i].status = -1;
    return;
  }
  out[i].status = sc->status;
  out[i].active = sc->active;
  out[i].n_steps = sc->n_steps;
  out[i].t = sc->t;
  if (sc->status == kRunning) atomicAdd(nrun, 1);
}

}  // namespace frg

using namespace frg;
using namespace frg::rt;

struct frg_batch {
  frg_ctx* ctx = nullptr;
  int cap = 0;
  std::vector<frg_solve*> slot;  // nullptr: free
  std::vector<char> running;
  BatchInst* d_insts = nullptr;
  BatchStatus* d_status = nullptr;
  BatchStatus* h_status = nullptr;  // pinned
  int* d_nrun = nullptr;
  int* h_nrun = nullptr;  // pinned
  struct Group {
    int dim, np, flux, av, variant;
    int hook = 0;     // post-step hook id shared by the members (kHookNone: none)
    int tx = 1, ty = 1;  // tile shape of the batched kernels
    // solo: one instance large enough to fill the device by itself, stepped
    // with the single-solve stage kernels (its own tuned tile shape)
    bool solo = false;
    HostOps ops;  // the group's tables (copied: members come and go)
    std::vector<BatchTile> tiles;
    std::vector<int> members;
    size_t ndof = 0;
    int reps = 1;  // steps per round
    void* d_buf = nullptr;  // tiles, then members
    size_t d_bytes = 0;
    const BatchTile* d_tiles() const { return (const BatchTile*)d_buf; }
    const int* d_members() const { return (const int*)((const char*)d_buf + sizeof(BatchTile) * tiles.size()); }
  };
  std::vector<Group> groups;
  std::vector<BatchInst> h_insts;  // the instance table as last uploaded
  // groups advance as parallel branches: an instance's stages depend only on
  // its own previous stage
  static constexpr int kAux = 16;
  cudaStream_t aux[kAux] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kAux] = {};
  cudaGraphExec_t graph = nullptr;
  int graph_rounds = 0;
  bool dirty = true;
  bool multirate = false;
  size_t budget = 0, used = 0;  // HBM admission budget (bytes, 0 = none)
};

namespace {

constexpr int kMaxReps = 32;  // multirate: most steps per round of one group
// An instance with at least a full wave of resident batched tiles (148 SMs
// times the batched kernel's CTAs per SM) gains nothing from sharing launches
// and runs solo.
constexpr int kSMs = 148;

int bcheck(frg_batch* b, cudaError_t e, const char* what) { return cuda_err(b->ctx, e, what); }

BatchInst inst_of(frg_solve* s) {
  BatchInst I;
  std::memset(&I, 0, sizeof(I));
  if (!s) return I;
  I.M2 = s->L2.mesh;
  I.M1 = s->L1.mesh;
  I.P = s->dim == 2 ? s->L2.phys : s->L1.phys;
  for (int k = 0; k < 3; ++k) {
    I.U[k] = s->U[k];
    I.E[k] = s->E[k];
  }
  I.sc = s->sc;
  I.rk2 = s->time_scheme == FRG_TIME_SSP_RK2;
  I.dim = s->dim;
  I.hook = s->post_step_id;
  I.hook_params[0] = s->post_step_params[0];
  I.hook_params[1] = s->post_step_params[1];
  return I;
}

bool same_tables(const HostOps& a, const HostOps& b) {
  if (a.np != b.np) return false;
  const int n = a.np;
  for (int i = 0; i < n; ++i) {
    if (a.xi[i] != b.xi[i] || a.w[i] != b.w[i] || a.lL[i] != b.lL[i] || a.lR[i] != b.lR[i] || a.gLxi[i] != b.gLxi[i] ||
        a.gRxi[i] != b.gRxi[i] || a.lLD[i] != b.lLD[i] || a.lRD[i] != b.lRD[i])
      return false;
    for (int k = 0; k < n; ++k)
      if (a.Dt[i][k] != b.Dt[i][k] || a.DtD[i][k] != b.DtD[i][k] || a.DD[i][k] != b.DD[i][k] ||
          a.Vinv[i][k] != b.Vinv[i][k])
        return false;
  }
  return true;
}

// Rebuild the instance table, the groups and their tile lists.
int rebuild(frg_batch* b) {
  std::vector<BatchInst>& insts = b->h_insts;
  insts.assign(b->cap, BatchInst{});
  for (int i = 0; i < b->cap; ++i) insts[i] = inst_of(b->slot[i]);
  int rc = bcheck(b, cudaMemcpyAsync(b->d_insts, insts.data(), sizeof(BatchInst) * b->cap,
                                     cudaMemcpyHostToDevice, b->ctx->stream), "batch instances");
  if (rc) return rc;
  for (auto& g : b->groups) {
    g.tiles.clear();
    g.members.clear();
    g.ndof = 0;
  }
  for (int i = 0; i < b->cap; ++i) {
    frg_solve* s = b->slot[i];
    if (!s) continue;
    const int av = s->dim == 2 ? s->L2.av : s->L1.av;
    const int flux = s->dim == 2 ? s->L2.flux : s->L1.flux;
    // the key's variant from the autotune table, else the fixed default tile
    int variant = -1;
    if (s->dim == 2 && !autotune_table_lookup(s->np - 1, flux, av, s->L2.mesh.curved ? 1 : 0, &variant))
      variant = -1;
    int tx = 1, ty = 1;
    const int per_sm = batch_tile_shape(s->dim, s->np, variant, &tx, &ty);
    // the choice depends on the instance alone, so its results do not
    // depend on what else is in the batch
    const bool solo =
        s->dim == 2 && (long)((s->nx + tx - 1) / tx) * ((s->ny + ty - 1) / ty) >= (long)kSMs * per_sm;
    frg_batch::Group* grp = nullptr;
    if (!solo)
      for (auto& g : b->groups)
        if (!g.solo && g.dim == s->dim && g.np == s->np && g.flux == flux && g.av == av && g.variant == variant &&
            g.hook == s->post_step_id && same_tables(g.ops, s->ops)) {
          grp = &g;
          break;
        }
    if (!grp)
      for (auto& g : b->groups)  // reuse an emptied group's device buffer
        if (g.members.empty()) {
          grp = &g;
          break;
        }
    if (!grp) {
      b->groups.emplace_back();
      grp = &b->groups.back();
    }
    if (grp->members.empty()) {
      grp->dim = s->dim;
      grp->np = s->np;
      grp->flux = flux;
      grp->av = av;
      grp->variant = variant;
      grp->solo = solo;
      grp->hook = s->post_step_id;
      grp->tx = tx;
      grp->ty = ty;
      grp->ops = s->ops;
    }
    grp->members.push_back(i);
    grp->ndof += s->ndof;
    if (solo) continue;
    if (s->dim == 2) {
      for (int y = 0; y < s->ny; y += ty)
        for (int x = 0; x < s->nx; x += tx) grp->tiles.push_back(BatchTile{i, x, y, 0});
    } else {
      for (int x = 0; x < s->nx; x += tx) grp->tiles.push_back(BatchTile{i, x, 0, 0});
    }
  }
  // drop empty groups, upload tile and member lists
  b->groups.erase(std::remove_if(b->groups.begin(), b->groups.end(),
                                 [](const frg_batch::Group& g) {
                                   if (g.members.empty() && g.d_buf) cudaFree(g.d_buf);
                                   return g.members.empty();
                                 }),
                  b->groups.end());
  for (auto& g : b->groups) {
    const size_t need = sizeof(BatchTile) * g.tiles.size() + sizeof(int) * g.members.size();
    if (need > g.d_bytes) {
      if (g.d_buf) cudaFree(g.d_buf);
      g.d_buf = nullptr;
      g.d_bytes = 0;
      if ((rc = bcheck(b, cudaMalloc(&g.d_buf, 2 * need), "tile list"))) return rc;
      g.d_bytes = 2 * need;
    }
    std::vector<char> host(need);
    std::memcpy(host.data(), g.tiles.data(), sizeof(BatchTile) * g.tiles.size());
    std::memcpy(host.data() + sizeof(BatchTile) * g.tiles.size(), g.members.data(),
                sizeof(int) * g.members.size());
    if ((rc = bcheck(b, cudaMemcpy(g.d_buf, host.data(), need, cudaMemcpyHostToDevice), "tile list upload")))
      return rc;
  }
  // steps per round: lockstep, or inversely proportional to the modelled
  // step time of the group (a fixed launch floor plus a per-DOF cost)
  double tmax = 0.0;
  auto step_us = [](const frg_batch::Group& g) { return 25.0 + 3.0 * (double)g.ndof / 30e3; };
  for (auto& g : b->groups) tmax = std::max(tmax, step_us(g));
  for (auto& g : b->groups) {
    g.reps = 1;
    if (b->multirate) g.reps = std::max(1, std::min(kMaxReps, (int)(tmax / step_us(g))));
  }
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->dirty = false;
  return FRG_OK;
}

int enqueue_group_step(frg_batch* b, const frg_batch::Group& g, cudaStream_t st) {
  const int m = (int)g.members.size();
  const int nb = (m + 127) / 128;
  batch_begin_kernel<<<nb, 128, 0, st>>>(b->d_insts, g.d_members(), m);
  if (g.solo) {
    const frg_solve* s = b->slot[g.members[0]];
    const int ns = s->time_scheme == FRG_TIME_SSP_RK2 ? 2 : 3;
    for (int stage = 1; stage <= ns; ++stage) {
      const int e = launch_stage2d(s->L2, stage_bufs(s, stage, true), st);
      if (e) return bcheck(b, (cudaError_t)e, "solo stage launch");
    }
    batch_end_kernel<<<nb, 128, 0, st>>>(b->d_insts, g.d_members(), m);
    const int rc = bcheck(b, cudaGetLastError(), "batch control kernels");
    // post_step! of a completed step (SSP_RK3.jl:162), as a single solve runs it
    return rc ? rc : enqueue_post_step_on(b->slot[g.members[0]], false, st);
  }
  for (int stage = 1; stage <= 3; ++stage) {
    const int e = g.dim == 2 ? launch_batch2d(&g.ops, g.flux, g.av, g.variant, b->d_insts, g.d_tiles(),
                                              (int)g.tiles.size(), stage, kModeStage, st)
                             : launch_batch1d(&g.ops, g.flux, g.av, b->d_insts, g.d_tiles(),
                                              (int)g.tiles.size(), stage, kModeStage, st);
    if (e) return bcheck(b, (cudaError_t)e, "batched stage launch");
  }
  batch_end_kernel<<<nb, 128, 0, st>>>(b->d_insts, g.d_members(), m);
  int rc = bcheck(b, cudaGetLastError(), "batch control kernels");
  if (rc || !g.hook) return rc;
  // post_step! of the members whose step completed (SSP_RK3.jl:162), then the
  // element viscosity and CFL wave speed of their limited states
  int e = enqueue_batch_post_step(g.ops, g.tx, g.ty, b->d_insts, g.d_tiles(), (int)g.tiles.size(), st);
  if (!e)
    e = g.dim == 2 ? launch_batch2d(&g.ops, g.flux, g.av, g.variant, b->d_insts, g.d_tiles(), (int)g.tiles.size(),
                                    0, kModePrime, st)
                   : launch_batch1d(&g.ops, g.flux, g.av, b->d_insts, g.d_tiles(), (int)g.tiles.size(), 0,
                                    kModePrime, st);
  return e ? bcheck(b, (cudaError_t)e, "batched post-step hook") : FRG_OK;
}

// `rounds` rounds of every group (group g takes rounds * reps_g steps); the
// groups are parallel branches forked from and joined back to the stream.
int enqueue_rounds(frg_batch* b, int rounds) {
  cudaStream_t main = b->ctx->stream;
  const int ng = (int)b->groups.size();
  const int nbr = ng < frg_batch::kAux ? ng : frg_batch::kAux;
  int rc;
  if (nbr <= 1) {
    for (int r = 0; r < rounds; ++r)
      for (auto& g : b->groups)
        for (int k = 0; k < g.reps; ++k)
          if ((rc = enqueue_group_step(b, g, main))) return rc;
    return FRG_OK;
  }
  if ((rc = bcheck(b, cudaEventRecord(b->fork, main), "fork"))) return rc;
  for (int k = 0; k < nbr; ++k)
    if ((rc = bcheck(b, cudaStreamWaitEvent(b->aux[k], b->fork, 0), "fork wait"))) return rc;
  // heaviest groups first, dealt round-robin over the branches
  std::vector<int> order(ng);
  for (int k = 0; k < ng; ++k) order[k] = k;
  std::sort(order.begin(), order.end(), [&](int x, int y) {
    return b->groups[x].ndof * b->groups[x].reps > b->groups[y].ndof * b->groups[y].reps;
  });
  for (int r = 0; r < rounds; ++r)
    for (int k = 0; k < ng; ++k) {
      const frg_batch::Group& g = b->groups[order[k]];
      for (int q = 0; q < g.reps; ++q)
        if ((rc = enqueue_group_step(b, g, b->aux[k % nbr]))) return rc;
    }
  for (int k = 0; k < nbr; ++k) {
    if ((rc = bcheck(b, cudaEventRecord(b->join[k], b->aux[k]), "join"))) return rc;
    if ((rc = bcheck(b, cudaStreamWaitEvent(main, b->join[k], 0), "join wait"))) return rc;
  }
  return FRG_OK;
}

int poll(frg_batch* b, int* nrun) {
  int rc = bcheck(b, cudaMemsetAsync(b->d_nrun, 0, sizeof(int), b->ctx->stream), "poll");
  if (rc) return rc;
  batch_status_kernel<<<(b->cap + 127) / 128, 128, 0, b->ctx->stream>>>(b->d_insts, b->cap, b->d_status,
                                                                        b->d_nrun);
  if ((rc = bcheck(b, cudaMemcpyAsync(b->h_status, b->d_status, sizeof(BatchStatus) * b->cap,
                                      cudaMemcpyDeviceToHost, b->ctx->stream), "poll copy")))
    return rc;
  if ((rc = bcheck(b, cudaMemcpyAsync(b->h_nrun, b->d_nrun, sizeof(int), cudaMemcpyDeviceToHost,
                                      b->ctx->stream), "poll copy")))
    return rc;
  if ((rc = bcheck(b, cudaStreamSynchronize(b->ctx->stream), "poll sync"))) return rc;
  *nrun = *b->h_nrun;
  return FRG_OK;
}

void release_batch(frg_batch* b) {
  for (auto& g : b->groups)
    if (g.d_buf) cudaFree(g.d_buf);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (int k = 0; k < frg_batch::kAux; ++k) {
    if (b->aux[k]) cudaStreamDestroy(b->aux[k]);
    if (b->join[k]) cudaEventDestroy(b->join[k]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  cudaFree(b->d_insts);
  cudaFree(b->d_status);
  cudaFree(b->d_nrun);
  cudaFreeHost(b->h_status);
  cudaFreeHost(b->h_nrun);
  delete b;
}

}  // namespace

extern "C" {

int frg_batch_create(frg_ctx* ctx, int capacity, size_t hbm_budget, frg_batch** out) {
  if (!ctx || !out || capacity < 1) return FRG_ERR_INVALID_ARG;
  *out = nullptr;
  cudaSetDevice(ctx->device);
  frg_batch* b = new (std::nothrow) frg_batch();
  if (!b) return FRG_ERR_OOM;
  b->ctx = ctx;
  b->cap = capacity;
  b->budget = hbm_budget;
  b->slot.assign(capacity, nullptr);
  b->running.assign(capacity, 0);
  int rc = bcheck(b, cudaMalloc((void**)&b->d_insts, sizeof(BatchInst) * capacity), "batch table");
  if (!rc) rc = bcheck(b, cudaMalloc((void**)&b->d_status, sizeof(BatchStatus) * capacity), "batch status");
  if (!rc) rc = bcheck(b, cudaMalloc((void**)&b->d_nrun, sizeof(int)), "batch counter");
  if (!rc) rc = bcheck(b, cudaMallocHost((void**)&b->h_status, sizeof(BatchStatus) * capacity), "pinned status");
  if (!rc) rc = bcheck(b, cudaMallocHost((void**)&b->h_nrun, sizeof(int)), "pinned counter");
  if (!rc) rc = bcheck(b, cudaMemset(b->d_insts, 0, sizeof(BatchInst) * capacity), "batch table");
  for (int k = 0; k < frg_batch::kAux && !rc; ++k) {
    rc = bcheck(b, cudaStreamCreateWithFlags(&b->aux[k], cudaStreamNonBlocking), "branch stream");
    if (!rc) rc = bcheck(b, cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming), "branch event");
  }
  if (!rc) rc = bcheck(b, cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "fork event");
  if (rc) {
    release_batch(b);
    return rc;
  }
  *out = b;
  return FRG_OK;
}

int frg_batch_destroy(frg_batch* b) {
  if (!b) return FRG_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  for (frg_solve* s : b->slot)
    if (s) frg_solve_destroy(s);
  release_batch(b);
  return FRG_OK;
}

int frg_batch_add(frg_batch* b, const frg_solve_desc* desc, int* slot) {
  if (!b || !desc || !slot) return FRG_ERR_INVALID_ARG;
  int free_slot = -1;
  for (int i = 0; i < b->cap; ++i)
    if (!b->slot[i]) {
      free_slot = i;
      break;
    }
  if (free_slot < 0) return set_err(b->ctx, FRG_ERR_OOM, "batch is full");
  frg_solve* s = nullptr;
  int rc = frg_solve_create(b->ctx, desc, &s);
  if (rc) return rc;
  if (b->budget && b->used + s->bytes > b->budget) {
    frg_solve_destroy(s);
    return set_err(b->ctx, FRG_ERR_OOM, "HBM budget of the batch exceeded");
  }
  // idle until frg_batch_start: the batch's step kernels skip it
  s->hsc->status = kFinished;
  if ((rc = push_scalars(s))) {
    frg_solve_destroy(s);
    return rc;
  }
  b->used += s->bytes;
  b->slot[free_slot] = s;
  b->running[free_slot] = 0;
  b->dirty = true;
  *slot = free_slot;
  return FRG_OK;
}

int frg_batch_remove(frg_batch* b, int i) {
  if (!b || i < 0 || i >= b->cap || !b->slot[i]) return FRG_ERR_INVALID_ARG;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  b->used -= b->slot[i]->bytes;
  frg_solve_destroy(b->slot[i]);
  b->slot[i] = nullptr;
  b->running[i] = 0;
  b->dirty = true;
  return FRG_OK;
}

// Upper bound of the device bytes a solve of this descriptor holds while it
// advances (state buffers, viscosity buffers, mesh arrays, status block): the
// admission test of a served batch.
int frg_solve_bytes(const frg_solve_desc* d, size_t* bytes) {
  if (!d || !bytes || d->nx < 1 || d->p < 1 || d->p > FRG_MAX_NP - 1) return FRG_ERR_INVALID_ARG;
  const size_t np = (size_t)d->p + 1;
  const size_t nx = (size_t)d->nx, ny = d->dim == 2 ? (size_t)(d->ny < 1 ? 1 : d->ny) : 1;
  const size_t nel = nx * ny;
  const size_t ndof = d->dim == 2 ? nel * np * np * 4 : nel * np * 3;
  size_t n = 3 * ndof + 3 * nel + (sizeof(DevScalars) + 7) / 8;  // U[3], E[3], scalars
  if (d->dim == 2) {
    n += 3 * (nx + ny) + nel;  // column / row spacing, h_char
    if (d->solid) n += nel / 8 + 1;
    if (d->geometry != FRG_GEOM_AFFINE) n += nel * (5 * np * np + 12 * np);  // SP metrics, face normals
  } else {
    n += 4 * nel;  // centres, J, dx, h
  }
  *bytes = 8 * n + 16 * 24;  // allocation padding
  return FRG_OK;
}

// Lockstep (0, default) or multirate (1) scheduling of the groups.
int frg_batch_set_multirate(frg_batch* b, int on) {
  if (!b) return FRG_ERR_INVALID_ARG;
  b->multirate = on != 0;
  b->dirty = true;
  return FRG_OK;
}

int frg_batch_get_solve(frg_batch* b, int i, frg_solve** s) {
  if (!b || i < 0 || i >= b->cap || !s) return FRG_ERR_INVALID_ARG;
  *s = b->slot[i];
  return *s ? FRG_OK : FRG_ERR_INVALID_ARG;
}

int frg_batch_slot_group(frg_batch* b, int i, int* variant, int* solo) {
  if (!b || i < 0 || i >= b->cap || !b->slot[i]) return FRG_ERR_INVALID_ARG;
  for (const auto& g : b->groups)
    for (int m : g.members)
      if (m == i) {
        if (variant) *variant = g.variant;
        if (solo) *solo = g.solo ? 1 : 0;
        return FRG_OK;
      }
  return FRG_ERR_STATE;  // not grouped yet: no frg_batch_run since it was added
}

// Configure an instance's run (integrate! arguments) and mark it running.
int frg_batch_start(frg_batch* b, int i, double t_final, double cfl, double fixed_dt, int64_t max_steps) {
  if (!b || i < 0 || i >= b->cap || !b->slot[i]) return FRG_ERR_INVALID_ARG;
  if (b->slot[i]->pre_id)
    return set_err(b->ctx, FRG_ERR_UNSUPPORTED_HOOK, "batched solves do not run preprocess_state hooks");
  frg_solve* s = b->slot[i];
  if (!s->have_state) return set_err(b->ctx, FRG_ERR_STATE, "no state uploaded");
  if (max_steps < 1 || (!(fixed_dt > 0.0) && !(cfl > 0.0))) return set_err(b->ctx, FRG_ERR_INVALID_ARG, "run");
  cudaSetDevice(b->ctx->device);
  int rc = make_current_canonical(s);
  if (rc) return rc;
  init_run_scalars(s, t_final, cfl, fixed_dt, max_steps);
  if ((rc = push_scalars(s))) return rc;
  if ((rc = prime(s, 0, true))) return rc;  // eps of the state, CFL wave speed
  // a hook selected after the last rebuild regroups the instance
  const BatchInst I = inst_of(s);
  if (i >= (int)b->h_insts.size() || b->h_insts[i].hook != I.hook ||
      b->h_insts[i].hook_params[0] != I.hook_params[0] || b->h_insts[i].hook_params[1] != I.hook_params[1] ||
      b->h_insts[i].P.flux_alpha != I.P.flux_alpha || b->h_insts[i].P.trace_hook != I.P.trace_hook ||
      b->h_insts[i].P.trace_p0 != I.P.trace_p0 || b->h_insts[i].P.trace_p1 != I.P.trace_p1)
    b->dirty = true;
  b->running[i] = 1;
  return FRG_OK;
}

// Advance every running instance by up to `max_steps` rounds (lockstep: one
// step per round; multirate: reps_g steps per round for group g), or until
// all have stopped.  results (capacity entries, may be NULL) receive each
// slot's status; *n_running the number still running.
int frg_batch_run(frg_batch* b, int64_t max_steps, frg_result* results, int* n_running) {
  if (!b || max_steps < 1) return FRG_ERR_INVALID_ARG;
  cudaSetDevice(b->ctx->device);
  int rc;
  if (b->dirty && (rc = rebuild(b))) return rc;
  int64_t total = 0;
  int nrun = 0;
  for (int i = 0; i < b->cap; ++i) nrun += b->running[i] ? 1 : 0;
  // rounds per graph: a few milliseconds of work and at most ~600 kernels
  size_t work = 0;
  int nodes = 0;
  for (auto& g : b->groups) {
    work += g.ndof * (size_t)g.reps;
    nodes += (g.hook ? 7 : 5) * g.reps;
  }
  int K = work > 4000000 ? 4 : (work > 400000 ? 8 : 16);
  while (K > 1 && K * nodes > 600) K /= 2;
  while (nrun > 0 && total < max_steps) {
    const int k = (int)std::min<int64_t>(K, max_steps - total);
    if (k == K) {
      if (!b->graph || b->graph_rounds != K) {
        if (b->graph) cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        cudaGraph_t g;
        if ((rc = bcheck(b, cudaStreamBeginCapture(b->ctx->stream, cudaStreamCaptureModeThreadLocal),
                         "batch capture")))
          return rc;
        const int crc = enqueue_rounds(b, K);
        cudaError_t ce = cudaStreamEndCapture(b->ctx->stream, &g);
        if (crc) return crc;
        if ((rc = bcheck(b, ce, "batch capture end"))) return rc;
        ce = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if ((rc = bcheck(b, ce, "batch graph"))) return rc;
        b->graph_rounds = K;
      }
      if ((rc = bcheck(b, cudaGraphLaunch(b->graph, b->ctx->stream), "batch graph launch"))) return rc;
    } else if ((rc = enqueue_rounds(b, k))) {
      return rc;
    }
    total += k;
    if ((rc = poll(b, &nrun))) return rc;
    for (int i = 0; i < b->cap; ++i) {
      if (!b->running[i] || !b->slot[i]) continue;
      if (b->h_status[i].status != kRunning) {
        b->running[i] = 0;
        if ((rc = finish_run(b->slot[i]))) return rc;
      }
    }
  }
  if (total == 0 && (rc = poll(b, &nrun))) return rc;
  if (results)
    for (int i = 0; i < b->cap; ++i) {
      results[i].status = FRG_ERR_STATE;  // empty slot
      results[i].n_steps = 0;
      results[i].t = 0.0;
      if (!b->slot[i] || b->h_status[i].status < 0) continue;
      const int st = b->h_status[i].status;
      results[i].status = st == kFinished ? FRG_OK : (st == kRunning ? FRG_RUNNING : st);
      results[i].n_steps = b->h_status[i].n_steps;
      results[i].t = b->h_status[i].t;
    }
  if (n_running) *n_running = nrun;
  return FRG_OK;
}

}  // extern "C"
