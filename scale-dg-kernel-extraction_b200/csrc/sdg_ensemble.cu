// Ensembles of independent DG advection instances on one GPU: the batched
// form (fixed membership, CUDA-graph RK steps, autotuned tile shapes) and
// the serving loop (requests admitted by free memory while others run).
//
// Each instance is a periodic box of NeX x NeY x NeZ elements of order p with
// its own state, velocity and dt, stored exactly like a single handle's
// resident state.  Instances with the same order and precision form a group;
// one RK stage of a group is ONE persistent launch of the pipelined fused
// kernel over a tile table (instance, first element, count) with
// per-instance array pointers and dt.  A batch step runs its groups one
// after another on the ensemble stream: each persistent launch deals its
// tiles out round-robin over a grid sized for the whole GPU, and concurrent
// groups (measured on the 96-instance ensemble: FP64 79.2 against 85.5 G
// DOF-updates/s sequential, mixed 113.9 against 124.2 G) left blocks that
// started late holding the tail.  The serving loop's groups are smaller and
// their launches' tails longer: they run on their own streams, forked from
// and joined back to the ensemble stream, so the tails overlap (busy
// throughput on 200 served requests 78.0 against 75.9 G sequential).
// Per-instance arithmetic does not depend on the group, its tiling or the
// chosen kernel variant (all variants compute bit-identical results), so an
// instance's result is the same alone, in a batch or in a served mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "sdg_gpu.h"
#include "sdg_internal.h"
#include "sdg_launch.h"
#include "sdg_tend.cuh"

namespace sdg {
namespace {

#define ENS_CUDA(call)                                                     \
  do {                                                                     \
    cudaError_t err_ = (call);                                             \
    if (err_ != cudaSuccess)                                               \
      return fail(SDG_ERR_CUDA, "%s failed: %s", #call,                    \
                  cudaGetErrorString(err_));                               \
  } while (0)

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

__global__ void ens_to_f32(float* __restrict__ out, const double* __restrict__ in, long n) {
  for (long x = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<long>(gridDim.x) * blockDim.x)
    out[x] = static_cast<float>(in[x]);
}

// Operators of one order, shared by every instance of that order.
struct Ops {
  int nq = 0;
  std::vector<double> D;      // row-major D(i,l)
  std::vector<double> lift;   // Lift_mat(Np,6)
  double* lift64 = nullptr;   // verbatim (exact kernels)
  double* lift64f = nullptr;  // factored when Lift_mat factorises (fast kernels)
  float* lift32 = nullptr;    // the fast table in FP32 (mixed kernels)
  std::vector<double> lift_z; // z-face factors (2, Nq); empty: not factored
};

enum InstState { kQueued = 0, kRunning = 1, kDone = 2, kFailed = 3 };

struct Inst {
  int id = 0;
  int nex = 0, ney = 0, nez = 0, p = 0, nq = 0, np = 0, ne = 0;
  double dt = 0;
  bool mixed = false;
  // Device state (stream-ordered pool allocations).
  double* q0 = nullptr;
  void* qa = nullptr;
  void* qb = nullptr;
  void* vel[3] = {nullptr, nullptr, nullptr};
  double* vel64 = nullptr;  // upload staging for mixed velocity
  int* pbase = nullptr;
  void* esc = nullptr;
  void* fsc = nullptr;
  size_t bytes = 0;
  // Serving bookkeeping.
  long long steps_left = 0;
  long long steps_total = 0;
  int state = kQueued;
  double t_submit = 0, t_admit = 0, t_done = 0;
  std::vector<double> host[4];   // q, u, v, w (Np, Ne) until admitted
  std::vector<double> result;    // q (Np, Ne) once done
};

size_t inst_bytes(int np, int ne, bool mixed) {
  const size_t n = static_cast<size_t>(np) * ne;
  const size_t es = mixed ? 4 : 8;
  return n * 8 + 2 * n * es + 3 * n * es + (mixed ? n * 8 : 0) + 6 * ne * 4 +
         9 * ne * 8 + 16 * 16;
}

// Compressed tables of the periodic unit box, identical to what sdg_init
// derives from mesh_setup's VMapM/VMapP/Escale/Fscale (mod_mesh.f90:74-193)
// in direct-periodic mode.
void box_tables(int nex, int ney, int nez, int np, std::vector<int>* pb,
                std::vector<double>* esc, std::vector<double>* fsc) {
  const int ne = nex * ney * nez;
  const double dx = 1.0 / static_cast<double>(nex);
  const double dy = 1.0 / static_cast<double>(ney);
  const double dz = 1.0 / static_cast<double>(nez);
  const double h[3] = {dx, dy, dz};
  pb->resize(6L * ne);
  esc->resize(3L * ne);
  fsc->resize(6L * ne);
  for (int k = 0; k < nez; ++k)
    for (int j = 0; j < ney; ++j)
      for (int i = 0; i < nex; ++i) {
        const long e = i + static_cast<long>(nex) * (j + static_cast<long>(ney) * k);
        const int nb[6] = {
            i + nex * ((j + ney - 1) % ney + ney * k),  // -y
            (i + 1) % nex + nex * (j + ney * k),        // +x
            i + nex * ((j + 1) % ney + ney * k),        // +y
            (i + nex - 1) % nex + nex * (j + ney * k),  // -x
            i + nex * (j + ney * ((k + nez - 1) % nez)),  // -z
            i + nex * (j + ney * ((k + 1) % nez))};       // +z
        for (int f = 0; f < 6; ++f) {
          (*pb)[6 * e + f] = nb[f] * np;
          (*fsc)[6 * e + f] = 2.0 / h[kFaceAxis[f]];
        }
        for (int d = 0; d < 3; ++d) (*esc)[3 * e + d] = 2.0 / h[d];
      }
}

template <typename T>
int pool_alloc(T** p, size_t bytes, cudaStream_t st) {
  void* v = nullptr;
  cudaError_t e = cudaMallocAsync(&v, bytes + 16, st);
  if (e != cudaSuccess)
    return fail(SDG_ERR_CUDA, "device allocation of %zu bytes failed: %s", bytes,
                cudaGetErrorString(e));
  *p = static_cast<T*>(v);
  return SDG_OK;
}

// One order and precision: members, tile tables, chosen kernel variant.
struct Group {
  int nq = 0;
  bool mixed = false;
  int flags = 0;
  Ops* ops = nullptr;
  std::vector<Inst*> members;
  int epb = 1;
  int variant = kVariantAuto;   // set by the autotuner
  bool dirty = true;
  // Device tables, two buffers: a rebuild writes the buffer that no launch
  // still in flight reads (at most two chunks of steps are in flight in the
  // serving loop) and makes it current.
  BatchInst* d_insts_buf[2] = {nullptr, nullptr};  // [3][inst_cap]
  BatchTile* d_tiles_buf[2] = {nullptr, nullptr};
  int inst_cap_buf[2] = {0, 0}, tile_cap_buf[2] = {0, 0};
  int cur = 0;
  BatchInst* d_insts = nullptr;  // the current buffer
  BatchTile* d_tiles = nullptr;
  int inst_cap = 0, tile_cap = 0, ntiles = 0;
  std::vector<BatchInst> h_insts;
  std::vector<BatchTile> h_tiles;
  cudaStream_t stream = nullptr;  // concurrent steps, autotuning, set-up
  cudaEvent_t done = nullptr;
  double tuned_ms[5] = {0, 0, 0, 0, 0};  // by KernelVariant
};

struct Ensemble {
  int flags = 0;  // SDG_FLAG_EXACT | SDG_FLAG_ORDER_GENERAL (FP64 arithmetic)
  int dev = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  int* status = nullptr;
  unsigned wait_spins = 0;  // bounded-wait spin limit (0: default)
  int inject_skip = 0;      // test hook: tile + 1 left without copies
  std::map<int, std::unique_ptr<Ops>> ops;              // by nq
  std::map<std::pair<int, bool>, std::unique_ptr<Group>> groups;

  ~Ensemble() {
    cudaSetDevice(dev);
    if (stream) cudaStreamSynchronize(stream);
    for (auto& g : groups) {
      for (int b = 0; b < 2; ++b) {
        if (g.second->d_insts_buf[b]) cudaFree(g.second->d_insts_buf[b]);
        if (g.second->d_tiles_buf[b]) cudaFree(g.second->d_tiles_buf[b]);
      }
      if (g.second->stream) cudaStreamDestroy(g.second->stream);
      if (g.second->done) cudaEventDestroy(g.second->done);
    }
    for (auto& o : ops) {
      if (o.second->lift64) cudaFree(o.second->lift64);
      if (o.second->lift64f) cudaFree(o.second->lift64f);
      if (o.second->lift32) cudaFree(o.second->lift32);
    }
    if (status) cudaFree(status);
    if (fork) cudaEventDestroy(fork);
    if (stream) cudaStreamDestroy(stream);
  }

  int init(int fl) {
    flags = fl;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      return fail(SDG_ERR_CUDA, "no CUDA device available; this library has no CPU path");
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) num_sms = prop.multiProcessorCount;
    ENS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    ENS_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    ENS_CUDA(cudaMalloc(&status, sizeof(int)));
    ENS_CUDA(cudaMemset(status, 0, sizeof(int)));
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;  // keep freed blocks cached for reuse
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    return SDG_OK;
  }

  int ops_for(int p, const double* D1D, const double* Lift, Ops** out) {
    const int nq = p + 1, np = nq * nq * nq;
    auto it = ops.find(nq);
    if (it != ops.end()) {
      Ops* o = it->second.get();
      for (int i = 0; i < nq; ++i)
        for (int l = 0; l < nq; ++l)
          if (o->D[i * nq + l] != D1D[i + nq * l])
            return fail(SDG_ERR_ARG, "instances of order %d must share one D1D", p);
      for (long x = 0; x < 6L * np; ++x)
        if (o->lift[x] != Lift[x])
          return fail(SDG_ERR_ARG, "instances of order %d must share one Lift_mat", p);
      *out = o;
      return SDG_OK;
    }
    auto o = std::make_unique<Ops>();
    o->nq = nq;
    o->D.resize(nq * nq);
    for (int i = 0; i < nq; ++i)
      for (int l = 0; l < nq; ++l) o->D[i * nq + l] = D1D[i + nq * l];
    o->lift.assign(Lift, Lift + 6L * np);
    std::vector<double> fact;
    if (!lift_factor(Lift, nq, &fact, &o->lift_z)) fact.clear();
    const double* fast = fact.empty() ? Lift : fact.data();
    std::vector<float> l32(6L * np);
    for (long x = 0; x < 6L * np; ++x) l32[x] = static_cast<float>(fast[x]);
    ENS_CUDA(cudaMalloc(&o->lift64, 6L * np * sizeof(double)));
    ENS_CUDA(cudaMalloc(&o->lift64f, 6L * np * sizeof(double)));
    ENS_CUDA(cudaMalloc(&o->lift32, 6L * np * sizeof(float)));
    ENS_CUDA(cudaMemcpy(o->lift64, Lift, 6L * np * sizeof(double), cudaMemcpyHostToDevice));
    ENS_CUDA(cudaMemcpy(o->lift64f, fast, 6L * np * sizeof(double), cudaMemcpyHostToDevice));
    ENS_CUDA(cudaMemcpy(o->lift32, l32.data(), 6L * np * sizeof(float),
                        cudaMemcpyHostToDevice));
    *out = o.get();
    ops[nq] = std::move(o);
    return SDG_OK;
  }

  int group_for(int nq, bool mixed, Ops* o, Group** out) {
    auto key = std::make_pair(nq, mixed);
    auto it = groups.find(key);
    if (it != groups.end()) {
      *out = it->second.get();
      return SDG_OK;
    }
    auto g = std::make_unique<Group>();
    g->nq = nq;
    g->mixed = mixed;
    g->flags = mixed ? 0 : flags;
    g->ops = o;
    g->epb = pipe_elems_per_tile(nq);
    // The fast pipelined kernels need the factored lift.
    const bool exact = !mixed && (flags & SDG_FLAG_EXACT);
    const bool can_pipe = pipe_supported(nq, mixed ? kStageMixed2 : kStageF64) &&
                          pipe_supported(nq, mixed ? kStageMixed1 : kStageF64) &&
                          pipe_supported(nq, mixed ? kStageMixed3 : kStageF64) &&
                          (exact || !o->lift_z.empty());
    g->variant = can_pipe ? kVariantPipe : kVariantBlock;
    ENS_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    ENS_CUDA(cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming));
    *out = g.get();
    groups[key] = std::move(g);
    return SDG_OK;
  }

  // Allocates and uploads an instance (host arrays (Np, Ne) or (Np, NeA)).
  int upload(Inst* I, const double* q, const double* u, const double* v, const double* w,
             cudaStream_t st) {
    const size_t n = static_cast<size_t>(I->np) * I->ne;
    const size_t es = I->mixed ? sizeof(float) : sizeof(double);
    int rc;
    if ((rc = pool_alloc(&I->q0, n * 8, st)) || (rc = pool_alloc(&I->qa, n * es, st)) ||
        (rc = pool_alloc(&I->qb, n * es, st)))
      return rc;
    for (int d = 0; d < 3; ++d)
      if ((rc = pool_alloc(&I->vel[d], n * es, st))) return rc;
    if (I->mixed && (rc = pool_alloc(&I->vel64, n * 8, st))) return rc;
    std::vector<int> pb;
    std::vector<double> esc, fsc;
    box_tables(I->nex, I->ney, I->nez, I->np, &pb, &esc, &fsc);
    if ((rc = pool_alloc(&I->pbase, pb.size() * 4, st)) ||
        (rc = pool_alloc(&I->esc, esc.size() * es, st)) ||
        (rc = pool_alloc(&I->fsc, fsc.size() * es, st)))
      return rc;
    ENS_CUDA(cudaMemcpyAsync(I->pbase, pb.data(), pb.size() * 4, cudaMemcpyHostToDevice, st));
    if (I->mixed) {
      std::vector<float> e32(esc.begin(), esc.end()), f32(fsc.begin(), fsc.end());
      ENS_CUDA(cudaMemcpyAsync(I->esc, e32.data(), e32.size() * 4, cudaMemcpyHostToDevice, st));
      ENS_CUDA(cudaMemcpyAsync(I->fsc, f32.data(), f32.size() * 4, cudaMemcpyHostToDevice, st));
      ENS_CUDA(cudaStreamSynchronize(st));  // the host vectors die here
    } else {
      ENS_CUDA(cudaMemcpyAsync(I->esc, esc.data(), esc.size() * 8, cudaMemcpyHostToDevice, st));
      ENS_CUDA(cudaMemcpyAsync(I->fsc, fsc.data(), fsc.size() * 8, cudaMemcpyHostToDevice, st));
    }
    ENS_CUDA(cudaMemcpyAsync(I->q0, q, n * 8, cudaMemcpyHostToDevice, st));
    ENS_CUDA(cudaMemsetAsync(I->qa, 0, n * es, st));
    ENS_CUDA(cudaMemsetAsync(I->qb, 0, n * es, st));
    const double* vh[3] = {u, v, w};
    for (int d = 0; d < 3; ++d) {
      if (I->mixed) {
        ENS_CUDA(cudaMemcpyAsync(I->vel64, vh[d], n * 8, cudaMemcpyHostToDevice, st));
        ens_to_f32<<<num_sms * 4, 256, 0, st>>>(static_cast<float*>(I->vel[d]), I->vel64,
                                                static_cast<long>(n));
        ENS_CUDA(cudaGetLastError());
      } else {
        ENS_CUDA(cudaMemcpyAsync(I->vel[d], vh[d], n * 8, cudaMemcpyHostToDevice, st));
      }
    }
    ENS_CUDA(cudaStreamSynchronize(st));
    if (I->mixed) {
      cudaFreeAsync(I->vel64, st);
      I->vel64 = nullptr;
    }
    I->bytes = inst_bytes(I->np, I->ne, I->mixed);
    return SDG_OK;
  }

  void release(Inst* I, cudaStream_t st) {
    void* ptrs[] = {I->q0, I->qa, I->qb, I->vel[0], I->vel[1], I->vel[2], I->vel64,
                    I->pbase, I->esc, I->fsc};
    for (void* p : ptrs)
      if (p) cudaFreeAsync(p, st);
    I->q0 = nullptr;
    I->qa = I->qb = nullptr;
    I->vel[0] = I->vel[1] = I->vel[2] = nullptr;
    I->vel64 = nullptr;
    I->pbase = nullptr;
    I->esc = I->fsc = nullptr;
  }

  void join(Inst* I, Group* g) {
    g->members.push_back(I);
    g->dirty = true;
  }

  void leave(Inst* I) {
    for (auto& kv : groups) {
      auto& m = kv.second->members;
      auto it = std::find(m.begin(), m.end(), I);
      if (it != m.end()) {
        m.erase(it);
        kv.second->dirty = true;
      }
    }
  }

  // Rebuilds a group's tile table and per-stage instance tables.
  int rebuild(Group* g) {
    if (!g->dirty) return SDG_OK;
    const int ni = static_cast<int>(g->members.size());
    g->h_insts.assign(3L * std::max(ni, 1), BatchInst{});
    g->h_tiles.clear();
    for (int m = 0; m < ni; ++m) {
      Inst* I = g->members[m];
      const void* in[3] = {I->q0, I->qa, I->qb};
      void* out[3] = {I->qa, I->qb, I->q0};
      for (int st = 0; st < 3; ++st) {
        BatchInst& b = g->h_insts[st * ni + m];
        b.q = in[st];
        b.u = I->vel[0];
        b.v = I->vel[1];
        b.w = I->vel[2];
        b.q0 = I->q0;
        b.out = out[st];
        b.pbase = I->pbase;
        b.escale = I->esc;
        b.fscale = I->fsc;
        b.dt = I->dt;
      }
      for (int e0 = 0; e0 < I->ne; e0 += g->epb)
        g->h_tiles.push_back(BatchTile{m, e0, std::min(g->epb, I->ne - e0), 0});
    }
    g->ntiles = static_cast<int>(g->h_tiles.size());
    const int b = g->cur ^ 1;  // the buffer no launch in flight reads
    if (ni > g->inst_cap_buf[b]) {
      if (g->d_insts_buf[b]) cudaFree(g->d_insts_buf[b]);
      g->inst_cap_buf[b] = std::max(ni, 2 * g->inst_cap_buf[b]);
      ENS_CUDA(cudaMalloc(&g->d_insts_buf[b], 3L * g->inst_cap_buf[b] * sizeof(BatchInst)));
    }
    if (g->ntiles > g->tile_cap_buf[b]) {
      if (g->d_tiles_buf[b]) cudaFree(g->d_tiles_buf[b]);
      g->tile_cap_buf[b] = std::max(g->ntiles, 2 * g->tile_cap_buf[b]);
      ENS_CUDA(cudaMalloc(&g->d_tiles_buf[b],
                          static_cast<size_t>(g->tile_cap_buf[b]) * sizeof(BatchTile)));
    }
    g->cur = b;
    g->d_insts = g->d_insts_buf[b];
    g->d_tiles = g->d_tiles_buf[b];
    g->inst_cap = g->inst_cap_buf[b];
    g->tile_cap = g->tile_cap_buf[b];
    if (ni > 0) {
      // Instance tables are laid out [stage][inst_cap]; pad each stage.
      std::vector<BatchInst> padded(3L * g->inst_cap);
      for (int st = 0; st < 3; ++st)
        for (int m = 0; m < ni; ++m) padded[st * g->inst_cap + m] = g->h_insts[st * ni + m];
      ENS_CUDA(cudaMemcpy(g->d_insts, padded.data(), padded.size() * sizeof(BatchInst),
                          cudaMemcpyHostToDevice));
      ENS_CUDA(cudaMemcpy(g->d_tiles, g->h_tiles.data(), g->h_tiles.size() * sizeof(BatchTile),
                          cudaMemcpyHostToDevice));
    }
    g->dirty = false;
    return SDG_OK;
  }

  LaunchSpec spec(Group* g, int st, cudaStream_t s) {
    LaunchSpec l;
    std::memset(&l, 0, sizeof(l));
    l.nq = g->nq;
    l.kind = g->mixed ? (kStageMixed1 + st) : kStageF64;
    l.exact = (g->flags & SDG_FLAG_EXACT) != 0;
    l.order = (g->flags & SDG_FLAG_ORDER_GENERAL) ? kOrderGeneral : kOrderOpt1;
    l.lift = g->mixed  ? static_cast<const void*>(g->ops->lift32)
             : l.exact ? g->ops->lift64
                       : g->ops->lift64f;
    l.D = g->ops->D.data();
    l.lift_z = g->ops->lift_z.empty() ? nullptr : g->ops->lift_z.data();
    l.stream = s;
    l.variant = g->variant;
    l.status = status;
    l.wait_spins = wait_spins;
    l.inject_skip = inject_skip;
    l.num_sms = num_sms;
    const double ra[3] = {0.0, 0.75, 1.0 / 3.0};
    const double rb[3] = {1.0, 0.25, 2.0 / 3.0};
    l.rk_a = ra[st];
    l.rk_b = rb[st];
    return l;
  }

  // One RK stage of a group: one batched launch, or one launch per member
  // for the one-tile-per-block variants.
  int stage(Group* g, int st, cudaStream_t s, int variant) {
    if (g->members.empty()) return SDG_OK;
    LaunchSpec l = spec(g, st, s);
    l.variant = variant;
    if (variant == kVariantPipe || variant == kVariantSplit) {
      l.batch_insts = g->d_insts + st * g->inst_cap;
      l.batch_tiles = g->d_tiles;
      l.batch_ntiles = g->ntiles;
      l.nelem = 1;  // the tile table defines the work
      return launch_tend(l);
    }
    for (Inst* I : g->members) {
      const void* in[3] = {I->q0, I->qa, I->qb};
      void* out[3] = {I->qa, I->qb, I->q0};
      l.q = in[st];
      l.u = I->vel[0];
      l.v = I->vel[1];
      l.w = I->vel[2];
      l.q0 = I->q0;
      l.out = out[st];
      l.pbase = I->pbase;
      l.escale = I->esc;
      l.fscale = I->fsc;
      l.Ne = I->ne;
      l.elem0 = 0;
      l.nelem = I->ne;
      l.dt = I->dt;
      int rc = launch_tend(l);
      if (rc) return rc;
    }
    return SDG_OK;
  }

  // Enqueues one RK step of every member of every group on `s`: with
  // `concurrent`, each group on its own stream, forked from and joined back
  // to `s`; otherwise one group after another on `s`, each alone.
  int step(cudaStream_t s, bool concurrent) {
    for (auto& kv : groups) {
      int rc = rebuild(kv.second.get());
      if (rc) return rc;
    }
    if (concurrent) ENS_CUDA(cudaEventRecord(fork, s));
    for (auto& kv : groups) {
      Group* g = kv.second.get();
      if (g->members.empty()) continue;
      cudaStream_t gs = concurrent ? g->stream : s;
      if (concurrent) ENS_CUDA(cudaStreamWaitEvent(gs, fork, 0));
      for (int st = 0; st < 3; ++st) {
        int rc = stage(g, st, gs, g->variant);
        if (rc) return rc;
      }
      if (concurrent) {
        ENS_CUDA(cudaEventRecord(g->done, gs));
        ENS_CUDA(cudaStreamWaitEvent(s, g->done, 0));
      }
    }
    return SDG_OK;
  }

  // Times the candidate tile shapes of each group on its current members
  // (RK stage 2, which reads q1 and q0 and writes q2; q2 is rewritten by
  // every real step before it is read) and keeps the fastest.
  // The kernel variants a group's launches support.
  std::vector<int> candidates(const Group* g) const {
    std::vector<int> cands;
    const bool can_pipe = pipe_supported(g->nq, g->mixed ? kStageMixed2 : kStageF64) &&
                          pipe_supported(g->nq, g->mixed ? kStageMixed1 : kStageF64) &&
                          pipe_supported(g->nq, g->mixed ? kStageMixed3 : kStageF64);
    if (can_pipe) cands.push_back(kVariantPipe);
    const bool can_split = split_supported(g->nq, g->mixed ? kStageMixed2 : kStageF64) &&
                           split_supported(g->nq, g->mixed ? kStageMixed1 : kStageF64) &&
                           split_supported(g->nq, g->mixed ? kStageMixed3 : kStageF64) &&
                           ((g->flags & SDG_FLAG_EXACT) || !g->ops->lift_z.empty());
    if (can_split) cands.push_back(kVariantSplit);
    cands.push_back(kVariantBlock);
    if (g->nq >= 4 && g->nq <= 8) cands.push_back(kVariantBlockOcc);
    return cands;
  }

  // SDG_KERNEL=block|pipe|blockocc|split, as for a handle: every group whose
  // order supports that variant takes it in place of the autotuner's choice.
  void force_variant() {
    const char* kv = std::getenv("SDG_KERNEL");
    if (!kv) return;
    int v = -1;
    if (std::strcmp(kv, "block") == 0) v = kVariantBlock;
    else if (std::strcmp(kv, "pipe") == 0) v = kVariantPipe;
    else if (std::strcmp(kv, "blockocc") == 0) v = kVariantBlockOcc;
    else if (std::strcmp(kv, "split") == 0) v = kVariantSplit;
    if (v < 0) return;
    for (auto& kvp : groups) {
      Group* g = kvp.second.get();
      const std::vector<int> c = candidates(g);
      if (std::find(c.begin(), c.end(), v) != c.end()) g->variant = v;
    }
  }

  int autotune(int reps) {
    for (auto& kv : groups) {
      Group* g = kv.second.get();
      if (g->members.empty()) continue;
      int rc = rebuild(g);
      if (rc) return rc;
      const std::vector<int> cands = candidates(g);
      cudaEvent_t e0, e1;
      ENS_CUDA(cudaEventCreate(&e0));
      ENS_CUDA(cudaEventCreate(&e1));
      double best = 1e30;
      int best_v = cands[0];
      for (int v : cands) {
        for (int w = 0; w < 2; ++w)
          if ((rc = stage(g, 1, g->stream, v))) return rc;
        ENS_CUDA(cudaEventRecord(e0, g->stream));
        for (int r = 0; r < reps; ++r)
          if ((rc = stage(g, 1, g->stream, v))) return rc;
        ENS_CUDA(cudaEventRecord(e1, g->stream));
        ENS_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double t = ms / reps;
        if (v >= 0 && v < 5) g->tuned_ms[v] = t;
        if (t < best) {
          best = t;
          best_v = v;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      g->variant = best_v;
    }
    return check_status();
  }

  // Runs the kernels' one-time attribute/occupancy set-up (zero-work
  // launches) so that a later stream capture contains only launches.
  int prime() {
    for (auto& kv : groups) {
      Group* g = kv.second.get();
      if (g->members.empty()) continue;
      int rc = rebuild(g);
      if (rc) return rc;
      for (int st = 0; st < 3; ++st) {
        LaunchSpec l = spec(g, st, g->stream);
        l.variant = g->variant;
        if (g->variant == kVariantPipe || g->variant == kVariantSplit) {
          l.batch_insts = g->d_insts;
          l.batch_tiles = g->d_tiles;
          l.batch_ntiles = 0;
        } else {
          l.nelem = 0;
        }
        if ((rc = launch_tend(l))) return rc;
      }
    }
    return SDG_OK;
  }

  int check_status() {
    int st = 0;
    ENS_CUDA(cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) {
      cudaMemset(status, 0, sizeof(int));
      return fail(SDG_ERR_CUDA, "a fused kernel's bounded wait timed out (status %d)", st);
    }
    return SDG_OK;
  }
};

int make_inst(int id, int nex, int ney, int nez, int p, double dt, bool mixed,
              std::unique_ptr<Inst>* out) {
  int sz[6];
  int rc = sdg_mesh_sizes(nex, ney, nez, p, sz);
  if (rc) return rc;
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(SDG_ERR_ARG, "dt must be positive");
  auto I = std::make_unique<Inst>();
  I->id = id;
  I->nex = nex;
  I->ney = ney;
  I->nez = nez;
  I->p = p;
  I->nq = p + 1;
  I->np = sz[4];
  I->ne = sz[0];
  I->dt = dt;
  I->mixed = mixed;
  *out = std::move(I);
  return SDG_OK;
}

}  // namespace
}  // namespace sdg

using namespace sdg;

// ===========================================================================
// Batched form
// ===========================================================================
struct sdg_batch {
  Ensemble ens;
  std::vector<std::unique_ptr<Inst>> insts;
  bool committed = false;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double t_run = 0;
  long long dof_steps = 0;
};

namespace {

// Captures one RK step of every group as the batch's step graph (replayed
// per step).
int capture_step(sdg_batch* b) {
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaGraph_t g;
  ENS_CUDA(cudaStreamBeginCapture(b->ens.stream, cudaStreamCaptureModeThreadLocal));
  int rc = b->ens.step(b->ens.stream, false);
  cudaError_t ee = cudaStreamEndCapture(b->ens.stream, &g);
  if (rc) return rc;
  if (ee != cudaSuccess)
    return fail(SDG_ERR_CUDA, "batch graph capture failed: %s", cudaGetErrorString(ee));
  ee = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (ee != cudaSuccess)
    return fail(SDG_ERR_CUDA, "batch graph instantiate failed: %s", cudaGetErrorString(ee));
  return SDG_OK;
}

}  // namespace

extern "C" {

int sdg_batch_create(sdg_batch** out, int flags) {
  if (!out) return fail(SDG_ERR_ARG, "null batch pointer");
  *out = nullptr;
  if (flags & ~(SDG_FLAG_EXACT | SDG_FLAG_ORDER_GENERAL | SDG_FLAG_MIXED))
    return fail(SDG_ERR_ARG, "unknown flag bits 0x%x", flags);
  if ((flags & SDG_FLAG_MIXED) && (flags & SDG_FLAG_EXACT))
    return fail(SDG_ERR_ARG, "SDG_FLAG_EXACT applies to the FP64 form only");
  auto b = std::make_unique<sdg_batch>();
  int rc = b->ens.init(flags & ~SDG_FLAG_MIXED);
  if (rc) return rc;
  b->ens.flags = flags;
  *out = b.release();
  return SDG_OK;
}

int sdg_batch_add(sdg_batch* b, int NeX, int NeY, int NeZ, int p, const double* D1D,
                  const double* Lift_mat, const double* q, const double* u, const double* v,
                  const double* w, double dt, int* id) {
  if (!b) return fail(SDG_ERR_ARG, "null batch");
  if (b->committed) return fail(SDG_ERR_STATE, "batch already committed");
  if (!D1D || !Lift_mat || !q || !u || !v || !w)
    return fail(SDG_ERR_ARG, "sdg_batch_add: null array");
  const bool mixed = (b->ens.flags & SDG_FLAG_MIXED) != 0;
  std::unique_ptr<Inst> I;
  int rc = make_inst(static_cast<int>(b->insts.size()), NeX, NeY, NeZ, p, dt, mixed, &I);
  if (rc) return rc;
  Ops* o;
  Group* g;
  cudaSetDevice(b->ens.dev);
  if ((rc = b->ens.ops_for(p, D1D, Lift_mat, &o))) return rc;
  if ((rc = b->ens.group_for(p + 1, mixed, o, &g))) return rc;
  if ((rc = b->ens.upload(I.get(), q, u, v, w, b->ens.stream))) return rc;
  b->ens.join(I.get(), g);
  if (id) *id = I->id;
  b->insts.push_back(std::move(I));
  return SDG_OK;
}

int sdg_batch_commit(sdg_batch* b, int autotune) {
  if (!b) return fail(SDG_ERR_ARG, "null batch");
  if (b->committed) return SDG_OK;
  if (b->insts.empty()) return fail(SDG_ERR_STATE, "empty batch");
  cudaSetDevice(b->ens.dev);
  int rc;
  if (autotune && (rc = b->ens.autotune(5))) return rc;
  b->ens.force_variant();
  if ((rc = b->ens.prime())) return rc;
  if ((rc = capture_step(b))) return rc;
  ENS_CUDA(cudaEventCreate(&b->ev0));
  ENS_CUDA(cudaEventCreate(&b->ev1));
  b->committed = true;
  return SDG_OK;
}

int sdg_batch_run(sdg_batch* b, int nsteps) {
  if (!b) return fail(SDG_ERR_ARG, "null batch");
  if (!b->committed) return fail(SDG_ERR_STATE, "commit the batch first");
  if (nsteps < 0) return fail(SDG_ERR_ARG, "nsteps must be >= 0");
  cudaSetDevice(b->ens.dev);
  ENS_CUDA(cudaEventRecord(b->ev0, b->ens.stream));
  for (int i = 0; i < nsteps; ++i) ENS_CUDA(cudaGraphLaunch(b->graph, b->ens.stream));
  ENS_CUDA(cudaEventRecord(b->ev1, b->ens.stream));
  ENS_CUDA(cudaEventSynchronize(b->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  b->t_run += 1e-3 * ms;
  long long dof = 0;
  for (auto& I : b->insts) dof += static_cast<long long>(I->np) * I->ne;
  b->dof_steps += dof * nsteps;
  return b->ens.check_status();
}

int sdg_batch_get(sdg_batch* b, int id, double* q) {
  if (!b || !q) return fail(SDG_ERR_ARG, "null argument");
  if (id < 0 || id >= static_cast<int>(b->insts.size()))
    return fail(SDG_ERR_ARG, "no instance %d", id);
  cudaSetDevice(b->ens.dev);
  Inst* I = b->insts[id].get();
  ENS_CUDA(cudaStreamSynchronize(b->ens.stream));
  ENS_CUDA(cudaMemcpy(q, I->q0, static_cast<size_t>(I->np) * I->ne * sizeof(double),
                      cudaMemcpyDeviceToHost));
  return SDG_OK;
}

int sdg_batch_info(sdg_batch* b, double* out, int n) {
  // out: [instances, total DOF, run seconds, DOF-steps run, groups,
  //       then per group (p, mixed, tiles, variant, t_pipe, t_block, t_block8,
  //       t_split)]
  if (!b || !out) return fail(SDG_ERR_ARG, "null argument");
  std::vector<double> v;
  long long dof = 0;
  for (auto& I : b->insts) dof += static_cast<long long>(I->np) * I->ne;
  v.push_back(static_cast<double>(b->insts.size()));
  v.push_back(static_cast<double>(dof));
  v.push_back(b->t_run);
  v.push_back(static_cast<double>(b->dof_steps));
  v.push_back(static_cast<double>(b->ens.groups.size()));
  for (auto& kv : b->ens.groups) {
    Group* g = kv.second.get();
    v.push_back(g->nq - 1);
    v.push_back(g->mixed ? 1 : 0);
    v.push_back(g->ntiles);
    v.push_back(g->variant);
    v.push_back(g->tuned_ms[kVariantPipe]);
    v.push_back(g->tuned_ms[kVariantBlock]);
    v.push_back(g->tuned_ms[kVariantBlockOcc]);
    v.push_back(g->tuned_ms[kVariantSplit]);
  }
  for (int i = 0; i < n && i < static_cast<int>(v.size()); ++i) out[i] = v[i];
  return static_cast<int>(v.size());
}

int sdg_batch_debug_inject_wait_timeout(sdg_batch* b, int tile, int spins) {
  if (!b) return fail(SDG_ERR_ARG, "null batch");
  if (spins < 0) return fail(SDG_ERR_ARG, "spins must be >= 0");
  cudaSetDevice(b->ens.dev);
  ENS_CUDA(cudaStreamSynchronize(b->ens.stream));
  b->ens.inject_skip = tile >= 0 ? tile + 1 : 0;
  b->ens.wait_spins = static_cast<unsigned>(spins);
  return b->committed ? capture_step(b) : SDG_OK;
}

int sdg_batch_destroy(sdg_batch* b) {
  if (!b) return fail(SDG_ERR_ARG, "null batch");
  cudaSetDevice(b->ens.dev);
  cudaStreamSynchronize(b->ens.stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  for (auto& I : b->insts) b->ens.release(I.get(), b->ens.stream);
  cudaStreamSynchronize(b->ens.stream);
  delete b;
  return SDG_OK;
}

}  // extern "C"

// ===========================================================================
// Serving loop
// ===========================================================================
// Three threads own the GPU side.  The uploader admits queued requests in
// arrival order while their device memory fits under the byte cap and
// uploads each on a stream of its own, so neither the GPU nor the worker
// waits for host-to-device copies.  The worker advances the admitted requests
// in chunks of RK steps: one chunk enqueues n RK steps of the current
// membership (every order and precision in one fork/join of batched launches
// per step), n = min(steps that fit in about kChunkMs of device time, the
// fewest steps any member has left), so no member overruns.  Up to two
// chunks are in flight: the worker enqueues the next chunk before it waits
// for the oldest, so the GPU does not idle while the host turns around.  A
// member whose steps end with a chunk leaves the membership when that chunk
// is enqueued; once the chunk completes (its status word checked), the
// retirer copies the results out on a stream of its own and returns the
// memory.  Requests uploaded meanwhile join the next chunk.  Membership
// changes rewrite a group's tile tables into the table buffer that no chunk
// in flight reads (Group keeps two).
constexpr int kChunkSteps = 16;
constexpr double kChunkMs = 8.0;

// Operators submitted with a request, kept until its admission (ops_for
// needs the arrays).
struct PendingOps {
  std::vector<double> D, L;
};

struct sdg_server {
  Ensemble ens;
  size_t cap = 0;
  size_t used = 0;
  std::mutex mu;
  std::condition_variable cv;      // worker: uploaded requests, stop
  std::condition_variable up_cv;   // uploader: a request queued, memory freed, stop
  std::condition_variable done_cv; // a request finished
  std::condition_variable ret_cv;  // retirer: finished requests to copy out
  std::deque<Inst*> queue;
  std::vector<Inst*> to_retire;    // finished, waiting for the retirer
  std::vector<Inst*> active;       // members of the next chunk
  std::vector<Inst*> joining;      // uploaded, joining at the next chunk
  int uploading = 0;               // admitted, upload in progress
  int retiring = 0;                // finished, results being copied out
  bool chunk_running = false;
  std::map<int, std::unique_ptr<Inst>> all;
  // Operators of queued requests, by request (guarded by mu, like queue).
  std::map<const Inst*, PendingOps> pending_ops;
  int next_id = 0;
  bool stop = false;
  int error = SDG_OK;
  std::string error_msg;
  std::thread worker, uploader, retirer;
  double busy = 0;            // seconds of device time of the chunks
  long long dof_steps = 0;    // DOF x RK steps completed
  long long steps_run = 0;    // RK steps run (over all chunks)
  long long chunks = 0;
  // The ensemble's operator and group tables: ops_for and group_for (the
  // uploader) against the worker's use of the groups.
  std::mutex ens_mu;

  // Worker-only state.
  cudaStream_t up_stream = nullptr;  // uploads (uploader thread)
  cudaStream_t out_stream = nullptr; // result downloads (retirer thread)
  // A chunk in flight: its events, steps, DOF per step and the members whose
  // steps end with it.
  struct Chunk {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int steps = 0;
    long long dof = 0;
    std::vector<Inst*> finishing;
  };
  Chunk chunk[2];
  int oldest = 0;                    // ring position of the oldest chunk
  int in_flight = 0;                 // chunks enqueued, not yet completed
  double step_ms = 0;                // device time per step of the last chunk

  ~sdg_server() {
    for (auto& c : chunk) {
      if (c.e0) cudaEventDestroy(c.e0);
      if (c.e1) cudaEventDestroy(c.e1);
    }
    if (up_stream) cudaStreamDestroy(up_stream);
    if (out_stream) cudaStreamDestroy(out_stream);
  }

  int init_worker_state() {
    ENS_CUDA(cudaStreamCreateWithFlags(&up_stream, cudaStreamNonBlocking));
    ENS_CUDA(cudaStreamCreateWithFlags(&out_stream, cudaStreamNonBlocking));
    for (auto& c : chunk) {
      ENS_CUDA(cudaEventCreate(&c.e0));
      ENS_CUDA(cudaEventCreate(&c.e1));
    }
    return SDG_OK;
  }

  bool idle() const {
    return queue.empty() && uploading == 0 && joining.empty() && active.empty() &&
           !chunk_running && retiring == 0;
  }

  void upload_loop();

  void loop() {
    cudaSetDevice(ens.dev);
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] {
          return stop || !active.empty() || !joining.empty() || in_flight > 0;
        });
        if (stop) return;
      }
      // Only the worker changes the membership and launches; the uploader
      // only adds operators and groups (under ens_mu) and uploads.
      join_uploaded();
      if (!active.empty() && in_flight < 2) launch_chunk();
      // Complete the oldest chunk once the next one is queued (or nothing
      // else can be queued).
      if (in_flight == 2 || (in_flight == 1 && active.empty())) complete_oldest();
    }
  }

  // Copies finished requests' results to the host and returns their memory,
  // so that neither the worker nor the GPU waits for those copies.
  void retire_loop() {
    cudaSetDevice(ens.dev);
    for (;;) {
      std::vector<Inst*> done;
      {
        std::unique_lock<std::mutex> lk(mu);
        ret_cv.wait(lk, [&] { return stop || !to_retire.empty(); });
        if (stop) return;
        done.swap(to_retire);
      }
      retire(done);
    }
  }

  void fail_all(int rc);
  void join_uploaded();
  void launch_chunk();
  void complete_oldest();
  void retire(std::vector<Inst*>& done);
};

// Admits queued requests in arrival order while they fit under the cap and
// uploads them; uploaded requests join at the worker's next chunk boundary.
void sdg_server::upload_loop() {
  cudaSetDevice(ens.dev);
  for (;;) {
    Inst* I = nullptr;
    PendingOps po;
    {
      std::unique_lock<std::mutex> lk(mu);
      up_cv.wait(lk, [&] {
        return stop || (!queue.empty() && used + queue.front()->bytes <= cap);
      });
      if (stop) return;
      I = queue.front();
      queue.pop_front();
      used += I->bytes;
      ++uploading;
      I->t_admit = now_s();
      po = std::move(pending_ops[I]);
      pending_ops.erase(I);
    }
    int rc;
    {
      std::lock_guard<std::mutex> lk(ens_mu);
      Ops* o = nullptr;
      Group* g = nullptr;
      rc = ens.ops_for(I->p, po.D.data(), po.L.data(), &o);
      if (!rc) rc = ens.group_for(I->nq, I->mixed, o, &g);
    }
    if (!rc) rc = ens.upload(I, I->host[0].data(), I->host[1].data(), I->host[2].data(),
                             I->host[3].data(), up_stream);
    std::lock_guard<std::mutex> lk(mu);
    --uploading;
    if (rc) {
      ens.release(I, up_stream);
      I->state = kFailed;
      used -= I->bytes;
      error = rc;
      error_msg = last_error();
      done_cv.notify_all();
      continue;
    }
    for (auto& h : I->host) std::vector<double>().swap(h);
    I->state = kRunning;
    joining.push_back(I);
    cv.notify_all();
  }
}

// Fails every request on the device after an error (the worker keeps
// serving later submissions).
void sdg_server::fail_all(int rc) {
  cudaStreamSynchronize(ens.stream);
  std::lock_guard<std::mutex> el(ens_mu);
  std::lock_guard<std::mutex> lk(mu);
  error = rc;
  error_msg = last_error();
  for (auto* list : {&active, &joining})
    for (Inst* I : *list) {
      ens.leave(I);
      ens.release(I, out_stream);
      used -= I->bytes;
      I->state = kFailed;
    }
  for (auto& c : chunk) {
    for (Inst* I : c.finishing) {
      ens.release(I, out_stream);
      used -= I->bytes;
      I->state = kFailed;
    }
    retiring -= static_cast<int>(c.finishing.size());
    c.finishing.clear();
  }
  active.clear();
  joining.clear();
  in_flight = 0;
  chunk_running = false;
  up_cv.notify_all();
  done_cv.notify_all();
}

// Lets the uploaded requests join the membership of the next chunk.
void sdg_server::join_uploaded() {
  std::vector<Inst*> join;
  {
    std::lock_guard<std::mutex> lk(mu);
    join.swap(joining);
  }
  if (join.empty()) return;
  std::lock_guard<std::mutex> el(ens_mu);
  for (Inst* I : join) ens.join(I, ens.groups.at(std::make_pair(I->nq, I->mixed)).get());
  std::lock_guard<std::mutex> lk(mu);
  active.insert(active.end(), join.begin(), join.end());
}

// Waits for the oldest chunk in flight, accounts it, checks the status word
// and hands the members it finished to the retirer.
void sdg_server::complete_oldest() {
  Chunk& c = chunk[oldest];
  cudaError_t ce = cudaEventSynchronize(c.e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, c.e0, c.e1);
  int rc = ce == cudaSuccess ? SDG_OK
                             : fail(SDG_ERR_CUDA, "serving chunk failed: %s",
                                    cudaGetErrorString(ce));
  if (!rc) rc = ens.check_status();
  if (c.steps > 0) step_ms = ms / c.steps;
  std::vector<Inst*> done;
  done.swap(c.finishing);
  {
    std::lock_guard<std::mutex> lk(mu);
    busy += 1e-3 * ms;
    steps_run += c.steps;
    dof_steps += c.dof * c.steps;
    ++chunks;
    --in_flight;
    oldest ^= 1;
    if (!rc) {
      to_retire.insert(to_retire.end(), done.begin(), done.end());
      ret_cv.notify_all();
    }
    chunk_running = in_flight > 0;
  }
  if (rc) {
    {
      std::lock_guard<std::mutex> lk(mu);
      chunk[oldest ^ 1].finishing.swap(done);  // fail these with the rest
    }
    fail_all(rc);
  }
}

// Enqueues the next chunk: n RK steps of the current membership.  Members
// whose steps end with it leave the membership now (their results are final
// once the chunk completes).
void sdg_server::launch_chunk() {
  long long n = kChunkSteps;
  if (step_ms > 0) n = std::max(1LL, std::min(n, static_cast<long long>(kChunkMs / step_ms)));
  for (Inst* I : active) n = std::min(n, I->steps_left);
  Chunk& c = chunk[oldest ^ in_flight];
  c.steps = static_cast<int>(n);
  c.dof = 0;
  c.finishing.clear();
  int rc = SDG_OK;
  {
    std::lock_guard<std::mutex> el(ens_mu);
    // Tables of changed groups (into the buffer no chunk in flight reads)
    // and the kernels' one-time set-up.
    rc = ens.prime();
    cudaEventRecord(c.e0, ens.stream);
    for (int k = 0; k < c.steps && !rc; ++k) rc = ens.step(ens.stream, true);
    cudaEventRecord(c.e1, ens.stream);
  }
  if (rc) {
    fail_all(rc);
    return;
  }
  std::vector<Inst*> keep;
  for (Inst* I : active) {
    c.dof += static_cast<long long>(I->np) * I->ne;
    I->steps_left -= n;
    (I->steps_left > 0 ? keep : c.finishing).push_back(I);
  }
  if (!c.finishing.empty()) {
    std::lock_guard<std::mutex> el(ens_mu);
    for (Inst* I : c.finishing) ens.leave(I);
  }
  std::lock_guard<std::mutex> lk(mu);
  active.swap(keep);
  retiring += static_cast<int>(c.finishing.size());
  ++in_flight;
  chunk_running = true;
}

// Copies the finished members' results to the host on the output stream and
// returns their memory; the running chunks no longer touch them.  The pool
// free is ordered after the copy on the same stream, and Ensemble::release
// touches no shared tables.
void sdg_server::retire(std::vector<Inst*>& done) {
  if (done.empty()) return;
  for (Inst* I : done) {
    I->result.resize(static_cast<size_t>(I->np) * I->ne);
    cudaMemcpyAsync(I->result.data(), I->q0, I->result.size() * sizeof(double),
                    cudaMemcpyDeviceToHost, out_stream);
    ens.release(I, out_stream);
  }
  cudaStreamSynchronize(out_stream);
  std::lock_guard<std::mutex> lk(mu);
  for (Inst* I : done) {
    used -= I->bytes;
    I->t_done = now_s();
    I->state = kDone;
  }
  retiring -= static_cast<int>(done.size());
  up_cv.notify_all();
  done_cv.notify_all();
}

extern "C" {

int sdg_serve_create(sdg_server** out, double max_bytes) {
  if (!out) return fail(SDG_ERR_ARG, "null server pointer");
  *out = nullptr;
  auto s = std::make_unique<sdg_server>();
  int rc = s->ens.init(0);
  if (rc) return rc;
  size_t free_b = 0, total_b = 0;
  ENS_CUDA(cudaMemGetInfo(&free_b, &total_b));
  // Default cap: 85% of the device memory free now.
  s->cap = max_bytes > 0 ? static_cast<size_t>(max_bytes)
                         : static_cast<size_t>(0.85 * static_cast<double>(free_b));
  if ((rc = s->init_worker_state())) return rc;
  sdg_server* raw = s.release();
  raw->worker = std::thread([raw] { raw->loop(); });
  raw->uploader = std::thread([raw] { raw->upload_loop(); });
  raw->retirer = std::thread([raw] { raw->retire_loop(); });
  *out = raw;
  return SDG_OK;
}

int sdg_serve_submit(sdg_server* s, int NeX, int NeY, int NeZ, int p, const double* D1D,
                     const double* Lift_mat, const double* q, const double* u,
                     const double* v, const double* w, double dt, int nsteps, int flags,
                     int* id) {
  if (!s || !D1D || !Lift_mat || !q || !u || !v || !w || !id)
    return fail(SDG_ERR_ARG, "sdg_serve_submit: null argument");
  if (nsteps < 1) return fail(SDG_ERR_ARG, "nsteps must be >= 1");
  if (flags & ~SDG_FLAG_MIXED)
    return fail(SDG_ERR_ARG, "requests take SDG_FLAG_MIXED or 0 (FMA FP64)");
  std::unique_ptr<Inst> I;
  int rc = make_inst(0, NeX, NeY, NeZ, p, dt, (flags & SDG_FLAG_MIXED) != 0, &I);
  if (rc) return rc;
  I->bytes = inst_bytes(I->np, I->ne, I->mixed);
  if (I->bytes > s->cap)
    return fail(SDG_ERR_ARG, "request needs %zu bytes of device memory, above the server's "
                "cap of %zu", I->bytes, s->cap);
  const size_t n = static_cast<size_t>(I->np) * I->ne;
  const double* src[4] = {q, u, v, w};
  for (int k = 0; k < 4; ++k) I->host[k].assign(src[k], src[k] + n);
  I->steps_left = I->steps_total = nsteps;
  PendingOps po;
  const int nq = p + 1;
  po.D.assign(D1D, D1D + nq * nq);
  po.L.assign(Lift_mat, Lift_mat + 6L * nq * nq * nq);
  std::lock_guard<std::mutex> lk(s->mu);
  I->id = s->next_id++;
  I->t_submit = now_s();
  I->state = kQueued;
  s->pending_ops[I.get()] = std::move(po);
  s->queue.push_back(I.get());
  *id = I->id;
  s->all[I->id] = std::move(I);
  s->up_cv.notify_all();
  return SDG_OK;
}

int sdg_serve_poll(sdg_server* s, int id, int* state, double* times) {
  // times: [queue wait (admit - submit), time to solution (done - submit)]
  if (!s || !state) return fail(SDG_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return fail(SDG_ERR_ARG, "no request %d", id);
  Inst* I = it->second.get();
  *state = I->state;
  if (times) {
    times[0] = I->t_admit > 0 ? I->t_admit - I->t_submit : -1.0;
    times[1] = I->state == kDone ? I->t_done - I->t_submit : -1.0;
  }
  return SDG_OK;
}

int sdg_serve_result(sdg_server* s, int id, double* q) {
  if (!s || !q) return fail(SDG_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return fail(SDG_ERR_ARG, "no request %d", id);
  Inst* I = it->second.get();
  if (I->state == kFailed) return fail(SDG_ERR_CUDA, "request %d failed: %s", id,
                                       s->error_msg.c_str());
  if (I->state != kDone) return fail(SDG_ERR_STATE, "request %d is not done", id);
  std::copy(I->result.begin(), I->result.end(), q);
  s->all.erase(it);
  return SDG_OK;
}

int sdg_serve_wait(sdg_server* s, double timeout_s) {
  if (!s) return fail(SDG_ERR_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  const auto deadline = std::chrono::steady_clock::now() +
                        std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
  auto idle = [&] { return s->idle(); };
  if (!s->done_cv.wait_until(lk, deadline, idle))
    return fail(SDG_ERR_STATE, "requests still pending after %.1f s", timeout_s);
  if (s->error) return fail(s->error, "%s", s->error_msg.c_str());
  return SDG_OK;
}

int sdg_serve_stats(sdg_server* s, double* out4) {
  // out4: [device-busy seconds, DOF x RK steps done, RK iterations, bytes in use]
  if (!s || !out4) return fail(SDG_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  out4[0] = s->busy;
  out4[1] = static_cast<double>(s->dof_steps);
  out4[2] = static_cast<double>(s->steps_run);
  out4[3] = static_cast<double>(s->used);
  return SDG_OK;
}

int sdg_serve_destroy(sdg_server* s) {
  if (!s) return fail(SDG_ERR_ARG, "null server");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
    s->up_cv.notify_all();
    s->ret_cv.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  if (s->uploader.joinable()) s->uploader.join();
  if (s->retirer.joinable()) s->retirer.join();
  cudaSetDevice(s->ens.dev);
  cudaStreamSynchronize(s->ens.stream);
  cudaStreamSynchronize(s->up_stream);
  for (Inst* I : s->active) s->ens.release(I, s->ens.stream);
  for (Inst* I : s->joining) s->ens.release(I, s->ens.stream);
  for (Inst* I : s->to_retire) s->ens.release(I, s->ens.stream);
  for (auto& c : s->chunk)
    for (Inst* I : c.finishing) s->ens.release(I, s->ens.stream);
  cudaStreamSynchronize(s->ens.stream);
  delete s;
  return SDG_OK;
}

}  // extern "C"
