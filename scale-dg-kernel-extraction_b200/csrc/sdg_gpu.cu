// GPU core of the SCALE-DG advection library: the handle, validation and
// compression of the reference's mesh tables, the resident SSP-RK3 path and
// the small auxiliary kernels (halo gather, precision conversion, reductions).
// The fused tendency kernel itself lives in sdg_tend.cuh and is instantiated
// per polynomial order by sdg_tend_inst.cu.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sdg_gpu.h"
#include "sdg_internal.h"
#include "sdg_launch.h"

namespace sdg {

int pipe_info(int nq, int kind, int* epb) {
  typedef int (*Fn)(int, int*);
  static const Fn table[17] = {nullptr,       nullptr,       pipe_info_nq2,  pipe_info_nq3,
                               pipe_info_nq4, pipe_info_nq5, pipe_info_nq6,  pipe_info_nq7,
                               pipe_info_nq8, pipe_info_nq9, pipe_info_nq10, pipe_info_nq11,
                               pipe_info_nq12, pipe_info_nq13, pipe_info_nq14, pipe_info_nq15,
                               pipe_info_nq16};
  *epb = 1;
  if (nq < 2 || nq > 16) return 0;
  return table[nq](kind, epb);
}

int pipe_elems_per_tile(int nq) {
  int epb = 1;
  pipe_info(nq, kTendF64, &epb);
  return epb;
}

bool pipe_supported(int nq, int kind) {
  int epb = 1;
  return (pipe_info(nq, kind, &epb) & 1) != 0;
}

bool split_supported(int nq, int kind) {
  int epb = 1;
  return (pipe_info(nq, kind, &epb) & 2) != 0;
}

int launch_tend(const LaunchSpec& s) {
  typedef int (*Fn)(const LaunchSpec&);
  static const Fn table[17] = {nullptr,          nullptr,          launch_tend_nq2,
                               launch_tend_nq3,  launch_tend_nq4,  launch_tend_nq5,
                               launch_tend_nq6,  launch_tend_nq7,  launch_tend_nq8,
                               launch_tend_nq9,  launch_tend_nq10, launch_tend_nq11,
                               launch_tend_nq12, launch_tend_nq13, launch_tend_nq14,
                               launch_tend_nq15, launch_tend_nq16};
  if (s.nq < 2 || s.nq > 16) return fail(SDG_ERR_ARG, "Nq %d outside 2..16", s.nq);
  const int rc = table[s.nq](s);
  if (rc != 0)
    return fail(SDG_ERR_CUDA, "fused tendency launch (Nq=%d) failed: %s", s.nq,
                cudaGetErrorString(static_cast<cudaError_t>(rc)));
  return SDG_OK;
}

namespace {

#define SDG_CUDA(call)                                                     \
  do {                                                                     \
    cudaError_t err_ = (call);                                             \
    if (err_ != cudaSuccess)                                               \
      return fail(SDG_ERR_CUDA, "%s failed: %s", #call,                    \
                  cudaGetErrorString(err_));                               \
  } while (0)

// ---------------------------------------------------------------------------
// Auxiliary kernels
// ---------------------------------------------------------------------------

// f(Np*Ne + b) = f(src(b)), src 0-based (update_halo, mod_mesh.f90:216-218).
template <typename T>
__global__ void halo_kernel(T* __restrict__ f, const int* __restrict__ src,
                            long base, int n) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n;
       b += gridDim.x * blockDim.x)
    f[base + b] = f[src[b]];
}

__global__ void to_f32_kernel(float* __restrict__ out,
                              const double* __restrict__ in, long n) {
  for (long x = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<long>(gridDim.x) * blockDim.x)
    out[x] = static_cast<float>(in[x]);
}

constexpr int kRedThreads = 256;

// Block-level reduction of NV values per thread; the last block to finish
// folds the per-block partials (in block order, so the result is
// deterministic) and resets the arrival counter.
template <int NV, typename Op>
__device__ void reduce_finish(double (&v)[NV], Op op, double* partials,
                              unsigned int* counter, double* result) {
  __shared__ double sh[NV][kRedThreads / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double x = v[i];
    for (int o = 16; o > 0; o >>= 1) x = op(i, x, __shfl_down_sync(0xffffffffu, x, o));
    if (lane == 0) sh[i][wid] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double x = sh[i][0];
      for (int w = 1; w < kRedThreads / 32; ++w) x = op(i, x, sh[i][w]);
      partials[NV * blockIdx.x + i] = x;
    }
    __threadfence();
    const unsigned int done = atomicAdd(counter, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double x = partials[i];
      for (unsigned int bk = 1; bk < gridDim.x; ++bk)
        x = op(i, x, partials[NV * bk + i]);
      result[i] = x;
    }
    *counter = 0u;
  }
}

__global__ void __launch_bounds__(kRedThreads)
    minmax_kernel(const double* __restrict__ q, long n, double* partials,
                  unsigned int* counter, double* result) {
  double v[2] = {INFINITY, -INFINITY};
  for (long x = blockIdx.x * static_cast<long>(kRedThreads) + threadIdx.x; x < n;
       x += static_cast<long>(gridDim.x) * kRedThreads) {
    const double y = q[x];
    v[0] = fmin(v[0], y);
    v[1] = fmax(v[1], y);
  }
  reduce_finish<2>(v, [](int i, double a, double b) { return i == 0 ? fmin(a, b) : fmax(a, b); },
                   partials, counter, result);
}

// mass = sum W(n) jac q, sumsq = sum W(n) jac q^2 with W(n) = w_i w_j w_k.
__global__ void __launch_bounds__(kRedThreads)
    moments_kernel(const double* __restrict__ q, const double* __restrict__ wn,
                   int Np, long n, double jac, double* partials,
                   unsigned int* counter, double* result) {
  double v[2] = {0.0, 0.0};
  for (long x = blockIdx.x * static_cast<long>(kRedThreads) + threadIdx.x; x < n;
       x += static_cast<long>(gridDim.x) * kRedThreads) {
    const double y = q[x];
    const double wj = wn[x % Np] * jac;
    v[0] += wj * y;
    v[1] += wj * y * y;
  }
  reduce_finish<2>(v, [](int, double a, double b) { return a + b; }, partials,
                   counter, result);
}

template <typename T>
T* dev_alloc(size_t n, int* rc) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T) + 16);
  if (e != cudaSuccess) {
    *rc = fail(SDG_ERR_CUDA, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T),
               cudaGetErrorString(e));
    return nullptr;
  }
  return static_cast<T*>(p);
}

}  // namespace
}  // namespace sdg

using namespace sdg;

struct sdg_handle {
  int dev = 0;
  int Nq = 0, Np = 0, NfpTot = 0, Ne = 0, NeA = 0, NhaloNode = 0;
  int flags = 0;
  bool direct_ok = false;
  int variant = kVariantAuto;  // KernelVariant of the fused kernel
  int num_sms = 148;
  int* status = nullptr;       // device status word of bounded waits
  unsigned wait_spins = 0;     // bounded-wait spin limit (0: default)
  int inject_skip = 0;         // test hook: tile + 1 left without copies
  bool primed = false;
  cudaStream_t stream = nullptr;
  std::vector<double> D;  // row-major D(i,l)
  // z-face factors of the factored lift (2, Nq); empty when Lift_mat has no
  // tensor-product factorisation (the fast kernels then read it verbatim).
  std::vector<double> lift_z;

  // Compressed tables (device).
  double* lift64 = nullptr;
  float* lift32 = nullptr;
  int* pb_halo = nullptr;
  int* pb_direct = nullptr;
  double* esc64 = nullptr;
  float* esc32 = nullptr;
  double* fsc64 = nullptr;
  float* fsc32 = nullptr;
  int* hsrc = nullptr;  // halo_src_map, 0-based

  // sdg_cal_tend staging (lazy).
  double* io[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};

  // Resident state (lazy): FP64 Q0 always; stage buffers FP64 or FP32.
  double* q0 = nullptr;
  void* qa = nullptr;
  void* qb = nullptr;
  void* vel[3] = {nullptr, nullptr, nullptr};
  double* vel64[3] = {nullptr, nullptr, nullptr};  // FP64 upload staging
  bool have_vel[3] = {false, false, false};
  bool have_q = false;

  // Reductions.
  double* red_partials = nullptr;
  unsigned int* red_counter = nullptr;
  double* red_result = nullptr;
  double* lgl_wn = nullptr;
  int red_blocks = 0;

  // Step graph.
  cudaGraphExec_t graph = nullptr;
  double graph_dt = 0.0;
  // Graph of an sdg_rk3_steps_host call of host_graph_steps steps (uploads,
  // chunked stages and downloads) for the pinned host array host_graph_q
  // and host_graph_dt, and the number of kernels it launches.
  cudaGraphExec_t host_graph = nullptr;
  const double* host_graph_q = nullptr;
  double host_graph_dt = 0.0;
  int host_graph_steps = 0;
  long long host_graph_launches = 0;

  // sdg_rk3_steps_host and sdg_cal_tend (lazy): element chunks (boundaries,
  // S + 1 of them; empty when the mesh is too small to pipeline), each
  // chunk's face-neighbour chunks (itself included) through the direct
  // table (empty when a face reads the halo) and through the halo table
  // (with chunk_halo[j]: a face of chunk j reads the halo buffer), the copy
  // streams and per-chunk events.
  bool chunks_built = false;
  std::vector<int> chunk_e0;
  std::vector<std::vector<int>> chunk_nbr;
  std::vector<std::vector<int>> chunk_nbr_h;
  std::vector<char> chunk_halo;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  std::vector<cudaEvent_t> ev_up, ev_fin;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool rk_pending = false;   // ev0/ev1 bracket an unaccounted rk3 batch
  double t_tend = 0, t_rk = 0, t_halo = 0, t_copy = 0;
  long long launches = 0;
};

namespace {

void free_handle(sdg_handle* h) {
  if (!h) return;
  cudaSetDevice(h->dev);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->host_graph) cudaGraphExecDestroy(h->host_graph);
  void* ptrs[] = {h->lift64, h->lift32, h->pb_halo, h->pb_direct, h->esc64,
                  h->esc32,  h->fsc64,  h->fsc32,   h->hsrc,      h->io[0],
                  h->io[1],  h->io[2],  h->io[3],   h->io[4],     h->q0,
                  h->qa,     h->qb,     h->vel[0],  h->vel[1],    h->vel[2],
                  h->vel64[0], h->vel64[1], h->vel64[2], h->red_partials,
                  h->red_counter, h->red_result, h->lgl_wn, h->status};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (cudaEvent_t e : h->ev_up) cudaEventDestroy(e);
  for (cudaEvent_t e : h->ev_fin) cudaEventDestroy(e);
  if (h->ev_in) cudaEventDestroy(h->ev_in);
  if (h->ev_out) cudaEventDestroy(h->ev_out);
  if (h->copy_in) cudaStreamDestroy(h->copy_in);
  if (h->copy_out) cudaStreamDestroy(h->copy_out);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

bool mixed(const sdg_handle* h) { return (h->flags & SDG_FLAG_MIXED) != 0; }

LaunchSpec base_spec(const sdg_handle* h, bool f32) {
  LaunchSpec s;
  std::memset(&s, 0, sizeof(s));
  s.nq = h->Nq;
  s.exact = (h->flags & SDG_FLAG_EXACT) != 0;
  s.order = (h->flags & SDG_FLAG_ORDER_GENERAL) ? kOrderGeneral : kOrderOpt1;
  s.lift = f32 ? static_cast<const void*>(h->lift32) : h->lift64;
  s.escale = f32 ? static_cast<const void*>(h->esc32) : h->esc64;
  s.fscale = f32 ? static_cast<const void*>(h->fsc32) : h->fsc64;
  s.Ne = h->Ne;
  s.elem0 = 0;
  s.nelem = h->Ne;
  s.D = h->D.data();
  s.lift_z = h->lift_z.empty() ? nullptr : h->lift_z.data();
  s.stream = h->stream;
  s.variant = h->variant;
  s.status = h->status;
  s.wait_spins = h->wait_spins;
  s.inject_skip = h->inject_skip;
  s.num_sms = h->num_sms;
  return s;
}

// Reads and clears the device status word after the stream has drained.
int check_status(sdg_handle* h) {
  int st = 0;
  cudaError_t e = cudaMemcpy(&st, h->status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess)
    return fail(SDG_ERR_CUDA, "status read failed: %s", cudaGetErrorString(e));
  if (st != 0) {
    cudaMemset(h->status, 0, sizeof(int));
    return fail(SDG_ERR_CUDA, "a fused kernel's bounded wait on its bulk copies timed out "
                "(status %d); results of that launch are invalid", st);
  }
  return SDG_OK;
}

int launch_halo(sdg_handle* h, void* f, bool f32, cudaStream_t st) {
  if (h->NhaloNode == 0) return SDG_OK;
  const int threads = 256;
  const int blocks = std::min((h->NhaloNode + threads - 1) / threads, 148 * 8);
  const long base = static_cast<long>(h->Np) * h->Ne;
  if (f32)
    halo_kernel<float><<<blocks, threads, 0, st>>>(static_cast<float*>(f), h->hsrc,
                                                   base, h->NhaloNode);
  else
    halo_kernel<double><<<blocks, threads, 0, st>>>(static_cast<double*>(f), h->hsrc,
                                                    base, h->NhaloNode);
  SDG_CUDA(cudaGetLastError());
  return SDG_OK;
}

// Validates the verbatim tables of advect3d_eq_cal_tend against the
// structured form the fused kernel uses, and builds the compressed tables.
int compress_tables(sdg_handle* h, const int* VMapM, const int* VMapP,
                    const int* hmap, const double* nfn, const double* Esc,
                    const double* Fsc, std::vector<int>* pbh,
                    std::vector<int>* pbd, std::vector<double>* esc,
                    std::vector<double>* fsc) {
  const int Nq = h->Nq, Nfp = Nq * Nq, Np = h->Np, NfpTot = h->NfpTot, Ne = h->Ne;
  const long NEf = static_cast<long>(NfpTot) * Ne, NEp = static_cast<long>(Np) * Ne;
  const long halo0 = static_cast<long>(Np) * Ne;   // first halo DOF, 0-based
  pbh->assign(6L * Ne, 0);
  pbd->assign(6L * Ne, 0);
  esc->assign(3L * Ne, 0.0);
  fsc->assign(6L * Ne, 0.0);
  bool direct = true;
  for (long e = 0; e < Ne; ++e) {
    for (int d = 0; d < 3; ++d) {
      const double* col = Esc + e * Np + d * NEp;
      for (int n = 1; n < Np; ++n)
        if (col[n] != col[0])
          return fail(SDG_ERR_MESH, "Escale(:,%ld,%d) is not constant over the "
                      "element", e + 1, d + 1);
      (*esc)[3 * e + d] = col[0];
    }
    for (int f = 0; f < 6; ++f) {
      const long s0 = f * Nfp + NfpTot * e;
      for (int fp = 0; fp < Nfp; ++fp) {
        const long s = s0 + fp;
        if (VMapM[s] != face_node(Nq, f, fp) + 1 + e * Np)
          return fail(SDG_ERR_MESH, "VMapM(%ld,%ld) is not the element's own face "
                      "node", s0 - NfpTot * e + fp + 1, e + 1);
        for (int d = 0; d < 3; ++d) {
          const double want = (d == kFaceAxis[f]) ? kFaceSign[f] : 0.0;
          if (nfn[s + d * NEf] != want)
            return fail(SDG_ERR_MESH, "normal_fn of face %d of element %ld is not "
                        "the axis-aligned normal", f + 1, e + 1);
        }
        if (Fsc[s] != Fsc[s0])
          return fail(SDG_ERR_MESH, "Fscale is not constant over face %d of "
                      "element %ld", f + 1, e + 1);
      }
      (*fsc)[6 * e + f] = Fsc[s0];
      const int opp = kOppFace[f];
      const long p1 = static_cast<long>(VMapP[s0]) - 1;  // 0-based
      if (p1 < 0 || p1 >= static_cast<long>(Np) * h->NeA)
        return fail(SDG_ERR_MESH, "VMapP(%d,%ld) = %ld out of range", f * Nfp + 1,
                    e + 1, p1 + 1);
      if (p1 < halo0) {
        const long pb = p1 - face_node(Nq, opp, 0);
        if (pb < 0 || pb % Np != 0)
          return fail(SDG_ERR_MESH, "VMapP of face %d of element %ld does not "
                      "point at the opposite face of one element", f + 1, e + 1);
        for (int fp = 0; fp < Nfp; ++fp)
          if (static_cast<long>(VMapP[s0 + fp]) - 1 != pb + face_node(Nq, opp, fp))
            return fail(SDG_ERR_MESH, "VMapP of face %d of element %ld is not "
                        "node-for-node the opposite face", f + 1, e + 1);
        (*pbh)[6 * e + f] = static_cast<int>(pb);
        (*pbd)[6 * e + f] = static_cast<int>(pb);
      } else {
        for (int fp = 0; fp < Nfp; ++fp)
          if (static_cast<long>(VMapP[s0 + fp]) - 1 != p1 + fp)
            return fail(SDG_ERR_MESH, "halo slots of face %d of element %ld are "
                        "not contiguous", f + 1, e + 1);
        if (p1 + Nfp > halo0 + h->NhaloNode)
          return fail(SDG_ERR_MESH, "halo slots of face %d of element %ld exceed "
                      "NhaloNode", f + 1, e + 1);
        (*pbh)[6 * e + f] = static_cast<int>(-1 - p1);
        // Direct mode: read the halo's source (the periodic neighbour) itself.
        if (direct && hmap) {
          const long h0 = p1 - halo0;
          const long src0 = static_cast<long>(hmap[h0]) - 1;
          const long pb = src0 - face_node(Nq, opp, 0);
          bool ok = pb >= 0 && pb % Np == 0 && pb < static_cast<long>(Np) * Ne;
          for (int fp = 0; ok && fp < Nfp; ++fp)
            ok = static_cast<long>(hmap[h0 + fp]) - 1 == pb + face_node(Nq, opp, fp);
          if (ok) (*pbd)[6 * e + f] = static_cast<int>(pb);
          else direct = false;
        } else {
          direct = false;
        }
      }
    }
  }
  // A subdomain whose halo the caller fills reads every boundary face
  // through the halo.
  h->direct_ok = direct && !(h->flags & SDG_FLAG_EXTERNAL_HALO);
  return SDG_OK;
}

template <typename T>
int upload(T** dst, const T* src, size_t n) {
  int rc = SDG_OK;
  *dst = dev_alloc<T>(n, &rc);
  if (!*dst) return rc;
  SDG_CUDA(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return SDG_OK;
}

int ensure_state(sdg_handle* h) {
  if (h->q0) return SDG_OK;
  int rc = SDG_OK;
  const size_t NA = static_cast<size_t>(h->Np) * h->NeA;
  const size_t es = mixed(h) ? sizeof(float) : sizeof(double);
  if (!(h->q0 = dev_alloc<double>(NA, &rc))) return rc;
  if (!(h->qa = dev_alloc<char>(NA * es, &rc))) return rc;
  if (!(h->qb = dev_alloc<char>(NA * es, &rc))) return rc;
  for (int d = 0; d < 3; ++d)
    if (!(h->vel[d] = dev_alloc<char>(NA * es, &rc))) return rc;
  if (mixed(h))
    for (int d = 0; d < 3; ++d)
      if (!(h->vel64[d] = dev_alloc<double>(NA, &rc))) return rc;
  SDG_CUDA(cudaMemsetAsync(h->q0, 0, NA * sizeof(double), h->stream));
  return SDG_OK;
}

// Enqueues stage st (0..2) of one SSP-RK3 step on the handle's stream.
// Stage 1: q1 = q0 + dt*L(q0); stage 2: q2 = 3/4 q0 + 1/4 (q1 + dt*L(q1));
// stage 3: q0 <- 1/3 q0 + 2/3 (q2 + dt*L(q2))  (main.f90:58-74 with the
// coefficients of mod_common.f90:29-30).  The step-start copy q0 = q of
// main.f90:53-56 disappears: q0 is the step's input buffer.
int enqueue_stage_range(sdg_handle* h, int st, double dt, int e0, int n) {
  const bool f32 = mixed(h);
  const int* pb = h->direct_ok ? h->pb_direct : h->pb_halo;
  const double ra[3] = {0.0, 0.75, 1.0 / 3.0};
  const double rb[3] = {1.0, 0.25, 2.0 / 3.0};
  const void* in[3] = {h->q0, h->qa, h->qb};
  void* out[3] = {h->qa, h->qb, h->q0};
  if (!h->direct_ok && !(h->flags & SDG_FLAG_EXTERNAL_HALO)) {
    const bool in32 = f32 && st > 0;
    int rc = launch_halo(h, const_cast<void*>(in[st]), in32, h->stream);
    if (rc) return rc;
  }
  LaunchSpec s = base_spec(h, f32);
  s.kind = f32 ? (kStageMixed1 + st) : kStageF64;
  s.q = in[st];
  s.u = h->vel[0];
  s.v = h->vel[1];
  s.w = h->vel[2];
  s.q0 = h->q0;
  s.out = out[st];
  s.pbase = pb;
  s.rk_a = ra[st];
  s.rk_b = rb[st];
  s.dt = dt;
  s.elem0 = e0;
  s.nelem = n;
  return launch_tend(s);
}

int enqueue_stage(sdg_handle* h, int st, double dt) {
  return enqueue_stage_range(h, st, dt, 0, h->Ne);
}

// Runs the one-time attribute/occupancy set-up of the three stage kernels
// outside any stream capture.
int prime_stages(sdg_handle* h) {
  if (h->primed) return SDG_OK;
  for (int st = 0; st < 3; ++st) {
    LaunchSpec s = base_spec(h, mixed(h));
    s.kind = mixed(h) ? (kStageMixed1 + st) : kStageF64;
    s.q = st == 0 ? static_cast<const void*>(h->q0) : (st == 1 ? h->qa : h->qb);
    s.u = h->vel[0];
    s.v = h->vel[1];
    s.w = h->vel[2];
    s.q0 = h->q0;
    s.out = h->qa;
    s.pbase = h->direct_ok ? h->pb_direct : h->pb_halo;
    s.rk_a = st == 0 ? 0.0 : 0.5;
    s.nelem = 0;
    int rc = launch_tend(s);
    if (rc) return rc;
  }
  h->primed = true;
  return SDG_OK;
}

// Enqueues one SSP-RK3 step (main.f90:51-74) on the handle's stream.
int enqueue_step(sdg_handle* h, double dt) {
  for (int st = 0; st < 3; ++st) {
    int rc = enqueue_stage(h, st, dt);
    if (rc) return rc;
  }
  return SDG_OK;
}

int check_handle(sdg_handle* h) {
  if (!h) return fail(SDG_ERR_ARG, "null handle");
  SDG_CUDA(cudaSetDevice(h->dev));
  return SDG_OK;
}

// Adds the device time of the last rk3 batch to its timer once the stream
// has passed it.
void account_rk(sdg_handle* h) {
  if (!h->rk_pending) return;
  float ms = 0;
  if (cudaEventSynchronize(h->ev1) == cudaSuccess &&
      cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess)
    h->t_rk += 1e-3 * ms;
  h->rk_pending = false;
}

// The CUDA graph of one RK3 step of size dt (captured on first use).
int ensure_graph(sdg_handle* h, double dt) {
  if (h->graph && h->graph_dt == dt) return SDG_OK;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  cudaGraph_t g;
  SDG_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(h, dt);
  cudaError_t ee = cudaStreamEndCapture(h->stream, &g);
  if (ee == cudaSuccess && rc) cudaGraphDestroy(g);
  if (rc) return rc;
  if (ee != cudaSuccess)
    return fail(SDG_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ee));
  ee = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (ee != cudaSuccess)
    return fail(SDG_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ee));
  h->graph_dt = dt;
  return SDG_OK;
}

// Releases the graphs (they hold kernel arguments: variant, test hooks).
void drop_graphs(sdg_handle* h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->host_graph) cudaGraphExecDestroy(h->host_graph);
  h->graph = nullptr;
  h->host_graph = nullptr;
  h->host_graph_q = nullptr;
}

// Chunk boundaries e0[0..S] of Ne elements of Np nodes whose face
// neighbours lie within cyclic index distance `reach` (empty: fewer than 4
// chunks, no pipelining).  Smallest chunk: 512 elements, or 2^18 nodes
// (2 MB of FP64 state) where that is fewer.  The chunk the last upload
// lands in and its neighbours to a depth of three (one per stage) finish
// after it, so the three first and four last chunks are thin, one reach
// each, and the ones between them about Ne/16.
std::vector<int> chunk_bounds(int Ne, int Np, int reach) {
  const int min_chunk = std::max(1, std::min(512, (1 << 18) / Np));
  const int thin = std::max(min_chunk, reach);
  std::vector<int> e0;
  if (Ne < 9 * thin) {
    const int S = std::min(16, Ne / min_chunk);
    if (S < 4) return e0;
    for (int j = 0; j <= S; ++j) e0.push_back(static_cast<int>(static_cast<long>(Ne) * j / S));
  } else {
    const int mid = Ne - 7 * thin;
    const int target = std::max(min_chunk, Ne / 16);
    const int M = std::max(1, (mid + target / 2) / target);
    for (int j = 0; j <= 3; ++j) e0.push_back(j * thin);
    for (int j = 1; j <= M; ++j)
      e0.push_back(3 * thin + static_cast<int>(static_cast<long>(mid) * j / M));
    for (int j = 1; j <= 4; ++j) e0.push_back(3 * thin + mid + j * thin);
  }
  return e0;
}

// One launch of chunked RK steps: stage g (0 .. 3 * steps - 1; RK stage
// g % 3 of step g / 3) over chunks j0..j1, after the upload of chunk `need`
// (stage 0 with uploads; -1: no upload to wait for).
struct StepOp {
  int g, j0, j1, need;
};

// The launches of `steps` chunked RK steps, in enqueue order.  Stage g of
// chunk j needs stage g-1 of every chunk in nbr[j] (which holds j and is
// symmetric); stage 0 needs those chunks uploaded, in chunk order, when
// `uploads` is set.  Stage g + 3 overwrites stage g's output buffer (and
// the last stage of a step q0, which stage 0 of that step reads from the
// neighbour chunks); it follows stage g + 2 of the neighbour chunks and so,
// through them, every stage g + 1 that reads it.  Ready work goes first,
// the latest stage first, so that chunks finish (and go back) early.  With
// uploads, the chunks after the first ready one that are ready for the
// same stage join its launch: the last chunks, whose stages all wait for
// the last upload.  Empty when the lists admit no schedule (a neighbour
// index outside 0..S-1).
std::vector<StepOp> plan_steps(int S, const std::vector<std::vector<int>>& nbr, int steps,
                               bool uploads);

// sdg_rk3_steps_host plans up to this many steps as one: the final state of
// a chunk then depends on the chunks within 3 * steps of it, so with more
// steps nearly every chunk waits for the last upload and the plan buys no
// overlap of the two copy directions.
constexpr int kPlanSteps = 3;

std::vector<StepOp> plan_steps(int S, const std::vector<std::vector<int>>& nbr, int steps,
                               bool uploads) {
  std::vector<StepOp> ops;
  const int G = 3 * steps;
  std::vector<char> done(G * static_cast<size_t>(S), 0);
  for (const auto& l : nbr)
    for (int c : l)
      if (c < 0 || c >= S) return ops;
  auto ready = [&](int g, int j, int avail, int* need) {
    for (int c : nbr[j]) {
      if (g == 0) {
        *need = std::max(*need, c);
        if (c > avail) return false;
      } else if (!done[(g - 1) * S + c]) {
        return false;
      }
    }
    return true;
  };
  int avail = uploads ? -1 : S - 1;  // uploads the stream may rely on
  int left = G * S;
  while (left > 0) {
    int bg = -1, bj = -1, need = -1;
    for (int g = G - 1; g >= 0 && bg < 0; --g)
      for (int j = 0; j < S && bg < 0; ++j) {
        int nu = -1;
        if (!done[g * S + j] && ready(g, j, avail, &nu)) {
          bg = g;
          bj = j;
          need = nu;
        }
      }
    if (bg < 0) {  // nothing ready: rely on the next upload
      if (++avail >= S) return {};
      continue;
    }
    int bl = bj;
    while (uploads && bl + 1 < S && !done[bg * S + bl + 1]) {
      int nu = need;
      if (!ready(bg, bl + 1, avail, &nu)) break;
      need = nu;
      ++bl;
    }
    ops.push_back({bg, bj, bl, bg == 0 && uploads ? need : -1});
    for (int j = bj; j <= bl; ++j) done[bg * S + j] = 1;
    left -= bl - bj + 1;
  }
  return ops;
}

// Element chunks of sdg_rk3_steps_host and sdg_cal_tend: S contiguous
// element ranges (fewer than 4 chunks do not pipeline) and, per chunk, the
// chunks that hold a face neighbour of one of its elements, through the
// direct table (the RK path; it does not pipeline when a boundary face
// reads the halo buffer) and through the halo table (the tendency call,
// which reads the caller's halo).  Elements are numbered x fastest, so in a
// box each chunk is a run of z-layers and its neighbours are the chunks
// before and after it (cyclically).  The last upload's chunk and its
// neighbours to a depth of three finish after it and go back last, so the
// three first and four last chunks are one z-layer thin and the chunks
// between them about Ne/16.  One step from pinned memory (ms; the three
// calls 5.31 at FP64 32^3 p = 7):
//
//   chunks                       FP64 32^3 p7   mixed 32^3 p7   mixed 16^3 p15
//   16 equal                     4.17           4.10            4.71 (8 equal)
//   32 equal                     4.32           4.16            -
//   7 thin + 6 of Ne/8           4.24           4.21            -
//   7 thin + 13 of Ne/16         3.97           3.93            4.18
//
// The copies in the two directions share the bus: alone 55 / 52 GB/s, both
// at once 43 GB/s each (134 MB each way in 3.15 ms).
int build_chunks(sdg_handle* h) {
  if (h->chunks_built) return SDG_OK;
  h->chunks_built = true;
  const int Ne = h->Ne;
  const size_t Np = static_cast<size_t>(h->Np);
  std::vector<int> pbh(6 * static_cast<size_t>(Ne)), pbd;
  if (cudaMemcpy(pbh.data(), h->pb_halo, pbh.size() * sizeof(int), cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return fail(SDG_ERR_CUDA, "reading the face-neighbour table failed");
  if (h->direct_ok) {
    pbd.resize(pbh.size());
    if (cudaMemcpy(pbd.data(), h->pb_direct, pbd.size() * sizeof(int),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(SDG_ERR_CUDA, "reading the face-neighbour table failed");
  }
  // Reach: the largest cyclic index distance between an element and a face
  // neighbour (a z-layer, NeX * NeY, in a periodic box).
  int reach = 1;
  for (int e = 0; e < Ne; ++e)
    for (int f = 0; f < 6; ++f) {
      const int p = pbh[6 * static_cast<size_t>(e) + f];
      if (p < 0) continue;
      const int d = std::abs(static_cast<int>(p / Np) - e);
      reach = std::max(reach, std::min(d, Ne - d));
    }
  const std::vector<int> e0 = chunk_bounds(Ne, h->Np, reach);
  if (e0.empty()) return SDG_OK;
  const int S = static_cast<int>(e0.size()) - 1;
  auto chunk_of = [&](int e) {
    return static_cast<int>(std::upper_bound(e0.begin(), e0.end(), e) - e0.begin()) - 1;
  };
  // hit[j][c]: chunk c holds a face neighbour of an element of chunk j, or
  // the other way round (the relation is made symmetric, so that every
  // chunk that reads a chunk's stage input in stage g precedes that chunk's
  // stage g + 2, which overwrites its q0 in stage 3).
  auto neighbours = [&](const std::vector<int>& pb, bool halo_ok,
                        std::vector<std::vector<int>>* nbr, std::vector<char>* halo) -> bool {
    std::vector<std::vector<char>> hit(S, std::vector<char>(S, 0));
    halo->assign(S, 0);
    for (int j = 0; j < S; ++j) {
      hit[j][j] = 1;
      for (int e = e0[j]; e < e0[j + 1]; ++e)
        for (int f = 0; f < 6; ++f) {
          const int p = pb[6 * static_cast<size_t>(e) + f];
          if (p < 0) {
            if (!halo_ok) return false;
            (*halo)[j] = 1;
            continue;
          }
          const int c = chunk_of(static_cast<int>(p / Np));
          hit[j][c] = hit[c][j] = 1;
        }
    }
    nbr->assign(S, {});
    for (int j = 0; j < S; ++j)
      for (int c = 0; c < S; ++c)
        if (hit[j][c]) (*nbr)[j].push_back(c);
    return true;
  };
  std::vector<std::vector<int>> nbr, nbr_h;
  std::vector<char> unused, halo;
  neighbours(pbh, true, &nbr_h, &halo);
  if (!h->direct_ok || !neighbours(pbd, false, &nbr, &unused)) nbr.clear();
  if (!h->copy_in) {
    SDG_CUDA(cudaStreamCreateWithFlags(&h->copy_in, cudaStreamNonBlocking));
    SDG_CUDA(cudaStreamCreateWithFlags(&h->copy_out, cudaStreamNonBlocking));
    SDG_CUDA(cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming));
    SDG_CUDA(cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming));
  }
  h->ev_up.resize(S, nullptr);
  h->ev_fin.resize(S, nullptr);
  for (int j = 0; j < S; ++j) {
    SDG_CUDA(cudaEventCreateWithFlags(&h->ev_up[j], cudaEventDisableTiming));
    SDG_CUDA(cudaEventCreateWithFlags(&h->ev_fin[j], cudaEventDisableTiming));
  }
  h->chunk_e0 = e0;
  h->chunk_nbr = nbr;
  h->chunk_nbr_h = nbr_h;
  h->chunk_halo = halo;
  return SDG_OK;
}

// sdg_cal_tend by element chunks: the halo parts of q, u, v, w go up first,
// then the chunks in order on copy_in; each chunk's tendency starts once the
// chunks it reads are up, and its dqdt goes back on copy_out as soon as it
// is computed, so the copies overlap each other and the kernels.
int cal_tend_chunked(sdg_handle* h, double* dqdt, const double* const src[4]) {
  const int S = static_cast<int>(h->chunk_e0.size()) - 1;
  const size_t Np = static_cast<size_t>(h->Np);
  const size_t NE = Np * h->Ne, NA = Np * h->NeA;
  cudaEvent_t ek0, ek1;
  SDG_CUDA(cudaEventCreate(&ek0));
  SDG_CUDA(cudaEventCreate(&ek1));
  SDG_CUDA(cudaEventRecord(h->ev0, h->stream));
  SDG_CUDA(cudaEventRecord(h->ev_in, h->stream));
  SDG_CUDA(cudaStreamWaitEvent(h->copy_in, h->ev_in, 0));
  SDG_CUDA(cudaStreamWaitEvent(h->copy_out, h->ev_in, 0));
  if (NA > NE)
    for (int i = 0; i < 4; ++i)
      SDG_CUDA(cudaMemcpyAsync(h->io[i] + NE, src[i] + NE, (NA - NE) * sizeof(double),
                               cudaMemcpyHostToDevice, h->copy_in));
  for (int j = 0; j < S; ++j) {
    const size_t a = h->chunk_e0[j] * Np, n = (h->chunk_e0[j + 1] - h->chunk_e0[j]) * Np;
    for (int i = 0; i < 4; ++i)
      SDG_CUDA(cudaMemcpyAsync(h->io[i] + a, src[i] + a, n * sizeof(double),
                               cudaMemcpyHostToDevice, h->copy_in));
    SDG_CUDA(cudaEventRecord(h->ev_up[j], h->copy_in));
  }
  // Chunk j needs the uploads up to the last chunk it reads (the halo went
  // first); chunks go in the order their inputs arrive.
  std::vector<std::pair<int, int>> order(S);
  for (int j = 0; j < S; ++j) order[j] = {h->chunk_nbr_h[j].back(), j};
  std::stable_sort(order.begin(), order.end());
  int waited = -1, rc = SDG_OK;
  for (int k = 0; k < S && !rc; ++k) {
    const int need = order[k].first, j = order[k].second;
    if (need > waited) {
      SDG_CUDA(cudaStreamWaitEvent(h->stream, h->ev_up[need], 0));
      waited = need;
    }
    if (k == 0) SDG_CUDA(cudaEventRecord(ek0, h->stream));
    LaunchSpec s = base_spec(h, false);
    s.kind = kTendF64;
    s.q = h->io[0];
    s.u = h->io[1];
    s.v = h->io[2];
    s.w = h->io[3];
    s.out = h->io[4];
    s.pbase = h->pb_halo;
    s.elem0 = h->chunk_e0[j];
    s.nelem = h->chunk_e0[j + 1] - h->chunk_e0[j];
    rc = launch_tend(s);
    if (rc) break;
    ++h->launches;
    const size_t a = s.elem0 * Np, n = s.nelem * Np;
    SDG_CUDA(cudaEventRecord(h->ev_fin[j], h->stream));
    SDG_CUDA(cudaStreamWaitEvent(h->copy_out, h->ev_fin[j], 0));
    SDG_CUDA(cudaMemcpyAsync(dqdt + a, h->io[4] + a, n * sizeof(double),
                             cudaMemcpyDeviceToHost, h->copy_out));
  }
  cudaEventRecord(ek1, h->stream);
  cudaEventRecord(h->ev_out, h->copy_out);
  cudaStreamWaitEvent(h->stream, h->ev_out, 0);
  cudaEventRecord(h->ev1, h->stream);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (!rc && e != cudaSuccess)
    rc = fail(SDG_ERR_CUDA, "sdg_cal_tend: %s", cudaGetErrorString(e));
  if (!rc) rc = check_status(h);
  if (!rc) {
    float all = 0, kern = 0;
    cudaEventElapsedTime(&all, h->ev0, h->ev1);
    cudaEventElapsedTime(&kern, ek0, ek1);
    h->t_tend += 1e-3 * kern;
    h->t_copy += 1e-3 * (all - kern);
  }
  cudaEventDestroy(ek0);
  cudaEventDestroy(ek1);
  return rc;
}

// Enqueues `steps` RK3 steps chunk by chunk on the handle's stream, in the
// order of plan_steps; stage-1 launches wait for the uploads they need
// (ev_up events of copy_in).  With `host`, each chunk's final state is
// copied to host[] on copy_out once its last stage is done.
int enqueue_steps_chunked(sdg_handle* h, double dt, int steps, bool uploads, double* host) {
  const int S = static_cast<int>(h->chunk_e0.size()) - 1;
  const size_t Np = static_cast<size_t>(h->Np);
  const std::vector<StepOp> ops = plan_steps(S, h->chunk_nbr, steps, uploads);
  if (ops.empty()) return fail(SDG_ERR_STATE, "no schedule for the element chunks");
  int waited = -1;  // uploads the stream already waits for
  for (const StepOp& op : ops) {
    if (op.need > waited) {
      SDG_CUDA(cudaStreamWaitEvent(h->stream, h->ev_up[op.need], 0));
      waited = op.need;
    }
    const int e0 = h->chunk_e0[op.j0], n = h->chunk_e0[op.j1 + 1] - e0;
    int rc = enqueue_stage_range(h, op.g % 3, dt, e0, n);
    if (rc) return rc;
    ++h->launches;
    if (op.g == 3 * steps - 1 && host) {
      SDG_CUDA(cudaEventRecord(h->ev_fin[op.j0], h->stream));
      SDG_CUDA(cudaStreamWaitEvent(h->copy_out, h->ev_fin[op.j0], 0));
      SDG_CUDA(cudaMemcpyAsync(host + e0 * Np, h->q0 + e0 * Np, n * Np * sizeof(double),
                               cudaMemcpyDeviceToHost, h->copy_out));
    }
  }
  return SDG_OK;
}

// Enqueues nsteps >= 1 RK3 steps of sdg_rk3_steps_host: the chunk uploads
// of q on copy_in, the steps by chunks (up to kPlanSteps of them as one
// plan; beyond, the first and last steps by chunks and the ones between
// through the step graph), the chunk downloads into q on copy_out, and the
// join of both copy streams into the handle's stream, so that later work
// there (which may overwrite q0) follows the download.
int enqueue_host_steps(sdg_handle* h, double* q, double dt, int nsteps) {
  const int S = static_cast<int>(h->chunk_e0.size()) - 1;
  const size_t Np = static_cast<size_t>(h->Np);
  // The uploads overwrite q0: after everything already on the stream.
  SDG_CUDA(cudaEventRecord(h->ev_in, h->stream));
  SDG_CUDA(cudaStreamWaitEvent(h->copy_in, h->ev_in, 0));
  SDG_CUDA(cudaStreamWaitEvent(h->copy_out, h->ev_in, 0));
  for (int j = 0; j < S; ++j) {
    const int e0 = h->chunk_e0[j], n = h->chunk_e0[j + 1] - e0;
    SDG_CUDA(cudaMemcpyAsync(h->q0 + e0 * Np, q + e0 * Np, n * Np * sizeof(double),
                             cudaMemcpyHostToDevice, h->copy_in));
    SDG_CUDA(cudaEventRecord(h->ev_up[j], h->copy_in));
  }
  // Up to kPlanSteps steps as one plan, so that the last chunks' downloads
  // overlap the uploads; beyond, the first and last steps by chunks and the
  // ones between through the step graph.
  int rc;
  if (nsteps <= kPlanSteps) {
    rc = enqueue_steps_chunked(h, dt, nsteps, true, q);
  } else {
    rc = enqueue_steps_chunked(h, dt, 1, true, nullptr);
    for (int i = 0; i < nsteps - 2 && !rc; ++i)
      if (cudaGraphLaunch(h->graph, h->stream) != cudaSuccess)
        rc = fail(SDG_ERR_CUDA, "graph launch failed");
    h->launches += 3LL * (nsteps - 2);
    if (!rc) rc = enqueue_steps_chunked(h, dt, 1, false, q);
  }
  cudaEventRecord(h->ev_out, h->copy_out);
  cudaStreamWaitEvent(h->stream, h->ev_out, 0);
  cudaEventRecord(h->ev_in, h->copy_in);
  cudaStreamWaitEvent(h->stream, h->ev_in, 0);
  return rc;
}

// An sdg_rk3_steps_host call of up to kPlanSteps steps from pinned host
// array q as a CUDA graph (captured on first use for q, dt and nsteps): one
// submission instead of ~60 launches, copies and event operations per step.  While the copies run, a chunk's
// stage kernel takes about twice its time alone (FP64 32^3 p = 7: median
// 44 against 21 us, with ~26 against 3 us between launches); the graph
// takes back little of that (one step 3.95 against 3.99 ms).
int ensure_host_graph(sdg_handle* h, double* q, double dt, int nsteps) {
  if (h->host_graph && h->host_graph_q == q && h->host_graph_dt == dt &&
      h->host_graph_steps == nsteps)
    return SDG_OK;
  if (h->host_graph) cudaGraphExecDestroy(h->host_graph);
  h->host_graph = nullptr;
  h->host_graph_q = nullptr;
  const long long l0 = h->launches;
  cudaGraph_t g;
  SDG_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_host_steps(h, q, dt, nsteps);
  cudaError_t ee = cudaStreamEndCapture(h->stream, &g);
  h->host_graph_launches = h->launches - l0;
  h->launches = l0;
  if (ee == cudaSuccess && rc) cudaGraphDestroy(g);
  if (rc) return rc;
  if (ee != cudaSuccess)
    return fail(SDG_ERR_CUDA, "host-step graph capture failed: %s", cudaGetErrorString(ee));
  ee = cudaGraphInstantiate(&h->host_graph, g, 0);
  cudaGraphDestroy(g);
  if (ee != cudaSuccess) {
    h->host_graph = nullptr;
    return fail(SDG_ERR_CUDA, "host-step graph instantiate failed: %s",
                cudaGetErrorString(ee));
  }
  h->host_graph_q = q;
  h->host_graph_dt = dt;
  h->host_graph_steps = nsteps;
  return SDG_OK;
}

// Page-locked (or registered) host memory, which a captured copy needs.
bool pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace

extern "C" {

int sdg_init(sdg_handle** out, int Nq, int Np, int NfpTot, int Ne, int NeA,
             int NhaloNode, const double* D1D, const double* Lift_mat,
             const int* VMapM, const int* VMapP, const int* halo_src_map,
             const double* normal_fn, const double* Escale,
             const double* Fscale, int flags) {
  if (!out) return fail(SDG_ERR_ARG, "sdg_init: null handle pointer");
  *out = nullptr;
  if (Nq < 2 || Nq > 16)
    return fail(SDG_ERR_ARG, "Nq = %d: PolyOrder must be 1..15", Nq);
  if (Np != Nq * Nq * Nq || NfpTot != 6 * Nq * Nq)
    return fail(SDG_ERR_ARG, "Np/NfpTot inconsistent with Nq = %d", Nq);
  if (Ne < 1 || NeA < Ne || NhaloNode < 0 ||
      static_cast<long long>(Np) * NeA > 2147483647LL ||
      static_cast<long long>(Np) * Ne + NhaloNode > static_cast<long long>(Np) * NeA)
    return fail(SDG_ERR_ARG, "inconsistent sizes Ne=%d NeA=%d NhaloNode=%d", Ne,
                NeA, NhaloNode);
  if (!D1D || !Lift_mat || !VMapM || !VMapP || !normal_fn || !Escale || !Fscale ||
      (NhaloNode > 0 && !halo_src_map))
    return fail(SDG_ERR_ARG, "sdg_init: null array argument");
  if (flags & ~(SDG_FLAG_EXACT | SDG_FLAG_ORDER_GENERAL | SDG_FLAG_MIXED |
                SDG_FLAG_EXTERNAL_HALO))
    return fail(SDG_ERR_ARG, "sdg_init: unknown flag bits 0x%x", flags);
  if ((flags & SDG_FLAG_MIXED) && (flags & SDG_FLAG_EXACT))
    return fail(SDG_ERR_ARG, "SDG_FLAG_EXACT applies to the FP64 form only");
  sdg_handle* h = new sdg_handle();
  h->Nq = Nq;
  h->Np = Np;
  h->NfpTot = NfpTot;
  h->Ne = Ne;
  h->NeA = NeA;
  h->NhaloNode = NhaloNode;
  h->flags = flags;
  h->D.resize(Nq * Nq);
  for (int i = 0; i < Nq; ++i)
    for (int l = 0; l < Nq; ++l) h->D[i * Nq + l] = D1D[i + Nq * l];

  std::vector<int> pbh, pbd;
  std::vector<double> esc, fsc;
  int rc = compress_tables(h, VMapM, VMapP, halo_src_map, normal_fn, Escale, Fscale,
                           &pbh, &pbd, &esc, &fsc);
  if (rc) { delete h; return rc; }
  for (int b = 0; b < NhaloNode; ++b)
    if (halo_src_map[b] < 1 || static_cast<long>(halo_src_map[b]) > static_cast<long>(Np) * Ne) {
      delete h;
      return fail(SDG_ERR_MESH, "halo_src_map(%d) = %d out of range", b + 1,
                  halo_src_map[b]);
    }
  // The tables are valid; from here on a device is required.
  int ndev = 0;
  cudaError_t ce = cudaGetDeviceCount(&ndev);
  if (ce != cudaSuccess || ndev == 0) {
    delete h;
    return fail(SDG_ERR_CUDA, "no CUDA device available (%s); this library has no "
                "CPU path", cudaGetErrorString(ce));
  }
  cudaGetDevice(&h->dev);
  {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, h->dev) == cudaSuccess)
      h->num_sms = prop.multiProcessorCount;
    const char* kv = std::getenv("SDG_KERNEL");
    if (kv && std::strcmp(kv, "block") == 0) h->variant = kVariantBlock;
    else if (kv && std::strcmp(kv, "pipe") == 0) h->variant = kVariantPipe;
    else if (kv && std::strcmp(kv, "blockocc") == 0) h->variant = kVariantBlockOcc;
    else if (kv && std::strcmp(kv, "split") == 0) h->variant = kVariantSplit;
    else if (kv && std::strcmp(kv, "tensor") == 0) h->variant = kVariantTensor;
  }

  auto bail = [&](int code) { free_handle(h); return code; };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess)
    return bail(fail(SDG_ERR_CUDA, "stream/event creation failed"));

  std::vector<int> hs(NhaloNode);
  for (int b = 0; b < NhaloNode; ++b) hs[b] = halo_src_map[b] - 1;
  // The exact FP64 kernels read the verbatim Lift_mat; the fast ones (FP64
  // and mixed) read its tensor-product factorisation when the table has one.
  std::vector<double> lift_fact;
  if (!lift_factor(Lift_mat, Nq, &lift_fact, &h->lift_z)) lift_fact.clear();
  const double* lift_fast = lift_fact.empty() ? Lift_mat : lift_fact.data();
  const double* lift_f64 = (flags & SDG_FLAG_EXACT) ? Lift_mat : lift_fast;
  if ((rc = upload(&h->lift64, lift_f64, 6L * Np)) ||
      (rc = upload(&h->pb_halo, pbh.data(), pbh.size())) ||
      (rc = upload(&h->pb_direct, pbd.data(), pbd.size())) ||
      (rc = upload(&h->esc64, esc.data(), esc.size())) ||
      (rc = upload(&h->fsc64, fsc.data(), fsc.size())) ||
      (NhaloNode > 0 && (rc = upload(&h->hsrc, hs.data(), hs.size()))))
    return bail(rc);
  {
    std::vector<float> l32(6L * Np), e32(esc.size()), f32v(fsc.size());
    for (size_t i = 0; i < l32.size(); ++i) l32[i] = static_cast<float>(lift_fast[i]);
    for (size_t i = 0; i < e32.size(); ++i) e32[i] = static_cast<float>(esc[i]);
    for (size_t i = 0; i < f32v.size(); ++i) f32v[i] = static_cast<float>(fsc[i]);
    if ((rc = upload(&h->lift32, l32.data(), l32.size())) ||
        (rc = upload(&h->esc32, e32.data(), e32.size())) ||
        (rc = upload(&h->fsc32, f32v.data(), f32v.size())))
      return bail(rc);
  }
  h->red_blocks = 148 * 4;
  if (!(h->red_partials = dev_alloc<double>(2 * h->red_blocks, &rc)) ||
      !(h->red_counter = dev_alloc<unsigned int>(1, &rc)) ||
      !(h->red_result = dev_alloc<double>(2, &rc)) ||
      !(h->lgl_wn = dev_alloc<double>(Np, &rc)))
    return bail(rc);
  if (!(h->status = dev_alloc<int>(1, &rc))) return bail(rc);
  if (cudaMemset(h->red_counter, 0, sizeof(unsigned int)) != cudaSuccess ||
      cudaMemset(h->status, 0, sizeof(int)) != cudaSuccess)
    return bail(fail(SDG_ERR_CUDA, "cudaMemset failed"));
  *out = h;
  return SDG_OK;
}

int sdg_finalize(sdg_handle* h) {
  if (!h) return fail(SDG_ERR_ARG, "null handle");
  free_handle(h);
  return SDG_OK;
}

int sdg_cal_tend_dev(sdg_handle* h, double* dqdt, const double* q,
                     const double* u, const double* v, const double* w,
                     void* stream) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (!dqdt || !q || !u || !v || !w) return fail(SDG_ERR_ARG, "null device array");
  LaunchSpec s = base_spec(h, false);
  s.kind = kTendF64;
  s.q = q;
  s.u = u;
  s.v = v;
  s.w = w;
  s.out = dqdt;
  s.pbase = h->pb_halo;
  if (stream) s.stream = static_cast<cudaStream_t>(stream);
  rc = launch_tend(s);
  if (!rc) ++h->launches;
  return rc;
}

int sdg_cal_tend(sdg_handle* h, double* dqdt, const double* q,
                 const double* u, const double* v, const double* w) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (!dqdt || !q || !u || !v || !w) return fail(SDG_ERR_ARG, "null host array");
  const size_t NA = static_cast<size_t>(h->Np) * h->NeA;
  const size_t NE = static_cast<size_t>(h->Np) * h->Ne;
  for (int i = 0; i < 5; ++i)
    if (!h->io[i] && !(h->io[i] = dev_alloc<double>(NA, &rc))) return rc;
  const double* src[4] = {q, u, v, w};
  account_rk(h);
  if ((rc = build_chunks(h))) return rc;
  if (!h->chunk_nbr_h.empty()) return cal_tend_chunked(h, dqdt, src);
  cudaEvent_t e2, e3;
  SDG_CUDA(cudaEventCreate(&e2));
  SDG_CUDA(cudaEventCreate(&e3));
  SDG_CUDA(cudaEventRecord(h->ev0, h->stream));
  for (int i = 0; i < 4; ++i)
    SDG_CUDA(cudaMemcpyAsync(h->io[i], src[i], NA * sizeof(double),
                             cudaMemcpyHostToDevice, h->stream));
  SDG_CUDA(cudaEventRecord(e2, h->stream));
  rc = sdg_cal_tend_dev(h, h->io[4], h->io[0], h->io[1], h->io[2], h->io[3], nullptr);
  if (rc) return rc;
  SDG_CUDA(cudaEventRecord(e3, h->stream));
  SDG_CUDA(cudaMemcpyAsync(dqdt, h->io[4], NE * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream));
  SDG_CUDA(cudaEventRecord(h->ev1, h->stream));
  SDG_CUDA(cudaStreamSynchronize(h->stream));
  if ((rc = check_status(h))) return rc;
  float a = 0, b = 0, c = 0;
  cudaEventElapsedTime(&a, h->ev0, e2);
  cudaEventElapsedTime(&b, e2, e3);
  cudaEventElapsedTime(&c, e3, h->ev1);
  h->t_copy += 1e-3 * (a + c);
  h->t_tend += 1e-3 * b;
  cudaEventDestroy(e2);
  cudaEventDestroy(e3);
  return SDG_OK;
}

int sdg_update_halo_dev(sdg_handle* h, double* f, void* stream) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (!f) return fail(SDG_ERR_ARG, "null device array");
  return launch_halo(h, f, false, stream ? static_cast<cudaStream_t>(stream) : h->stream);
}

int sdg_set_field(sdg_handle* h, int which, const double* host) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (which < SDG_FIELD_Q || which > SDG_FIELD_W || !host)
    return fail(SDG_ERR_ARG, "sdg_set_field: bad field or null array");
  if ((rc = ensure_state(h))) return rc;
  const size_t NE = static_cast<size_t>(h->Np) * h->Ne;
  const size_t NA = static_cast<size_t>(h->Np) * h->NeA;
  if (which == SDG_FIELD_Q) {
    SDG_CUDA(cudaMemcpyAsync(h->q0, host, NE * sizeof(double), cudaMemcpyHostToDevice,
                             h->stream));
    if ((rc = launch_halo(h, h->q0, false, h->stream))) return rc;
    h->have_q = true;
  } else {
    const int d = which - SDG_FIELD_U;
    double* dst = mixed(h) ? h->vel64[d] : static_cast<double*>(h->vel[d]);
    SDG_CUDA(cudaMemcpyAsync(dst, host, NE * sizeof(double), cudaMemcpyHostToDevice,
                             h->stream));
    if ((rc = launch_halo(h, dst, false, h->stream))) return rc;
    if (mixed(h)) {
      to_f32_kernel<<<148 * 8, 256, 0, h->stream>>>(static_cast<float*>(h->vel[d]), dst,
                                                    static_cast<long>(NA));
      SDG_CUDA(cudaGetLastError());
    }
    h->have_vel[d] = true;
  }
  SDG_CUDA(cudaStreamSynchronize(h->stream));
  return SDG_OK;
}

int sdg_get_field(sdg_handle* h, int which, double* host) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (which < SDG_FIELD_Q || which > SDG_FIELD_W || !host)
    return fail(SDG_ERR_ARG, "sdg_get_field: bad field or null array");
  if (!h->q0) return fail(SDG_ERR_STATE, "no resident state: call sdg_set_field first");
  const size_t NE = static_cast<size_t>(h->Np) * h->Ne;
  const double* src = h->q0;
  if (which != SDG_FIELD_Q) {
    const int d = which - SDG_FIELD_U;
    src = mixed(h) ? h->vel64[d] : static_cast<const double*>(h->vel[d]);
  }
  SDG_CUDA(cudaMemcpyAsync(host, src, NE * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream));
  SDG_CUDA(cudaStreamSynchronize(h->stream));
  return check_status(h);
}

int sdg_rk3_steps(sdg_handle* h, double dt, int nsteps) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (nsteps < 0) return fail(SDG_ERR_ARG, "nsteps must be >= 0");
  if (!h->have_q || !h->have_vel[0] || !h->have_vel[1] || !h->have_vel[2])
    return fail(SDG_ERR_STATE, "upload q, u, v and w with sdg_set_field first");
  if (h->flags & SDG_FLAG_EXTERNAL_HALO)
    return fail(SDG_ERR_STATE, "SDG_FLAG_EXTERNAL_HALO: the caller fills the halo between "
                "stages; run sdg_update_halo_stage, the exchange and sdg_rk3_stage");
  if (nsteps == 0) return SDG_OK;
  if ((rc = prime_stages(h))) return rc;
  if ((rc = ensure_graph(h, dt))) return rc;
  account_rk(h);
  SDG_CUDA(cudaEventRecord(h->ev0, h->stream));
  for (int i = 0; i < nsteps; ++i) SDG_CUDA(cudaGraphLaunch(h->graph, h->stream));
  SDG_CUDA(cudaEventRecord(h->ev1, h->stream));
  h->rk_pending = true;
  h->launches += 3LL * nsteps;
  return SDG_OK;
}

int sdg_rk3_steps_host(sdg_handle* h, double* q, double dt, int nsteps) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (!q) return fail(SDG_ERR_ARG, "sdg_rk3_steps_host: null array");
  if (nsteps < 0) return fail(SDG_ERR_ARG, "nsteps must be >= 0");
  if (!h->have_vel[0] || !h->have_vel[1] || !h->have_vel[2])
    return fail(SDG_ERR_STATE, "upload u, v and w with sdg_set_field first");
  if (h->flags & SDG_FLAG_EXTERNAL_HALO)
    return fail(SDG_ERR_STATE, "SDG_FLAG_EXTERNAL_HALO: the caller fills the halo between "
                "stages; run sdg_update_halo_stage, the exchange and sdg_rk3_stage");
  if ((rc = ensure_state(h))) return rc;
  if ((rc = build_chunks(h))) return rc;
  if (h->chunk_nbr.empty() || nsteps == 0) {
    if ((rc = sdg_set_field(h, SDG_FIELD_Q, q))) return rc;
    if ((rc = sdg_rk3_steps(h, dt, nsteps))) return rc;
    return sdg_get_field(h, SDG_FIELD_Q, q);
  }
  if ((rc = prime_stages(h))) return rc;
  if (nsteps > kPlanSteps && (rc = ensure_graph(h, dt))) return rc;
  account_rk(h);
  h->have_q = true;
  const size_t NE = static_cast<size_t>(h->Np) * h->Ne;
  if (nsteps <= kPlanSteps && pinned(q) && pinned(q + NE - 1)) {
    if ((rc = ensure_host_graph(h, q, dt, nsteps))) return rc;
    SDG_CUDA(cudaGraphLaunch(h->host_graph, h->stream));
    h->launches += h->host_graph_launches;
  } else if ((rc = enqueue_host_steps(h, q, dt, nsteps))) {
    cudaStreamSynchronize(h->stream);
    return rc;
  }
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return fail(SDG_ERR_CUDA, "sdg_rk3_steps_host: %s", cudaGetErrorString(e));
  return check_status(h);
}

int sdg_rk3_stage(sdg_handle* h, int stage, double dt) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (stage < 1 || stage > 3) return fail(SDG_ERR_ARG, "stage must be 1..3");
  if (!h->have_q || !h->have_vel[0] || !h->have_vel[1] || !h->have_vel[2])
    return fail(SDG_ERR_STATE, "upload q, u, v and w with sdg_set_field first");
  rc = enqueue_stage(h, stage - 1, dt);
  if (!rc) ++h->launches;
  return rc;
}

int sdg_get_stream(sdg_handle* h, void** stream) {
  if (!h || !stream) return fail(SDG_ERR_ARG, "null argument");
  *stream = h->stream;
  return SDG_OK;
}

int sdg_synchronize(sdg_handle* h) {
  int rc = check_handle(h);
  if (rc) return rc;
  SDG_CUDA(cudaStreamSynchronize(h->stream));
  account_rk(h);
  return check_status(h);
}

int sdg_minmax(sdg_handle* h, double* qmin, double* qmax) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (!h->have_q) return fail(SDG_ERR_STATE, "no resident state");
  const long n = static_cast<long>(h->Np) * h->Ne;
  minmax_kernel<<<h->red_blocks, kRedThreads, 0, h->stream>>>(
      h->q0, n, h->red_partials, h->red_counter, h->red_result);
  SDG_CUDA(cudaGetLastError());
  double r[2];
  SDG_CUDA(cudaMemcpyAsync(r, h->red_result, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
  SDG_CUDA(cudaStreamSynchronize(h->stream));
  if ((rc = check_status(h))) return rc;
  if (qmin) *qmin = r[0];
  if (qmax) *qmax = r[1];
  return SDG_OK;
}

int sdg_diagnostics(sdg_handle* h, const double* lgl_w, double jac, double* mass,
                    double* l2) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (!h->have_q) return fail(SDG_ERR_STATE, "no resident state");
  if (!lgl_w) return fail(SDG_ERR_ARG, "null weights");
  const int Nq = h->Nq;
  std::vector<double> wn(h->Np);
  for (int k = 0; k < Nq; ++k)
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) wn[i + Nq * j + Nq * Nq * k] = lgl_w[i] * lgl_w[j] * lgl_w[k];
  SDG_CUDA(cudaMemcpyAsync(h->lgl_wn, wn.data(), h->Np * sizeof(double),
                           cudaMemcpyHostToDevice, h->stream));
  const long n = static_cast<long>(h->Np) * h->Ne;
  moments_kernel<<<h->red_blocks, kRedThreads, 0, h->stream>>>(
      h->q0, h->lgl_wn, h->Np, n, jac, h->red_partials, h->red_counter, h->red_result);
  SDG_CUDA(cudaGetLastError());
  double r[2];
  SDG_CUDA(cudaMemcpyAsync(r, h->red_result, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
  SDG_CUDA(cudaStreamSynchronize(h->stream));
  if (mass) *mass = r[0];
  if (l2) *l2 = std::sqrt(r[1]);
  return SDG_OK;
}

int sdg_field_dev_ptr(sdg_handle* h, int which, void** ptr) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (!ptr || which < SDG_FIELD_Q || which > SDG_FIELD_W)
    return fail(SDG_ERR_ARG, "sdg_field_dev_ptr: bad argument");
  if ((rc = ensure_state(h))) return rc;
  *ptr = which == SDG_FIELD_Q ? static_cast<void*>(h->q0) : h->vel[which - SDG_FIELD_U];
  return SDG_OK;
}

int sdg_resident_array(sdg_handle* h, int which, void** ptr, int* elem_bytes) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (!ptr || which < SDG_FIELD_Q || which > SDG_ARRAY_STAGE3)
    return fail(SDG_ERR_ARG, "sdg_resident_array: bad argument");
  if ((rc = ensure_state(h))) return rc;
  const int es = mixed(h) ? 4 : 8;
  void* arrays[6] = {h->q0, h->vel[0], h->vel[1], h->vel[2], h->qa, h->qb};
  *ptr = arrays[which];
  if (elem_bytes) *elem_bytes = which == SDG_FIELD_Q ? 8 : es;
  return SDG_OK;
}

int sdg_update_halo_stage(sdg_handle* h, int stage) {
  int rc = check_handle(h);
  if (rc) return rc;
  if (stage < 1 || stage > 3) return fail(SDG_ERR_ARG, "stage must be 1..3");
  if ((rc = ensure_state(h))) return rc;
  void* in[3] = {h->q0, h->qa, h->qb};
  return launch_halo(h, in[stage - 1], mixed(h) && stage > 1, h->stream);
}

int sdg_timers(sdg_handle* h, double* t4) {
  if (!h || !t4) return fail(SDG_ERR_ARG, "null argument");
  account_rk(h);
  t4[0] = h->t_tend;
  t4[1] = h->t_rk;
  t4[2] = h->t_halo;
  t4[3] = h->t_copy;
  return SDG_OK;
}

long long sdg_launch_count(sdg_handle* h) { return h ? h->launches : -1; }

int sdg_set_kernel_variant(sdg_handle* h, int variant) {
  if (!h) return fail(SDG_ERR_ARG, "null handle");
  if (variant < kVariantAuto || variant > kVariantTensor)
    return fail(SDG_ERR_ARG, "kernel variant must be 0 (auto), 1 (block), 2 (pipelined), "
                "3 (block, 8 blocks per SM), 4 (pipelined, split columns) or 5 "
                "(pipelined, tensor-core lines of the mixed form at p = 7)");
  if (variant != h->variant) drop_graphs(h);
  h->variant = variant;
  h->primed = false;
  return SDG_OK;
}

int sdg_debug_chunk_bounds(int Ne, int Np, int reach, int* e0, int cap, int* nchunks) {
  if (Ne < 1 || Np < 1 || reach < 1 || reach > Ne || !nchunks || cap < 0 || (cap > 0 && !e0))
    return fail(SDG_ERR_ARG, "sdg_debug_chunk_bounds: bad argument");
  const std::vector<int> b = chunk_bounds(Ne, Np, reach);
  *nchunks = b.empty() ? 0 : static_cast<int>(b.size()) - 1;
  if (static_cast<int>(b.size()) > cap)
    return fail(SDG_ERR_ARG, "sdg_debug_chunk_bounds: %d boundaries, room for %d",
                static_cast<int>(b.size()), cap);
  std::copy(b.begin(), b.end(), e0);
  return SDG_OK;
}

int sdg_debug_step_plan(int S, const int* nbr_ptr, const int* nbr_idx, int steps, int uploads,
                        int* ops, int cap, int* nops) {
  if (S < 1 || steps < 1 || steps > 64 || !nbr_ptr || !nbr_idx || !nops || cap < 0 ||
      (cap > 0 && !ops))
    return fail(SDG_ERR_ARG, "sdg_debug_step_plan: bad argument");
  std::vector<std::vector<int>> nbr(S);
  for (int j = 0; j < S; ++j) {
    if (nbr_ptr[j + 1] < nbr_ptr[j])
      return fail(SDG_ERR_ARG, "sdg_debug_step_plan: nbr_ptr decreases at %d", j);
    nbr[j].assign(nbr_idx + nbr_ptr[j], nbr_idx + nbr_ptr[j + 1]);
  }
  const std::vector<StepOp> p = plan_steps(S, nbr, steps, uploads != 0);
  if (p.empty()) return fail(SDG_ERR_ARG, "sdg_debug_step_plan: the lists admit no schedule");
  *nops = static_cast<int>(p.size());
  if (4 * *nops > cap)
    return fail(SDG_ERR_ARG, "sdg_debug_step_plan: %d launches, room for %d", *nops, cap / 4);
  for (size_t i = 0; i < p.size(); ++i) {
    ops[4 * i] = p[i].g;
    ops[4 * i + 1] = p[i].j0;
    ops[4 * i + 2] = p[i].j1;
    ops[4 * i + 3] = p[i].need;
  }
  return SDG_OK;
}

int sdg_debug_inject_wait_timeout(sdg_handle* h, int tile, int spins) {
  if (!h) return fail(SDG_ERR_ARG, "null handle");
  if (spins < 0) return fail(SDG_ERR_ARG, "spins must be >= 0");
  cudaSetDevice(h->dev);
  cudaStreamSynchronize(h->stream);
  drop_graphs(h);  // the graphs hold the old kernel arguments
  h->inject_skip = tile >= 0 ? tile + 1 : 0;
  h->wait_spins = static_cast<unsigned>(spins);
  return SDG_OK;
}

}  // extern "C"
