// Host-side launch description shared by the per-order instantiation units
// (sdg_tend_inst.cu, compiled once per NQ) and the library core.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

namespace sdg {

// Per-device cache of a kernel's one-time launch set-up: function
// attributes and occupancy queries act on the current device only, so a
// process that drives several devices sets each one up.  One static
// instance per kernel instantiation; a slot holds 0 until set up.
constexpr int kMaxSetupDevices = 64;
struct DeviceSetup {
  std::atomic<int> slot[kMaxSetupDevices];
};

// The current device, or -1 when it cannot be read or lies beyond the cache.
inline int setup_device() {
  int d = -1;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxSetupDevices) return -1;
  return d;
}

// Largest dynamic shared memory a block of the current device may opt in to
// (cudaDevAttrMaxSharedMemoryPerBlockOptin), read once per device; 0 when it
// cannot be read.  A kernel plan above it falls back to a smaller kernel.
inline size_t device_smem_optin() {
  static DeviceSetup cache;
  const int d = setup_device();
  if (d < 0) return 0;
  int v = cache.slot[d].load(std::memory_order_relaxed);
  if (v == 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, d) != cudaSuccess ||
        v <= 0)
      return 0;
    cache.slot[d].store(v, std::memory_order_relaxed);
  }
  return static_cast<size_t>(v);
}

// Summation order of the contractions for NQ > 8: OPT1's three partial sums
// (mod_dg_optr_kernel_opt1.F90.erb:242-274) or GENERAL's sequential loop
// (mod_dg_optr_kernel.f90:221-257).  Identical for NQ <= 8.
enum SumOrder { kOrderOpt1 = 0, kOrderGeneral = 1 };

// Which typed variant of the fused kernel to run.
enum TendKind {
  kTendF64 = 0,       // dqdt = L(q), all FP64
  kStageF64 = 1,      // q_new = a*q0 + b*(q + dt*L(q)), all FP64
  kStageMixed1 = 2,   // FP64 q in, FP32 velocity/compute, FP32 q out
  kStageMixed2 = 3,   // FP32 q in, FP64 q0, FP32 q out
  kStageMixed3 = 4,   // FP32 q in, FP64 q0, FP64 q out
};

struct LaunchSpec {
  int nq;
  int kind;          // TendKind
  bool exact;        // separate roundings, reference order (FP64 kinds)
  int order;         // SumOrder (matters for exact FP64 and NQ > 8)
  const void* q;
  const void* u;
  const void* v;
  const void* w;
  const double* q0;
  void* out;
  const void* lift;    // FP64 or FP32 by kind
  const int* pbase;
  const void* escale;
  const void* fscale;
  int Ne;
  int elem0;
  int nelem;
  double rk_a, rk_b, dt;
  const double* D;     // row-major D(i,l), NQ*NQ
  // Factored lift of the fast kernels: the z-face factors lz(k, f) for
  // f = -z, +z ((2, NQ), host memory), given when `lift` holds the
  // tensor-product factorisation of Lift_mat; null for the verbatim table.
  const double* lift_z;
  cudaStream_t stream;
  int variant;         // KernelVariant
  int* status;         // device status word (bounded-wait timeouts)
  unsigned wait_spins; // spin limit of a bounded wait; 0: the default
  int inject_skip;     // test hook: tile + 1 whose copies are skipped; 0: none
  int num_sms;         // multiprocessors of the device
  // Batched launch (pipelined kernel only): device arrays of BatchInst and
  // BatchTile (sdg_tend.cuh) and the tile count; null for one instance.
  const void* batch_insts;
  const void* batch_tiles;
  int batch_ntiles;
};

// Elements per tile of the pipelined kernel for a given order (the tile
// size a batch's tile table must use).
int pipe_elems_per_tile(int nq);

// Whether the pipelined kernel can run kind `kind` at this order (its
// shared-memory plan fits).
bool pipe_supported(int nq, int kind);

// Whether the split-column kernel exists at this order and its plan fits.
bool split_supported(int nq, int kind);

// Launches the fused kernel described by `s`; returns SDG_OK or an SDG_ERR_*
// status with the thread's last error set.
int launch_tend(const LaunchSpec& s);

// Kernel variants: the one-tile-per-block kernel (tend_kernel) and the
// persistent bulk-copy pipelined kernel (tend_pipe_kernel); identical
// arithmetic.  Auto picks the split-column kernel at the orders where it
// measured faster (kSplitAuto), else the pipelined one when its
// shared-memory plan fits one block (kPipeMaxSmem) and every array is
// 16-byte aligned, else the one-tile-per-block kernel.
// kVariantBlockOcc is the one-tile-per-block kernel built for eight resident
// blocks per SM (p = 3..7; other orders use kVariantBlock).
// kVariantSplit is the persistent ring kernel with each z-column split over
// two threads (tend_split_kernel), for the orders with one element per tile
// (Nq >= 9).  kVariantTensor is the pipelined kernel of the mixed form at
// Nq = 8 with its x/y lines on the tensor cores (TF32, three hi/lo passes);
// its rounding differs from the other variants', so it is never chosen
// automatically (other orders and forms run their automatic variant).
enum KernelVariant {
  kVariantAuto = 0,
  kVariantBlock = 1,
  kVariantPipe = 2,
  kVariantBlockOcc = 3,
  kVariantSplit = 4,
  kVariantTensor = 5
};

// Returns 0 when launched, -1 when this unit does not hold spec.nq,
// otherwise a cudaError_t value.
int launch_tend_nq2(const LaunchSpec&);
int launch_tend_nq3(const LaunchSpec&);
int launch_tend_nq4(const LaunchSpec&);
int launch_tend_nq5(const LaunchSpec&);
int launch_tend_nq6(const LaunchSpec&);
int launch_tend_nq7(const LaunchSpec&);
int launch_tend_nq8(const LaunchSpec&);
int launch_tend_nq9(const LaunchSpec&);
int launch_tend_nq10(const LaunchSpec&);
int launch_tend_nq11(const LaunchSpec&);
int launch_tend_nq12(const LaunchSpec&);
int launch_tend_nq13(const LaunchSpec&);
int launch_tend_nq14(const LaunchSpec&);
int launch_tend_nq15(const LaunchSpec&);
int launch_tend_nq16(const LaunchSpec&);

// Per order: elements per tile of the pipelined kernel (*epb) and which
// persistent kernels' shared-memory plans fit for `kind` (return value: bit 0
// the pipelined kernel, bit 1 the split-column kernel).
int pipe_info_nq2(int kind, int* epb);
int pipe_info_nq3(int kind, int* epb);
int pipe_info_nq4(int kind, int* epb);
int pipe_info_nq5(int kind, int* epb);
int pipe_info_nq6(int kind, int* epb);
int pipe_info_nq7(int kind, int* epb);
int pipe_info_nq8(int kind, int* epb);
int pipe_info_nq9(int kind, int* epb);
int pipe_info_nq10(int kind, int* epb);
int pipe_info_nq11(int kind, int* epb);
int pipe_info_nq12(int kind, int* epb);
int pipe_info_nq13(int kind, int* epb);
int pipe_info_nq14(int kind, int* epb);
int pipe_info_nq15(int kind, int* epb);
int pipe_info_nq16(int kind, int* epb);

// Shared-memory bytes and threads per block of the fused kernel.
void tend_block_shape(int nq, bool fp32, int* threads, size_t* smem,
                      int* elems_per_block);

}  // namespace sdg
