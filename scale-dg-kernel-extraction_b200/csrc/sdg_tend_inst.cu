// Instantiates the fused tendency kernel for one polynomial order.
// Compiled once per NQ = p+1 (2..16) with -DSDG_NQ=<NQ>, so the fifteen
// fully unrolled variants build in parallel.
#include <stdint.h>

#include <algorithm>

#include "sdg_launch.h"
#include "sdg_tend.cuh"
#include "sdg_tend_pipe.cuh"
#include "sdg_tend_split.cuh"

#ifndef SDG_NQ
#error "SDG_NQ must be defined"
#endif

namespace sdg {
namespace {

constexpr int NQ = SDG_NQ;

// Launches a persistent pipelined kernel: attribute and occupancy set-up on
// the first call of each instantiation (a call with no tiles only primes
// it, e.g. before a stream capture), then one block per resident slot.  The
// kernel is a template argument so that the set-up state belongs to that
// kernel: kernels of one signature (tendency and stage forms) differ in
// their shared-memory plans.
// floor_blocks: resident blocks per SM to launch at least (the occupancy
// query reports one block per SM for kernels that allocate tensor memory,
// whose shared memory, registers and 32 TMEM columns allow more).
template <auto KERN, int THREADS = PipeGeo<NQ>::THREADS, typename Args, typename Dm>
int launch_pipe(size_t smem, int ntiles, const LaunchSpec& s, const Args& a, const Dm& d,
                int floor_blocks = 0) {
  constexpr auto kern = KERN;
  static DeviceSetup setup;  // blocks per SM, per kernel and device
  const int dev = setup_device();
  if (dev < 0) return static_cast<int>(cudaErrorInvalidDevice);
  int blocks_per_sm = setup.slot[dev].load(std::memory_order_relaxed);
  if (blocks_per_sm == 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int nb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, THREADS, smem);
    if (e != cudaSuccess) return static_cast<int>(e);
    blocks_per_sm = std::max(nb > 0 ? nb : 1, floor_blocks);
    setup.slot[dev].store(blocks_per_sm, std::memory_order_relaxed);
  }
  if (ntiles <= 0) return 0;
  const int grid = std::min(ntiles, blocks_per_sm * (s.num_sms > 0 ? s.num_sms : 148));
  kern<<<grid, THREADS, smem, s.stream>>>(a, d);
  return static_cast<int>(cudaGetLastError());
}

template <typename TQ, typename TV, typename TO, typename TC, bool EXACT,
          int ORDER, bool STAGE>
int run(const LaunchSpec& s) {
  using G = Geo<NQ>;
  TendArgs<TQ, TV, TO, TC> a;
  a.q = static_cast<const TQ*>(s.q);
  a.u = static_cast<const TV*>(s.u);
  a.v = static_cast<const TV*>(s.v);
  a.w = static_cast<const TV*>(s.w);
  a.q0 = s.q0;
  a.out = static_cast<TO*>(s.out);
  a.lift = static_cast<const TC*>(s.lift);
  a.pbase = s.pbase;
  a.escale = static_cast<const TC*>(s.escale);
  a.fscale = static_cast<const TC*>(s.fscale);
  a.Ne = s.Ne;
  a.elem0 = s.elem0;
  a.nelem = s.nelem;
  a.rk_a = s.rk_a;
  a.rk_b = s.rk_b;
  a.dt = s.dt;
  a.status = s.status;
  a.wait_spins = s.wait_spins ? s.wait_spins : kWaitSpins;
  a.inject_skip = s.inject_skip;
  a.prefetch_dist = 0;
  a.insts = static_cast<const BatchInst*>(s.batch_insts);
  a.tiles = static_cast<const BatchTile*>(s.batch_tiles);
  a.ntiles = s.batch_ntiles;
  DMat<NQ, TC> d;
  for (int i = 0; i < NQ * NQ; ++i) d.d[i] = static_cast<TC>(s.D[i]);
  for (int i = 0; i < 2 * NQ; ++i)
    d.lz[i] = s.lift_z ? static_cast<TC>(s.lift_z[i]) : TC(0);
  using P = PipePlan<NQ, TQ, TV, TC, STAGE>;
  using PB = PipePlan<NQ, TQ, TV, TC, STAGE, false, true>;  // batched launches
  auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  const bool batch = s.batch_tiles != nullptr;
  // Batched arrays are allocated 256-byte aligned by the batch itself.  The
  // fast pipelined kernels need the factored lift; with a verbatim table a
  // fast launch takes the one-tile-per-block kernel.
  const size_t pipe_bytes = batch ? PB::BYTES : P::BYTES;
  const bool can_pipe = pipe_bytes <= kPipeMaxSmem && pipe_bytes <= device_smem_optin() &&
                        (EXACT || s.lift_z != nullptr) &&
                        (batch || (aligned(s.q) && aligned(s.u) && aligned(s.v) &&
                                   aligned(s.w) && aligned(s.escale) && aligned(s.fscale)));
  // The split-column kernel: orders with one element per tile.
  if constexpr (NQ >= 9) {
    constexpr int H = kSplitH<NQ>;
    using SP = SplitPlan<NQ, H, TQ, TV, TC, STAGE>;
    const bool can_split = SP::BYTES <= kPipeMaxSmem && SP::BYTES <= device_smem_optin() &&
                           (EXACT || s.lift_z != nullptr) &&
                           (batch || (aligned(s.q) && aligned(s.u) && aligned(s.v) &&
                                      aligned(s.w) && aligned(s.escale) &&
                                      aligned(s.fscale) && aligned(s.pbase) &&
                                      (s.q0 == nullptr || aligned(s.q0))));
    const bool want_split =
        s.variant == kVariantSplit ||
        (s.variant == kVariantAuto && !batch && kSplitAuto<NQ, TC, EXACT>);
    if (want_split) {
      if (!can_split) {
        if (batch) return static_cast<int>(cudaErrorNotSupported);
      } else {
        constexpr int T = SplitGeo<NQ, H>::THREADS;
        const int ntiles = batch ? s.batch_ntiles : s.nelem;
        if (batch)
          return launch_pipe<tend_split_kernel<NQ, H, TQ, TV, TO, TC, EXACT, ORDER, STAGE, true>,
                             T>(SP::BYTES, ntiles, s, a, d);
        return launch_pipe<tend_split_kernel<NQ, H, TQ, TV, TO, TC, EXACT, ORDER, STAGE, false>,
                           T>(SP::BYTES, ntiles, s, a, d);
      }
    }
  }
  // Tensor-core lines (mixed form, Nq = 8, single instance).
  if constexpr (NQ == 8 && sizeof(TC) == 4 && !EXACT && STAGE) {
    using TP = PipePlan<NQ, TQ, TV, TC, STAGE, true>;
    if (s.variant == kVariantTensor && !batch && can_pipe && TP::BYTES <= device_smem_optin()) {
      const int ntiles = (s.nelem + PipeGeo<NQ>::EPB - 1) / PipeGeo<NQ>::EPB;
      // Blocks per SM of the plan and the launch bounds: 4 x 32 TMEM columns
      // of the SM's 512.
      constexpr int fb = pipe_min_blocks<NQ, TQ, TV, TC, EXACT, STAGE, true>();
      return launch_pipe<tend_pipe_kernel<NQ, TQ, TV, TO, TC, EXACT, ORDER, STAGE, false, true>>(
          TP::BYTES, ntiles, s, a, d, fb);
    }
  }
  if (batch && !can_pipe) return static_cast<int>(cudaErrorNotSupported);
  const bool pipe =
      batch || ((s.variant == kVariantPipe || s.variant == kVariantAuto ||
                 s.variant == kVariantSplit || s.variant == kVariantTensor) && can_pipe);
  if (pipe) {
    const int ntiles =
        batch ? s.batch_ntiles : (s.nelem + PipeGeo<NQ>::EPB - 1) / PipeGeo<NQ>::EPB;
    if (batch)
      return launch_pipe<tend_pipe_kernel<NQ, TQ, TV, TO, TC, EXACT, ORDER, STAGE, true>>(
          PB::BYTES, ntiles, s, a, d);
    return launch_pipe<tend_pipe_kernel<NQ, TQ, TV, TO, TC, EXACT, ORDER, STAGE, false>>(
        P::BYTES, ntiles, s, a, d);
  }

  const size_t smem = SmemLayout<NQ, TC>::BYTES;
  if constexpr (NQ >= 4 && NQ <= 8) {
    // One tile per block, built for 8 resident 128-thread blocks per SM
    // (64 registers per thread) with the largest shared-memory carveout.
    if (s.variant == kVariantBlockOcc) {
      auto kern = tend_kernel<NQ, TQ, TV, TO, TC, EXACT, ORDER, STAGE, 8>;
      static DeviceSetup carve;  // per device
      const int dev = setup_device();
      if (dev < 0) return static_cast<int>(cudaErrorInvalidDevice);
      if (carve.slot[dev].load(std::memory_order_relaxed) == 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        carve.slot[dev].store(1, std::memory_order_relaxed);
      }
      if (s.nelem <= 0) return 0;
      a.prefetch_dist = 8 * (s.num_sms > 0 ? s.num_sms : 148);
      const int blocks = (s.nelem + G::EPB - 1) / G::EPB;
      kern<<<blocks, G::THREADS, smem, s.stream>>>(a, d);
      return static_cast<int>(cudaGetLastError());
    }
  }
  // The fast FP64 kernels with columns of 12 or more nodes are built for two
  // resident blocks: left free they take 160-254 registers, one block of
  // 144-256 threads per SM; capped they spill but measured 1.1-1.6x faster
  // (p = 11: 29.5 -> 48.5 G DOF-updates/s, p = 15: 47.5 -> 53.0).
  constexpr int MB = (!EXACT && NQ >= 12) ? 2 : 1;
  auto kern = tend_kernel<NQ, TQ, TV, TO, TC, EXACT, ORDER, STAGE, MB>;
  static DeviceSetup setup;  // blocks per SM, per instantiation and device
  const int dev = setup_device();
  if (dev < 0) return static_cast<int>(cudaErrorInvalidDevice);
  int resident = setup.slot[dev].load(std::memory_order_relaxed);
  if (resident == 0) {
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(
          kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e != cudaSuccess) return static_cast<int>(e);
    }
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int nb = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, G::THREADS, smem);
    if (e != cudaSuccess) return static_cast<int>(e);
    resident = nb > 0 ? nb : 1;
    setup.slot[dev].store(resident, std::memory_order_relaxed);
  }
  if (s.nelem <= 0) return 0;
  a.prefetch_dist = resident * (s.num_sms > 0 ? s.num_sms : 148);
  const int blocks = (s.nelem + G::EPB - 1) / G::EPB;
  kern<<<blocks, G::THREADS, smem, s.stream>>>(a, d);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace

#define SDG_CAT2(a, b) a##b
#define SDG_CAT(a, b) SDG_CAT2(a, b)

// Which persistent plans fit both the build's limit and the current
// device's per-block opt-in: bit 0 the pipelined kernel, bit 1 the
// split-column kernel (orders with one element per tile).
template <typename TQ, typename TV, typename TC, bool STAGE>
int pipe_fits() {
  const size_t optin = device_smem_optin();
  // Batched plans (the ensemble asks): the tile context travels in the slot.
  constexpr size_t bytes = PipePlan<NQ, TQ, TV, TC, STAGE, false, true>::BYTES;
  int r = (bytes <= kPipeMaxSmem && bytes <= optin) ? 1 : 0;
  if constexpr (NQ >= 9) {
    constexpr size_t sb = SplitPlan<NQ, kSplitH<NQ>, TQ, TV, TC, STAGE>::BYTES;
    if (sb <= kPipeMaxSmem && sb <= optin) r |= 2;
  }
  return r;
}

// Pipelined-kernel facts for this order: elements per tile, and whether the
// shared-memory plan of each kind fits.
int SDG_CAT(pipe_info_nq, SDG_NQ)(int kind, int* epb) {
  *epb = PipeGeo<NQ>::EPB;
  switch (kind) {
    case kTendF64: return pipe_fits<double, double, double, false>();
    case kStageF64: return pipe_fits<double, double, double, true>();
    case kStageMixed1: return pipe_fits<double, float, float, true>();
    case kStageMixed2: return pipe_fits<float, float, float, true>();
    case kStageMixed3: return pipe_fits<float, float, float, true>();
    default: return 0;
  }
}

int SDG_CAT(launch_tend_nq, SDG_NQ)(const LaunchSpec& s) {
  if (s.nq != NQ) return -1;
  // Orders only differ for NQ > 8; below that both map to one variant.
  const bool gen = (NQ > 8) && s.order == kOrderGeneral;
  switch (s.kind) {
    case kTendF64:
      if (!s.exact) return run<double, double, double, double, false, kOrderOpt1, false>(s);
      if (gen) return run<double, double, double, double, true, kOrderGeneral, false>(s);
      return run<double, double, double, double, true, kOrderOpt1, false>(s);
    case kStageF64:
      if (!s.exact) return run<double, double, double, double, false, kOrderOpt1, true>(s);
      if (gen) return run<double, double, double, double, true, kOrderGeneral, true>(s);
      return run<double, double, double, double, true, kOrderOpt1, true>(s);
    case kStageMixed1:
      return run<double, float, float, float, false, kOrderOpt1, true>(s);
    case kStageMixed2:
      return run<float, float, float, float, false, kOrderOpt1, true>(s);
    case kStageMixed3:
      return run<float, float, double, float, false, kOrderOpt1, true>(s);
    default:
      return static_cast<int>(cudaErrorInvalidValue);
  }
}

}  // namespace sdg
