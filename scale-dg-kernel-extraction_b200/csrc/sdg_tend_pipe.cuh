// Persistent, software-pipelined variant of the fused tendency / RK-stage
// kernel (same arithmetic as tend_kernel in sdg_tend.cuh, same results).
//
// Each block loops over tiles of EPB consecutive elements.  The element data
// a tile needs (q, u, v, w and, for RK stages, q0) are contiguous in HBM, so
// one elected thread moves them into a shared-memory ring of NSTAGE tiles
// with cp.async.bulk (the TMA bulk-copy engine), completing on an mbarrier
// per ring slot; the copy of tile i+NSTAGE is issued as soon as tile i has
// been read out of its slot.  Compute threads never stall on their own
// loads: the bytes in flight per SM are set by the ring, not by occupancy.
// The plus-side face values, which live in neighbouring elements, are
// gathered with ordinary loads issued before the ring wait so that their
// L2 latency overlaps it.  For p <= 7 each column thread keeps its 6*NQ
// lift coefficients in registers for the whole persistent loop.
//
// Every wait is bounded.  A wait that runs out sets *status and the block
// drains its own copies (again bounded) and returns; the host reports the
// status as an error.  Decisions after a wait are made block-uniform with
// __syncthreads_and so that no thread can skip a barrier another reaches.
#pragma once

#include "sdg_tend.cuh"

namespace sdg {

constexpr int kStatusWaitTimeout = 1;
constexpr unsigned kWaitSpins = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of `bar` with the given parity.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (unsigned it = 0; it < kWaitSpins; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Global -> shared bulk copy on the TMA engine (no multicast), completing
// `bytes` of transaction count on `bar`.  dst, src and bytes are multiples
// of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Shared-memory plan of the pipelined kernel.
template <int NQ, typename TQ, typename TV, typename TC, bool STAGE>
struct PipePlan {
  using G = Geo<NQ>;
  static constexpr int EPB = G::EPB;
  static constexpr int NP = G::NP;
  static constexpr int NSTAGE = 2;
  static constexpr size_t r16(size_t x) { return (x + 15) & ~size_t(15); }
  // Each array region holds EPB elements plus 32 bytes of slack: the source
  // range is widened to 16-byte boundaries at both ends (at most 12 bytes
  // each for 4- and 8-byte elements).
  static constexpr size_t QB = r16(sizeof(TQ) * EPB * NP + 32);
  static constexpr size_t VB = r16(sizeof(TV) * EPB * NP + 32);
  static constexpr size_t Q0B = STAGE ? r16(sizeof(double) * EPB * NP + 32) : 0;
  static constexpr size_t SLOT = QB + 3 * VB + Q0B;
  static constexpr size_t WORK = r16(sizeof(TC) * SmemLayout<NQ, TC>::PER_ELEM * EPB);
  static constexpr size_t BARS = 16 * NSTAGE;
  static constexpr size_t BYTES = NSTAGE * SLOT + WORK + BARS;
  // Lift coefficients kept in registers when the column is short.
  static constexpr bool LIFT_REGS = NQ <= 8;
};

template <int NQ, typename TQ, typename TV, typename TO, typename TC, bool EXACT,
          int ORDER, bool STAGE>
__global__ void __launch_bounds__(Geo<NQ>::THREADS)
    tend_pipe_kernel(const __grid_constant__ TendArgs<TQ, TV, TO, TC> A,
                     const __grid_constant__ DMat<NQ, TC> D) {
  using G = Geo<NQ>;
  using P = PipePlan<NQ, TQ, TV, TC, STAGE>;
  using AR = Ar<TC, EXACT>;
  constexpr int NQ2 = G::NQ2;
  constexpr int NP = G::NP;
  constexpr int RS = G::RS;
  constexpr int PS = G::PS;
  constexpr int EPB = G::EPB;
  constexpr int NS = P::NSTAGE;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* slots = smem_raw;
  TC* work = reinterpret_cast<TC*>(smem_raw + NS * P::SLOT);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + NS * P::SLOT + P::WORK);

  const int s = threadIdx.x / NQ2;
  const int t = threadIdx.x - s * NQ2;
  const int a = t % NQ;
  const int b = t / NQ;
  const int ntiles = (A.nelem + EPB - 1) / EPB;

  TC* sX = work + s * SmemLayout<NQ, TC>::PER_ELEM;
  TC* sY = sX + G::SBUF;
  TC* fQ = sY + G::SBUF;
  TC* fU = fQ + 4 * NQ2;

  // Byte range of the tile's elements in an array of element size `sz`,
  // widened to 16-byte boundaries.
  auto range = [&](int tile, size_t sz, size_t* lo16, uint32_t* bytes, uint32_t* shift) {
    const int e0 = A.elem0 + tile * EPB;
    const int n = min(EPB, A.nelem - tile * EPB);
    const size_t lo = static_cast<size_t>(e0) * NP * sz;
    const size_t hi = static_cast<size_t>(e0 + n) * NP * sz;
    *lo16 = lo & ~size_t(15);
    *bytes = static_cast<uint32_t>(((hi + 15) & ~size_t(15)) - *lo16);
    *shift = static_cast<uint32_t>(lo - *lo16);
  };

  // Producer: one thread fills ring slot `slot` with tile `tile`.
  auto issue = [&](int tile, int slot) {
    unsigned char* base = slots + slot * P::SLOT;
    const void* src[5] = {A.q, A.u, A.v, A.w, A.q0};
    const size_t sz[5] = {sizeof(TQ), sizeof(TV), sizeof(TV), sizeof(TV), sizeof(double)};
    const size_t off[5] = {0, P::QB, P::QB + P::VB, P::QB + 2 * P::VB, P::QB + 3 * P::VB};
    const int narr = (STAGE && A.rk_a != 0.0) ? 5 : 4;
    size_t lo[5];
    uint32_t by[5], sh[5], total = 0;
    for (int k = 0; k < narr; ++k) {
      range(tile, sz[k], &lo[k], &by[k], &sh[k]);
      total += by[k];
    }
    mbar_arrive_expect_tx(&bars[slot], total);
    for (int k = 0; k < narr; ++k)
      bulk_g2s(base + off[k], static_cast<const unsigned char*>(src[k]) + lo[k], by[k],
               &bars[slot]);
  };

  if (threadIdx.x == 0) {
    for (int k = 0; k < NS; ++k) mbar_init(&bars[k], 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < NS; ++k) {
      const int tile = blockIdx.x + k * gridDim.x;
      if (tile < ntiles) issue(tile, k);
    }

  // Lift coefficients of this column, kept for the whole loop (p <= 7).
  constexpr int LR = P::LIFT_REGS ? 6 * NQ : 1;
  TC lreg[LR];
  if constexpr (P::LIFT_REGS) {
#pragma unroll
    for (int k = 0; k < NQ; ++k)
#pragma unroll
      for (int f = 0; f < 6; ++f) lreg[6 * k + f] = ldro(A.lift + t + NQ2 * k + NP * f);
  }

  for (int it = 0;; ++it) {
    const int tile = blockIdx.x + it * gridDim.x;
    if (tile >= ntiles) break;
    const int slot = it % NS;
    const uint32_t parity = (it / NS) & 1;
    const int el = tile * EPB + s;
    const bool active = el < A.nelem;
    const int e = A.elem0 + (active ? el : 0);
    const long base = static_cast<long>(e) * NP;

    // ---- Plus-side face gathers, issued before the ring wait ---------------
    TC qP[4], unP[4], q5 = TC(0), w5 = TC(0), q6 = TC(0), w6 = TC(0);
    if (active) {
      const int* pb = A.pbase + 6 * static_cast<long>(e);
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const int p = pb[f];
        long idx;
        if (p >= 0) {
          const int off = (f == 0)   ? a + NQ * (NQ - 1) + NQ2 * b
                          : (f == 1) ? NQ * a + NQ2 * b
                          : (f == 2) ? a + NQ2 * b
                                     : (NQ - 1) + NQ * a + NQ2 * b;
          idx = static_cast<long>(p) + off;
        } else {
          idx = static_cast<long>(-1 - p) + t;
        }
        qP[f] = static_cast<TC>(ldro(A.q + idx));
        unP[f] = static_cast<TC>((f == 1 || f == 3) ? ldro(A.u + idx) : ldro(A.v + idx));
      }
      const int p5 = pb[4];
      const long i5 = (p5 >= 0) ? static_cast<long>(p5) + t + NQ2 * (NQ - 1)
                                : static_cast<long>(-1 - p5) + t;
      q5 = static_cast<TC>(ldro(A.q + i5));
      w5 = static_cast<TC>(ldro(A.w + i5));
      const int p6 = pb[5];
      const long i6 = (p6 >= 0) ? static_cast<long>(p6) + t : static_cast<long>(-1 - p6) + t;
      q6 = static_cast<TC>(ldro(A.q + i6));
      w6 = static_cast<TC>(ldro(A.w + i6));
    }

    // ---- Wait for the tile's slot (bounded, block-uniform) -----------------
    const bool ok = __syncthreads_and(mbar_wait_bounded(&bars[slot], parity));
    if (!ok) {
      if (threadIdx.x == 0) {
        atomicExch(A.status, kStatusWaitTimeout);
        // Drain this block's copies still in flight (this slot included)
        // before leaving.
        for (int k = 0; k < NS; ++k) {
          const int tk = blockIdx.x + (it + k) * gridDim.x;
          if (tk < ntiles) mbar_wait_bounded(&bars[(it + k) % NS], ((it + k) / NS) & 1);
        }
      }
      return;
    }

    // ---- Phase 1: read the column out of the slot -------------------------
    unsigned char* sb = slots + slot * P::SLOT;
    size_t lo;
    uint32_t by, shq, shv, sh0 = 0;
    range(tile, sizeof(TQ), &lo, &by, &shq);
    range(tile, sizeof(TV), &lo, &by, &shv);
    if (STAGE) range(tile, sizeof(double), &lo, &by, &sh0);
    const TQ* sq = reinterpret_cast<const TQ*>(sb + shq) + s * NP;
    const TV* su = reinterpret_cast<const TV*>(sb + P::QB + shv) + s * NP;
    const TV* sv = reinterpret_cast<const TV*>(sb + P::QB + P::VB + shv) + s * NP;
    const TV* sw = reinterpret_cast<const TV*>(sb + P::QB + 2 * P::VB + shv) + s * NP;
    const double* sq0 =
        reinterpret_cast<const double*>(sb + P::QB + 3 * P::VB + sh0) + s * NP;

    TC qc[NQ], fz[NQ];
    double qs[STAGE && sizeof(TQ) != sizeof(TC) ? NQ : 1];
    double q0v[STAGE ? NQ : 1];
    TC wlo = TC(0), whi = TC(0);
    if (active) {
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        const int n = t + NQ2 * k;
        const TC qv = static_cast<TC>(sq[n]);
        const TC uv = static_cast<TC>(su[n]);
        const TC vv = static_cast<TC>(sv[n]);
        const TC wv = static_cast<TC>(sw[n]);
        if constexpr (STAGE && sizeof(TQ) != sizeof(TC)) qs[k] = static_cast<double>(sq[n]);
        if constexpr (STAGE) q0v[k] = (A.rk_a != 0.0) ? sq0[n] : 0.0;
        qc[k] = qv;
        sX[a + RS * b + PS * k] = AR::mul(qv, uv);
        sY[a + RS * b + PS * k] = AR::mul(qv, vv);
        fz[k] = AR::mul(qv, wv);
        if (k == 0) wlo = wv;
        if (k == NQ - 1) whi = wv;
        if (b == 0)      { fQ[0 * NQ2 + a + NQ * k] = qv; fU[0 * NQ2 + a + NQ * k] = vv; }
        if (a == NQ - 1) { fQ[1 * NQ2 + b + NQ * k] = qv; fU[1 * NQ2 + b + NQ * k] = uv; }
        if (b == NQ - 1) { fQ[2 * NQ2 + a + NQ * k] = qv; fU[2 * NQ2 + a + NQ * k] = vv; }
        if (a == 0)      { fQ[3 * NQ2 + b + NQ * k] = qv; fU[3 * NQ2 + b + NQ * k] = uv; }
      }
    }
    __syncthreads();
    // The slot has been read out: refill it with the tile NS iterations on.
    if (threadIdx.x == 0) {
      const int nt = blockIdx.x + (it + NS) * gridDim.x;
      if (nt < ntiles) issue(nt, slot);
    }

    TC f5 = TC(0), f6 = TC(0);
    if (active) {
      const TC* fs = A.fscale + 6 * static_cast<long>(e);
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const TC sg = (f == 0 || f == 3) ? TC(-1) : TC(1);
        fQ[f * NQ2 + t] =
            upwind_flux<AR, TC>(fQ[f * NQ2 + t], fU[f * NQ2 + t], qP[f], unP[f], sg, fs[f]);
      }
      f5 = upwind_flux<AR, TC>(qc[0], wlo, q5, w5, TC(-1), fs[4]);
      f6 = upwind_flux<AR, TC>(qc[NQ - 1], whi, q6, w6, TC(1), fs[5]);
      TC line[NQ];
#pragma unroll
      for (int l = 0; l < NQ; ++l) line[l] = sX[l + RS * a + PS * b];
#pragma unroll
      for (int i = 0; i < NQ; ++i)
        sX[i + RS * a + PS * b] = contract<NQ, ORDER, AR, TC>(
            [&](int l) { return D.d[i * NQ + l]; }, [&](int l) { return line[l]; });
#pragma unroll
      for (int l = 0; l < NQ; ++l) line[l] = sY[a + RS * l + PS * b];
#pragma unroll
      for (int j = 0; j < NQ; ++j)
        sY[a + RS * j + PS * b] = contract<NQ, ORDER, AR, TC>(
            [&](int l) { return line[l]; }, [&](int l) { return D.d[j * NQ + l]; });
    }
    __syncthreads();

    if (active) {
      TC dz[NQ];
#pragma unroll
      for (int k = 0; k < NQ; ++k)
        dz[k] = contract<NQ, ORDER, AR, TC>([&](int l) { return fz[l]; },
                                            [&](int l) { return D.d[k * NQ + l]; });
      const TC* es = A.escale + 3 * static_cast<long>(e);
      const TC e1 = es[0], e2 = es[1], e3 = es[2];
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        TC L[6];
#pragma unroll
        for (int f = 0; f < 6; ++f) {
          if constexpr (P::LIFT_REGS) L[f] = lreg[6 * k + f];
          else L[f] = ldro(A.lift + t + NQ2 * k + NP * f);
        }
        TC lf = AR::mul(L[0], fQ[0 * NQ2 + a + NQ * k]);
        lf = AR::mad(L[1], fQ[1 * NQ2 + b + NQ * k], lf);
        lf = AR::mad(L[2], fQ[2 * NQ2 + a + NQ * k], lf);
        lf = AR::mad(L[3], fQ[3 * NQ2 + b + NQ * k], lf);
        lf = AR::mad(L[4], f5, lf);
        lf = AR::mad(L[5], f6, lf);
        TC acc = AR::mul(e1, sX[a + RS * b + PS * k]);
        acc = AR::mad(e2, sY[a + RS * b + PS * k], acc);
        acc = AR::mad(e3, dz[k], acc);
        acc = AR::add(acc, lf);
        const TC dqdt = -acc;
        const long n = base + t + NQ2 * k;
        if constexpr (!STAGE) {
          A.out[n] = static_cast<TO>(dqdt);
        } else {
          using AD = Ar<double, EXACT>;
          double qd;
          if constexpr (sizeof(TQ) == sizeof(TC)) qd = static_cast<double>(qc[k]);
          else qd = qs[k];
          double r = AD::mul(A.rk_b, AD::mad(A.dt, static_cast<double>(dqdt), qd));
          if (A.rk_a != 0.0) r = AD::mad(A.rk_a, q0v[k], r);
          A.out[n] = static_cast<TO>(r);
        }
      }
    }
  }
}

}  // namespace sdg
