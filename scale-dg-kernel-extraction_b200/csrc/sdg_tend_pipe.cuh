// Persistent, software-pipelined variant of the fused tendency / RK-stage
// kernel (same arithmetic as tend_kernel in sdg_tend.cuh, same results).
//
// Each block loops over tiles of EPB consecutive elements.  The element data
// a tile needs (q, u, v, w and, for RK stages 2-3, q0) are contiguous in
// HBM, so one elected thread moves them into a shared-memory ring of NSTAGE
// tiles with cp.async.bulk (the TMA bulk-copy engine), completing on an
// mbarrier per ring slot.  A slot stays resident for its whole tile (the
// epilogue re-reads q and q0 from it instead of holding them in registers)
// and is refilled, with the tile NSTAGE iterations on, as the block starts
// the next tile.  Compute threads never stall on their own element loads:
// the bytes in flight per SM are set by the ring, not by occupancy.  The
// plus-side face values (in neighbouring elements) are gathered with
// ordinary loads issued before the ring wait, so their latency overlaps it.
//
// Thread mapping.  Column (a,b) of an element (its z-line) is owned by H
// threads.  With H = 2 (Nq^2 a multiple of 32, i.e. p = 7 and p = 15) the two
// owners sit in different warps, so the half index h is warp-uniform:
//   h = 0: nodes k < Nq/2, the x-line (j,k) = (a,b), faces 1-2 at node
//          (a,b), the -z face;
//   h = 1: nodes k >= Nq/2, the y-line (i,k) = (a,b), faces 3-4, the +z face.
// The two halves of a z-column meet in shared memory for the z-derivative.
// With H = 1 one thread plays every role, as in tend_kernel.  Splitting
// halves the registers per thread and doubles the warps per SM for the same
// shared memory; each output's summation chain is unchanged.
//
// For p <= 7 each thread keeps the lift coefficients of its column nodes in
// registers for the whole persistent loop.
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
// Largest shared-memory plan the pipelined kernel is used with: two blocks
// of it fit on one SM (228 KB).
constexpr size_t kPipeMaxSmem = 110 * 1024;

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

// Thread geometry of the pipelined kernel.
// kSplitColumns enables the two-owners-per-column mapping (H = 2) where
// Nq^2 is a multiple of 32.  Measured on B200 at p = 7 it doubles the warps
// per SM but is slower (60.9 vs 70.6 G DOF-updates/s FP64): the kernel is
// limited by the shared-memory pipe, and the split adds 15% wavefronts and
// barrier stalls.  Kept for experiments; off by default.
#ifndef SDG_SPLIT_COLUMNS
#define SDG_SPLIT_COLUMNS 0
#endif
constexpr bool kSplitColumns = SDG_SPLIT_COLUMNS != 0;

// Placement of node (i,j,k) in the x-line and y-line buffers.  Generic
// orders use the padded layout of tend_kernel.  For Nq = 8 an XOR swizzle
// over the 16 eight-byte bank pairs makes every access pattern of the
// kernel conflict-free: column (i fastest, two j per half-warp), x-line
// (fixed i, j and two k per half-warp) and y-line (fixed j, i and two k):
//   x(i,j,k) = 16*((j + 8k) >> 1) + ((i ^ j) & 7) + 8*((j + k) & 1)
//   y(i,j,k) = 16*((i + 8k) >> 1) + ((i ^ j) & 7) + 8*((i + k) & 1)
// (bijections onto 0..511).  The padded layout costs two wavefronts more
// per column access.
template <int NQ>
struct LineIdx {
  static constexpr int SIZE = Geo<NQ>::SBUF;
  static __device__ __forceinline__ int x(int i, int j, int k) {
    return i + Geo<NQ>::RS * j + Geo<NQ>::PS * k;
  }
  static __device__ __forceinline__ int y(int i, int j, int k) {
    return i + Geo<NQ>::RS * j + Geo<NQ>::PS * k;
  }
};
template <>
struct LineIdx<8> {
  static constexpr int SIZE = 512;
  static __device__ __forceinline__ int x(int i, int j, int k) {
    return 16 * ((j + 8 * k) >> 1) + ((i ^ j) & 7) + 8 * ((j + k) & 1);
  }
  static __device__ __forceinline__ int y(int i, int j, int k) {
    return 16 * ((i + 8 * k) >> 1) + ((i ^ j) & 7) + 8 * ((i + k) & 1);
  }
};

// A (q_minus, un_minus) pair of a face node, stored in one 8- or 16-byte word.
template <typename T>
struct Pair2;
template <>
struct Pair2<double> {
  using type = double2;
};
template <>
struct Pair2<float> {
  using type = float2;
};

template <int NQ>
struct PipeGeo {
  static constexpr int NQ2 = NQ * NQ;
  static constexpr int NP = NQ2 * NQ;
  static constexpr int H = (kSplitColumns && NQ2 % 32 == 0) ? 2 : 1;  // owners per column
  static constexpr int KH = NQ / H;                  // column nodes per thread
  static constexpr int TPE = H * NQ2;                // threads per element
  static constexpr int TARGET = (H == 2) ? 256 : 128;
  static constexpr int EPB = TPE >= TARGET ? 1 : TARGET / TPE;
  static constexpr int THREADS = EPB * TPE;
  static constexpr int SBUF = LineIdx<NQ>::SIZE;
  // Per-element work area (in compute-type words): x- and y-line buffers,
  // the four x/y faces' (q_minus, un_minus) pairs (each face flux
  // overwrites its q_minus), the two z-face fluxes and, when H = 2, the
  // z-column exchange buffer.
  static constexpr int WORK_ELEM = 2 * SBUF + 8 * NQ2 + 2 * NQ2 + (H == 2 ? NP : 0);
};

// Shared-memory plan of the pipelined kernel.
template <int NQ, typename TQ, typename TV, typename TC, bool STAGE>
struct PipePlan {
  using G = PipeGeo<NQ>;
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
  static constexpr size_t WORK = r16(sizeof(TC) * G::WORK_ELEM * EPB);
  static constexpr size_t BARS = 16 * NSTAGE;
  static constexpr size_t BYTES = NSTAGE * SLOT + WORK + BARS;
  // Lift coefficients kept in registers when the column is short.
  static constexpr bool LIFT_REGS = NQ <= 8;
};

// Arrays and element range of one tile.
template <typename TQ, typename TV, typename TO, typename TC>
struct TileCtx {
  const TQ* q;
  const TV* u;
  const TV* v;
  const TV* w;
  const double* q0;
  TO* out;
  const int* pbase;
  const TC* escale;
  const TC* fscale;
  double dt;
  int e0;  // first element (index into the arrays)
  int n;   // elements in the tile (1..EPB)
};

// BATCH is a compile-time property of the kernel, so a single-instance
// launch keeps its pointers in the parameter bank instead of registers.
template <int EPB, bool BATCH, typename TQ, typename TV, typename TO, typename TC>
__device__ __forceinline__ TileCtx<TQ, TV, TO, TC> tile_ctx(const TendArgs<TQ, TV, TO, TC>& A,
                                                            int tile) {
  TileCtx<TQ, TV, TO, TC> c;
  if constexpr (!BATCH) {
    c.q = A.q;
    c.u = A.u;
    c.v = A.v;
    c.w = A.w;
    c.q0 = A.q0;
    c.out = A.out;
    c.pbase = A.pbase;
    c.escale = A.escale;
    c.fscale = A.fscale;
    c.dt = A.dt;
    c.e0 = A.elem0 + tile * EPB;
    c.n = min(EPB, A.nelem - tile * EPB);
  } else {
    const BatchTile t = A.tiles[tile];
    const BatchInst& I = A.insts[t.inst];
    c.q = static_cast<const TQ*>(I.q);
    c.u = static_cast<const TV*>(I.u);
    c.v = static_cast<const TV*>(I.v);
    c.w = static_cast<const TV*>(I.w);
    c.q0 = I.q0;
    c.out = static_cast<TO*>(I.out);
    c.pbase = I.pbase;
    c.escale = static_cast<const TC*>(I.escale);
    c.fscale = static_cast<const TC*>(I.fscale);
    c.dt = I.dt;
    c.e0 = t.e0;
    c.n = t.n;
  }
  return c;
}

// Plus-side node of face f (0-based) at face node (a,b) of the neighbour
// starting at node p >= 0: Fmask(fp, oppface) - 1 (mod_mesh.f90:278-324).
template <int NQ>
__device__ __forceinline__ int opp_offset(int f, int a, int b) {
  constexpr int NQ2 = NQ * NQ;
  switch (f) {
    case 0: return a + NQ * (NQ - 1) + NQ2 * b;   // opposite face 3 (j = Nq)
    case 1: return NQ * a + NQ2 * b;              // opposite face 4 (i = 1)
    case 2: return a + NQ2 * b;                   // opposite face 1 (j = 1)
    case 3: return (NQ - 1) + NQ * a + NQ2 * b;   // opposite face 2 (i = Nq)
    case 4: return a + NQ * b + NQ2 * (NQ - 1);   // opposite face 6 (k = Nq)
    default: return a + NQ * b;                   // opposite face 5 (k = 1)
  }
}

// Phase 4 of one thread: z-derivative, lift, combine and store for the
// column nodes k = K0 .. K0+KH-1 (K0 compile-time, so D's rows are
// immediate constant-bank operands).
template <int NQ, int K0, int KH, int ORDER, bool STAGE, bool LIFT_REGS, bool EXACT,
          typename TQ, typename TV, typename TO, typename TC>
__device__ __forceinline__ void column_epilogue(
    const TendArgs<TQ, TV, TO, TC>& A, const DMat<NQ, TC>& D,
    const TileCtx<TQ, TV, TO, TC>& C, int e, long base, int t, int a, int b, const TC* zcol,
    const TC* sX, const TC* sY, const TC* fQ, TC f5, TC f6, const TQ* sq,
    const double* sq0, const TC* lreg) {
  constexpr int NQ2 = NQ * NQ;
  constexpr int NP = NQ2 * NQ;
  using LI = LineIdx<NQ>;
  using AR = Ar<TC, EXACT>;
  const TC* es = C.escale + 3 * static_cast<long>(e);
  const TC e1 = es[0], e2 = es[1], e3 = es[2];
#pragma unroll
  for (int kk = 0; kk < KH; ++kk) {
    const int k = K0 + kk;
    const TC dz = contract<NQ, ORDER, AR, TC>([&](int l) { return zcol[l]; },
                                              [&](int l) { return D.d[k * NQ + l]; });
    TC L[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if constexpr (LIFT_REGS) L[f] = lreg[6 * kk + f];
      else L[f] = ldro(A.lift + t + NQ2 * k + NP * f);
    }
    // x/y face fluxes sit at stride 2 (the .x of each (q, un) pair).
    TC lf = AR::mul(L[0], fQ[2 * (0 * NQ2 + a + NQ * k)]);
    lf = AR::mad(L[1], fQ[2 * (1 * NQ2 + b + NQ * k)], lf);
    lf = AR::mad(L[2], fQ[2 * (2 * NQ2 + a + NQ * k)], lf);
    lf = AR::mad(L[3], fQ[2 * (3 * NQ2 + b + NQ * k)], lf);
    lf = AR::mad(L[4], f5, lf);
    lf = AR::mad(L[5], f6, lf);
    TC acc = AR::mul(e1, sX[LI::x(a, b, k)]);
    acc = AR::mad(e2, sY[LI::y(a, b, k)], acc);
    acc = AR::mad(e3, dz, acc);
    acc = AR::add(acc, lf);
    const TC dqdt = -acc;
    const long n = base + t + NQ2 * k;
    if constexpr (!STAGE) {
      C.out[n] = static_cast<TO>(dqdt);
    } else {
      using AD = Ar<double, EXACT>;
      double qd;
      // The stage input at its stored precision, from the tile's ring slot.
      qd = static_cast<double>(sq[t + NQ2 * k]);
      double r = AD::mul(A.rk_b, AD::mad(C.dt, static_cast<double>(dqdt), qd));
      // q0 is read from the tile's ring slot (still resident in phase 4).
      if (A.rk_a != 0.0) r = AD::mad(A.rk_a, sq0[t + NQ2 * k], r);
      C.out[n] = static_cast<TO>(r);
    }
  }
}

template <int NQ, typename TQ, typename TV, typename TO, typename TC, bool EXACT,
          int ORDER, bool STAGE, bool BATCH>
__global__ void __launch_bounds__(PipeGeo<NQ>::THREADS, 2)
    tend_pipe_kernel(const __grid_constant__ TendArgs<TQ, TV, TO, TC> A,
                     const __grid_constant__ DMat<NQ, TC> D) {
  using G = PipeGeo<NQ>;
  using P = PipePlan<NQ, TQ, TV, TC, STAGE>;
  using AR = Ar<TC, EXACT>;
  using Ctx = TileCtx<TQ, TV, TO, TC>;
  constexpr int NQ2 = G::NQ2;
  constexpr int NP = G::NP;
  constexpr int EPB = G::EPB;
  constexpr int H = G::H;
  constexpr int KH = G::KH;
  constexpr int NS = P::NSTAGE;
  constexpr int NFACE = 4 / H;   // x/y faces evaluated per thread
  constexpr int NZF = 2 / H;     // z faces evaluated per thread

  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* slots = smem_raw;
  TC* work = reinterpret_cast<TC*>(smem_raw + NS * P::SLOT);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + NS * P::SLOT + P::WORK);

  const int s = threadIdx.x / G::TPE;            // element slot
  const int r = threadIdx.x - s * G::TPE;
  const int h = (H == 2) ? r / NQ2 : 0;          // warp-uniform half
  const int t = r - h * NQ2;                     // column index a + NQ*b
  const int a = t % NQ;
  const int b = t / NQ;
  const int k0 = h * KH;
  const int ntiles = BATCH ? A.ntiles : (A.nelem + EPB - 1) / EPB;

  using V2 = typename Pair2<TC>::type;
  using LI = LineIdx<NQ>;
  TC* sX = work + s * G::WORK_ELEM;
  TC* sY = sX + G::SBUF;
  // [4][NQ2] (q, un) of the minus side; phase 2 overwrites q with the flux,
  // so the lift reads the x/y face fluxes at stride 2 from fQ.
  V2* fM = reinterpret_cast<V2*>(sY + G::SBUF);
  TC* fQ = sY + G::SBUF;
  TC* fZ = fQ + 8 * NQ2;       // [2][NQ2] z-face fluxes
  TC* sZ = fZ + 2 * NQ2;       // [NQ][NQ2] z-column exchange (H = 2)

  // Byte range of elements [e0, e0+n) in an array of element size `sz`,
  // widened to 16-byte boundaries.
  auto range = [&](int e0, int n, size_t sz, size_t* lo16, uint32_t* bytes,
                   uint32_t* shift) {
    const size_t lo = static_cast<size_t>(e0) * NP * sz;
    const size_t hi = static_cast<size_t>(e0 + n) * NP * sz;
    *lo16 = lo & ~size_t(15);
    *bytes = static_cast<uint32_t>(((hi + 15) & ~size_t(15)) - *lo16);
    *shift = static_cast<uint32_t>(lo - *lo16);
  };

  // Producer: one thread fills ring slot `slot` with tile `tile`.
  auto issue = [&](int tile, int slot) {
    const Ctx c = tile_ctx<EPB, BATCH>(A, tile);
    unsigned char* base = slots + slot * P::SLOT;
    const void* src[5] = {c.q, c.u, c.v, c.w, c.q0};
    const size_t sz[5] = {sizeof(TQ), sizeof(TV), sizeof(TV), sizeof(TV), sizeof(double)};
    const size_t off[5] = {0, P::QB, P::QB + P::VB, P::QB + 2 * P::VB, P::QB + 3 * P::VB};
    const int narr = (STAGE && A.rk_a != 0.0) ? 5 : 4;
    size_t lo[5];
    uint32_t by[5], sh[5], total = 0;
    for (int k = 0; k < narr; ++k) {
      range(c.e0, c.n, sz[k], &lo[k], &by[k], &sh[k]);
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

  // Lift coefficients of this thread's column nodes, kept for the loop.
  constexpr int LR = P::LIFT_REGS ? 6 * KH : 1;
  TC lreg[LR];
  if constexpr (P::LIFT_REGS) {
#pragma unroll
    for (int kk = 0; kk < KH; ++kk)
#pragma unroll
      for (int f = 0; f < 6; ++f)
        lreg[6 * kk + f] = ldro(A.lift + t + NQ2 * (k0 + kk) + NP * f);
  }

  for (int it = 0;; ++it) {
    const int tile = blockIdx.x + it * gridDim.x;
    if (tile >= ntiles) break;
    const int slot = it % NS;
    const uint32_t parity = (it / NS) & 1;
    const Ctx C = tile_ctx<EPB, BATCH>(A, tile);
    const bool active = s < C.n;
    const int e = C.e0 + (active ? s : 0);
    const long base = static_cast<long>(e) * NP;

    // ---- Plus-side face gathers, issued before the ring wait -------------
    TC qP[NFACE], unP[NFACE], qZ[NZF], wZ[NZF];
    if (active) {
      const int* pb = C.pbase + 6 * static_cast<long>(e);
#pragma unroll
      for (int ff = 0; ff < NFACE; ++ff) {
        const int f = h * NFACE + ff;
        const int p = pb[f];
        const long idx = (p >= 0) ? static_cast<long>(p) + opp_offset<NQ>(f, a, b)
                                  : static_cast<long>(-1 - p) + t;
        qP[ff] = static_cast<TC>(ldro(C.q + idx));
        unP[ff] = static_cast<TC>((f == 1 || f == 3) ? ldro(C.u + idx) : ldro(C.v + idx));
      }
#pragma unroll
      for (int zz = 0; zz < NZF; ++zz) {
        const int f = 4 + h * NZF + zz;
        const int p = pb[f];
        const long idx = (p >= 0) ? static_cast<long>(p) + opp_offset<NQ>(f, a, b)
                                  : static_cast<long>(-1 - p) + t;
        qZ[zz] = static_cast<TC>(ldro(C.q + idx));
        wZ[zz] = static_cast<TC>(ldro(C.w + idx));
      }
    }

    // ---- Wait for the tile's slot (bounded, block-uniform) -----------------
    const bool ok = __syncthreads_and(mbar_wait_bounded(&bars[slot], parity));
    if (!ok) {
      if (threadIdx.x == 0) {
        atomicExch(A.status, kStatusWaitTimeout);
        // Drain this block's copies still in flight before leaving: tile it
        // and, before the first refill, the prologue's other tiles.  A tile
        // T >= NS is issued in iteration T - NS + 1.
        for (int k = 0; k < NS; ++k) {
          const int T = it + k;
          const int tk = blockIdx.x + T * gridDim.x;
          if (tk < ntiles && (T < NS || T - NS + 1 <= it - 1))
            mbar_wait_bounded(&bars[T % NS], (T / NS) & 1);
        }
      }
      return;
    }
    // Every thread finished the previous tile (the barrier above), so its
    // slot is free: refill it with the tile NS iterations on from it.
    if (threadIdx.x == 0 && it > 0) {
      const int nt = blockIdx.x + (it - 1 + NS) * gridDim.x;
      if (nt < ntiles) issue(nt, (it - 1) % NS);
    }

    // ---- Phase 1: read this thread's column nodes out of the slot ---------
    unsigned char* sb = slots + slot * P::SLOT;
    size_t lo;
    uint32_t by, shq, shv;
    range(C.e0, C.n, sizeof(TQ), &lo, &by, &shq);
    range(C.e0, C.n, sizeof(TV), &lo, &by, &shv);
    const TQ* sq = reinterpret_cast<const TQ*>(sb + shq) + s * NP;
    const TV* su = reinterpret_cast<const TV*>(sb + P::QB + shv) + s * NP;
    const TV* sv = reinterpret_cast<const TV*>(sb + P::QB + P::VB + shv) + s * NP;
    const TV* sw = reinterpret_cast<const TV*>(sb + P::QB + 2 * P::VB + shv) + s * NP;
    uint32_t sh0 = 0;
    if constexpr (STAGE) range(C.e0, C.n, sizeof(double), &lo, &by, &sh0);
    const double* sq0 =
        reinterpret_cast<const double*>(sb + P::QB + 3 * P::VB + sh0) + s * NP;

    TC fz[KH];
    TC qlo = TC(0), qhi = TC(0);   // q on the -z and +z faces
    TC wM[NZF];
    if (active) {
#pragma unroll
      for (int kk = 0; kk < KH; ++kk) {
        const int k = k0 + kk;
        const int n = t + NQ2 * k;
        const TC qv = static_cast<TC>(sq[n]);
        const TC uv = static_cast<TC>(su[n]);
        const TC vv = static_cast<TC>(sv[n]);
        const TC wv = static_cast<TC>(sw[n]);
        if (kk == 0) qlo = qv;
        if (kk == KH - 1) qhi = qv;
        sX[LI::x(a, b, k)] = AR::mul(qv, uv);
        sY[LI::y(a, b, k)] = AR::mul(qv, vv);
        fz[kk] = AR::mul(qv, wv);
        if constexpr (H == 2) sZ[t + NQ2 * k] = fz[kk];
        if (kk == 0 && k == 0) wM[0] = wv;                 // -z face (k = 1)
        if (kk == KH - 1 && k == NQ - 1) wM[NZF - 1] = wv;  // +z face (k = Nq)
        if (b == 0) fM[0 * NQ2 + a + NQ * k] = V2{qv, vv};
        if (a == NQ - 1) fM[1 * NQ2 + b + NQ * k] = V2{qv, uv};
        if (b == NQ - 1) fM[2 * NQ2 + a + NQ * k] = V2{qv, vv};
        if (a == 0) fM[3 * NQ2 + b + NQ * k] = V2{qv, uv};
      }
    }
    __syncthreads();

    if (active) {
      // ---- Phase 2: face fluxes -------------------------------------------
      const TC* fs = C.fscale + 6 * static_cast<long>(e);
#pragma unroll
      for (int ff = 0; ff < NFACE; ++ff) {
        const int f = h * NFACE + ff;
        const TC sg = (f == 0 || f == 3) ? TC(-1) : TC(1);
        const V2 m = fM[f * NQ2 + t];
        fQ[2 * (f * NQ2 + t)] = upwind_flux<AR, TC>(m.x, m.y, qP[ff], unP[ff], sg, fs[f]);
      }
#pragma unroll
      for (int zz = 0; zz < NZF; ++zz) {
        const int f = 4 + h * NZF + zz;   // 4: -z (k = 1), 5: +z (k = Nq)
        const TC qm = (f == 4) ? qlo : qhi;
        fZ[(f - 4) * NQ2 + t] =
            upwind_flux<AR, TC>(qm, wM[zz], qZ[zz], wZ[zz], f == 4 ? TC(-1) : TC(1), fs[f]);
      }
      // ---- Phase 3: line contractions (x-line for h = 0, y-line for h = 1)
      TC line[NQ];
      if (H == 1 || h == 0) {
#pragma unroll
        for (int l = 0; l < NQ; ++l) line[l] = sX[LI::x(l, a, b)];
#pragma unroll
        for (int i = 0; i < NQ; ++i)
          sX[LI::x(i, a, b)] = contract<NQ, ORDER, AR, TC>(
              [&](int l) { return D.d[i * NQ + l]; }, [&](int l) { return line[l]; });
      }
      if (H == 1 || h == 1) {
#pragma unroll
        for (int l = 0; l < NQ; ++l) line[l] = sY[LI::y(a, l, b)];
#pragma unroll
        for (int j = 0; j < NQ; ++j)
          sY[LI::y(a, j, b)] = contract<NQ, ORDER, AR, TC>(
              [&](int l) { return line[l]; }, [&](int l) { return D.d[j * NQ + l]; });
      }
    }
    __syncthreads();

    if (active) {
      // ---- Phase 4: z-derivative, lift, combine, store ---------------------
      TC zcol[NQ];
      if constexpr (H == 2) {
#pragma unroll
        for (int l = 0; l < NQ; ++l) zcol[l] = sZ[t + NQ2 * l];
      } else {
#pragma unroll
        for (int l = 0; l < NQ; ++l) zcol[l] = fz[l];
      }
      const TC f5 = fZ[t], f6 = fZ[NQ2 + t];
      if (H == 1 || h == 0)
        column_epilogue<NQ, 0, KH, ORDER, STAGE, P::LIFT_REGS, EXACT>(
            A, D, C, e, base, t, a, b, zcol, sX, sY, fQ, f5, f6, sq, sq0, lreg);
      else
        column_epilogue<NQ, (H == 2 ? KH : 0), KH, ORDER, STAGE, P::LIFT_REGS, EXACT>(
            A, D, C, e, base, t, a, b, zcol, sX, sY, fQ, f5, f6, sq, sq0, lreg);
    }
  }
}

}  // namespace sdg
