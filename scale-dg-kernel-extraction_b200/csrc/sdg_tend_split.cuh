// Split-column variant of the persistent fused kernel, for the high orders
// (one element per tile, Nq >= 9).
//
// In tend_pipe_kernel one element is handled by Nq^2 threads, each owning a
// whole z-column of Nq nodes.  From Nq = 9 on a tile is one element, and the
// element's shared-memory ring allows one to three blocks per SM, so an SM
// holds only 5-7 warps: too few to cover the latency of the column loads,
// line contractions and face gathers.  Here each column is split over H
// threads, H = 2 (thread T = c + Nq^2 h owns nodes k in [h*KZ, (h+1)*KZ) of
// column c, KZ = ceil(Nq/H)), so a tile has H*Nq^2 threads, each with half
// the column's registers, and the other phases are shared out by h:
//
//   phase 1   every thread: its nodes' volume fluxes, q*w in place of w,
//             minus-side face values;
//   lines     h = 0 contracts x-line c, h = 1 y-line c;
//   faces     h = 0: the two y faces at face node c and the -z face of
//             column c (it owns node k = 0); h = 1: the two x faces and
//             the +z face (it owns node k = Nq-1);
//   epilogue  every thread: z-derivative (from the whole q*w column in
//             shared memory), lift, combine and RK stage of its nodes.
//
// Every node goes through exactly the operations, operands and order of
// tend_pipe_kernel and tend_kernel, so all variants compute identical bits.
// The ring (cp.async.bulk of q, u, v, w, escale and fscale into NSTAGE
// slots, bounded mbarrier waits, status word on a timeout) is the one of
// tend_pipe_kernel with one element per tile.
#pragma once

#include "sdg_tend_pipe.cuh"

namespace sdg {

// Orders whose column parts each take a whole number of warps (Nq^2 threads
// rounded up to a multiple of 32, the rest idle), so that no warp holds
// threads of both parts and every phase is one pass per warp (the warp that
// straddles the parts otherwise contracts both an x and a y line and
// evaluates both kinds of face).  Measured (RK stage 2, ~16.8 M DOF, ms
// padded / not): FP64 p = 8 0.223 / 0.253, p = 11 0.251 / 0.291, p = 12
// 0.246 / 0.273; mixed p = 8 0.129 / 0.149, p = 11 0.132 / 0.142.  Slower
// at FP64 p = 9 (0.274 / 0.223: a whole warp more for four columns) and
// p = 13 (0.267 / 0.252: 132 bytes of spill at 448 threads).
template <int NQ>
constexpr bool kSplitPadParts = NQ == 9 || NQ == 11 || NQ == 12 || NQ == 13 || NQ == 15;

template <int NQ, int H>
struct SplitGeo {
  static constexpr int NQ2 = NQ * NQ;
  static constexpr int NP = NQ2 * NQ;
  static constexpr bool PAD = kSplitPadParts<NQ>;
  static constexpr int PT = PAD ? (NQ2 + 31) / 32 * 32 : NQ2;  // threads per part
  static constexpr int THREADS = H * PT;
  static constexpr int KZ = (NQ + H - 1) / H;  // column nodes per thread
};

// Registers a thread keeps at least, which caps the resident blocks: 128 for
// FP64 and 80 for FP32.  (FP64 at Nq = 10 with 80: three blocks of 224
// threads per SM, 8 bytes of spill, measured 0.252 against 0.234 ms per RK
// stage 2 with two blocks.)
template <int NQ, typename TC>
constexpr int kSplitRegFloor = sizeof(TC) == 8 ? 128 : 80;

// Where the RK base state q0 may travel in the ring slot (a bulk copy with
// the tile's other inputs, read from shared memory by the epilogue) rather
// than be loaded into registers from L2: it frees KZ registers for the
// whole tile.  Measured (RK stage 2, ~16.8 M DOF, ms in the slot / from L2):
// FP64 p = 8 0.255 / 0.264, p = 11 0.290 / 0.296, p = 12 0.274 / 0.294;
// mixed p = 9 0.143 / 0.151; slower at FP64 p = 9 (0.230 / 0.226).  The plan
// takes it where it costs no resident block and no separate line buffers.
template <int NQ, typename TC>
constexpr bool kSplitRingQ0 = !(sizeof(TC) == 8 && NQ == 10);

// Shared-memory plan: the ring of one-element slots (q, u, v, w and the
// element's escale, fscale and face-neighbour rows), the x- and y-line
// buffers, the minus-side face values (FaceArea), the face fluxes ((f1, f3)
// and (f2, f4) pairs per face node, f5 and f6 per column), the factored
// lift's x/y factors, barriers; q0 in the slot where RING_Q0.  The line
// buffers have space of their own (SEP) where the plan fits, so phase 1
// writes them directly; otherwise they reuse the slot's u and v regions once
// every thread holds its column, which costs a barrier.  Where it gains a
// resident block the face fluxes overwrite the minus-side values they were
// computed from (FLUX_ALIAS): each thread writes only the face-area words it
// alone has read.
template <int NQ, int H, typename TQ, typename TV, typename TC, bool STAGE>
struct SplitPlan {
  static constexpr int NQ2 = NQ * NQ;
  static constexpr int NP = NQ2 * NQ;
  static constexpr int NSTAGE = 2;
  static constexpr size_t r16(size_t x) { return (x + 15) & ~size_t(15); }
  static constexpr size_t mx(size_t a, size_t b) { return a > b ? a : b; }
  static constexpr size_t LINE =
      r16(sizeof(TC) * LineIdx<NQ, static_cast<int>(sizeof(TC))>::SIZE);
  static constexpr size_t QB = r16(sizeof(TQ) * NP + 32);
  static constexpr size_t VB0 = r16(sizeof(TV) * NP + 32);
  static constexpr size_t EB = r16(sizeof(TC) * 3 + 32);
  static constexpr size_t FB = r16(sizeof(TC) * 6 + 32);
  static constexpr size_t PB = r16(sizeof(int) * 6 + 32);
  static constexpr size_t CB = 128;  // a batched tile's TileCtx
  static constexpr size_t FACE = r16(sizeof(TC) * FaceArea<NQ, sizeof(TC) == 8>::ELEM);
  static constexpr size_t FLUX = r16(sizeof(TC) * 6 * NQ2);
  static constexpr size_t LIFTB = r16(sizeof(TC) * 4 * NQ);
  static constexpr size_t BARS = 16 * NSTAGE;
  // The RK base state q0 of the tile (stages 2-3), when it travels in the
  // slot.
  static constexpr size_t Q0B = STAGE ? r16(sizeof(double) * NP + 32) : 0;
  // Bytes of the plan with separate line buffers (sep), with the face
  // fluxes in the face area (fal) and with q0 in the slot (rq).  Without sep
  // the u and v regions hold the line buffers; w holds q*w either way.
  static constexpr size_t bytes_of(bool sep, bool fal, bool rq) {
    return NSTAGE * (QB + 2 * (sep ? VB0 : mx(VB0, LINE)) + VB0 + EB + FB + PB + CB +
                     (rq ? Q0B : 0)) +
           (sep ? 2 * LINE : 0) + FACE + (fal ? 0 : FLUX) + LIFTB + BARS;
  }
  static constexpr size_t SEP_BYTES = bytes_of(true, false, false);
  static constexpr size_t ALIAS_BYTES = bytes_of(false, false, false);
  static constexpr int blocks(size_t bytes) {
    return bytes > kPipeMaxSmem
               ? 0
               : static_cast<int>(kSmemPerSM / (bytes + kSmemPerBlockReserved));
  }
  // Resident blocks the registers allow (kSplitRegFloor registers a thread).
  static constexpr int REG_BLOCKS =
      65536 / (((SplitGeo<NQ, H>::THREADS + 31) / 32 * 32) * kSplitRegFloor<NQ, TC>);
  static constexpr int cap(int b) { return b < REG_BLOCKS ? b : REG_BLOCKS; }
  // The most resident blocks any layout reaches, and the first layout that
  // reaches it in the order of preference: separate line buffers, then q0
  // in the slot, then separate fluxes.  Layout index L: bit 2 sep, bit 1 rq,
  // bit 0 !fal.
  static constexpr int blocks_of(int L) {
    return cap(blocks(bytes_of((L & 4) != 0, (L & 1) == 0, (L & 2) != 0)));
  }
  static constexpr int best_blocks() {
    int b = 0;
    for (int L = 0; L < 8; ++L) b = blocks_of(L) > b ? blocks_of(L) : b;
    return b;
  }
  static constexpr int BEST = best_blocks();
  static constexpr int pick() {
    for (int L = 7; L >= 0; --L) {
      if (!kSplitRingQ0<NQ, TC> && (L & 2)) continue;
      if (blocks_of(L) == BEST) return L;
    }
    return 0;
  }
  static constexpr int LAYOUT = pick();
  static constexpr bool SEP = (LAYOUT & 4) != 0;
  static constexpr bool RING_Q0 = STAGE && (LAYOUT & 2) != 0;
  static constexpr bool FLUX_ALIAS = (LAYOUT & 1) == 0;
  static constexpr size_t VB = SEP ? VB0 : mx(VB0, LINE);
  static constexpr size_t OFF_U = QB;
  static constexpr size_t OFF_V = QB + VB;
  static constexpr size_t OFF_W = QB + 2 * VB;
  static constexpr size_t OFF_E = OFF_W + VB0;
  static constexpr size_t OFF_F = OFF_E + EB;
  static constexpr size_t OFF_P = OFF_F + FB;
  static constexpr size_t OFF_C = OFF_P + PB;
  static constexpr size_t OFF_Q0 = OFF_C + CB;
  static constexpr size_t SLOT = OFF_Q0 + (RING_Q0 ? Q0B : 0);
  static constexpr size_t LINES = SEP ? 2 * LINE : 0;
  static constexpr size_t REST = FACE + (FLUX_ALIAS ? 0 : FLUX) + LIFTB + BARS;
  static constexpr size_t BYTES = NSTAGE * SLOT + LINES + REST;
  static_assert(BYTES == bytes_of(SEP, FLUX_ALIAS, RING_Q0), "slot layout");
  static constexpr int BLOCKS_PER_SM_SMEM = static_cast<int>(
      kSmemPerSM / (BYTES + kSmemPerBlockReserved) > 4
          ? 4
          : (kSmemPerSM / (BYTES + kSmemPerBlockReserved) < 1
                 ? 1
                 : kSmemPerSM / (BYTES + kSmemPerBlockReserved)));
};

// A part of the column, as a type (the per-node phases are compiled once per
// part; -1: the part known at run time only).
template <int HH>
struct Part {
  static constexpr int value = HH;
};

// Orders whose per-node phases are compiled once per part, with node k a
// compile-time constant, for the warps whose threads all hold the same part
// (the one warp that straddles the two parts runs the run-time copy, so it
// does not do both).  At Nq = 12 and 16 the copies make the register
// allocator spill (0.8-4 KB a thread), so those keep the run-time copy.
template <int NQ>
constexpr bool kSplitPartCopies = NQ != 12 && NQ != 16;

// Columns split in two from Nq = 9 on.
template <int NQ>
constexpr int kSplitH = 2;

// Where the automatic variant takes the split-column kernel: the orders at
// which it measured faster than tend_pipe_kernel (RK stage 2, ~16.8 M DOF,
// ms split / pipelined): fast FP64 p = 8 0.223 / 0.261, p = 9 0.223 / 0.253,
// p = 11 0.251 / 0.325, p = 12 0.246 / 0.316, p = 13 0.252 / 0.295; mixed
// p = 8 0.129 / 0.146, p = 9 0.144 / 0.158, p = 11 0.132 / 0.146.  Slower at
// FP64 p = 10 and 14 (0.232 / 0.230, 0.332 / 0.313) and the other mixed
// orders.
template <int NQ, typename TC, bool EXACT>
constexpr bool kSplitAuto =
    !EXACT && (sizeof(TC) == 8 ? (NQ == 9 || NQ == 10 || (NQ >= 12 && NQ <= 14))
                               : (NQ == 9 || NQ == 10 || NQ == 12));

// Blocks per SM the kernel is built for: what the shared memory allows,
// capped so that a thread keeps at least kSplitRegFloor registers.
template <int NQ, int H, typename TQ, typename TV, typename TC, bool STAGE>
constexpr int split_min_blocks() {
  constexpr int m = SplitPlan<NQ, H, TQ, TV, TC, STAGE>::BLOCKS_PER_SM_SMEM;
  constexpr int thr = (SplitGeo<NQ, H>::THREADS + 31) / 32 * 32;
  constexpr int floor_regs = kSplitRegFloor<NQ, TC>;
  constexpr int by_regs = 65536 / (thr * floor_regs);
  constexpr int r = m < by_regs ? m : by_regs;
  return r < 1 ? 1 : r;
}

template <int NQ, int H, typename TQ, typename TV, typename TO, typename TC, bool EXACT,
          int ORDER, bool STAGE, bool BATCH>
__global__ void __launch_bounds__((SplitGeo<NQ, H>::THREADS + 31) / 32 * 32,
                                  (split_min_blocks<NQ, H, TQ, TV, TC, STAGE>()))
    tend_split_kernel(const __grid_constant__ TendArgs<TQ, TV, TO, TC> A,
                      const __grid_constant__ DMat<NQ, TC> D) {
  using G = SplitGeo<NQ, H>;
  using P = SplitPlan<NQ, H, TQ, TV, TC, STAGE>;
  using AR = Ar<TC, EXACT>;
  using Ctx = TileCtx<TQ, TV, TO, TC>;
  using V2 = typename Pair2<TC>::type;
  using LI = LineIdx<NQ, static_cast<int>(sizeof(TC))>;
  constexpr int NQ2 = G::NQ2;
  constexpr int NP = G::NP;
  constexpr int KZ = G::KZ;
  constexpr int NS = P::NSTAGE;
  static_assert(H == 2, "columns split in two parts");

  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* slots = smem_raw;
  unsigned char* rest = smem_raw + NS * P::SLOT + P::LINES;
  TC* fa = reinterpret_cast<TC*>(rest);
  constexpr size_t FLUXB = P::FLUX_ALIAS ? 0 : P::FLUX;
  TC* flux = reinterpret_cast<TC*>(rest + P::FACE);
  TC* sL = reinterpret_cast<TC*>(rest + P::FACE + FLUXB);
  uint64_t* bars = reinterpret_cast<uint64_t*>(rest + P::FACE + FLUXB + P::LIFTB);
  constexpr bool SEP = P::SEP;

  constexpr int PT = G::PT;
  const int h = threadIdx.x / PT;       // part of the column
  const int c = threadIdx.x - h * PT;   // column a + NQ*b
  const bool valid = !G::PAD || c < NQ2;  // padded parts: idle beyond Nq^2
  const int a = c % NQ;
  const int b = c / NQ;
  const int k0 = h * KZ;                // first node of this thread's part
  const int ntiles = BATCH ? A.ntiles : A.nelem;
  const bool own_y = h == 0 && valid;      // y faces and the -z face
  const bool own_x = h == H - 1 && valid;  // x faces and the +z face
  const unsigned spins = A.wait_spins;
  // The part of this warp's threads, or -1 when the warp holds both.
  auto part_of_warp = [&]() {
    const int t0 = threadIdx.x & ~31;
    const int t1 = min(t0 + 31, static_cast<int>(blockDim.x) - 1);
    return (t0 / PT == t1 / PT) ? t0 / PT : -1;
  };

  // Minus-side face values (FaceArea): FP64 keeps the x faces in two scalar
  // arrays and the y faces as (q, v) pairs; FP32 keeps (q, un) pairs of the
  // four faces, face-major.
  constexpr bool XSPLIT = sizeof(TC) == 8;
  using FA = FaceArea<NQ, XSPLIT>;
  TC* xq = fa;
  TC* xu = fa + FA::XA;
  V2* ypair = reinterpret_cast<V2*>(fa + FA::Y0);
  V2* fM = reinterpret_cast<V2*>(fa);
  // Face fluxes: (f1, f3) and (f2, f4) at face node n, f5 and f6 at column n.
  // With FLUX_ALIAS, in the face area: (f1, f3) over the -y pair of face
  // node n, f5 over the +y pair's first word; FP64: f2, f4 and f6 over the
  // x arrays' words xq[n], xq[XOFF + n] and xu[n]; FP32: (f2, f4) over the
  // +x pair, f6 over the -x pair's first word.
  constexpr bool FAL = P::FLUX_ALIAS;
  V2* fl13 = FAL ? (XSPLIT ? ypair : fM) : reinterpret_cast<V2*>(flux);
  V2* fl24 = FAL ? fM + NQ2 : reinterpret_cast<V2*>(flux) + NQ2;
  TC* fl5 = FAL ? reinterpret_cast<TC*>(XSPLIT ? ypair + NQ2 : fM + 2 * NQ2) : flux + 4 * NQ2;
  TC* fl6 = FAL ? (XSPLIT ? xu : reinterpret_cast<TC*>(fM + FA::F3)) : flux + 5 * NQ2;
  // Word stride of f5 and f6 between columns (pairs in the aliased form).
  constexpr int S5 = FAL ? 2 : 1;
  constexpr int S6 = (FAL && !XSPLIT) ? 2 : 1;

  // Producer: one thread fills ring slot `slot` with tile (element) `tile`.
  auto issue = [&](int tile, int slot) {
    // Test hook (host-set): leave this tile's slot empty.
    if (tile + 1 == A.inject_skip) return;
    const Ctx cx = tile_ctx<1, BATCH>(A, tile, ntiles);
    unsigned char* base = slots + slot * P::SLOT;
    // A batched tile's context goes with it (read by the consumers from
    // shared memory instead of the tile and instance tables).
    if constexpr (BATCH) *reinterpret_cast<Ctx*>(base + P::OFF_C) = cx;
    const void* src[7] = {cx.q, cx.u, cx.v, cx.w, cx.escale, cx.fscale, cx.pbase};
    const size_t per[7] = {sizeof(TQ) * NP, sizeof(TV) * NP, sizeof(TV) * NP,
                           sizeof(TV) * NP, sizeof(TC) * 3,  sizeof(TC) * 6,
                           sizeof(int) * 6};
    const size_t off[7] = {0, P::OFF_U, P::OFF_V, P::OFF_W, P::OFF_E, P::OFF_F, P::OFF_P};
    size_t lo[7];
    uint32_t by[7], sh[7], total = 0;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      tile_range(cx.e0, cx.n, per[k], &lo[k], &by[k], &sh[k]);
      total += by[k];
    }
    // q0 (RK stages 2-3): into the slot where the plan holds it, else
    // into L2 for the epilogue's loads.
    size_t l0 = 0;
    uint32_t b0 = 0, s0 = 0;
    const bool q0_used = STAGE && A.rk_a != 0.0;
    if (q0_used) {
      tile_range(cx.e0, cx.n, sizeof(double) * NP, &l0, &b0, &s0);
      if constexpr (P::RING_Q0) total += b0;
    }
    mbar_arrive_expect_tx(&bars[slot], total);
#pragma unroll
    for (int k = 0; k < 7; ++k)
      bulk_g2s(base + off[k], static_cast<const unsigned char*>(src[k]) + lo[k], by[k],
               &bars[slot]);
    if (q0_used) {
      const unsigned char* q0src = reinterpret_cast<const unsigned char*>(cx.q0) + l0;
      if constexpr (P::RING_Q0)
        bulk_g2s(base + P::OFF_Q0, q0src, b0, &bars[slot]);
      else
        bulk_prefetch_l2(q0src, b0);
    }
  };

  if (threadIdx.x == 0) {
    for (int k = 0; k < NS; ++k) mbar_init(&bars[k], 1);
    fence_barrier_init();
  }
  if constexpr (!EXACT) {
    for (int x = threadIdx.x; x < 4 * NQ; x += blockDim.x) {
      const int f = x / NQ, n = x - f * NQ;
      sL[x] = ldro(A.lift + NP * f + ((f & 1) ? n : NQ * n));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < NS; ++k) {
      const int tile = blockIdx.x + k * gridDim.x;
      if (tile < ntiles) issue(tile, k);
    }

  for (int it = 0;; ++it) {
    const int tile = blockIdx.x + it * gridDim.x;
    if (tile >= ntiles) break;
    const int slot = it % NS;
    const uint32_t parity = (it / NS) & 1;
    Ctx C;
    if constexpr (!BATCH) C = tile_ctx<1, false>(A, tile, ntiles);

    // ---- Wait for the tile's slot (bounded, block-uniform) ---------------
    const bool ok = __syncthreads_and(mbar_wait_bounded(&bars[slot], parity, spins));
    if (!ok) {
      if (threadIdx.x == 0) {
        atomicExch(A.status, kStatusWaitTimeout);
        for (int k = 0; k < NS; ++k) {
          const int T = it + k;
          const int tk = blockIdx.x + T * gridDim.x;
          if (tk < ntiles && (T < NS || T - NS + 1 <= it - 1))
            mbar_wait_bounded(&bars[T % NS], (T / NS) & 1, spins);
        }
      }
      return;
    }
    unsigned char* sb = slots + slot * P::SLOT;
    if constexpr (BATCH) C = *reinterpret_cast<const Ctx*>(sb + P::OFF_C);
    const int e = C.e0;
    const long base = static_cast<long>(e) * NP;
    if (threadIdx.x == 0 && it > 0) {
      const int nt = blockIdx.x + (it - 1 + NS) * gridDim.x;
      if (nt < ntiles) issue(nt, (it - 1) % NS);
    }

    const TQ* sq = reinterpret_cast<const TQ*>(sb + tile_shift(C.e0, sizeof(TQ) * NP));
    const uint32_t shv = tile_shift(C.e0, sizeof(TV) * NP);
    const TV* su = reinterpret_cast<const TV*>(sb + P::OFF_U + shv);
    const TV* sv = reinterpret_cast<const TV*>(sb + P::OFF_V + shv);
    const TV* sw = reinterpret_cast<const TV*>(sb + P::OFF_W + shv);
    const TC* ses = reinterpret_cast<const TC*>(sb + P::OFF_E + tile_shift(C.e0, sizeof(TC) * 3));
    const TC* sfs = reinterpret_cast<const TC*>(sb + P::OFF_F + tile_shift(C.e0, sizeof(TC) * 6));
    const int* spb = reinterpret_cast<const int*>(sb + P::OFF_P + tile_shift(C.e0, 24));
    const double* sq0 = reinterpret_cast<const double*>(
        sb + P::OFF_Q0 + tile_shift(C.e0, sizeof(double) * NP));
    static_assert(sizeof(TV) == sizeof(TC), "w and q*w share their slots");
    TC* sz = reinterpret_cast<TC*>(sb + P::OFF_W + shv);
    TC* sX = SEP ? reinterpret_cast<TC*>(smem_raw + NS * P::SLOT)
                 : reinterpret_cast<TC*>(sb + P::OFF_U);
    TC* sY = SEP ? reinterpret_cast<TC*>(smem_raw + NS * P::SLOT + P::LINE)
                 : reinterpret_cast<TC*>(sb + P::OFF_V);

    // ---- Plus-side face values (L2) and q0, issued first ------------------
    // The face-neighbour row came with the tile.  Slots 0, 1: the two x or y
    // faces of this thread; 2: its z face.
    TC qP[3], unP[3];
    {
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const bool mine = (f == 0 || f == 2 || f == 4) ? own_y : own_x;
        if (!mine) continue;
        const int pb = spb[f];
        // slot of face f among this thread's faces
        const int sl = (f >= 4) ? 2 : ((f == 0 || f == 1) ? 0 : 1);
        const long idx = (pb >= 0) ? static_cast<long>(pb) + opp_offset<NQ>(f, a, b)
                                   : static_cast<long>(-1 - pb) + c;
        qP[sl] = static_cast<TC>(ldro(C.q + idx));
        unP[sl] = static_cast<TC>((f == 1 || f == 3) ? ldro(C.u + idx)
                                                     : ((f >= 4) ? ldro(C.w + idx)
                                                                 : ldro(C.v + idx)));
      }
    }
    // q0 (RK stages 2-3, in L2 since the tile's copies were issued): loaded
    // here where the separate line buffers leave registers to spare, after
    // the lines otherwise (measured: FP64 p = 10, aliased plan, 0.33 against
    // 0.25 ms with the early loads).
    double q0r[STAGE ? KZ : 1];
    const bool use_q0 = STAGE && A.rk_a != 0.0;
    auto load_q0 = [&]() {
      if constexpr (STAGE && !P::RING_Q0) {
        if (use_q0 && valid) {
#pragma unroll
          for (int kk = 0; kk < KZ; ++kk) {
            const int k = k0 + kk;
            if (KZ * H != NQ && k >= NQ) break;
            q0r[kk] = ld_stream(C.q0 + base + c + NQ2 * k);
          }
        }
      }
    };
    if constexpr (SEP) load_q0();

    // ---- Phase 1: this thread's nodes of column c -------------------------
    // The per-node phases run in a copy per part h (kSplitPartCopies), so
    // that node k is a compile-time constant: the coefficients D(k, l) and
    // the z-lift factors are then immediate constant-bank operands, not
    // indexed constant loads.
    constexpr bool PC = kSplitPartCopies<NQ>;
    const int hw = PC ? part_of_warp() : -1;  // the warp's part, -1: mixed
    TC fx[KZ], fy[KZ];
    TC wlo = TC(0), whi = TC(0), qlo = TC(0), qhi = TC(0);
    auto phase1 = [&](auto part) __attribute__((always_inline)) {
      const int K0 = decltype(part)::value >= 0 ? decltype(part)::value * KZ : k0;
      const bool onx = (a == 0) || (a == NQ - 1);
      const bool ony = (b == 0) || (b == NQ - 1);
      [[maybe_unused]] const int xo = (a == 0 ? FA::XOFF : 0) + b;
      [[maybe_unused]] V2* fmx = fM + (a == 0 ? FA::F3 : NQ2) + b;
      V2* fmy = XSPLIT ? ypair + (b == 0 ? 0 : NQ2) + a : fM + (b == 0 ? 0 : 2) * NQ2 + a;
#pragma unroll
      for (int kk = 0; kk < KZ; ++kk) {
        const int k = K0 + kk;
        if (KZ * H != NQ && k >= NQ) break;
        const int n = c + NQ2 * k;
        const TC qv = static_cast<TC>(sq[n]);
        const TC uv = static_cast<TC>(su[n]);
        const TC vv = static_cast<TC>(sv[n]);
        const TC wv = static_cast<TC>(sw[n]);
        if (k == 0) {
          wlo = wv;
          qlo = qv;
        }
        if (k == NQ - 1) {
          whi = wv;
          qhi = qv;
        }
        fx[kk] = AR::mul(qv, uv);
        fy[kk] = AR::mul(qv, vv);
        sz[n] = AR::mul(qv, wv);
        if constexpr (SEP) {
          sX[LI::colx(a, b, k)] = fx[kk];
          sY[LI::coly(a, b, k)] = fy[kk];
        }
        if constexpr (XSPLIT) {
          if (onx) {
            xq[xo + NQ * k] = qv;
            xu[xo + NQ * k] = uv;
          }
        } else {
          if (onx) fmx[NQ * k] = V2{qv, uv};
        }
        if (ony) fmy[NQ * k] = V2{qv, vv};
      }
    };
    if (!valid) {
    } else if (hw < 0) {
      phase1(Part<-1>{});
    } else if (hw == 0) {
      phase1(Part<0>{});
    } else {
      phase1(Part<1>{});
    }
    // The slot's writes (q*w; line buffers in u, v without SEP) come before
    // the refill that overwrites it.
    fence_proxy_async_smem();
    __syncthreads();
    if constexpr (!SEP) {
      // The slot's u, v are dead: reuse them as line buffers.
#pragma unroll
      for (int kk = 0; kk < KZ; ++kk) {
        const int k = k0 + kk;
        if ((KZ * H != NQ && k >= NQ) || !valid) break;
        sX[LI::colx(a, b, k)] = fx[kk];
        sY[LI::coly(a, b, k)] = fy[kk];
      }
      __syncthreads();
    }

    // ---- Lines: x-line c (h = 0) and y-line c (h = 1), in place ----------
    {
      const int lbx = LI::xl_base(a, b), lby = LI::yl_base(a, b);
      if (h == 0 && valid) {
        TC line[NQ];
#pragma unroll
        for (int l = 0; l < NQ; ++l) line[l] = sX[LI::xl(lbx, l)];
#pragma unroll
        for (int i = 0; i < NQ; ++i)
          sX[LI::xl(lbx, i)] = contract<NQ, ORDER, AR, TC>(
              [&](int l) { return D.d[i * NQ + l]; }, [&](int l) { return line[l]; });
      }
      if (h == H - 1 && valid) {
        TC line[NQ];
#pragma unroll
        for (int l = 0; l < NQ; ++l) line[l] = sY[LI::yl(lby, l)];
#pragma unroll
        for (int j = 0; j < NQ; ++j)
          sY[LI::yl(lby, j)] = contract<NQ, ORDER, AR, TC>(
              [&](int l) { return line[l]; }, [&](int l) { return D.d[j * NQ + l]; });
      }
    }
    // Without SEP the line buffers live in the slot that the next refill
    // overwrites.
    if constexpr (!SEP) {
      fence_proxy_async_smem();
      load_q0();
    }
    // ---- Face fluxes ------------------------------------------------------
    if (own_y) {
      // y faces at face node c: -y (1) and +y (3); -z (5) of column c.
      V2 m1, m3;
      if constexpr (XSPLIT) {
        m1 = ypair[c];
        m3 = ypair[NQ2 + c];
      } else {
        m1 = fM[c];
        m3 = fM[2 * NQ2 + c];
      }
      const TC f1 = upwind_flux<AR, TC>(m1.x, m1.y, qP[0], unP[0], TC(-1), sfs[0]);
      const TC f3 = upwind_flux<AR, TC>(m3.x, m3.y, qP[1], unP[1], TC(1), sfs[2]);
      fl13[c] = V2{f1, f3};
      fl5[S5 * c] = upwind_flux<AR, TC>(qlo, wlo, qP[2], unP[2], TC(-1), sfs[4]);
    }
    if (own_x) {
      // x faces at face node c: +x (2) and -x (4); +z (6) of column c.
      TC q2, u2, q4, u4;
      if constexpr (XSPLIT) {
        const int xn = NQ * b + a;
        q2 = xq[xn];
        u2 = xu[xn];
        q4 = xq[FA::XOFF + xn];
        u4 = xu[FA::XOFF + xn];
      } else {
        const V2 m2 = fM[NQ2 + c], m4 = fM[FA::F3 + c];
        q2 = m2.x;
        u2 = m2.y;
        q4 = m4.x;
        u4 = m4.y;
      }
      const TC f2 = upwind_flux<AR, TC>(q2, u2, qP[0], unP[0], TC(1), sfs[1]);
      const TC f4 = upwind_flux<AR, TC>(q4, u4, qP[1], unP[1], TC(-1), sfs[3]);
      if constexpr (FAL && XSPLIT) {
        xq[c] = f2;
        xq[FA::XOFF + c] = f4;
      } else {
        fl24[c] = V2{f2, f4};
      }
      fl6[S6 * c] = upwind_flux<AR, TC>(qhi, whi, qP[2], unP[2], TC(1), sfs[5]);
    }
    __syncthreads();

    // ---- Epilogue: z-derivative, lift, combine, store ---------------------
    auto epilogue = [&](auto part) __attribute__((always_inline)) {
      const int K0 = decltype(part)::value >= 0 ? decltype(part)::value * KZ : k0;
      const TC e1 = ses[0], e2 = ses[1], e3 = ses[2];
      [[maybe_unused]] TC lxy[4];
      if constexpr (!EXACT) {
        lxy[0] = sL[b];
        lxy[1] = sL[NQ + a];
        lxy[2] = sL[2 * NQ + b];
        lxy[3] = sL[3 * NQ + a];
      }
      const TC f5 = fl5[S5 * c], f6 = fl6[S6 * c];
      TC fz[NQ];
#pragma unroll
      for (int l = 0; l < NQ; ++l) fz[l] = sz[c + NQ2 * l];
#pragma unroll
      for (int kk = 0; kk < KZ; ++kk) {
        const int k = K0 + kk;
        if (KZ * H != NQ && k >= NQ) break;
        const TC dz = contract<NQ, ORDER, AR, TC>([&](int l) { return fz[l]; },
                                                  [&](int l) { return D.d[k * NQ + l]; });
        TC L[6];
        if constexpr (!EXACT) {
#pragma unroll
          for (int f = 0; f < 4; ++f) L[f] = lxy[f];
          L[4] = D.lz[k];
          L[5] = D.lz[NQ + k];
        } else {
#pragma unroll
          for (int f = 0; f < 6; ++f) L[f] = ldro(A.lift + c + NQ2 * k + NP * f);
        }
        // tensorprod_Lift_hexahedral (kern:278-283), face order 1..6.
        const V2 f13 = fl13[a + NQ * k];
        V2 f24;
        if constexpr (FAL && XSPLIT) {
          f24.x = xq[b + NQ * k];
          f24.y = xq[FA::XOFF + b + NQ * k];
        } else {
          f24 = fl24[b + NQ * k];
        }
        TC lf = AR::mul(L[0], f13.x);
        lf = AR::mad(L[1], f24.x, lf);
        lf = AR::mad(L[2], f13.y, lf);
        lf = AR::mad(L[3], f24.y, lf);
        lf = AR::mad(L[4], f5, lf);
        lf = AR::mad(L[5], f6, lf);
        // dqdt = -(Escale1*DxF + Escale2*DyF + Escale3*DzF + Lift), eq:194-198.
        TC acc = AR::mul(e1, sX[LI::colx(a, b, k)]);
        acc = AR::mad(e2, sY[LI::coly(a, b, k)], acc);
        acc = AR::mad(e3, dz, acc);
        acc = AR::add(acc, lf);
        const TC dqdt = -acc;
        const long n = base + c + NQ2 * k;
        if constexpr (!STAGE) {
          C.out[n] = static_cast<TO>(dqdt);
        } else {
          // q = rk_a*q0 + rk_b*(q + dt*dqdt), main.f90:70-71, in FP64.
          using AD = Ar<double, EXACT>;
          const double qd = static_cast<double>(sq[c + NQ2 * k]);
          double r = AD::mul(A.rk_b, AD::mad(C.dt, static_cast<double>(dqdt), qd));
          if (use_q0) {
            if constexpr (P::RING_Q0)
              r = AD::mad(A.rk_a, sq0[c + NQ2 * k], r);
            else
              r = AD::mad(A.rk_a, q0r[kk], r);
          }
          C.out[n] = static_cast<TO>(r);
        }
      }
    };
    if (!valid) {
    } else if (hw < 0) {
      epilogue(Part<-1>{});
    } else if (hw == 0) {
      epilogue(Part<0>{});
    } else {
      epilogue(Part<1>{});
    }
  }
}

}  // namespace sdg
