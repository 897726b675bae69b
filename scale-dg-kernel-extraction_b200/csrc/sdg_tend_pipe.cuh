// Persistent, software-pipelined variant of the fused tendency / RK-stage
// kernel (same arithmetic as tend_kernel in sdg_tend.cuh, same results).
//
// Each block loops over tiles of EPB consecutive elements.  The element data
// a tile needs (q, u, v, w and the tile's rows of escale and fscale) are
// contiguous in HBM, so one elected thread moves them into a shared-memory
// ring of NSTAGE tiles with cp.async.bulk (the TMA bulk-copy engine),
// completing on an mbarrier per ring slot.  A slot stays resident for its
// whole tile and is refilled, with the tile NSTAGE iterations on, as the
// block starts the next tile.  Compute threads never stall on their own
// element loads: the bytes in flight per SM are set by the ring, not by
// occupancy.
//
// Loads that are not contiguous per tile are issued early, as ordinary
// loads whose latency later work covers: the plus-side face values in
// neighbouring elements (from a face-neighbour row loaded before the ring
// wait) are issued before the line contractions, and the face fluxes come
// after them; for RK stages 2-3, the column's q0 values, which a bulk
// prefetch issued with the tile's ring copies has brought into L2, are
// loaded before the face fluxes and used in the epilogue.
//
// Shared memory per block: the ring, plus one area for the minus side of the
// four x/y faces and their fluxes (FaceArea).  The x- and y-line buffers of the
// derivative reuse the current slot's u and v regions: those are dead once
// every thread holds its column, so a barrier separates the column reads
// from the line-buffer writes.  At p = 7 this keeps an FP64 block at 73 KB,
// three blocks (12 warps) per SM.
//
// Thread mapping, as in tend_kernel: thread t = a + Nq*b of an element owns
// the z-column (a,b) in registers (z-derivative, z faces, combine), the
// x-line (j,k) = (a,b) and y-line (i,k) = (a,b), and node t of each x/y face.
//
// Lift.  The fast kernels use the tensor-product factorisation of Lift_mat
// (the host checks it against the table): the x/y-face factors from a small
// shared table and the z-face factors from the parameter bank.  The exact
// kernels read the verbatim table through the read-only path.
//
// Every wait is bounded.  A wait that runs out sets *status and the block
// drains its own copies (again bounded) and returns; the host reports the
// status as an error.  Decisions after a wait are made block-uniform with
// __syncthreads_and so that no thread can skip a barrier another reaches.
#pragma once

#include "sdg_tcgen05.cuh"
#include "sdg_tend.cuh"

namespace sdg {

constexpr int kStatusWaitTimeout = 1;
// Default spin limit of a bounded wait (polls of mbarrier.try_wait).
constexpr unsigned kWaitSpins = 1u << 22;
// Largest shared-memory plan the pipelined kernel is used with: the 227 KB a
// block may opt in to (one block plus the 1 KB per-block reservation fits the
// SM's 228 KB).  Plans above 110 KB run one block per SM; its copy ring still
// overlaps the next tile's loads with compute, which measured faster than the
// one-tile-per-block kernel there (G DOF-updates/s, one-block pipelined / one
// tile per block: FP64 p = 12 54.7 / 46.9, p = 13 47.5 / 38.9; mixed p = 13
// 104.7 / 80.0, p = 14 91.2 / 82.3, p = 15 107.2 / 92.2; FP64 p = 11 about
// equal; FP64 p = 14, whose plan is 231,648 bytes, stage time 0.326 / 0.368 ms).
constexpr size_t kPipeMaxSmem = 227 * 1024;
// Shared memory of one SM and the per-block reservation of the driver.
constexpr size_t kSmemPerSM = 228 * 1024;
constexpr size_t kSmemPerBlockReserved = 1024;

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

// Bounded wait for the phase of `bar` with the given parity: at most
// `spins` polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  unsigned spins) {
  for (unsigned it = 0; it < spins; ++it)
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

// Orders this thread's shared-memory writes before later bulk copies (async
// proxy) into the same bytes.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Streaming load (read once: evict-first in the caches).
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) {
  return __ldcs(p);
}

// Placement of node (i,j,k) in the x-line and y-line buffers.  A thread
// (a,b) touches them in three patterns: its column (a,b,k) for k = 0..Nq-1,
// its x-line (l,a,b) and its y-line (a,l,b) for l = 0..Nq-1.  Each pattern
// has a per-thread part and a compile-time part (k or l unrolled), so the
// accesses cost a register plus an immediate or one XOR:
//   column   x: colx(a,b,k)              y: coly(a,b,k)
//   x-line   xl(xl_base(a,b), l)         y-line  yl(yl_base(a,b), l)
// Generic orders use the padded layout of tend_kernel (row stride RS,
// plane stride PS).  At Nq = 8 the layout depends on the word size, because
// a warp's 32 accesses must fall in distinct banks: 16 eight-byte bank pairs
// per half-warp for FP64, 32 four-byte banks for FP32.
//   FP64: an XOR swizzle with x and y buffers of their own,
//     x(i,j,k) = 16*((j + 8k) >> 1) + ((i ^ j) & 7) + 8*((j + k) & 1)
//     y(i,j,k) = 16*((i + 8k) >> 1) + ((i ^ j) & 7) + 8*((i + k) & 1)
//   so that both line patterns reduce to
//   x(l,a,b) = y(a,l,b) = (64b + 16(a>>1) + 8((a+b)&1) + a) ^ l.
//   FP32: one layout for both buffers,
//     f(i,j,k) = 64k + 8(j ^ k) + (i ^ (4(j>>2) + (k&3))),
//   whose three bit fields are disjoint, so that
//     column (a,b,k): ((8b + (a ^ 4(b>>2))) ^ (8k + (k&3))) + 64k,
//     x-line (l,a,b): (64b | 8(a^b) | (4(a>>2) + (b&3))) ^ l,
//     y-line (a,l,b): (72b + (a ^ (b&3))) ^ (8l + 4(l>>2)).
//   (The FP64 swizzle, read with four-byte banks, conflicts two ways on
//   every x-line access; this one is conflict-free on all three patterns.)
// All are bijections onto 0..511.  The padded layout costs two wavefronts
// more per column access.
//   Nq = 4, FP64: f(i,j,k) = 16k + 4(j ^ k) + (i ^ k), so that
//     column (a,b,k): 16k + (t ^ 5k) with t = a + 4b,
//     x-line (l,a,b): (16b + 4(a^b) + b) ^ l,
//     y-line (a,l,b): (20b + (a^b)) ^ 4l,
//   each 16 distinct eight-byte bank pairs over an element (a half-warp);
//   the padded layout conflicts two ways on column accesses there (FP64
//   p = 3: 78.2 -> 80.7 G with this one).  The same map is conflict-free for
//   FP32 as well (elements 80 words apart, 16 mod 32), but its XOR
//   addressing took the FP32 kernels from 96 to 111 registers and one
//   resident block fewer: 101.5 against 104.0 G, so FP32 uses a skewed linear
//   layout at Nq = 4 instead (SkewIdx below).
template <int NQ, int WORD>
struct LineIdx {
  static constexpr int SIZE = Geo<NQ>::SBUF;
  static constexpr int RS = Geo<NQ>::RS;
  static constexpr int PS = Geo<NQ>::PS;
  static __device__ __forceinline__ int colx(int a, int b, int k) { return a + RS * b + PS * k; }
  static __device__ __forceinline__ int coly(int a, int b, int k) { return a + RS * b + PS * k; }
  static __device__ __forceinline__ int xl_base(int a, int b) { return RS * a + PS * b; }
  static __device__ __forceinline__ int xl(int base, int l) { return base + l; }
  static __device__ __forceinline__ int yl_base(int a, int b) { return a + PS * b; }
  static __device__ __forceinline__ int yl(int base, int l) { return base + RS * l; }
};
template <>
struct LineIdx<8, 8> {
  static constexpr int SIZE = 512;
  static __device__ __forceinline__ int colx(int a, int b, int k) {
    return 16 * (b >> 1) + ((a ^ b) & 7) + 8 * ((b + k) & 1) + 64 * k;
  }
  static __device__ __forceinline__ int coly(int a, int b, int k) {
    return 16 * (a >> 1) + ((a ^ b) & 7) + 8 * ((a + k) & 1) + 64 * k;
  }
  static __device__ __forceinline__ int xl_base(int a, int b) {
    return (64 * b + 16 * (a >> 1) + 8 * ((a + b) & 1)) | a;
  }
  static __device__ __forceinline__ int xl(int base, int l) { return base ^ l; }
  static __device__ __forceinline__ int yl_base(int a, int b) { return xl_base(a, b); }
  static __device__ __forceinline__ int yl(int base, int l) { return base ^ l; }
};
// Skewed linear layouts (FP64, Nq = 6, 7): x(i,j,k) = QX*i_x + ..., a
// permutation of (i, j, k) weighted (Q, 1, Nq) per buffer, elements SIZE
// words apart.  Every pattern is a register plus an immediate.
template <int NQ, int X0, int X1, int X2, int QX, int Y0, int Y1, int Y2, int QY, int E>
struct SkewIdx {
  static constexpr int SIZE = E;
  template <int P0, int P1, int P2, int Q>
  static __device__ __forceinline__ int w(int i, int j, int k) {
    const int idx[3] = {i, j, k};
    return Q * idx[P0] + idx[P1] + NQ * idx[P2];
  }
  // Weight of i in the x layout and of j in the y layout (the line index).
  static constexpr int WXI = X0 == 0 ? QX : (X1 == 0 ? 1 : NQ);
  static constexpr int WYJ = Y0 == 1 ? QY : (Y1 == 1 ? 1 : NQ);
  static __device__ __forceinline__ int colx(int a, int b, int k) { return w<X0, X1, X2, QX>(a, b, k); }
  static __device__ __forceinline__ int coly(int a, int b, int k) { return w<Y0, Y1, Y2, QY>(a, b, k); }
  static __device__ __forceinline__ int xl_base(int a, int b) { return w<X0, X1, X2, QX>(0, a, b); }
  static __device__ __forceinline__ int xl(int base, int l) { return base + WXI * l; }
  static __device__ __forceinline__ int yl_base(int a, int b) { return w<Y0, Y1, Y2, QY>(a, 0, b); }
  static __device__ __forceinline__ int yl(int base, int l) { return base + WYJ * l; }
};
//   Nq = 6: x = 38i + j + 6k, y = 38j + i + 6k, 228 words per element;
//   Nq = 7: x = 49i + k + 7j, y = 49j + k + 7i, 343 words per element;
//   Nq = 9: x = 89i + j + 9k, y = 89j + i + 9k;
//   Nq = 10: x = 102i + j + 10k, y = 106j + i + 10k.
// Found by exhaustive search over permutations, Q and the element stride
// against the warp layout of each block (one element per tile from Nq = 9
// on), with the shared-memory plan kept at its resident-block count.  Line-
// buffer wavefronts per tile against the padded layout (ideal): Nq = 6
// 276 -> 204 (168), Nq = 7 294 -> 203 (196), Nq = 9 261 -> 216 (216),
// Nq = 10 460 -> 330 (280); measured FP64 p = 5 +5 %, p = 6 +11 %, p = 8
// +7 %, p = 9 +10 %.  FP32 (four-byte banks, 32-lane groups): Nq = 6
// x = 36i + j + 6k, y = 38j + i + 6k (150 -> 114, ideal 96) and Nq = 7
// x = 49k + i + 7j, y = 49j + k + 7i (168 -> 140, ideal 112); measured mixed
// p = 5 +2 %, p = 6 +2 %; Nq = 4 x = 20i + j + 4k, y = 20j + i + 4k (96 -> 64, its
// ideal), mixed p = 3 +6 % (the XOR map of FP64 is conflict-free for four-byte
// words too, but its addressing cost the FP32 kernel a resident block).  Layouts
// that reached their ideal but measured no gain
// were left out: FP64 Nq = 11 (429 -> 352; 66.6 against 67.6 G) and FP32
// Nq = 10 (250 -> 190; 109.2 against 112.9 G).
template <>
struct LineIdx<6, 8> : SkewIdx<6, 0, 1, 2, 38, 1, 0, 2, 38, 228> {};
template <>
struct LineIdx<7, 8> : SkewIdx<7, 0, 2, 1, 49, 1, 2, 0, 49, 343> {};
template <>
struct LineIdx<4, 4> : SkewIdx<4, 0, 1, 2, 20, 1, 0, 2, 20, 80> {};
template <>
struct LineIdx<6, 4> : SkewIdx<6, 0, 1, 2, 36, 1, 0, 2, 38, 228> {};
template <>
struct LineIdx<7, 4> : SkewIdx<7, 2, 0, 1, 49, 1, 2, 0, 49, 343> {};
template <>
struct LineIdx<9, 8> : SkewIdx<9, 0, 1, 2, 89, 1, 0, 2, 89, 794> {};
template <>
struct LineIdx<10, 8> : SkewIdx<10, 0, 1, 2, 102, 1, 0, 2, 106, 1054> {};

template <>
struct LineIdx<4, 8> {
  static constexpr int SIZE = 80;
  static __device__ __forceinline__ int colx(int a, int b, int k) {
    return 16 * k + ((a + 4 * b) ^ (5 * k));
  }
  static __device__ __forceinline__ int coly(int a, int b, int k) { return colx(a, b, k); }
  static __device__ __forceinline__ int xl_base(int a, int b) { return 16 * b + 4 * (a ^ b) + b; }
  static __device__ __forceinline__ int xl(int base, int l) { return base ^ l; }
  static __device__ __forceinline__ int yl_base(int a, int b) { return 20 * b + (a ^ b); }
  static __device__ __forceinline__ int yl(int base, int l) { return base ^ (4 * l); }
};
template <>
struct LineIdx<8, 4> {
  static constexpr int SIZE = 512;
  static __device__ __forceinline__ int colx(int a, int b, int k) {
    return ((8 * b + (a ^ (4 * (b >> 2)))) ^ (8 * k + (k & 3))) + 64 * k;
  }
  static __device__ __forceinline__ int coly(int a, int b, int k) { return colx(a, b, k); }
  static __device__ __forceinline__ int xl_base(int a, int b) {
    return (64 * b) | (8 * (a ^ b)) | (4 * (a >> 2) + (b & 3));
  }
  static __device__ __forceinline__ int xl(int base, int l) { return base ^ l; }
  static __device__ __forceinline__ int yl_base(int a, int b) { return 72 * b + (a ^ (b & 3)); }
  static __device__ __forceinline__ int yl(int base, int l) { return base ^ (8 * l + 4 * (l >> 2)); }
};

// Line buffers of the tensor-core contractions (fast FP64, Nq = 8): eight
// k-planes of 64, each an 8x8 (i,j) block in which
//   x:  F_x(i,j) at px(i,j) = (j ^ h(i)) + 8i,  DxF(i,j) at qx(i,j) = (j ^ (i&6)) + 8i
//   y:  F_y(i,j) at py(i,j) = (i ^ h(j)) + 8j,  DyF(i,j) at qy(i,j) = (i ^ (j&6)) + 8j
// with h(n) = ((n&2) << 1) | ((n&4) >> 1).  The four patterns on each buffer
// (column writes of F, B-fragment loads, 16-byte C-fragment stores, column
// reads of the result) each put a half-warp's eight-byte accesses on 16
// distinct bank pairs.
struct TensorIdx8 {
  static __device__ __forceinline__ int h(int n) { return ((n & 2) << 1) | ((n & 4) >> 1); }
  static __device__ __forceinline__ int px(int i, int j) { return (j ^ h(i)) + 8 * i; }
  static __device__ __forceinline__ int qx(int i, int j) { return (j ^ (i & 6)) + 8 * i; }
  static __device__ __forceinline__ int py(int i, int j) { return (i ^ h(j)) + 8 * j; }
  static __device__ __forceinline__ int qy(int i, int j) { return (i ^ (j & 6)) + 8 * j; }
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

// Per-element area of minus-side face values and face fluxes (in
// compute-type words).  x faces (+x = 2, -x = 4): q and u in two arrays,
// entry (face, k, j) at XOFF*[face is -x] + Nq*k + j, the -x block shifted
// by Nq^2 + 4 so that the eight writers of one k (a = 0 or Nq-1) hit
// distinct banks.  y faces (-y = 1, +y = 3): (q, v) pairs, face-major, node
// a + Nq*k.  After the flux phase the pair of -y at node t holds
// (flux -y, flux +y) and the pair of +y at node t (flux +x, flux -x), so the
// lift reads two pairs per node.  Each
// scalar store of a warp then costs two wavefronts (one per half-warp), and
// a pair store of the y writers one (they fill one quarter-warp).
//
// The split x arrays pay off where a pair is 16 bytes (FP64, whose 128-bit
// shared accesses run in quarter-warp phases: the x writers span all four).
// With 8-byte FP32 pairs the x faces keep (q, u) pairs like the y faces
// (SPLIT = false), face-major in the order -y, +x, +y, -x; after the flux
// phase the pair of -y at node t holds (flux -y, flux +y) and the pair of +x
// (flux +x, flux -x).
template <int NQ, bool SPLIT>
struct FaceArea {
  static constexpr int NQ2 = NQ * NQ;
  static constexpr int XOFF = NQ2 + 4;
  static constexpr int XA = 2 * XOFF;                // one x array (q or u)
  static constexpr int Y0 = SPLIT ? 2 * XA : 4 * NQ2;  // start of the y pairs
  // Pairs (SPLIT = false): the -x block starts P3 pairs after 3 Nq^2, so that
  // the threads of a warp on the -x face (a = 0) and on the +x face
  // (a = Nq-1) store their (q, u) pairs 16 banks apart, not on the same ones.
  static constexpr int P3 = SPLIT ? 0 : ((8 - 2 * NQ2) % 16 + 16) % 16;
  static constexpr int F3 = 3 * NQ2 + P3;            // pair index of the -x block
  static constexpr int ELEM = SPLIT ? Y0 + 4 * NQ2 : 2 * (4 * NQ2 + P3);
  // Pair index of face block f (0: -y, 1: +x, 2: +y, 3: -x).
  static __host__ __device__ constexpr int block(int f) { return f == 3 ? F3 : f * NQ2; }
};

// Thread geometry: Nq^2 threads per element, EPB elements per block
// (128 threads where Nq^2 divides it).
template <int NQ>
struct PipeGeo {
  static constexpr int NQ2 = NQ * NQ;
  static constexpr int NP = NQ2 * NQ;
  static constexpr int EPB = NQ2 >= 128 ? 1 : 128 / NQ2;
  static constexpr int THREADS = EPB * NQ2;
};

// Shared-memory plan of the pipelined kernel.  TCG adds the operands of the
// tensor-core line contractions (sdg_tcgen05.cuh): x and y, hi and lo, the
// hi and lo halves of D, the TMEM address and the MMA completion barrier.
// BATCH adds to each slot the tile's face-neighbour rows and its TileCtx
// (instance pointers, first element, count), written by the producer, where
// kRingCtx allows.
template <int NQ, typename TC, bool BATCH>
constexpr bool kRingCtx =
    BATCH && (sizeof(TC) == 8 || (PipeGeo<NQ>::NQ2 >= 128 ? 1 : 128 / PipeGeo<NQ>::NQ2) <= 2);

template <int NQ, typename TQ, typename TV, typename TC, bool STAGE, bool TCG = false,
          bool BATCH = false>
struct PipePlan {
  using G = PipeGeo<NQ>;
  static constexpr int EPB = G::EPB;
  static constexpr int NP = G::NP;
  static constexpr int NSTAGE = 2;
  static constexpr size_t r16(size_t x) { return (x + 15) & ~size_t(15); }
  static constexpr size_t mx(size_t a, size_t b) { return a > b ? a : b; }
  // Each array region holds EPB elements plus 32 bytes of slack: the source
  // range is widened to 16-byte boundaries at both ends (at most 12 bytes
  // each for 4- and 8-byte elements).  The u and v regions double as the
  // x- and y-line buffers once the tile's columns are in registers.
  static constexpr size_t QB = r16(sizeof(TQ) * EPB * NP + 32);
  static constexpr size_t VB =
      mx(r16(sizeof(TV) * EPB * NP + 32),
         r16(sizeof(TC) * EPB * LineIdx<NQ, static_cast<int>(sizeof(TC))>::SIZE));
  static constexpr size_t EB = r16(sizeof(TC) * 3 * EPB + 32);  // escale rows
  static constexpr size_t FB = r16(sizeof(TC) * 6 * EPB + 32);  // fscale rows
  static constexpr bool RING_CTX = kRingCtx<NQ, TC, BATCH>;
  static constexpr size_t PB = RING_CTX ? r16(sizeof(int) * 6 * EPB + 32) : 0;  // pbase rows
  static constexpr size_t CB = RING_CTX ? 128 : 0;                   // TileCtx
  static constexpr size_t OFF_U = QB;
  static constexpr size_t OFF_V = QB + VB;
  static constexpr size_t OFF_W = QB + 2 * VB;
  static constexpr size_t OFF_E = QB + 3 * VB;
  static constexpr size_t OFF_F = OFF_E + EB;
  static constexpr size_t OFF_P = OFF_F + FB;
  static constexpr size_t OFF_C = OFF_P + PB;
  static constexpr size_t SLOT = OFF_C + CB;
  // (q, un) pairs of the four x/y faces' minus side, per element.
  static constexpr size_t FACE = r16(sizeof(TC) * FaceArea<NQ, sizeof(TC) == 8>::ELEM * EPB);
  // Per-face lift factors l_f(n) of the fast kernels, (4, Nq).
  static constexpr size_t LIFTB = r16(sizeof(TC) * 4 * NQ);
  static constexpr size_t BARS = 16 * NSTAGE;
  static constexpr size_t TCGB = TCG ? 4 * tc::kOperandBytes + 2 * tc::kBBytes + 32 : 0;
  static constexpr size_t BYTES = NSTAGE * SLOT + FACE + LIFTB + BARS + TCGB;
  // Blocks per SM that the shared memory allows (the register budget per
  // thread follows from it), at most 4.
  static constexpr int BLOCKS_PER_SM_SMEM = static_cast<int>(
      kSmemPerSM / (BYTES + kSmemPerBlockReserved) > 4
          ? 4
          : (kSmemPerSM / (BYTES + kSmemPerBlockReserved) < 1
                 ? 1
                 : kSmemPerSM / (BYTES + kSmemPerBlockReserved)));
  static constexpr int MIN_BLOCKS =
      (BLOCKS_PER_SM_SMEM * G::THREADS > 512) ? 512 / G::THREADS : BLOCKS_PER_SM_SMEM;
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
  int n;   // elements in the tile (0..EPB; 0 past the last tile)
};

// BATCH is a compile-time property of the kernel, so a single-instance
// launch keeps its pointers in the parameter bank instead of registers.
template <int EPB, bool BATCH, typename TQ, typename TV, typename TO, typename TC>
__device__ __forceinline__ TileCtx<TQ, TV, TO, TC> tile_ctx(const TendArgs<TQ, TV, TO, TC>& A,
                                                            int tile, int ntiles) {
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
    c.n = tile < ntiles ? min(EPB, A.nelem - tile * EPB) : 0;
  } else {
    const BatchTile t = A.tiles[tile < ntiles ? tile : 0];
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
    c.n = tile < ntiles ? t.n : 0;
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

// Byte range of elements [e0, e0+n) in an array of `per_elem` bytes per
// element, widened to 16-byte boundaries: start, length and the offset of
// element e0 inside the copied range.
__device__ __forceinline__ void tile_range(int e0, int n, size_t per_elem, size_t* lo16,
                                           uint32_t* bytes, uint32_t* shift) {
  const size_t lo = static_cast<size_t>(e0) * per_elem;
  const size_t hi = static_cast<size_t>(e0 + n) * per_elem;
  *lo16 = lo & ~size_t(15);
  *bytes = static_cast<uint32_t>(((hi + 15) & ~size_t(15)) - *lo16);
  *shift = static_cast<uint32_t>(lo - *lo16);
}

__device__ __forceinline__ uint32_t tile_shift(int e0, size_t per_elem) {
  return static_cast<uint32_t>((static_cast<size_t>(e0) * per_elem) & 15);
}

// Blocks per SM the kernel is compiled for: what its shared memory allows,
// but at most 2 for the exact kernels, whose separately rounded arithmetic
// needs the larger register budget, for FP64 columns of 9 or more nodes (at
// the three-block budget of 168 registers they spill 200-300 bytes; two
// blocks measured 13 % faster at Nq = 10, and four spilling blocks 8 % slower
// at Nq = 9) and for all columns of 12 or more nodes; and at most 3 for the
// fast FP64 kernels at Nq = 7 (at the four-block budget of 128 registers they
// spill 36 bytes; three blocks measured 10 % faster: 62.7 -> 69.1 G).
template <int NQ, typename TQ, typename TV, typename TC, bool EXACT, bool STAGE,
          bool TCG = false, bool BATCH = false>
constexpr int pipe_min_blocks() {
  constexpr int m = PipePlan<NQ, TQ, TV, TC, STAGE, TCG, BATCH>::MIN_BLOCKS;
  if constexpr (sizeof(TC) == 8 && !EXACT && NQ == 7) return m > 3 ? 3 : m;
  return ((EXACT || (sizeof(TC) == 8 && NQ >= 9) || NQ >= 12) && m > 2) ? 2 : m;
}

// The thread bound is the block size rounded up to whole warps (the
// compiler front end of CUDA 12.9 fails on this kernel with a bound of,
// e.g., 81 threads at Nq = 9).
//
// TCG (mixed form at Nq = 8 only, kernel variant kVariantTensor): the x and
// y line contractions on the tensor cores, TF32 in three hi/lo passes with
// the results in tensor memory (sdg_tcgen05.cuh); phase 1 writes the split
// operands, one thread issues the MMAs after the first barrier, and each
// line owner reads its eight results back into the line buffers.  Its
// rounding differs from the FP32 FMA lines of the other variants.
template <int NQ, typename TQ, typename TV, typename TO, typename TC, bool EXACT,
          int ORDER, bool STAGE, bool BATCH, bool TCG = false>
__global__ void __launch_bounds__((PipeGeo<NQ>::THREADS + 31) / 32 * 32,
                                  (pipe_min_blocks<NQ, TQ, TV, TC, EXACT, STAGE, TCG, BATCH>()))
    tend_pipe_kernel(const __grid_constant__ TendArgs<TQ, TV, TO, TC> A,
                     const __grid_constant__ DMat<NQ, TC> D) {
  using G = PipeGeo<NQ>;
  using P = PipePlan<NQ, TQ, TV, TC, STAGE, TCG, BATCH>;
  static_assert(sizeof(TileCtx<TQ, TV, TO, TC>) <= 128, "TileCtx fits its slot area");
  // Batched tiles whose context and face-neighbour rows travel in the ring
  // (measured: FP64 batched stages 4-10 % faster; FP32 with 3-8 elements
  // per tile 4-8 % slower, so those resolve the tables themselves).
  constexpr bool RCTX = P::RING_CTX;
  static_assert(!TCG || (NQ == 8 && sizeof(TC) == 4 && !EXACT && G::THREADS == 128),
                "tensor-core lines: fast FP32 at Nq = 8, 128 threads");
  using AR = Ar<TC, EXACT>;
  using Ctx = TileCtx<TQ, TV, TO, TC>;
  using V2 = typename Pair2<TC>::type;
  using LI = LineIdx<NQ, static_cast<int>(sizeof(TC))>;
  constexpr int NQ2 = G::NQ2;
  constexpr int NP = G::NP;
  constexpr int EPB = G::EPB;
  constexpr int NS = P::NSTAGE;
  // x/y line contractions on the tensor cores (fast FP64, Nq = 8).
  constexpr bool TENSOR = kTensorLines<NQ, TC, EXACT>;
  double da0 = 0.0, da1 = 0.0;  // this lane's A fragments of D
  if constexpr (TENSOR) dmma_dfrag(D, &da0, &da1);

  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* slots = smem_raw;
  TC* sL = reinterpret_cast<TC*>(smem_raw + NS * P::SLOT + P::FACE);
  uint64_t* bars =
      reinterpret_cast<uint64_t*>(smem_raw + NS * P::SLOT + P::FACE + P::LIFTB);
  // Tensor-core operands (TCG): A for x and y, hi and lo; B hi and lo; the
  // MMA barrier and the TMEM address.
  unsigned char* tcg = smem_raw + NS * P::SLOT + P::FACE + P::LIFTB + P::BARS;
  unsigned char* tA = tcg;                                      // [xhi, xlo, yhi, ylo]
  unsigned char* tB = tcg + 4 * tc::kOperandBytes;              // [hi, lo]
  uint64_t* mma_bar = reinterpret_cast<uint64_t*>(tB + 2 * tc::kBBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tB + 2 * tc::kBBytes + 16);

  const int s = threadIdx.x / NQ2;               // element slot of the tile
  const int t = threadIdx.x - s * NQ2;           // column index a + NQ*b
  const int a = t % NQ;
  const int b = t / NQ;
  const int ntiles = BATCH ? A.ntiles : (A.nelem + EPB - 1) / EPB;

  // Minus-side values of the x/y faces, replaced in phase 2 by the face
  // fluxes that the epilogue's lift reads (see FaceArea).
  constexpr bool XSPLIT = sizeof(TC) == 8;
  using FA = FaceArea<NQ, XSPLIT>;
  TC* fa = reinterpret_cast<TC*>(smem_raw + NS * P::SLOT) + s * FA::ELEM;
  TC* xq = fa;                                     // split x faces: q
  TC* xu = fa + FA::XA;                            // split x faces: u
  V2* ypair = reinterpret_cast<V2*>(fa + FA::Y0);  // y faces: (q, v) pairs
  // FP32: [4][NQ2] (q, un) pairs of the four faces, face-major.
  V2* fM = reinterpret_cast<V2*>(fa);

  // Producer: one thread fills ring slot `slot` with tile `tile`.
  auto issue = [&](int tile, int slot) {
    // Test hook (host-set): leave this tile's slot empty, so that its wait
    // runs out and the timeout path below is taken.
    if (tile + 1 == A.inject_skip) return;
    const Ctx c = tile_ctx<EPB, BATCH>(A, tile, ntiles);
    unsigned char* base = slots + slot * P::SLOT;
    const void* src[6] = {c.q, c.u, c.v, c.w, c.escale, c.fscale};
    const size_t per[6] = {sizeof(TQ) * NP, sizeof(TV) * NP, sizeof(TV) * NP,
                           sizeof(TV) * NP, sizeof(TC) * 3,  sizeof(TC) * 6};
    const size_t off[6] = {0, P::OFF_U, P::OFF_V, P::OFF_W, P::OFF_E, P::OFF_F};
    size_t lo[6];
    uint32_t by[6], sh[6], total = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      tile_range(c.e0, c.n, per[k], &lo[k], &by[k], &sh[k]);
      total += by[k];
    }
    // Batched tiles: the tile's context and its elements' face-neighbour
    // rows go with it, so that the consumers read them from shared memory
    // instead of the tile and instance tables.
    size_t plo = 0;
    uint32_t pby = 0, psh = 0;
    if constexpr (RCTX) {
      *reinterpret_cast<Ctx*>(base + P::OFF_C) = c;
      tile_range(c.e0, c.n, sizeof(int) * 6, &plo, &pby, &psh);
      total += pby;
    }
    mbar_arrive_expect_tx(&bars[slot], total);
#pragma unroll
    for (int k = 0; k < 6; ++k)
      bulk_g2s(base + off[k], static_cast<const unsigned char*>(src[k]) + lo[k], by[k],
               &bars[slot]);
    if constexpr (RCTX)
      bulk_g2s(base + P::OFF_P, reinterpret_cast<const unsigned char*>(c.pbase) + plo, pby,
               &bars[slot]);
    // q0 (RK stages 2-3) is read by the epilogue straight from global
    // memory; bring the tile's range into L2 now.
    if (STAGE && A.rk_a != 0.0) {
      size_t l0;
      uint32_t b0, s0;
      tile_range(c.e0, c.n, sizeof(double) * NP, &l0, &b0, &s0);
      bulk_prefetch_l2(reinterpret_cast<const unsigned char*>(c.q0) + l0, b0);
    }
  };

  if (threadIdx.x == 0) {
    for (int k = 0; k < NS; ++k) mbar_init(&bars[k], 1);
    if constexpr (TCG) mbar_init(mma_bar, 1);
    fence_barrier_init();
  }
  uint32_t tmem = 0;
  if constexpr (TCG) {
    if (threadIdx.x < 32) tc::tmem_alloc(tmem_slot);
    // B(l, i) = D(i, l), row i, K index l; hi and lo TF32 halves.
    if (threadIdx.x < 64) {
      const int i = threadIdx.x >> 3, l = threadIdx.x & 7;
      const float d = D.d[i * NQ + l];
      const float hi = tc::to_tf32(d);
      *reinterpret_cast<float*>(tB + tc::offset(i, l)) = hi;
      *reinterpret_cast<float*>(tB + tc::kBBytes + tc::offset(i, l)) = tc::to_tf32(d - hi);
    }
    fence_proxy_async_smem();
    tc::fence_before_sync();
  }
  // Factored lift of the fast kernels: l_f(n) is the factored table's entry
  // at normal index n, tangential indices 0 (faces 1, 3 lie along j, faces
  // 2, 4 along i).  The exact kernels read the verbatim table instead.
  if constexpr (!EXACT) {
    for (int x = threadIdx.x; x < 4 * NQ; x += blockDim.x) {
      const int f = x / NQ, n = x - f * NQ;
      sL[x] = ldro(A.lift + NP * f + ((f & 1) ? n : NQ * n));
    }
  }
  __syncthreads();
  if constexpr (TCG) {
    tc::fence_after_sync();
    tmem = *tmem_slot;
  }
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
    // A single instance's tile context comes from the parameters; the
    // element's face-neighbour row, needed after phase 1, is loaded before
    // the wait.  A batched tile's context and rows come with the tile.
    Ctx C = RCTX ? Ctx{} : tile_ctx<EPB, BATCH>(A, tile, ntiles);
    bool active = s < C.n;
    int e = C.e0 + (active ? s : 0);
    long base = static_cast<long>(e) * NP;

    // The element's face-neighbour row, needed after phase 1.
    int pbc[6];
#pragma unroll
    for (int f = 0; f < 6; ++f)
      pbc[f] = (!RCTX && active) ? ldro(C.pbase + 6 * static_cast<long>(e) + f) : 0;

    // ---- Wait for the tile's slot (bounded, block-uniform) -----------------
    const bool ok = __syncthreads_and(mbar_wait_bounded(&bars[slot], parity, A.wait_spins));
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
            mbar_wait_bounded(&bars[T % NS], (T / NS) & 1, A.wait_spins);
        }
      }
      if constexpr (TCG) {
        // No MMA is in flight (the previous tile's results were read).
        __syncwarp();
        if (threadIdx.x < 32) tc::tmem_dealloc(tmem);
      }
      return;
    }
    if constexpr (RCTX) {
      const unsigned char* sb0 = slots + slot * P::SLOT;
      C = *reinterpret_cast<const Ctx*>(sb0 + P::OFF_C);
      active = s < C.n;
      e = C.e0 + (active ? s : 0);
      const int* spb =
          reinterpret_cast<const int*>(sb0 + P::OFF_P + tile_shift(C.e0, 24)) + 6 * s;
#pragma unroll
      for (int f = 0; f < 6; ++f) pbc[f] = active ? spb[f] : 0;
      base = static_cast<long>(e) * NP;
    }
    // Every thread finished the previous tile (the barrier above), so its
    // slot is free: refill it with the tile NS iterations on from it.
    if (threadIdx.x == 0 && it > 0) {
      const int nt = blockIdx.x + (it - 1 + NS) * gridDim.x;
      if (nt < ntiles) issue(nt, (it - 1) % NS);
    }

    unsigned char* sb = slots + slot * P::SLOT;
    const TQ* sq =
        reinterpret_cast<const TQ*>(sb + tile_shift(C.e0, sizeof(TQ) * NP)) + s * NP;
    const uint32_t shv = tile_shift(C.e0, sizeof(TV) * NP);
    const TV* su = reinterpret_cast<const TV*>(sb + P::OFF_U + shv) + s * NP;
    const TV* sv = reinterpret_cast<const TV*>(sb + P::OFF_V + shv) + s * NP;
    const TV* sw = reinterpret_cast<const TV*>(sb + P::OFF_W + shv) + s * NP;
    const TC* ses =
        reinterpret_cast<const TC*>(sb + P::OFF_E + tile_shift(C.e0, sizeof(TC) * 3)) + 3 * s;
    const TC* sfs =
        reinterpret_cast<const TC*>(sb + P::OFF_F + tile_shift(C.e0, sizeof(TC) * 6)) + 6 * s;
    // z-flux column in place of w.
    static_assert(sizeof(TV) == sizeof(TC), "w and q*w share their slots");
    TC* sz = reinterpret_cast<TC*>(sb + P::OFF_W + shv) + s * NP;
    // Line buffers in the u and v regions (valid after the column reads).
    TC* sX = reinterpret_cast<TC*>(sb + P::OFF_U) + s * LI::SIZE;
    TC* sY = reinterpret_cast<TC*>(sb + P::OFF_V) + s * LI::SIZE;

    // ---- Plus-side face values ---------------------------------------------
    // x/y faces whose neighbour lies outside the tile (or in the caller's
    // halo) and the z faces come from global memory; a neighbour inside the
    // tile is read from shared memory after phase 1.  The global loads are
    // issued before phase 1, so that phase 1 and the line contractions cover
    // their latency, except in the FP32 kernels with one element per tile,
    // which measured faster (-4 % register pressure in phase 1) with the
    // loads after the line buffers are published.
    TC qP[4], unP[4], qZ[2], wZ[2];
    unsigned in_tile = 0;  // bit f: face f's neighbour is an element of this tile
    if constexpr (EPB > 1) {
      if (active) {
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          const int d = pbc[f] - C.e0 * NP;
          if (pbc[f] >= 0 && d >= 0 && d < C.n * NP) in_tile |= 1u << f;
        }
      }
    }
    auto gather = [&]() {
      if (!active) return;
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        if (in_tile & (1u << f)) continue;
        const long idx = (pbc[f] >= 0) ? static_cast<long>(pbc[f]) + opp_offset<NQ>(f, a, b)
                                       : static_cast<long>(-1 - pbc[f]) + t;
        qP[f] = static_cast<TC>(ldro(C.q + idx));
        unP[f] = static_cast<TC>((f == 1 || f == 3) ? ldro(C.u + idx) : ldro(C.v + idx));
      }
#pragma unroll
      for (int z = 0; z < 2; ++z) {
        const int f = 4 + z;
        const long idx = (pbc[f] >= 0) ? static_cast<long>(pbc[f]) + opp_offset<NQ>(f, a, b)
                                       : static_cast<long>(-1 - pbc[f]) + t;
        qZ[z] = static_cast<TC>(ldro(C.q + idx));
        wZ[z] = static_cast<TC>(ldro(C.w + idx));
      }
    };
    constexpr bool EARLY = EPB > 1 || sizeof(TC) == 8;
    if constexpr (EARLY) gather();

    // ---- Phase 1: the column's volume fluxes and minus-side face values ---
    // q*w replaces w in place: each thread reads and writes only its own
    // column there, so the z-flux column waits in shared memory for phase 4.
    TC fx[NQ], fy[NQ];
    TC wlo = TC(0), whi = TC(0), qlo = TC(0), qhi = TC(0);
    if (active) {
      // A thread on an x face (a = 0 or Nq-1) stores its (q, u) there, one on
      // a y face (b = 0 or Nq-1) its (q, v): faces -x/+x are 4/2, -y/+y 1/3.
      const bool onx = (a == 0) || (a == NQ - 1);
      const bool ony = (b == 0) || (b == NQ - 1);
      const int xo = (a == 0 ? FA::XOFF : 0) + b;
      V2* fmx = fM + (a == 0 ? FA::F3 : NQ2) + b;
      V2* fmy = XSPLIT ? ypair + (b == 0 ? 0 : NQ2) + a : fM + (b == 0 ? 0 : 2) * NQ2 + a;
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        const int n = t + NQ2 * k;
        const TC qv = static_cast<TC>(sq[n]);
        const TC uv = static_cast<TC>(su[n]);
        const TC vv = static_cast<TC>(sv[n]);
        const TC wv = static_cast<TC>(sw[n]);
        if (k == 0) wlo = wv;
        if (k == NQ - 1) whi = wv;
        fx[k] = AR::mul(qv, uv);
        fy[k] = AR::mul(qv, vv);
        sz[n] = AR::mul(qv, wv);
        if constexpr (TCG) {
          // x line (j, k, e) = (b, k, s) is row m of A_x with K index a; y
          // line (i, k, e) = (a, k, s) is row m of A_y with K index b.
          const uint32_t ox = tc::offset(b + 8 * k + 64 * s, a);
          const uint32_t oy = tc::offset(a + 8 * k + 64 * s, b);
          const float xh = tc::to_tf32(fx[k]), yh = tc::to_tf32(fy[k]);
          *reinterpret_cast<float*>(tA + ox) = xh;
          *reinterpret_cast<float*>(tA + tc::kOperandBytes + ox) = tc::to_tf32(fx[k] - xh);
          *reinterpret_cast<float*>(tA + 2 * tc::kOperandBytes + oy) = yh;
          *reinterpret_cast<float*>(tA + 3 * tc::kOperandBytes + oy) = tc::to_tf32(fy[k] - yh);
        }
        if constexpr (XSPLIT) {
          if (k == 0) qlo = qv;
          if (k == NQ - 1) qhi = qv;
          if (onx) {
            xq[xo + NQ * k] = qv;
            xu[xo + NQ * k] = uv;
          }
        } else {
          if (onx) fmx[NQ * k] = V2{qv, uv};
        }
        if (ony) fmy[NQ * k] = V2{qv, vv};
      }
    }
    if constexpr (TCG) fence_proxy_async_smem();  // A operands -> tensor cores
    __syncthreads();   // the slot's u, v are dead: reuse them as line buffers
    if constexpr (TCG) {
      if (threadIdx.x == 0) {
        tc::fence_after_sync();
        const uint64_t bh = tc::smem_desc(tB), bl = tc::smem_desc(tB + tc::kBBytes);
#pragma unroll
        for (int d = 0; d < 2; ++d) {
          const uint32_t acc = tmem + 8 * d;  // columns 0-7: x, 8-15: y
          const uint64_t ah = tc::smem_desc(tA + 2 * d * tc::kOperandBytes);
          const uint64_t al = tc::smem_desc(tA + (2 * d + 1) * tc::kOperandBytes);
          tc::mma_tf32(acc, ah, bh, false);
          tc::mma_tf32(acc, al, bh, true);
          tc::mma_tf32(acc, ah, bl, true);
        }
        tc::commit(mma_bar);
      }
    }
    if (active) {
      if constexpr (TCG) {
        // The lines come from the tensor cores; no column writes.
      } else if constexpr (TENSOR) {
        TC* px = sX + TensorIdx8::px(a, b);
        TC* py = sY + TensorIdx8::py(a, b);
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
          px[NQ2 * k] = fx[k];
          py[NQ2 * k] = fy[k];
        }
      } else {
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
          sX[LI::colx(a, b, k)] = fx[k];
          sY[LI::coly(a, b, k)] = fy[k];
        }
      }
      // A neighbour in this tile stored its minus-side values of the shared
      // face (the face opposite f: -y/+y and +x/-x swap) in its face area
      // before the barrier above; phase 2 replaces them with fluxes only
      // after the next barrier.  Read them here rather than gathering them
      // from global memory.  The values are the same, so are the results.
      if constexpr (EPB > 1) {
        TC* const fa0 = reinterpret_cast<TC*>(smem_raw + NS * P::SLOT);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          if (in_tile & (1u << f)) {
            const int d = pbc[f] - C.e0 * NP;
            const TC* nfa = fa0 + (d / NP) * FA::ELEM;
            if constexpr (XSPLIT) {
              if (f == 1 || f == 3) {
                const int xi = (f == 1 ? FA::XOFF : 0) + t;
                qP[f] = nfa[xi];
                unP[f] = nfa[FA::XA + xi];
              } else {
                const V2 m = reinterpret_cast<const V2*>(nfa + FA::Y0)[(f == 0 ? NQ2 : 0) + t];
                qP[f] = m.x;
                unP[f] = m.y;
              }
            } else {
              const V2 m = reinterpret_cast<const V2*>(nfa)[FA::block((f + 2) & 3) + t];
              qP[f] = m.x;
              unP[f] = m.y;
            }
          }
        }
      }
    }
    __syncthreads();
    if constexpr (!EARLY) gather();

    constexpr int NQ0 = STAGE ? NQ : 1;
    double q0r[NQ0];
    const bool use_q0 = STAGE && A.rk_a != 0.0;
    TC f5 = TC(0), f6 = TC(0);
    if (active) {
      // ---- Phase 3: x-line and y-line contractions, in place --------------
      if constexpr (TCG) {
        // Wait for this tile's MMAs (bounded), then each thread reads its
        // x line and y line (TMEM lane = thread) into the line buffers.
        const bool done = mbar_wait_bounded(mma_bar, it & 1, A.wait_spins);
        if (!done) atomicExch(A.status, kStatusWaitTimeout);
        tc::fence_after_sync();
        float rx[8], ry[8];
        const uint32_t lane = tmem + (static_cast<uint32_t>(threadIdx.x & ~31) << 16);
        tc::ld8(lane, rx);
        tc::ld8(lane + 8, ry);
        tc::fence_before_sync();
        const int lbx = LI::xl_base(a, b), lby = LI::yl_base(a, b);
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
          sX[LI::xl(lbx, i)] = rx[i];
          sY[LI::yl(lby, i)] = ry[i];
        }
      } else if constexpr (TENSOR) {
        // DMMA tiles: the element's two warps take four k-planes each; a
        // plane is read and rewritten only by its warp.
        const int lane = threadIdx.x & 31, g = lane >> 2, qd = lane & 3;
        const int we = t >> 5;  // warp of the element
        using TI = TensorIdx8;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          TC* px = sX + NQ2 * (4 * we + kk);
          TC* py = sY + NQ2 * (4 * we + kk);
          double d0, d1;
          // x: B(l, j) = F_x(l, j), C(i, j) = DxF(i, j) on this plane.
          dmma_tile8(da0, da1, px[TI::px(qd, g)], px[TI::px(4 + qd, g)], &d0, &d1);
          *reinterpret_cast<double2*>(px + TI::qx(g, 2 * qd)) = make_double2(d0, d1);
          // y: B(l, i) = F_y(i, l), C(j, i) = DyF(i, j).
          dmma_tile8(da0, da1, py[TI::py(g, qd)], py[TI::py(g, 4 + qd)], &d0, &d1);
          *reinterpret_cast<double2*>(py + TI::qy(2 * qd, g)) = make_double2(d0, d1);
        }
      } else {
        const int lbx = LI::xl_base(a, b), lby = LI::yl_base(a, b);
        if constexpr (sizeof(TC) == 4 && !EXACT && kPairedLinesPipe<NQ>) {
          // Fast FP32: the x line (a,b) and the y line (a,b) take the same
          // coefficient row D(i, .), so one packed FMA advances both.
          float2 ln[NQ];
#pragma unroll
          for (int l = 0; l < NQ; ++l) ln[l] = make_float2(sX[LI::xl(lbx, l)], sY[LI::yl(lby, l)]);
#pragma unroll
          for (int i = 0; i < NQ; ++i) {
            const float2 r = contract2<NQ, ORDER>([&](int l) { return D.d[i * NQ + l]; },
                                                  [&](int l) { return ln[l]; });
            sX[LI::xl(lbx, i)] = r.x;
            sY[LI::yl(lby, i)] = r.y;
          }
        } else {
          TC line[NQ];
#pragma unroll
          for (int l = 0; l < NQ; ++l) line[l] = sX[LI::xl(lbx, l)];
#pragma unroll
          for (int i = 0; i < NQ; ++i)
            sX[LI::xl(lbx, i)] = contract<NQ, ORDER, AR, TC>(
                [&](int l) { return D.d[i * NQ + l]; }, [&](int l) { return line[l]; });
#pragma unroll
          for (int l = 0; l < NQ; ++l) line[l] = sY[LI::yl(lby, l)];
#pragma unroll
          for (int j = 0; j < NQ; ++j)
            sY[LI::yl(lby, j)] = contract<NQ, ORDER, AR, TC>(
                [&](int l) { return line[l]; }, [&](int l) { return D.d[j * NQ + l]; });
        }
      }
      // The line buffers live in the slot that the next refill overwrites.
      fence_proxy_async_smem();
      // q0 of the column (RK stages 2-3), in L2 since the tile's copies were
      // issued.
      if constexpr (STAGE) {
        if (use_q0) {
#pragma unroll
          for (int k = 0; k < NQ; ++k) q0r[k] = ld_stream(C.q0 + base + t + NQ2 * k);
        }
      }
      // ---- Phase 2: face fluxes -------------------------------------------
      // Thread t is node t of every x/y face: x node (j,k) = (a,b) at
      // Nq*b + a of the x arrays, y node (i,k) = (a,b) at t of the pairs.
      if constexpr (XSPLIT) {
        const int xn = NQ * b + a;
        const V2 m1 = ypair[t], m3 = ypair[NQ2 + t];
        const TC f1 = upwind_flux<AR, TC>(m1.x, m1.y, qP[0], unP[0], TC(-1), sfs[0]);
        const TC f3 = upwind_flux<AR, TC>(m3.x, m3.y, qP[2], unP[2], TC(1), sfs[2]);
        const TC f2 = upwind_flux<AR, TC>(xq[xn], xu[xn], qP[1], unP[1], TC(1), sfs[1]);
        const TC f4 = upwind_flux<AR, TC>(xq[FA::XOFF + xn], xu[FA::XOFF + xn], qP[3],
                                          unP[3], TC(-1), sfs[3]);
        // The fluxes go to the two y pairs of node t, which only this thread
        // reads in this phase: (f1, f3) for the y faces, (f2, f4) for the x
        // faces, one 16-byte read each per node in the epilogue.
        ypair[t] = V2{f1, f3};
        ypair[NQ2 + t] = V2{f2, f4};
      } else {
        // Fluxes as two pairs in the slots of faces 1 and 2 of node t (only
        // this thread reads node t's minus sides in this phase): (f1, f3)
        // for the y faces, (f2, f4) for the x faces.
        TC fl[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          const TC sg = (f == 0 || f == 3) ? TC(-1) : TC(1);
          const V2 m = fM[FA::block(f) + t];
          fl[f] = upwind_flux<AR, TC>(m.x, m.y, qP[f], unP[f], sg, sfs[f]);
        }
        fM[t] = V2{fl[0], fl[2]};
        fM[NQ2 + t] = V2{fl[1], fl[3]};
        qlo = static_cast<TC>(sq[t]);
        qhi = static_cast<TC>(sq[t + NQ2 * (NQ - 1)]);
      }
      f5 = upwind_flux<AR, TC>(qlo, wlo, qZ[0], wZ[0], TC(-1), sfs[4]);
      f6 = upwind_flux<AR, TC>(qhi, whi, qZ[1], wZ[1], TC(1), sfs[5]);
    }
    __syncthreads();

    if (active) {
      // ---- Phase 4: z-derivative, lift, combine, store ---------------------
      const TC e1 = ses[0], e2 = ses[1], e3 = ses[2];
      // This column's entry of the x/y results at node k.
      auto xres = [&](int k) -> TC {
        if constexpr (TENSOR) return sX[TensorIdx8::qx(a, b) + NQ2 * k];
        else return sX[LI::colx(a, b, k)];
      };
      auto yres = [&](int k) -> TC {
        if constexpr (TENSOR) return sY[TensorIdx8::qy(a, b) + NQ2 * k];
        else return sY[LI::coly(a, b, k)];
      };
      TC lxy[4];
      if constexpr (!EXACT) {
        lxy[0] = sL[b];
        lxy[1] = sL[NQ + a];
        lxy[2] = sL[2 * NQ + b];
        lxy[3] = sL[3 * NQ + a];
      }
      TC fz[NQ];
#pragma unroll
      for (int l = 0; l < NQ; ++l) fz[l] = sz[t + NQ2 * l];
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
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
          for (int f = 0; f < 6; ++f) L[f] = ldro(A.lift + t + NQ2 * k + NP * f);
        }
        // tensorprod_Lift_hexahedral (kern:278-283): face order 1..6; the
        // x/y face fluxes as (f1, f3) at (i,k) = (a,k) and (f2, f4) at
        // (j,k) = (b,k).
        const V2* fp = XSPLIT ? ypair : fM;
        const V2 f13 = fp[a + NQ * k];
        const V2 f24 = fp[NQ2 + b + NQ * k];
        const TC fl1 = f13.x, fl3 = f13.y, fl2 = f24.x, fl4 = f24.y;
        TC lf = AR::mul(L[0], fl1);
        lf = AR::mad(L[1], fl2, lf);
        lf = AR::mad(L[2], fl3, lf);
        lf = AR::mad(L[3], fl4, lf);
        lf = AR::mad(L[4], f5, lf);
        lf = AR::mad(L[5], f6, lf);
        // dqdt = -(Escale1*DxF + Escale2*DyF + Escale3*DzF + Lift), eq:194-198.
        TC acc = AR::mul(e1, xres(k));
        acc = AR::mad(e2, yres(k), acc);
        acc = AR::mad(e3, dz, acc);
        acc = AR::add(acc, lf);
        const TC dqdt = -acc;
        const long n = base + t + NQ2 * k;
        if constexpr (!STAGE) {
          C.out[n] = static_cast<TO>(dqdt);
        } else {
          // q = rk_a*q0 + rk_b*(q + dt*dqdt), main.f90:70-71, in FP64, with
          // the stage input at its stored precision from the ring slot.
          using AD = Ar<double, EXACT>;
          const double qd = static_cast<double>(sq[t + NQ2 * k]);
          double r = AD::mul(A.rk_b, AD::mad(C.dt, static_cast<double>(dqdt), qd));
          if (use_q0) r = AD::mad(A.rk_a, q0r[k], r);
          C.out[n] = static_cast<TO>(r);
        }
      }
    }
  }
  if constexpr (TCG) {
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc(tmem);
  }
}

}  // namespace sdg
