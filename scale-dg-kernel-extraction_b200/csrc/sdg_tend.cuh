// Fused DG advection tendency / RK-stage kernel for sm_100a.
//
// One kernel computes, per hexahedral element, everything that
// advect3d_eq_cal_tend (mod_advect3d_eq.f90:41-85) computes in two OpenMP
// passes, and optionally the SSP-RK3 stage update of main.f90:69-73:
//
//   * the upwind face flux over the six faces (cal_elembnd_flux,
//     mod_advect3d_eq.f90:116-140), with the minus side read from the
//     element itself and the plus side gathered from the neighbour (or from
//     the packed halo buffer, exactly where VMapP points);
//   * the volume fluxes q*u, q*v, q*w and the sum-factorised derivative
//     along x, y and z (tensorprod_divlike_dirXYZ, mod_dg_optr_kernel.f90
//     :197-258 and mod_dg_optr_kernel_opt1.F90.erb:228-344);
//   * the lift of the face flux (tensorprod_Lift_hexahedral,
//     mod_dg_optr_kernel.f90:262-288);
//   * dqdt = -(Escale . D F + Lift) (mod_advect3d_eq.f90:194-198), written
//     out, or folded into q_new = a*q0 + b*(q + dt*dqdt).
//
// No ebnd_flux array is materialised: face fluxes live in shared memory.
//
// Thread mapping.  An element of NQ^3 nodes is handled by NQ^2 threads; a
// block holds EPB elements.  Thread t = a + NQ*b of an element plays four
// roles in turn:
//   column   (i,j) = (a,b): owns the z-line of q and q*w in registers, does
//                           the z-derivative and the final combine;
//   x-line   (j,k) = (a,b): contracts one x-line of q*u held in shared memory;
//   y-line   (i,k) = (a,b): contracts one y-line of q*v;
//   face     fp = t       : evaluates the flux at face node fp of the four
//                           x/y faces.  The two z-faces are evaluated by the
//                           column threads from registers.
// Shared-memory rows are padded (row stride NQ+1 for even NQ) so that the
// line, column and face accesses of a half-warp fall in distinct banks.
//
// The 1-D differentiation matrix travels as a kernel parameter, so the
// unrolled contractions read it from the parameter constant bank with
// compile-time offsets.  The lift matrix (NQ^3 x 6) is read through the
// read-only path; it stays cache-resident.
//
// Arithmetic policy EXACT=true rounds every product and sum separately
// (__dmul_rn/__dadd_rn: no FMA contraction) in the reference's order, so the
// result is bit-for-bit the reference's x86-64 result.  EXACT=false uses FMA
// chains (same order, one rounding fewer per term).  ORDER selects the
// summation of the contractions for NQ > 8: the OPT1 three-partial-sum split
// (erb:242-274) or the sequential GENERAL loop.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sdg_launch.h"

namespace sdg {

// ---------------------------------------------------------------------------
// Arithmetic policies
// ---------------------------------------------------------------------------
template <typename T, bool EXACT>
struct Ar;

template <>
struct Ar<double, true> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  // t + a*b with two roundings, in that order.
  static __device__ __forceinline__ double mad(double a, double b, double t) {
    return __dadd_rn(t, __dmul_rn(a, b));
  }
};
// The fast policies fuse exactly where `mad` is written and nowhere else
// (the _rn intrinsics keep the compiler from contracting on its own), so
// every kernel variant computes bit-identical results.
template <>
struct Ar<double, false> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mad(double a, double b, double t) { return fma(a, b, t); }
};
template <>
struct Ar<float, true> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mad(float a, float b, float t) {
    return __fadd_rn(t, __fmul_rn(a, b));
  }
};
template <>
struct Ar<float, false> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mad(float a, float b, float t) { return fmaf(a, b, t); }
};

// ---------------------------------------------------------------------------
// Geometry of one element and of a block
// ---------------------------------------------------------------------------
template <int NQ>
struct Geo {
  static constexpr int NQ2 = NQ * NQ;
  static constexpr int NP = NQ2 * NQ;
  // Padded shared-memory row and plane strides.
  static constexpr int RS = (NQ % 2 == 0) ? NQ + 1 : NQ;
  static constexpr int PS = RS * NQ;
  static constexpr int SBUF = PS * NQ;
  // Elements per block: about 128 threads, at least one element.
  static constexpr int EPB = (NQ2 >= 128) ? 1 : (128 / NQ2);
  static constexpr int THREADS = EPB * NQ2;
  // np_div3 of mod_dg_optr_kernel_opt1.F90.erb:43 for NQ > 8.
  static constexpr int N3 = (NQ + 1) / 3;
};

template <int NQ, typename TC>
struct SmemLayout {
  using G = Geo<NQ>;
  // Per element: x-line buffer, y-line buffer, 4 faces x (q_minus, un_minus).
  // The face flux overwrites q_minus in place.
  static constexpr int PER_ELEM = 2 * G::SBUF + 8 * G::NQ2;
  static constexpr size_t BYTES = sizeof(TC) * PER_ELEM * G::EPB;
};

// The 1-D differentiation matrix D(i,l) = D1D(i,l), row-major, by value.
template <int NQ, typename TC>
struct DMat {
  TC d[NQ * NQ];
  TC lz[2 * NQ];  // z-face lift factors (-z, +z) of the factored fast lift
};

// Sum_{l} A(l)*B(l) in the reference's order (see header comment).
template <int NQ, int ORDER, typename AR, typename T, typename FA, typename FB>
__device__ __forceinline__ T contract(FA A, FB B) {
  if constexpr (NQ <= 8 || ORDER == kOrderGeneral) {
    T t = AR::mul(A(0), B(0));
#pragma unroll
    for (int l = 1; l < NQ; ++l) t = AR::mad(A(l), B(l), t);
    return t;
  } else {
    constexpr int N3 = Geo<NQ>::N3;
    T t1 = AR::mul(A(0), B(0));
#pragma unroll
    for (int l = 1; l < N3; ++l) t1 = AR::mad(A(l), B(l), t1);
    T t2 = AR::mul(A(N3), B(N3));
#pragma unroll
    for (int l = N3 + 1; l < 2 * N3; ++l) t2 = AR::mad(A(l), B(l), t2);
    T t3 = AR::mul(A(2 * N3), B(2 * N3));
#pragma unroll
    for (int l = 2 * N3 + 1; l < NQ; ++l) t3 = AR::mad(A(l), B(l), t3);
    return AR::add(AR::add(t1, t2), t3);
  }
}

// Orders (NQ = p + 1) whose fast FP32 kernels advance the x and y lines of a
// thread together with packed FMAs (contract2).  Measured per order on the
// pipelined kernel (G DOF-updates/s, paired vs scalar): p = 3 104.2 / 102.5,
// p = 7 146.7 / 140.7, p = 10 128.5 / 121.2, p = 11 111.4 / 102.3, p = 12
// 119.9 / 99.4; slower at p = 4, 5, 8 (101.5 / 106.0, 106.7 / 114.1,
// 109.1 / 118.7), where the wider live range costs a resident block.
template <int NQ>
constexpr bool kPairedLinesPipe = NQ == 4 || NQ == 8 || NQ >= 11;
// The one-tile-per-block kernel, which the fast FP32 forms run at p >= 13:
// p = 13 78.2 / 63.5, p = 14 81.9 / 78.1, p = 15 92.7 / 86.9.
template <int NQ>
constexpr bool kPairedLinesBlock = NQ >= 14;

// Two fast FP32 contractions in one: component c of the result is
// contract<NQ, ORDER, Ar<float, false>, float>(A, B_c), step for step, where
// A(l) is shared and B(l) holds both second factors.  The packed sm_100
// instructions (__ffma2_rn, __fmul2_rn, __fadd2_rn) round each component
// exactly as the scalar fmaf/__fmul_rn/__fadd_rn, so the results are the
// scalar contraction's bits at half the instructions.
template <int NQ, int ORDER, typename FA, typename FB>
__device__ __forceinline__ float2 contract2(FA A, FB B) {
  auto dup = [](float x) { return make_float2(x, x); };
  if constexpr (NQ <= 8 || ORDER == kOrderGeneral) {
    float2 t = __fmul2_rn(dup(A(0)), B(0));
#pragma unroll
    for (int l = 1; l < NQ; ++l) t = __ffma2_rn(dup(A(l)), B(l), t);
    return t;
  } else {
    constexpr int N3 = Geo<NQ>::N3;
    float2 t1 = __fmul2_rn(dup(A(0)), B(0));
#pragma unroll
    for (int l = 1; l < N3; ++l) t1 = __ffma2_rn(dup(A(l)), B(l), t1);
    float2 t2 = __fmul2_rn(dup(A(N3)), B(N3));
#pragma unroll
    for (int l = N3 + 1; l < 2 * N3; ++l) t2 = __ffma2_rn(dup(A(l)), B(l), t2);
    float2 t3 = __fmul2_rn(dup(A(2 * N3)), B(2 * N3));
#pragma unroll
    for (int l = 2 * N3 + 1; l < NQ; ++l) t3 = __ffma2_rn(dup(A(l)), B(l), t3);
    return __fadd2_rn(__fadd2_rn(t1, t2), t3);
  }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core line contractions (fast FP64 kernels, Nq = 8)
// ---------------------------------------------------------------------------
// The x- and y-derivatives of an element are the 8x8-by-8x64 products
// D * F_x and D * F_y (over the 64 lines of each direction).  The fast FP64
// kernels at Nq = 8 compute them with mma.sync m8n8k4 (DMMA): one 8x8 output
// tile = one k-plane of the element, two chained k-steps (l = 0..3, then
// 4..7).  A DMMA does 256 FMAs in one warp instruction where the DFMA form
// needs 32 per instruction, at the same FP64 peak.  Fragments (PTX ISA,
// m8n8k4 .f64): lane L holds A(L>>2, L&3), B(L&3, L>>2) and
// C(L>>2, 2(L&3) + {0,1}).  Every kernel variant uses this same sequence,
// so their fast FP64 results stay bit-identical.
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b,
                                            double c0, double c1) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%4,%5};"
      : "=d"(d0), "=d"(d1)
      : "d"(a), "d"(b), "d"(c0), "d"(c1));
}

// This lane's A fragments of D for the two k-steps: D(L>>2, 4s + (L&3)).
template <typename DM>
__device__ __forceinline__ void dmma_dfrag(const DM& D, double* a0, double* a1) {
  const int lane = threadIdx.x & 31;
  *a0 = D.d[(lane >> 2) * 8 + (lane & 3)];
  *a1 = D.d[(lane >> 2) * 8 + 4 + (lane & 3)];
}

// The kernels that contract x- and y-lines on the tensor cores.
template <int NQ, typename TC, bool EXACT>
constexpr bool kTensorLines = (NQ == 8) && !EXACT && sizeof(TC) == 8;

// One 8x8 output tile: d = D * B, with this lane's B fragments b0 = B(L&3,
// L>>2) and b1 = B(4 + (L&3), L>>2).
__device__ __forceinline__ void dmma_tile8(double a0, double a1, double b0, double b1,
                                           double* d0, double* d1) {
  double c0, c1;
  dmma_m8n8k4(c0, c1, a0, b0, 0.0, 0.0);
  dmma_m8n8k4(*d0, *d1, a1, b1, c0, c1);
}

// Bulk prefetch of a global range into L2 (TMA engine); addr and bytes are
// multiples of 16.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes)
               : "memory");
}

// Prefetch of bytes [lo, hi) of an array into L2, shrunk to whole 16-byte
// words inside the range (so it never touches a byte outside it).
__device__ __forceinline__ void prefetch_l2_range(const void* base, size_t lo, size_t hi) {
  const uintptr_t b = reinterpret_cast<uintptr_t>(base);
  const uintptr_t a0 = (b + lo + 15) & ~uintptr_t(15);
  const uintptr_t a1 = (b + hi) & ~uintptr_t(15);
  if (a1 > a0) bulk_prefetch_l2(reinterpret_cast<const void*>(a0), static_cast<uint32_t>(a1 - a0));
}

__device__ __forceinline__ double absv(double x) { return fabs(x); }
__device__ __forceinline__ float absv(float x) { return fabsf(x); }

// Upwind flux of mod_advect3d_eq.f90:134-139 with an axis-aligned normal of
// sign sg: Vel = sg*u_n exactly (the other normal components are zero).
template <typename AR, typename T>
__device__ __forceinline__ T upwind_flux(T qM, T unM, T qP, T unP, T sg,
                                         T fscale) {
  const T velM = AR::mul(unM, sg);
  const T velP = AR::mul(unP, sg);
  const T alpha = AR::mul(T(0.5), absv(AR::add(velP, velM)));
  const T jump = AR::sub(AR::sub(AR::mul(qP, velP), AR::mul(qM, velM)),
                         AR::mul(alpha, AR::sub(qP, qM)));
  return AR::mul(AR::mul(T(0.5), fscale), jump);
}

template <typename T>
__device__ __forceinline__ T ldro(const T* p) {
  return __ldg(p);
}

// ---------------------------------------------------------------------------
// Kernel arguments
// ---------------------------------------------------------------------------
// Face-neighbour table pbase(f, e), f = 0..5 (reference faces 1..6):
//   >= 0 : 0-based first node of the neighbour element; the plus-side node
//          of face node fp is pbase + Fmask(fp, oppface) - 1;
//   <  0 : halo face; the plus-side nodes are contiguous from -1 - pbase.
template <typename TQ, typename TV, typename TO, typename TC>
struct TendArgs {
  const TQ* q;          // state read by the tendency, (Np, NeA)
  const TV* u;          // velocity, (Np, NeA)
  const TV* v;
  const TV* w;
  const double* q0;     // RK base state (stage mode, a != 0), (Np, Ne)
  TO* out;              // dqdt (tendency mode) or q_new (stage mode)
  const TC* lift;       // Lift_mat(Np, 6)
  const int* pbase;     // (6, Ne)
  const TC* escale;     // (3, Ne)  per-element 2/dx, 2/dy, 2/dz
  const TC* fscale;     // (6, Ne)  per-face 2/d_perp
  int Ne;
  int elem0;            // first element of this launch
  int nelem;            // elements in this launch
  double rk_a, rk_b, dt;
  int* status;          // device status word: nonzero after a timed-out wait
  // Spin limit of each bounded wait of the pipelined kernel (try_wait
  // polls), and a test hook: when inject_skip = T + 1, tile T's bulk copies
  // are never issued, so the wait for them runs out (0: none).
  unsigned wait_spins;
  int inject_skip;
  // One-tile-per-block kernel: block b prefetches into L2 the inputs of
  // block b + prefetch_dist (about one resident wave ahead); 0 disables.
  int prefetch_dist;
  // Batched launches (pipelined kernel only): per-instance arrays and a
  // table of element tiles.  Null for a single instance, whose tiles are
  // the consecutive elements elem0 .. elem0+nelem-1 of the arrays above.
  const struct BatchInst* insts;
  const struct BatchTile* tiles;
  int ntiles;
};

// One ensemble instance of a batched launch.  Arrays have the single
// instance's layout; q, u, v, w and q0 hold at least Np*Ne elements plus 16
// bytes of slack (the bulk copies read whole 16-byte words).
struct BatchInst {
  const void* q;
  const void* u;
  const void* v;
  const void* w;
  const double* q0;
  void* out;
  const int* pbase;
  const void* escale;
  const void* fscale;
  double dt;
};

// A tile: up to EPB consecutive elements e0 .. e0+n-1 of instance `inst`.
struct BatchTile {
  int inst;
  int e0;
  int n;
  int pad;
};

// ---------------------------------------------------------------------------
// The kernel
// ---------------------------------------------------------------------------
// MINB is the minimum number of resident blocks per SM the build must allow
// (it caps registers per thread); 1 leaves the compiler free.
template <int NQ, typename TQ, typename TV, typename TO, typename TC,
          bool EXACT, int ORDER, bool STAGE, int MINB = 1>
__global__ void __launch_bounds__(Geo<NQ>::THREADS, MINB)
    tend_kernel(const __grid_constant__ TendArgs<TQ, TV, TO, TC> A,
                const __grid_constant__ DMat<NQ, TC> D) {
  using G = Geo<NQ>;
  using AR = Ar<TC, EXACT>;
  constexpr int NQ2 = G::NQ2;
  constexpr int RS = G::RS;
  constexpr int PS = G::PS;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  TC* smem = reinterpret_cast<TC*>(smem_raw);

  const int s = threadIdx.x / NQ2;           // element slot in the block
  const int t = threadIdx.x - s * NQ2;       // thread within the element
  const int a = t % NQ;
  const int b = t / NQ;
  const int el = blockIdx.x * G::EPB + s;    // element index within launch
  const bool active = el < A.nelem;
  const int e = A.elem0 + (active ? el : 0);
  const long base = static_cast<long>(e) * G::NP;

  TC* sX = smem + s * SmemLayout<NQ, TC>::PER_ELEM;
  TC* sY = sX + G::SBUF;
  TC* fQ = sY + G::SBUF;       // [4][NQ2] minus-side q on faces 1..4
  TC* fU = fQ + 4 * NQ2;       // [4][NQ2] minus-side normal velocity

  TC qc[NQ];                   // column of q
  TC fz[NQ];                   // column of q*w
  TC wlo = TC(0), whi = TC(0);

  // Blocks run in launch order, so the block one resident wave later starts
  // about when this one ends: bring its inputs into L2 now.
  if (A.prefetch_dist > 0 && threadIdx.x == 0) {
    const long nb = (static_cast<long>(A.nelem) + G::EPB - 1) / G::EPB;
    const long pblk = static_cast<long>(blockIdx.x) + A.prefetch_dist;
    if (pblk < nb) {
      const long e0 = A.elem0 + pblk * G::EPB;
      const long e1 = A.elem0 + min(static_cast<long>(A.nelem), (pblk + 1) * G::EPB);
      prefetch_l2_range(A.q, e0 * G::NP * sizeof(TQ), e1 * G::NP * sizeof(TQ));
      prefetch_l2_range(A.u, e0 * G::NP * sizeof(TV), e1 * G::NP * sizeof(TV));
      prefetch_l2_range(A.v, e0 * G::NP * sizeof(TV), e1 * G::NP * sizeof(TV));
      prefetch_l2_range(A.w, e0 * G::NP * sizeof(TV), e1 * G::NP * sizeof(TV));
      if (STAGE && A.rk_a != 0.0)
        prefetch_l2_range(A.q0, e0 * G::NP * sizeof(double), e1 * G::NP * sizeof(double));
    }
  }

  // The element's face-neighbour row, needed after phase 1: loaded first so
  // that phase 1 covers its latency and the gathers of phase 2 wait on one
  // load, not two in a chain.
  int pb[6];
  if (active) {
#pragma unroll
    for (int f = 0; f < 6; ++f) pb[f] = ldro(A.pbase + 6 * static_cast<long>(e) + f);
  }

  // ---- Phase 1: load the column, form the volume fluxes ------------------
  if (active) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      const long n = base + t + NQ2 * k;
      const TC qv = static_cast<TC>(A.q[n]);
      const TC uv = static_cast<TC>(A.u[n]);
      const TC vv = static_cast<TC>(A.v[n]);
      const TC wv = static_cast<TC>(A.w[n]);
      qc[k] = qv;
      sX[a + RS * b + PS * k] = AR::mul(qv, uv);   // flux_x = q*u
      sY[a + RS * b + PS * k] = AR::mul(qv, vv);   // flux_y = q*v
      fz[k] = AR::mul(qv, wv);                     // flux_z = q*w
      if (k == 0) wlo = wv;
      if (k == NQ - 1) whi = wv;
      // Minus-side face values of the x/y faces (face fp orders of
      // mod_mesh.f90:278-308): face 1 (-y, j=0) and 3 (+y) index (i,k),
      // faces 2 (+x) and 4 (-x, i=0) index (j,k).
      if (b == 0)      { fQ[0 * NQ2 + a + NQ * k] = qv; fU[0 * NQ2 + a + NQ * k] = vv; }
      if (a == NQ - 1) { fQ[1 * NQ2 + b + NQ * k] = qv; fU[1 * NQ2 + b + NQ * k] = uv; }
      if (b == NQ - 1) { fQ[2 * NQ2 + a + NQ * k] = qv; fU[2 * NQ2 + a + NQ * k] = vv; }
      if (a == 0)      { fQ[3 * NQ2 + b + NQ * k] = qv; fU[3 * NQ2 + b + NQ * k] = uv; }
    }
  }
  __syncthreads();

  TC f5 = TC(0), f6 = TC(0);
  if (active) {
    // ---- Phase 2a: flux on the x/y faces, face node fp = t ---------------
    const TC* fs = A.fscale + 6 * static_cast<long>(e);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const int p = pb[f];
      long idx;
      if (p >= 0) {
        // Plus-side node Fmask(fp, oppface) of the neighbour.
        const int off = (f == 0)   ? a + NQ * (NQ - 1) + NQ2 * b   // opp 3
                        : (f == 1) ? NQ * a + NQ2 * b              // opp 4
                        : (f == 2) ? a + NQ2 * b                   // opp 1
                                   : (NQ - 1) + NQ * a + NQ2 * b;  // opp 2
        idx = static_cast<long>(p) + off;
      } else {
        idx = static_cast<long>(-1 - p) + t;
      }
      const TC qP = static_cast<TC>(ldro(A.q + idx));
      const TC unP = static_cast<TC>((f == 1 || f == 3) ? ldro(A.u + idx)
                                                        : ldro(A.v + idx));
      const TC sg = (f == 0 || f == 3) ? TC(-1) : TC(1);
      const TC fsc = fs[f];
      fQ[f * NQ2 + t] =
          upwind_flux<AR, TC>(fQ[f * NQ2 + t], fU[f * NQ2 + t], qP, unP, sg, fsc);
    }
    // ---- Phase 2b: flux on the z faces from the column registers ---------
    {
      const int p5 = pb[4];
      const long i5 = (p5 >= 0) ? static_cast<long>(p5) + t + NQ2 * (NQ - 1)
                                : static_cast<long>(-1 - p5) + t;
      const TC q5 = static_cast<TC>(ldro(A.q + i5));
      const TC w5 = static_cast<TC>(ldro(A.w + i5));
      f5 = upwind_flux<AR, TC>(qc[0], wlo, q5, w5, TC(-1), fs[4]);
      const int p6 = pb[5];
      const long i6 = (p6 >= 0) ? static_cast<long>(p6) + t
                                : static_cast<long>(-1 - p6) + t;
      const TC q6 = static_cast<TC>(ldro(A.q + i6));
      const TC w6 = static_cast<TC>(ldro(A.w + i6));
      f6 = upwind_flux<AR, TC>(qc[NQ - 1], whi, q6, w6, TC(1), fs[5]);
    }
    // ---- Phase 3: x-line and y-line contractions, in place --------------
    if constexpr (kTensorLines<NQ, TC, EXACT>) {
      // DMMA tiles: the element's two warps take four k-planes each; a
      // plane is read and rewritten only by its warp.
      double a0, a1;
      dmma_dfrag(D, &a0, &a1);
      const int lane = threadIdx.x & 31, g = lane >> 2, qd = lane & 3;
      const int we = (t >> 5);  // warp of the element
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const int T = 4 * we + kk;
        double d0, d1;
        // x: B(l, j) = F_x(i = l, j, k = T); C(i, j) = DxF(i, j, T).
        dmma_tile8(a0, a1, sX[qd + RS * g + PS * T], sX[4 + qd + RS * g + PS * T], &d0, &d1);
        sX[g + RS * (2 * qd) + PS * T] = d0;
        sX[g + RS * (2 * qd + 1) + PS * T] = d1;
        // y: B(l, i) = F_y(i, j = l, k = T); C(j, i) = DyF(i, j, T).
        dmma_tile8(a0, a1, sY[g + RS * qd + PS * T], sY[g + RS * (4 + qd) + PS * T], &d0,
                   &d1);
        sY[2 * qd + RS * g + PS * T] = d0;
        sY[2 * qd + 1 + RS * g + PS * T] = d1;
      }
    } else if constexpr (sizeof(TC) == 4 && !EXACT && kPairedLinesBlock<NQ>) {
      // x line (a,b) and y line (a,b) share the coefficient row D(i, .).
      float2 ln[NQ];
#pragma unroll
      for (int l = 0; l < NQ; ++l)
        ln[l] = make_float2(sX[l + RS * a + PS * b], sY[a + RS * l + PS * b]);
#pragma unroll
      for (int i = 0; i < NQ; ++i) {
        const float2 r = contract2<NQ, ORDER>([&](int l) { return D.d[i * NQ + l]; },
                                              [&](int l) { return ln[l]; });
        sX[i + RS * a + PS * b] = r.x;
        sY[a + RS * i + PS * b] = r.y;
      }
    } else {
      TC line[NQ];
#pragma unroll
      for (int l = 0; l < NQ; ++l) line[l] = sX[l + RS * a + PS * b];
#pragma unroll
      for (int i = 0; i < NQ; ++i)
        sX[i + RS * a + PS * b] = contract<NQ, ORDER, AR, TC>(
            [&](int l) { return D.d[i * NQ + l]; },   // Mat(i,l)
            [&](int l) { return line[l]; });          // vec_in_x(l,jk)
#pragma unroll
      for (int l = 0; l < NQ; ++l) line[l] = sY[a + RS * l + PS * b];
#pragma unroll
      for (int j = 0; j < NQ; ++j)
        sY[a + RS * j + PS * b] = contract<NQ, ORDER, AR, TC>(
            [&](int l) { return line[l]; },           // vec_in_y(i,l,k)
            [&](int l) { return D.d[j * NQ + l]; });  // Mat_tr(l,j)
    }
  }
  __syncthreads();

  if (!active) return;

  // ---- Phase 4: z-derivative, lift and combine in the column thread -------
  // The z-derivative of node k is formed where it is used, so no column of
  // results is held in registers (it matters for the long columns of p > 10).
  auto dz = [&](int k) {
    return contract<NQ, ORDER, AR, TC>(
        [&](int l) { return fz[l]; },                 // vec_in_z(i,j,l)
        [&](int l) { return D.d[k * NQ + l]; });      // Mat_tr(l,k)
  };

  const TC* es = A.escale + 3 * static_cast<long>(e);
  const TC e1 = es[0], e2 = es[1], e3 = es[2];
  const TC* L = A.lift + t;
#pragma unroll
  for (int k = 0; k < NQ; ++k) {
    const int nk = NQ2 * k;
    // tensorprod_Lift_hexahedral (kern:278-283): face order 1..6.
    TC lf = AR::mul(ldro(L + nk + 0 * G::NP), fQ[0 * NQ2 + a + NQ * k]);
    lf = AR::mad(ldro(L + nk + 1 * G::NP), fQ[1 * NQ2 + b + NQ * k], lf);
    lf = AR::mad(ldro(L + nk + 2 * G::NP), fQ[2 * NQ2 + a + NQ * k], lf);
    lf = AR::mad(ldro(L + nk + 3 * G::NP), fQ[3 * NQ2 + b + NQ * k], lf);
    lf = AR::mad(ldro(L + nk + 4 * G::NP), f5, lf);
    lf = AR::mad(ldro(L + nk + 5 * G::NP), f6, lf);
    // dqdt = -(Escale1*DxF + Escale2*DyF + Escale3*DzF + Lift), eq:194-198.
    TC acc = AR::mul(e1, sX[a + RS * b + PS * k]);
    acc = AR::mad(e2, sY[a + RS * b + PS * k], acc);
    acc = AR::mad(e3, dz(k), acc);
    acc = AR::add(acc, lf);
    const TC dqdt = -acc;
    const long n = base + t + NQ2 * k;
    if constexpr (!STAGE) {
      A.out[n] = static_cast<TO>(dqdt);
    } else {
      // q = rk_a*q0 + rk_b*(q + dt*dqdt), main.f90:70-71, in FP64.
      using AD = Ar<double, EXACT>;
      // The stage input at its stored precision (re-read when the compute
      // type is narrower than the stored state).
      double qd;
      if constexpr (sizeof(TQ) == sizeof(TC)) qd = static_cast<double>(qc[k]);
      else qd = static_cast<double>(A.q[n]);
      double r = AD::mul(A.rk_b, AD::mad(A.dt, static_cast<double>(dqdt), qd));
      if (A.rk_a != 0.0) r = AD::mad(A.rk_a, A.q0[n], r);
      A.out[n] = static_cast<TO>(r);
    }
  }
}

}  // namespace sdg
