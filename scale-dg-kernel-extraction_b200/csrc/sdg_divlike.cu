// Sum-factorised derivative operators on device arrays, for fields other than
// the advected q:
//
//   sdg_divlike_dev   element_operation_kernel_matvec_divlike_dirXYZ_var5_P<p>
//                     (mod_dg_optr_kernel_opt1.F90.erb:347-465): the x-, y-
//                     and z-derivatives of nvar fields per element, each
//                     direction from its own input (the flux components of a
//                     system, five for the Euler equations), three outputs;
//   sdg_gradlike_dev  element_operation_kernel_matvec_gradlike_dirXYZ_P<p>
//                     (erb:166-219): the three derivatives of one field.
//
// Both are the contraction of the advection kernel (tensorprod_divlike_dirXYZ,
// mod_dg_optr_kernel.f90:197-258, erb:228-344) without the flux, lift and
// combine: out_x(i,j,k) = sum_l D(i,l) in_x(l,j,k), out_y(i,j,k) =
// sum_l in_y(i,l,k) D(j,l), out_z(i,j,k) = sum_l in_z(i,j,l) D(k,l), in the
// OPT1 summation order (left to right for p <= 7, three partial sums split
// at np_div3 for p > 7) or, in exact mode on request, the GENERAL order.
// They compute what those reference routines are written to compute.  Two
// index slips in the reference text are not reproduced: the var5 y output
// index jkv = j + (kv-1)*np*5 (erb:400) runs past vec_out_y(np, np^2*5) for
// kv >= 3 (the intended jkv = j + (kv-1)*np is used), and the gradlike
// z-derivative's first term reads vec_in(i,1,k)*Mat_tr(1,j) (erb:209) where
// every other term reads vec_in(i,j,kk)*Mat_tr(kk,k) (the latter is used).
//
// Layout: element e, field v of nvar, node n = i + Nq*j + Nq^2*k (0-based)
// at n + Np*(v + nvar*e), as vec_in_x(np, np^2*5) of the reference holds the
// five fields of one element back to back.  One (element, field) pair is a
// unit of Np nodes; a block takes EPB units with Nq^2 threads each (the
// thread mapping of the tendency kernel).  Thread (a,b) of a unit loads its
// z-column of the three inputs (coalesced over a warp), keeps the z input in
// registers and puts the x and y inputs into shared line buffers in the
// layouts of the tendency kernel (LineIdx, conflict-free at p = 3, 5-9);
// after a barrier it contracts its x-line (j,k) = (a,b) and y-line
// (i,k) = (a,b) in place and its z-column in registers (at some orders the
// z-column first, before the barrier), and after a second barrier it stores
// its x and y output columns.  No scratch, no
// atomics: every unit reads and writes only its own Np nodes.
#include <cuda_runtime.h>

#include "sdg_gpu.h"
#include "sdg_internal.h"
#include "sdg_launch.h"
#include "sdg_tend.cuh"
#include "sdg_tend_pipe.cuh"

namespace sdg {
namespace {

template <int NQ, bool EXACT, int ORDER, bool ONE>
__global__ void __launch_bounds__((Geo<NQ>::THREADS + 31) / 32 * 32)
    derivative_kernel(const double* __restrict__ ix, const double* __restrict__ iy,
                      const double* __restrict__ iz, double* __restrict__ ox,
                      double* __restrict__ oy, double* __restrict__ oz, long long units,
                      const __grid_constant__ DMat<NQ, double> D) {
  using G = Geo<NQ>;
  using LI = LineIdx<NQ, 8>;
  using AR = Ar<double, EXACT>;
  constexpr int NQ2 = G::NQ2;
  constexpr int NP = G::NP;
  extern __shared__ __align__(16) double line_smem[];

  const int s = threadIdx.x / NQ2;  // unit slot of the block
  const int t = threadIdx.x - s * NQ2;
  const int a = t % NQ;
  const int b = t / NQ;
  const long long u = static_cast<long long>(blockIdx.x) * G::EPB + s;
  const bool active = s < G::EPB && u < units;
  double* sX = line_smem + s * 2 * LI::SIZE;
  double* sY = sX + LI::SIZE;
  const long long base = u * NP + t;

  // Column (a,b) of the three inputs; with one input for all three
  // directions (gradlike) it is read once.  The z-derivative needs only this
  // thread's column.  Where registers are tight it is done before the
  // barrier, so that the column leaves the registers before the line
  // contractions; elsewhere after the lines, which hides the column loads
  // behind the barrier.  Measured per order (G values/s, early / late z):
  // gradlike p = 8 149 / 126, p = 9 148 / 118; both operators p = 10-12
  // 109-146 / 93-133; five fields p = 7 125 / 144, p = 8 115 / 125, p = 9
  // 112 / 119; both p = 14 76-81 / 135-155.
  constexpr bool EARLYZ = (NQ >= 11 && NQ <= 13) || (ONE && (NQ == 9 || NQ == 10));
  auto zderiv = [&](const double (&col)[NQ]) {
    // Z-dir (erb:430-463): vec_in_z(i,j,l) * Mat_tr(l,k), stored straight
    // from registers (coalesced over the warp).
#pragma unroll
    for (int k = 0; k < NQ; ++k)
      oz[base + NQ2 * k] = contract<NQ, ORDER, AR, double>(
          [&](int l) { return col[l]; }, [&](int l) { return D.d[k * NQ + l]; });
  };
  double col[NQ];
  if (active) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      const double xv = ldro(ix + base + NQ2 * k);
      sX[LI::colx(a, b, k)] = xv;
      sY[LI::coly(a, b, k)] = ONE ? xv : ldro(iy + base + NQ2 * k);
      col[k] = ONE ? xv : ldro(iz + base + NQ2 * k);
    }
    if constexpr (EARLYZ) zderiv(col);
  }
  __syncthreads();
  if (active) {
    double line[NQ];
    const int lbx = LI::xl_base(a, b), lby = LI::yl_base(a, b);
    // X-dir (erb:366-394): Mat(i,l) * vec_in_x(l,jk)
#pragma unroll
    for (int l = 0; l < NQ; ++l) line[l] = sX[LI::xl(lbx, l)];
#pragma unroll
    for (int i = 0; i < NQ; ++i)
      sX[LI::xl(lbx, i)] = contract<NQ, ORDER, AR, double>(
          [&](int l) { return D.d[i * NQ + l]; }, [&](int l) { return line[l]; });
    // Y-dir (erb:397-427): vec_in_y(i,l,k) * Mat_tr(l,j)
#pragma unroll
    for (int l = 0; l < NQ; ++l) line[l] = sY[LI::yl(lby, l)];
#pragma unroll
    for (int j = 0; j < NQ; ++j)
      sY[LI::yl(lby, j)] = contract<NQ, ORDER, AR, double>(
          [&](int l) { return line[l]; }, [&](int l) { return D.d[j * NQ + l]; });
    if constexpr (!EARLYZ) zderiv(col);
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      ox[base + NQ2 * k] = sX[LI::colx(a, b, k)];
      oy[base + NQ2 * k] = sY[LI::coly(a, b, k)];
    }
  }
}

struct DerivCall {
  const double* ix;
  const double* iy;
  const double* iz;
  double* ox;
  double* oy;
  double* oz;
  long long units;
  const double* D1D;  // column-major (Nq,Nq), as read from operator_data
  cudaStream_t stream;
};

template <int NQ, bool EXACT, int ORDER, bool ONE>
int launch_derivative(const DerivCall& c) {
  using G = Geo<NQ>;
  auto kern = derivative_kernel<NQ, EXACT, ORDER, ONE>;
  const size_t smem = sizeof(double) * 2 * LineIdx<NQ, 8>::SIZE * G::EPB;
  static DeviceSetup setup;  // per instantiation and device
  const int dev = setup_device();
  if (dev < 0) return fail(SDG_ERR_CUDA, "derivative: no usable current device");
  if (setup.slot[dev].load(std::memory_order_relaxed) == 0) {
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem));
      if (e != cudaSuccess)
        return fail(SDG_ERR_CUDA, "derivative kernel set-up failed: %s", cudaGetErrorString(e));
    }
    setup.slot[dev].store(1, std::memory_order_relaxed);
  }
  if (c.units <= 0) return SDG_OK;
  DMat<NQ, double> d;
  for (int i = 0; i < NQ; ++i)
    for (int l = 0; l < NQ; ++l) d.d[i * NQ + l] = c.D1D[i + NQ * l];  // D(i,l)
  for (int i = 0; i < 2 * NQ; ++i) d.lz[i] = 0.0;
  const long long blocks = (c.units + G::EPB - 1) / G::EPB;
  if (blocks > 0x7fffffffLL) return fail(SDG_ERR_ARG, "derivative: too many elements");
  kern<<<static_cast<unsigned>(blocks), G::THREADS, smem, c.stream>>>(c.ix, c.iy, c.iz, c.ox,
                                                                      c.oy, c.oz, c.units, d);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(SDG_ERR_CUDA, "derivative kernel launch failed: %s", cudaGetErrorString(e));
  return SDG_OK;
}

template <int NQ>
int dispatch_order(const DerivCall& c, int flags, bool one) {
  const bool exact = flags & SDG_FLAG_EXACT;
  const bool general = flags & SDG_FLAG_ORDER_GENERAL;
  if (!exact) {
    return one ? launch_derivative<NQ, false, kOrderOpt1, true>(c)
               : launch_derivative<NQ, false, kOrderOpt1, false>(c);
  }
  if (general)
    return one ? launch_derivative<NQ, true, kOrderGeneral, true>(c)
               : launch_derivative<NQ, true, kOrderGeneral, false>(c);
  return one ? launch_derivative<NQ, true, kOrderOpt1, true>(c)
             : launch_derivative<NQ, true, kOrderOpt1, false>(c);
}

int dispatch(int Nq, const DerivCall& c, int flags, bool one) {
  switch (Nq) {
    case 2: return dispatch_order<2>(c, flags, one);
    case 3: return dispatch_order<3>(c, flags, one);
    case 4: return dispatch_order<4>(c, flags, one);
    case 5: return dispatch_order<5>(c, flags, one);
    case 6: return dispatch_order<6>(c, flags, one);
    case 7: return dispatch_order<7>(c, flags, one);
    case 8: return dispatch_order<8>(c, flags, one);
    case 9: return dispatch_order<9>(c, flags, one);
    case 10: return dispatch_order<10>(c, flags, one);
    case 11: return dispatch_order<11>(c, flags, one);
    case 12: return dispatch_order<12>(c, flags, one);
    case 13: return dispatch_order<13>(c, flags, one);
    case 14: return dispatch_order<14>(c, flags, one);
    case 15: return dispatch_order<15>(c, flags, one);
    case 16: return dispatch_order<16>(c, flags, one);
    default: return fail(SDG_ERR_ARG, "derivative: Nq must be 2..16 (p = 1..15), got %d", Nq);
  }
}

int check_common(const char* who, int Nq, long long Ne, const double* D1D, int flags) {
  if (Nq < 2 || Nq > 16) return fail(SDG_ERR_ARG, "%s: Nq must be 2..16, got %d", who, Nq);
  if (Ne < 0) return fail(SDG_ERR_ARG, "%s: Ne must be >= 0", who);
  if (!D1D) return fail(SDG_ERR_ARG, "%s: null D1D", who);
  if (flags & ~(SDG_FLAG_EXACT | SDG_FLAG_ORDER_GENERAL))
    return fail(SDG_ERR_ARG, "%s: flags may hold only SDG_FLAG_EXACT and SDG_FLAG_ORDER_GENERAL",
                who);
  if ((flags & SDG_FLAG_ORDER_GENERAL) && !(flags & SDG_FLAG_EXACT))
    return fail(SDG_ERR_ARG, "%s: SDG_FLAG_ORDER_GENERAL needs SDG_FLAG_EXACT", who);
  return SDG_OK;
}

}  // namespace
}  // namespace sdg

extern "C" int sdg_divlike_dev(int Nq, int nvar, long long Ne, const double* D1D,
                               const double* in_x, const double* in_y, const double* in_z,
                               double* out_x, double* out_y, double* out_z, int flags,
                               void* stream) {
  int rc = sdg::check_common("sdg_divlike_dev", Nq, Ne, D1D, flags);
  if (rc) return rc;
  if (nvar < 1) return sdg::fail(SDG_ERR_ARG, "sdg_divlike_dev: nvar must be >= 1");
  if (Ne > 0 && (!in_x || !in_y || !in_z || !out_x || !out_y || !out_z))
    return sdg::fail(SDG_ERR_ARG, "sdg_divlike_dev: null array");
  sdg::DerivCall c{in_x, in_y, in_z, out_x, out_y, out_z, Ne * nvar, D1D,
                   static_cast<cudaStream_t>(stream)};
  return sdg::dispatch(Nq, c, flags, in_x == in_y && in_y == in_z);
}

extern "C" int sdg_gradlike_dev(int Nq, long long Ne, const double* D1D, const double* in,
                                double* out_x, double* out_y, double* out_z, int flags,
                                void* stream) {
  int rc = sdg::check_common("sdg_gradlike_dev", Nq, Ne, D1D, flags);
  if (rc) return rc;
  if (Ne > 0 && (!in || !out_x || !out_y || !out_z))
    return sdg::fail(SDG_ERR_ARG, "sdg_gradlike_dev: null array");
  sdg::DerivCall c{in, in, in, out_x, out_y, out_z, Ne, D1D, static_cast<cudaStream_t>(stream)};
  return sdg::dispatch(Nq, c, flags, true);
}
