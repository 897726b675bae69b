// CPU oracle for the SCALE-DG 3D DG advection right-hand side.
//
// TEST INFRASTRUCTURE ONLY: a loop-for-loop C++/OpenMP restatement of the
// reference Fortran, used by the test-suite, the smoke check and the bench's
// CPU-baseline leg as the checker.  Nothing in the product links it.
// Built with -O3 -fopenmp -ffp-contract=off (see oracle/Makefile) so that
// products and sums round exactly as the reference's x86-64 gfortran build.
//
// Parity status: no reference binary can be built here (no Fortran
// compiler), so this restatement is pinned against golden vectors produced by
// mechanically translating and evaluating the reference's Fortran source, and
// by analytic known-answer tests.  See the header.
//
// Index conventions: arrays are Fortran column-major; a(i,j) with extents
// (n1,n2) lives at a[(i-1) + n1*(j-1)].  Maps hold 1-based values.

#include "sdg_oracle.h"

#include <omp.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

// mod_common.f90:25
const double kPI = 4.0 * std::atan(1.0);

// mod_common.f90:28-30
const double kRkA[3] = {0.0, 0.75, 1.0 / 3.0};
const double kRkB[3] = {1.0, 0.25, 2.0 / 3.0};

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Reads whitespace-separated reals the way a Fortran list-directed read of
// real(8) does for these files (plain E notation; D exponents accepted).
bool read_reals(FILE* f, double* out, long n) {
  char tok[128];
  for (long i = 0; i < n; ++i) {
    if (std::fscanf(f, "%127s", tok) != 1) return false;
    for (char* c = tok; *c; ++c)
      if (*c == 'D' || *c == 'd') *c = 'E';
    char* end = nullptr;
    out[i] = std::strtod(tok, &end);
    if (end == tok) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Tensor-product kernels.
// GENERAL: mod_dg_optr_kernel.f90:197-258 (accumulate from 0.0 in l order).
// OPT1:    mod_dg_optr_kernel_opt1.F90.erb:228-344 (left-to-right sum for
//          p<=7; for p>7 three partial sums split at np_div3, erb:43-44).
// ---------------------------------------------------------------------------

void divlike_general(double* ox, double* oy, double* oz, const double* Mat,
                     const double* Mat_tr, const double* ix, const double* iy,
                     const double* iz, int Nq) {
  const int Nq2 = Nq * Nq;
  const int Np = Nq2 * Nq;
  for (int n = 0; n < Np; ++n) {
    ox[n] = 0.0;
    oy[n] = 0.0;
    oz[n] = 0.0;
  }
  // x-direction, kern:221-230
  for (int jk = 0; jk < Nq2; ++jk)
    for (int i = 0; i < Nq; ++i)
      for (int l = 0; l < Nq; ++l)
        ox[i + Nq * jk] = ox[i + Nq * jk] + Mat[i + Nq * l] * ix[l + Nq * jk];
  // y-direction, kern:232-243
  for (int k = 0; k < Nq; ++k)
    for (int j = 0; j < Nq; ++j) {
      const int jk = j + k * Nq;
      for (int i = 0; i < Nq; ++i)
        for (int l = 0; l < Nq; ++l)
          oy[i + Nq * jk] =
              oy[i + Nq * jk] + iy[i + Nq * l + Nq2 * k] * Mat_tr[l + Nq * j];
    }
  // z-direction, kern:245-257
  for (int k = 0; k < Nq; ++k)
    for (int j = 0; j < Nq; ++j) {
      const int jk = j + k * Nq;
      for (int i = 0; i < Nq; ++i)
        for (int l = 0; l < Nq; ++l)
          oz[i + Nq * jk] =
              oz[i + Nq * jk] + iz[i + Nq * j + Nq2 * l] * Mat_tr[l + Nq * k];
    }
}

// One OPT1 contraction: terms t(l) = a(l)*b(l), l = 0..NQ-1, summed left to
// right (p<=7) or as ((sum 1..n3) + (sum n3+1..2n3)) + (sum 2n3+1..NQ).
template <int NQ>
inline double opt1_sum(const double* a, int sa, const double* b, int sb) {
  if (NQ <= 8) {
    double t = a[0] * b[0];
    for (int l = 1; l < NQ; ++l) t = t + a[l * sa] * b[l * sb];
    return t;
  } else {
    // np_div3 = ((p+1)/3.0).round (erb:43): Ruby rounds half away from
    // zero, and (NQ+1)/3 in integers equals it for NQ = 9..16.
    const int n3 = (NQ + 1) / 3;
    double t1 = a[0] * b[0];
    for (int l = 1; l < n3; ++l) t1 = t1 + a[l * sa] * b[l * sb];
    double t2 = a[n3 * sa] * b[n3 * sb];
    for (int l = n3 + 1; l < 2 * n3; ++l) t2 = t2 + a[l * sa] * b[l * sb];
    double t3 = a[2 * n3 * sa] * b[2 * n3 * sb];
    for (int l = 2 * n3 + 1; l < NQ; ++l) t3 = t3 + a[l * sa] * b[l * sb];
    return t1 + t2 + t3;
  }
}

template <int NQ>
void divlike_opt1(double* ox, double* oy, double* oz, const double* Mat,
                  const double* Mat_tr, const double* ix, const double* iy,
                  const double* iz) {
  constexpr int Nq2 = NQ * NQ;
  // X-dir (erb:249-276): Mat(i,l) * vec_in_x(l,jk)
  for (int jk = 0; jk < Nq2; ++jk)
    for (int i = 0; i < NQ; ++i)
      ox[i + NQ * jk] = opt1_sum<NQ>(Mat + i, NQ, ix + NQ * jk, 1);
  // Y-dir (erb:279-309): vec_in_y(i,l,k) * Mat_tr(l,j)
  for (int k = 0; k < NQ; ++k)
    for (int j = 0; j < NQ; ++j) {
      const int jk = j + NQ * k;
      for (int i = 0; i < NQ; ++i)
        oy[i + NQ * jk] =
            opt1_sum<NQ>(iy + i + Nq2 * k, NQ, Mat_tr + NQ * j, 1);
    }
  // Z-dir (erb:312-342): vec_in_z(i,j,l) * Mat_tr(l,k)
  for (int k = 0; k < NQ; ++k)
    for (int j = 0; j < NQ; ++j) {
      const int jk = j + NQ * k;
      for (int i = 0; i < NQ; ++i)
        oz[i + NQ * jk] = opt1_sum<NQ>(iz + i + NQ * j, Nq2, Mat_tr + NQ * k, 1);
    }
}

// tensorprod_Lift_hexahedral_general (kern:262-288); the OPT1 variant
// (erb:134-157) has the identical six-term expression.
void lift_hex(double* out, const double* Lift, const double* fin, int Nq) {
  const int Nq2 = Nq * Nq;
  const int Np = Nq2 * Nq;
  for (int k = 0; k < Nq; ++k)
    for (int j = 0; j < Nq; ++j)
      for (int i = 0; i < Nq; ++i) {
        const int n = i + Nq * j + Nq2 * k;
        out[n] = Lift[n + 0 * Np] * fin[i + Nq * k + 0 * Nq2] +
                 Lift[n + 1 * Np] * fin[j + Nq * k + 1 * Nq2] +
                 Lift[n + 2 * Np] * fin[i + Nq * k + 2 * Nq2] +
                 Lift[n + 3 * Np] * fin[j + Nq * k + 3 * Nq2] +
                 Lift[n + 4 * Np] * fin[i + Nq * j + 4 * Nq2] +
                 Lift[n + 5 * Np] * fin[i + Nq * j + 5 * Nq2];
      }
}

typedef void (*opt1_fn)(double*, double*, double*, const double*,
                        const double*, const double*, const double*,
                        const double*);

opt1_fn opt1_table(int Nq) {
  switch (Nq) {
    case 2: return divlike_opt1<2>;
    case 3: return divlike_opt1<3>;
    case 4: return divlike_opt1<4>;
    case 5: return divlike_opt1<5>;
    case 6: return divlike_opt1<6>;
    case 7: return divlike_opt1<7>;
    case 8: return divlike_opt1<8>;
    case 9: return divlike_opt1<9>;
    case 10: return divlike_opt1<10>;
    case 11: return divlike_opt1<11>;
    case 12: return divlike_opt1<12>;
    case 13: return divlike_opt1<13>;
    case 14: return divlike_opt1<14>;
    case 15: return divlike_opt1<15>;
    case 16: return divlike_opt1<16>;
    default: return nullptr;
  }
}

// cal_elembnd_flux, mod_advect3d_eq.f90:89-142
void cal_elembnd_flux(double* flux, const double* q_, const double* u_,
                      const double* v_, const double* w_, const int* VMapM,
                      const int* VMapP, const double* normal_fn,
                      const double* Fscale, int NfpTot, int Ne) {
  const long NN = static_cast<long>(NfpTot) * Ne;
#pragma omp parallel for schedule(static)
  for (int ke = 0; ke < Ne; ++ke) {
    const long b = static_cast<long>(NfpTot) * ke;
    for (int n = 0; n < NfpTot; ++n) {
      const long iM = VMapM[b + n] - 1;
      const long iP = VMapP[b + n] - 1;
      const double qM = q_[iM];
      const double qP = q_[iP];
      const double n1 = normal_fn[b + n];
      const double n2 = normal_fn[b + n + NN];
      const double n3 = normal_fn[b + n + 2 * NN];
      const double VelM = u_[iM] * n1 + v_[iM] * n2 + w_[iM] * n3;
      const double VelP = u_[iP] * n1 + v_[iP] * n2 + w_[iP] * n3;
      const double alpha = 0.5 * std::fabs(VelP + VelM);
      flux[b + n] = 0.5 * Fscale[b + n] *
                    (qP * VelP - qM * VelM - alpha * (qP - qM));
    }
  }
}

// cal_dqdt, mod_advect3d_eq.f90:146-201
void cal_dqdt(int evaltype, double* dqdt, const double* q, const double* u,
              const double* v, const double* w, const double* flux_bnd,
              const double* D1D, const double* D1D_tr, const double* Lift,
              const double* Escale, int Nq, int Np, int NfpTot, int Ne) {
  const long NE = static_cast<long>(Np) * Ne;
  opt1_fn opt1 = opt1_table(Nq);
#pragma omp parallel
  {
    std::vector<double> fx(Np), fy(Np), fz(Np), dx(Np), dy(Np), dz(Np),
        lift(Np);
#pragma omp for schedule(static)
    for (int ke = 0; ke < Ne; ++ke) {
      const long b = static_cast<long>(Np) * ke;
      for (int n = 0; n < Np; ++n) {
        fx[n] = q[b + n] * u[b + n];
        fy[n] = q[b + n] * v[b + n];
        fz[n] = q[b + n] * w[b + n];
      }
      if (evaltype == ORC_GENERAL)
        divlike_general(dx.data(), dy.data(), dz.data(), D1D, D1D_tr,
                        fx.data(), fy.data(), fz.data(), Nq);
      else
        opt1(dx.data(), dy.data(), dz.data(), D1D, D1D_tr, fx.data(),
             fy.data(), fz.data());
      lift_hex(lift.data(), Lift, flux_bnd + static_cast<long>(NfpTot) * ke,
               Nq);
      for (int n = 0; n < Np; ++n)
        dqdt[b + n] = -(Escale[b + n] * dx[n] + Escale[b + n + NE] * dy[n] +
                        Escale[b + n + 2 * NE] * dz[n] + lift[n]);
    }
  }
}

int elem_id(int i, int j, int k, int NeX, int NeY) {
  return i + (j - 1) * NeX + (k - 1) * NeX * NeY;
}

// eval_neighbor_element, mod_mesh.f90:407-483
void eval_neighbor_element(int i, int j, int k, int f, int NeX, int NeY,
                           int NeZ, int* keP, int* oppface, bool* is_bnd) {
  *is_bnd = false;
  switch (f) {
    case 1:
      *oppface = 3;
      if (j > 1) *keP = elem_id(i, j - 1, k, NeX, NeY);
      else { *keP = elem_id(i, NeY, k, NeX, NeY); *is_bnd = true; }
      break;
    case 2:
      *oppface = 4;
      if (i < NeX) *keP = elem_id(i + 1, j, k, NeX, NeY);
      else { *keP = elem_id(1, j, k, NeX, NeY); *is_bnd = true; }
      break;
    case 3:
      *oppface = 1;
      if (j < NeY) *keP = elem_id(i, j + 1, k, NeX, NeY);
      else { *keP = elem_id(i, 1, k, NeX, NeY); *is_bnd = true; }
      break;
    case 4:
      *oppface = 2;
      if (i > 1) *keP = elem_id(i - 1, j, k, NeX, NeY);
      else { *keP = elem_id(NeX, j, k, NeX, NeY); *is_bnd = true; }
      break;
    case 5:
      *oppface = 6;
      if (k > 1) *keP = elem_id(i, j, k - 1, NeX, NeY);
      else { *keP = elem_id(i, j, NeZ, NeX, NeY); *is_bnd = true; }
      break;
    case 6:
      *oppface = 5;
      if (k < NeZ) *keP = elem_id(i, j, k + 1, NeX, NeY);
      else { *keP = elem_id(i, j, 1, NeX, NeY); *is_bnd = true; }
      break;
  }
}

// splitmix64 stream for the seeded initial condition and velocities.
struct SplitMix {
  unsigned long long s;
  unsigned long long next() {
    s += 0x9E3779B97F4A7C15ULL;
    unsigned long long z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
  double normal() {
    const double u1 = 1.0 - uniform();
    const double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPI * u2);
  }
};

}  // namespace

extern "C" {

int orc_num_threads(void) { return omp_get_max_threads(); }

void orc_fmask(int Nq, int* Fmask) {
  // mod_mesh.f90:278-324; Fmask(fp,f) at Fmask[(fp-1) + Nfp*(f-1)].
  const int Nfp = Nq * Nq;
  const int Nq2 = Nq * Nq;
  int fp = 0;
  for (int k = 1; k <= Nq; ++k)
    for (int i = 1; i <= Nq; ++i) Fmask[fp++ + 0 * Nfp] = i + (k - 1) * Nq2;
  fp = 0;
  for (int k = 1; k <= Nq; ++k)
    for (int j = 1; j <= Nq; ++j)
      Fmask[fp++ + 1 * Nfp] = Nq + (j - 1) * Nq + (k - 1) * Nq2;
  fp = 0;
  for (int k = 1; k <= Nq; ++k)
    for (int i = 1; i <= Nq; ++i)
      Fmask[fp++ + 2 * Nfp] = i + (Nq - 1) * Nq + (k - 1) * Nq2;
  fp = 0;
  for (int k = 1; k <= Nq; ++k)
    for (int j = 1; j <= Nq; ++j)
      Fmask[fp++ + 3 * Nfp] = 1 + (j - 1) * Nq + (k - 1) * Nq2;
  fp = 0;
  for (int j = 1; j <= Nq; ++j)
    for (int i = 1; i <= Nq; ++i) Fmask[fp++ + 4 * Nfp] = i + (j - 1) * Nq;
  fp = 0;
  for (int j = 1; j <= Nq; ++j)
    for (int i = 1; i <= Nq; ++i)
      Fmask[fp++ + 5 * Nfp] = i + (j - 1) * Nq + (Nq - 1) * Nq2;
}

int orc_read_operators(const char* dir, int p, double* x1D, double* D1D,
                       double* Lift_mat) {
  if (p < 1) return 1;
  const int Nq = p + 1;
  std::string fname = std::string(dir) + "/p" + std::to_string(p) + ".dat";
  FILE* f = std::fopen(fname.c_str(), "r");
  if (!f) return 2;
  bool ok = read_reals(f, x1D, Nq) && read_reals(f, D1D, Nq * Nq) &&
            read_reals(f, Lift_mat, 6L * Nq * Nq * Nq);
  std::fclose(f);
  return ok ? 0 : 3;
}

int orc_mesh_sizes(int NeX, int NeY, int NeZ, int p, int* out) {
  const int Nq = p + 1;
  const int Nfp = Nq * Nq;
  const int Ne = NeX * NeY * NeZ;
  const int Nhalo = 2 * (NeY * NeZ + NeX * NeZ + NeX * NeY);
  out[0] = Ne;
  out[1] = Nhalo;
  out[2] = Ne + Nhalo;
  out[3] = Nfp * Nhalo;
  out[4] = Nfp * Nq;
  out[5] = 6 * Nfp;
  return 0;
}

int orc_mesh_setup(int NeX, int NeY, int NeZ, int p, double domx,
                   double domy, double domz, const double* x1D, int* VMapM,
                   int* VMapP, int* halo_src_map, double* normal_fn,
                   double* Escale, double* Fscale, double* pos_en) {
  const int Nq = p + 1;
  const int Nfp = Nq * Nq;
  const int Np = Nfp * Nq;
  const int NfpTot = 6 * Nfp;
  const int Ne = NeX * NeY * NeZ;
  std::vector<int> Fmask(Nfp * 6);
  orc_fmask(Nq, Fmask.data());

  const double dx = domx / static_cast<double>(NeX);
  const double dy = domy / static_cast<double>(NeY);
  const double dz = domz / static_cast<double>(NeZ);
  const long NEp = static_cast<long>(Np) * Ne;
  const long NEf = static_cast<long>(NfpTot) * Ne;

#pragma omp parallel for collapse(3) schedule(static)
  for (int k = 1; k <= NeZ; ++k)
    for (int j = 1; j <= NeY; ++j)
      for (int i = 1; i <= NeX; ++i) {
        const int ke = elem_id(i, j, k, NeX, NeY);
        const long e0 = ke - 1;
        const double xc = (static_cast<double>(i) - 0.5) * dx;
        const double yc = (static_cast<double>(j) - 0.5) * dy;
        const double zc = (static_cast<double>(k) - 0.5) * dz;
        // set_element_position, mod_mesh.f90:332-353
        for (int kk = 1; kk <= Nq; ++kk)
          for (int jj = 1; jj <= Nq; ++jj)
            for (int ii = 1; ii <= Nq; ++ii) {
              const long n = (ii - 1) + (jj - 1) * Nq + (kk - 1) * Nfp;
              pos_en[n + Np * e0] = xc + 0.5 * dx * x1D[ii - 1];
              pos_en[n + Np * e0 + NEp] = yc + 0.5 * dy * x1D[jj - 1];
              pos_en[n + Np * e0 + 2 * NEp] = zc + 0.5 * dz * x1D[kk - 1];
            }
        // mod_mesh.f90:147-149
        for (int n = 0; n < Np; ++n) {
          Escale[n + Np * e0] = 2.0 / dx;
          Escale[n + Np * e0 + NEp] = 2.0 / dy;
          Escale[n + Np * e0 + 2 * NEp] = 2.0 / dz;
        }
        // set_face_geometry, mod_mesh.f90:356-397
        for (int d = 0; d < 3; ++d)
          for (int n = 0; n < NfpTot; ++n)
            normal_fn[n + NfpTot * e0 + d * NEf] = 0.0;
        const int nd[6] = {1, 0, 1, 0, 2, 2};
        const double sg[6] = {-1.0, 1.0, 1.0, -1.0, -1.0, 1.0};
        const double fs[6] = {2.0 / dy, 2.0 / dx, 2.0 / dy,
                              2.0 / dx, 2.0 / dz, 2.0 / dz};
        for (int f = 0; f < 6; ++f)
          for (int fp = 0; fp < Nfp; ++fp) {
            normal_fn[f * Nfp + fp + NfpTot * e0 + nd[f] * NEf] = sg[f];
            Fscale[f * Nfp + fp + NfpTot * e0] = fs[f];
          }
        // mod_mesh.f90:153-166
        for (int f = 1; f <= 6; ++f) {
          int keP, opp;
          bool bnd;
          eval_neighbor_element(i, j, k, f, NeX, NeY, NeZ, &keP, &opp, &bnd);
          for (int fp = 1; fp <= Nfp; ++fp)
            VMapM[(f - 1) * Nfp + fp - 1 + NfpTot * e0] =
                Fmask[(fp - 1) + (f - 1) * Nfp] + (ke - 1) * Np;
          if (!bnd)
            for (int fp = 1; fp <= Nfp; ++fp)
              VMapP[(f - 1) * Nfp + fp - 1 + NfpTot * e0] =
                  Fmask[(fp - 1) + (opp - 1) * Nfp] + (keP - 1) * Np;
        }
      }

  // Serial boundary loop, mod_mesh.f90:171-190 (order defines the halo).
  int ibuf = 0;
  for (int k = 1; k <= NeZ; ++k)
    for (int j = 1; j <= NeY; ++j)
      for (int i = 1; i <= NeX; ++i) {
        const int ke = elem_id(i, j, k, NeX, NeY);
        for (int f = 1; f <= 6; ++f) {
          int keP, opp;
          bool bnd;
          eval_neighbor_element(i, j, k, f, NeX, NeY, NeZ, &keP, &opp, &bnd);
          for (int fp = 1; fp <= Nfp; ++fp)
            if (bnd) {
              ibuf = ibuf + 1;
              VMapP[(f - 1) * Nfp + fp - 1 + static_cast<long>(NfpTot) *
                                                  (ke - 1)] = Np * Ne + ibuf;
              halo_src_map[ibuf - 1] =
                  Fmask[(fp - 1) + (opp - 1) * Nfp] + (keP - 1) * Np;
            }
        }
      }
  return 0;
}

void orc_update_halo(double* f, int Np, int Ne, int NhaloNode,
                     const int* halo_src_map) {
  const long base = static_cast<long>(Np) * Ne;
  for (int ib = 0; ib < NhaloNode; ++ib)
    f[base + ib] = f[halo_src_map[ib] - 1];
}

int orc_cal_tend(int evaltype, double* dqdt, const double* q, const double* u,
                 const double* v, const double* w, const double* D1D,
                 const double* D1D_tr, const double* Lift_mat,
                 const int* VMapM, const int* VMapP, const double* normal_fn,
                 const double* Escale, const double* Fscale, int Nq, int Np,
                 int NfpTot, int Ne, int NeA, double* t_flux, double* t_dqdt) {
  (void)NeA;
  if (evaltype != ORC_GENERAL && evaltype != ORC_OPT1) return 1;
  if (evaltype == ORC_OPT1 && !opt1_table(Nq)) return 2;
  // The automatic array ebnd_flux(NfpTot,Ne) of mod_advect3d_eq.f90:66.
  std::vector<double> ebnd(static_cast<size_t>(NfpTot) * Ne);
  double t0 = now_s();
  cal_elembnd_flux(ebnd.data(), q, u, v, w, VMapM, VMapP, normal_fn, Fscale,
                   NfpTot, Ne);
  double t1 = now_s();
  cal_dqdt(evaltype, dqdt, q, u, v, w, ebnd.data(), D1D, D1D_tr, Lift_mat,
           Escale, Nq, Np, NfpTot, Ne);
  double t2 = now_s();
  if (t_flux) *t_flux += t1 - t0;
  if (t_dqdt) *t_dqdt += t2 - t1;
  return 0;
}

int orc_divlike_fields(int evaltype, int Nq, int nvar, long long Ne,
                       const double* D1D, const double* ix, const double* iy,
                       const double* iz, double* ox, double* oy, double* oz) {
  if (Nq < 2 || Nq > 16 || nvar < 1 || Ne < 0) return 1;
  if (evaltype != ORC_GENERAL && evaltype != ORC_OPT1) return 1;
  // D1D_tr = transpose(D1D) (mod_mesh.f90:263).
  std::vector<double> Dtr(static_cast<size_t>(Nq) * Nq);
  for (int i = 0; i < Nq; ++i)
    for (int l = 0; l < Nq; ++l) Dtr[l + Nq * i] = D1D[i + Nq * l];
  const long long Np = static_cast<long long>(Nq) * Nq * Nq;
  const long long units = Ne * nvar;
  opt1_fn opt1 = opt1_table(Nq);
#pragma omp parallel for schedule(static)
  for (long long u = 0; u < units; ++u) {
    const long long o = u * Np;
    if (evaltype == ORC_OPT1)
      opt1(ox + o, oy + o, oz + o, D1D, Dtr.data(), ix + o, iy + o, iz + o);
    else
      divlike_general(ox + o, oy + o, oz + o, D1D, Dtr.data(), ix + o, iy + o, iz + o, Nq);
  }
  return 0;
}

int orc_run_rk3(int evaltype, double* q, const double* u, const double* v,
                const double* w, const double* D1D, const double* Lift_mat,
                const int* VMapM, const int* VMapP, const int* halo_src_map,
                const double* normal_fn, const double* Escale,
                const double* Fscale, int Nq, int Ne, int NeA, int NhaloNode,
                double dt, int nstep, int output_interval, double* diag,
                double* times) {
  const int Np = Nq * Nq * Nq;
  const int NfpTot = 6 * Nq * Nq;
  const long NA = static_cast<long>(Np) * NeA;
  std::vector<double> q0(NA), dqdt(NA, 0.0), D1D_tr(Nq * Nq);
  // D1D_tr = transpose(D1D), mod_mesh.f90:263
  for (int a = 0; a < Nq; ++a)
    for (int b = 0; b < Nq; ++b) D1D_tr[a + Nq * b] = D1D[b + Nq * a];
  double t_tend = 0, t_flux = 0, t_dqdt = 0;
  const double t_start = now_s();
  int nd = 0;
  // main.f90:51-80
  for (int istep = 1; istep <= nstep; ++istep) {
#pragma omp parallel for schedule(static)
    for (int ke = 0; ke < Ne; ++ke)
      for (int n = 0; n < Np; ++n)
        q0[n + static_cast<long>(Np) * ke] = q[n + static_cast<long>(Np) * ke];
    for (int stage = 0; stage < 3; ++stage) {
      orc_update_halo(q, Np, Ne, NhaloNode, halo_src_map);
      const double ts = now_s();
      int rc = orc_cal_tend(evaltype, dqdt.data(), q, u, v, w, D1D,
                            D1D_tr.data(), Lift_mat, VMapM, VMapP, normal_fn,
                            Escale, Fscale, Nq, Np, NfpTot, Ne, NeA, &t_flux,
                            &t_dqdt);
      if (rc) return rc;
      t_tend += now_s() - ts;
      const double a = kRkA[stage], b = kRkB[stage];
#pragma omp parallel for schedule(static)
      for (int ke = 0; ke < Ne; ++ke)
        for (int n = 0; n < Np; ++n) {
          const long x = n + static_cast<long>(Np) * ke;
          q[x] = a * q0[x] + b * (q[x] + dt * dqdt[x]);
        }
    }
    if (output_interval > 0 && istep % output_interval == 0 && diag) {
      double mn = q[0], mx = q[0];
      const long NO = static_cast<long>(Np) * Ne;
      for (long x = 1; x < NO; ++x) {
        mn = q[x] < mn ? q[x] : mn;
        mx = q[x] > mx ? q[x] : mx;
      }
      diag[3 * nd + 0] = istep;
      diag[3 * nd + 1] = mn;
      diag[3 * nd + 2] = mx;
      ++nd;
    }
  }
  if (times) {
    times[0] = now_s() - t_start;
    times[1] = t_tend;
    times[2] = t_flux;
    times[3] = t_dqdt;
  }
  return 0;
}

void orc_random_velocity(unsigned long long seed, double* vel3) {
  SplitMix r{seed};
  for (int d = 0; d < 3; ++d) vel3[d] = 2.0 * r.uniform() - 1.0;
}

int orc_init_fields(int ic_kind, unsigned long long seed, int vel_kind,
                    double vx, double vy, double vz, const double* pos_en,
                    int Np, int Ne, int NeA, double* q, double* u, double* v,
                    double* w) {
  (void)NeA;
  const long NE = static_cast<long>(Np) * Ne;
  // Seeded Fourier modes: integer wavenumbers 1..4 per axis, amplitude
  // N(0, 0.01), phase U[0, 2*pi).
  double kx[8], ky[8], kz[8], amp[8], ph[8];
  SplitMix r{seed};
  for (int m = 0; m < 8; ++m) {
    kx[m] = static_cast<double>(1 + r.next() % 4);
    ky[m] = static_cast<double>(1 + r.next() % 4);
    kz[m] = static_cast<double>(1 + r.next() % 4);
    amp[m] = 0.01 * r.normal();
    ph[m] = 2.0 * kPI * r.uniform();
  }
  const double sig = 0.1;
  if (ic_kind != 0 && ic_kind != 1) return 1;
  if (vel_kind != 0 && vel_kind != 1) return 2;
#pragma omp parallel for schedule(static)
  for (long x = 0; x < NE; ++x) {
    const double px = pos_en[x], py = pos_en[x + NE], pz = pos_en[x + 2 * NE];
    if (ic_kind == 0) {
      // main.f90:149-151
      q[x] = std::sin(2.0 * kPI * px) * std::sin(2.0 * kPI * py) *
             std::sin(2.0 * kPI * pz);
    } else {
      const double r2 = (px - 0.5) * (px - 0.5) + (py - 0.5) * (py - 0.5) +
                        (pz - 0.5) * (pz - 0.5);
      double s = std::exp(-r2 / (2.0 * sig * sig));
      for (int m = 0; m < 8; ++m)
        s = s + amp[m] * std::cos(2.0 * kPI * (kx[m] * px + ky[m] * py +
                                               kz[m] * pz) + ph[m]);
      q[x] = s;
    }
    if (vel_kind == 0) {
      u[x] = vx;
      v[x] = vy;
      w[x] = vz;
    } else {
      u[x] = std::sin(2.0 * kPI * py);
      v[x] = std::sin(2.0 * kPI * pz);
      w[x] = std::sin(2.0 * kPI * px);
    }
  }
  return 0;
}

}  // extern "C"
