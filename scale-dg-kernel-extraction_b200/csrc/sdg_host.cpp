// Host-side set-up of the SCALE-DG advection library: operator files, the
// structured periodic mesh and its VMapM/VMapP/halo tables, and the initial
// fields.  These are the host duties of the reference's Fortran driver
// (element_init mod_mesh.f90:226-327, mesh_setup mod_mesh.f90:74-193,
// update_halo mod_mesh.f90:209-221, initial condition main.f90:146-157),
// restated in C++ so that a host program in any language can prepare the
// arrays that sdg_init takes.  Tables come out bit-identical to the
// reference's.
//
// Built with -ffp-contract=off: node coordinates and initial fields round
// exactly like the reference's x86-64 build.

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sdg_gpu.h"
#include "sdg_internal.h"

namespace sdg {

namespace {
thread_local std::string g_last_error;
}

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

const std::string& last_error() { return g_last_error; }

// Face f (0-based, reference face f+1): normal axis, sign, opposite face.
// Faces: 1 -y, 2 +x, 3 +y, 4 -x, 5 -z, 6 +z (mod_mesh.f90:269-275).
const int kFaceAxis[6] = {1, 0, 1, 0, 2, 2};
const double kFaceSign[6] = {-1.0, 1.0, 1.0, -1.0, -1.0, 1.0};
const int kOppFace[6] = {2, 3, 0, 1, 5, 4};

// 0-based node of face node fp (0-based) on face f (0-based), i.e.
// Fmask(fp+1, f+1) - 1, with fp enumerated as in mod_mesh.f90:278-324.
int face_node(int Nq, int f, int fp) {
  const int a = fp % Nq, b = fp / Nq, Nq2 = Nq * Nq;
  switch (f) {
    case 0: return a + Nq2 * b;                          // j = 1,  (i,k)
    case 1: return (Nq - 1) + Nq * a + Nq2 * b;          // i = Nq, (j,k)
    case 2: return a + Nq * (Nq - 1) + Nq2 * b;          // j = Nq, (i,k)
    case 3: return Nq * a + Nq2 * b;                     // i = 1,  (j,k)
    case 4: return a + Nq * b;                           // k = 1,  (i,j)
    default: return a + Nq * b + Nq2 * (Nq - 1);         // k = Nq, (i,j)
  }
}

bool lift_factor(const double* Lift, int Nq, std::vector<double>* expanded,
                 std::vector<double>* lift_z) {
  const long Nq2 = static_cast<long>(Nq) * Nq, Np = Nq2 * Nq;
  expanded->clear();
  lift_z->clear();
  double mx = 0.0;
  for (long x = 0; x < 6 * Np; ++x) mx = std::fmax(mx, std::fabs(Lift[x]));
  std::vector<double> ex(6 * Np);
  const long stride[3] = {1, Nq, Nq2};  // node offset of one step along i, j, k
  double spread = 0.0;
  for (int f = 0; f < 6; ++f)
    for (long n = 0; n < Np; ++n) {
      const long ijk[3] = {n % Nq, (n / Nq) % Nq, n / Nq2};
      const int ax = kFaceAxis[f];
      const double ref = Lift[Np * f + ijk[ax] * stride[ax]];  // tangential (0, 0)
      ex[Np * f + n] = ref;
      spread = std::fmax(spread, std::fabs(Lift[Np * f + n] - ref));
    }
  if (!(spread <= kLiftFactorTol * mx)) return false;
  lift_z->resize(2L * Nq);
  for (int k = 0; k < Nq; ++k) {
    (*lift_z)[k] = ex[Np * 4 + Nq2 * k];
    (*lift_z)[Nq + k] = ex[Np * 5 + Nq2 * k];
  }
  expanded->swap(ex);
  return true;
}

}  // namespace sdg

using namespace sdg;

namespace {

// splitmix64: the seeded stream of the synthetic workloads.
struct SplitMix64 {
  unsigned long long s;
  unsigned long long next() {
    s += 0x9E3779B97F4A7C15ULL;
    unsigned long long z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
  double gaussian(double two_pi) {
    const double r = std::sqrt(-2.0 * std::log(1.0 - uniform()));
    return r * std::cos(two_pi * uniform());
  }
};

bool parse_reals(FILE* f, double* out, long n) {
  char tok[96];
  for (long i = 0; i < n; ++i) {
    if (std::fscanf(f, "%95s", tok) != 1) return false;
    for (char* c = tok; *c; ++c)
      if (*c == 'd' || *c == 'D') *c = 'E';  // Fortran double exponent
    char* end = nullptr;
    out[i] = std::strtod(tok, &end);
    if (end == tok || *end != '\0') return false;
  }
  return true;
}

// Neighbour of element (i,j,k) (1-based) across face f (0-based) on the
// periodic box, as eval_neighbor_element (mod_mesh.f90:407-483).
void neighbour(int i, int j, int k, int f, int NeX, int NeY, int NeZ,
               int* keP, bool* wraps) {
  int ii = i, jj = j, kk = k;
  *wraps = false;
  switch (f) {
    case 0: if (j > 1) jj = j - 1; else { jj = NeY; *wraps = true; } break;
    case 1: if (i < NeX) ii = i + 1; else { ii = 1; *wraps = true; } break;
    case 2: if (j < NeY) jj = j + 1; else { jj = 1; *wraps = true; } break;
    case 3: if (i > 1) ii = i - 1; else { ii = NeX; *wraps = true; } break;
    case 4: if (k > 1) kk = k - 1; else { kk = NeZ; *wraps = true; } break;
    default: if (k < NeZ) kk = k + 1; else { kk = 1; *wraps = true; } break;
  }
  *keP = ii + (jj - 1) * NeX + (kk - 1) * NeX * NeY;  // elem_id
}

}  // namespace

extern "C" {

int sdg_last_error(char* buf, int buflen) {
  const std::string& e = last_error();
  if (buf && buflen > 0) {
    std::strncpy(buf, e.c_str(), static_cast<size_t>(buflen) - 1);
    buf[buflen - 1] = '\0';
  }
  return static_cast<int>(e.size());
}

const char* sdg_version(void) { return "0.1.0"; }

int sdg_read_operators(const char* dir, int p, double* x1D, double* D1D,
                       double* Lift_mat) {
  if (p < 1 || p > 15)
    return fail(SDG_ERR_ARG, "PolyOrder %d outside the supported 1..15", p);
  if (!dir || !x1D || !D1D || !Lift_mat)
    return fail(SDG_ERR_ARG, "sdg_read_operators: null argument");
  const int Nq = p + 1;
  const std::string path = std::string(dir) + "/p" + std::to_string(p) + ".dat";
  FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return fail(SDG_ERR_IO, "cannot open operator file %s", path.c_str());
  const bool ok = parse_reals(f, x1D, Nq) && parse_reals(f, D1D, Nq * Nq) &&
                  parse_reals(f, Lift_mat, 6L * Nq * Nq * Nq);
  std::fclose(f);
  if (!ok)
    return fail(SDG_ERR_IO,
                "operator file %s is short or malformed (expected %d + %d + %d "
                "reals)", path.c_str(), Nq, Nq * Nq, 6 * Nq * Nq * Nq);
  return SDG_OK;
}

int sdg_mesh_sizes(int NeX, int NeY, int NeZ, int p, int* sizes) {
  if (p < 1 || p > 15)
    return fail(SDG_ERR_ARG, "PolyOrder %d outside the supported 1..15", p);
  if (NeX < 1 || NeY < 1 || NeZ < 1)
    return fail(SDG_ERR_ARG, "element counts must be positive");
  const long long Nq = p + 1, Nfp = Nq * Nq, Np = Nfp * Nq;
  const long long Ne = 1LL * NeX * NeY * NeZ;
  const long long Nhalo = 2LL * (1LL * NeY * NeZ + 1LL * NeX * NeZ + 1LL * NeX * NeY);
  const long long NeA = Ne + Nhalo;
  if (Np * NeA > 2147483647LL)
    return fail(SDG_ERR_ARG,
                "Np*NeA = %lld overflows the int32 index space of VMapM/VMapP",
                Np * NeA);
  sizes[0] = static_cast<int>(Ne);
  sizes[1] = static_cast<int>(Nhalo);
  sizes[2] = static_cast<int>(NeA);
  sizes[3] = static_cast<int>(Nfp * Nhalo);
  sizes[4] = static_cast<int>(Np);
  sizes[5] = static_cast<int>(6 * Nfp);
  return SDG_OK;
}

int sdg_fmask(int p, int* Fmask) {
  if (p < 1 || p > 15) return fail(SDG_ERR_ARG, "PolyOrder %d outside 1..15", p);
  const int Nq = p + 1, Nfp = Nq * Nq;
  for (int f = 0; f < 6; ++f)
    for (int fp = 0; fp < Nfp; ++fp) Fmask[fp + Nfp * f] = face_node(Nq, f, fp) + 1;
  return SDG_OK;
}

int sdg_mesh_setup(int NeX, int NeY, int NeZ, int p, double domx, double domy,
                   double domz, const double* x1D, int* VMapM, int* VMapP,
                   int* halo_src_map, double* normal_fn, double* Escale,
                   double* Fscale, double* pos_en) {
  int sz[6];
  int rc = sdg_mesh_sizes(NeX, NeY, NeZ, p, sz);
  if (rc) return rc;
  const int Ne = sz[0], Np = sz[4], NfpTot = sz[5];
  const int Nq = p + 1, Nfp = Nq * Nq;
  const double dx = domx / static_cast<double>(NeX);
  const double dy = domy / static_cast<double>(NeY);
  const double dz = domz / static_cast<double>(NeZ);
  const double h[3] = {dx, dy, dz};
  const long NEp = static_cast<long>(Np) * Ne;
  const long NEf = static_cast<long>(NfpTot) * Ne;

  // Element order k, j, i (elem_id = i + (j-1)NeX + (k-1)NeX NeY); the halo
  // slots are numbered in exactly this traversal order, face by face and
  // node by node (the serialised loop of mod_mesh.f90:171-190).
  int ibuf = 0;
  for (int k = 1; k <= NeZ; ++k)
    for (int j = 1; j <= NeY; ++j)
      for (int i = 1; i <= NeX; ++i) {
        const int ke = i + (j - 1) * NeX + (k - 1) * NeX * NeY;
        const long e0 = ke - 1;
        const double ctr[3] = {(static_cast<double>(i) - 0.5) * dx,
                               (static_cast<double>(j) - 0.5) * dy,
                               (static_cast<double>(k) - 0.5) * dz};
        if (pos_en) {
          for (int n = 0; n < Np; ++n) {
            const int ix[3] = {n % Nq, (n / Nq) % Nq, n / Nfp};
            for (int d = 0; d < 3; ++d)
              pos_en[n + Np * e0 + d * NEp] = ctr[d] + 0.5 * h[d] * x1D[ix[d]];
          }
        }
        if (Escale)
          for (int d = 0; d < 3; ++d)
            for (int n = 0; n < Np; ++n) Escale[n + Np * e0 + d * NEp] = 2.0 / h[d];
        for (int f = 0; f < 6; ++f) {
          int keP;
          bool wraps;
          neighbour(i, j, k, f, NeX, NeY, NeZ, &keP, &wraps);
          const int opp = kOppFace[f];
          for (int fp = 0; fp < Nfp; ++fp) {
            const long slot = f * Nfp + fp + NfpTot * e0;
            if (VMapM) VMapM[slot] = face_node(Nq, f, fp) + 1 + (ke - 1) * Np;
            const int src = face_node(Nq, opp, fp) + 1 + (keP - 1) * Np;
            if (wraps) {
              ++ibuf;
              if (VMapP) VMapP[slot] = Np * Ne + ibuf;
              if (halo_src_map) halo_src_map[ibuf - 1] = src;
            } else if (VMapP) {
              VMapP[slot] = src;
            }
            if (normal_fn)
              for (int d = 0; d < 3; ++d)
                normal_fn[slot + d * NEf] = (d == kFaceAxis[f]) ? kFaceSign[f] : 0.0;
            if (Fscale) Fscale[slot] = 2.0 / h[kFaceAxis[f]];
          }
        }
      }
  return SDG_OK;
}

int sdg_update_halo_host(double* f, int Np, int Ne, int NhaloNode,
                         const int* halo_src_map) {
  if (!f || !halo_src_map || Np < 1 || Ne < 1 || NhaloNode < 0)
    return fail(SDG_ERR_ARG, "sdg_update_halo_host: bad argument");
  const long base = static_cast<long>(Np) * Ne;
  for (int b = 0; b < NhaloNode; ++b) f[base + b] = f[halo_src_map[b] - 1];
  return SDG_OK;
}

int sdg_random_velocity(unsigned long long seed, double* vel3) {
  if (!vel3) return fail(SDG_ERR_ARG, "sdg_random_velocity: null argument");
  SplitMix64 r{seed};
  for (int d = 0; d < 3; ++d) vel3[d] = 2.0 * r.uniform() - 1.0;
  return SDG_OK;
}

}  // extern "C"

namespace {

// The initial condition and velocity at every node x of [0, NE), the node
// position from pos(x, &px, &py, &pz).  Nodes are independent, so they are
// split over host threads (the values do not depend on the split).
template <typename Pos>
int fill_fields(int ic_kind, unsigned long long seed, int vel_kind, double vx, double vy,
                double vz, long NE, Pos pos, double* q, double* u, double* v, double* w) {
  if (ic_kind < 0 || ic_kind > 1)
    return fail(SDG_ERR_ARG, "unknown initial-condition kind %d", ic_kind);
  if (vel_kind < 0 || vel_kind > 1)
    return fail(SDG_ERR_ARG, "unknown velocity kind %d", vel_kind);
  const double pi = 4.0 * std::atan(1.0);  // mod_common.f90:25
  const double two_pi = 2.0 * pi;
  double kx[8], ky[8], kz[8], amp[8], ph[8];
  SplitMix64 r{seed};
  for (int m = 0; m < 8; ++m) {
    kx[m] = static_cast<double>(1 + r.next() % 4);
    ky[m] = static_cast<double>(1 + r.next() % 4);
    kz[m] = static_cast<double>(1 + r.next() % 4);
    amp[m] = 0.01 * r.gaussian(two_pi);
    ph[m] = two_pi * r.uniform();
  }
  const double two_s2 = 2.0 * 0.1 * 0.1;  // 2 sigma^2, sigma = 0.1
  auto fill = [&](long x0, long x1) {
    for (long x = x0; x < x1; ++x) {
      double px, py, pz;
      pos(x, &px, &py, &pz);
      if (ic_kind == 0) {
        q[x] = std::sin(two_pi * px) * std::sin(two_pi * py) * std::sin(two_pi * pz);
      } else {
        const double r2 = (px - 0.5) * (px - 0.5) + (py - 0.5) * (py - 0.5) +
                          (pz - 0.5) * (pz - 0.5);
        double s = std::exp(-r2 / two_s2);
        for (int m = 0; m < 8; ++m)
          s = s + amp[m] * std::cos(two_pi * (kx[m] * px + ky[m] * py + kz[m] * pz) + ph[m]);
        q[x] = s;
      }
      if (vel_kind == 0) {
        u[x] = vx;
        v[x] = vy;
        w[x] = vz;
      } else {
        u[x] = std::sin(two_pi * py);
        v[x] = std::sin(two_pi * pz);
        w[x] = std::sin(two_pi * px);
      }
    }
  };
  const unsigned hw = std::thread::hardware_concurrency();
  const long nthr = std::max(1L, std::min({static_cast<long>(hw ? hw : 1), 32L, NE / 65536}));
  if (nthr == 1) {
    fill(0, NE);
  } else {
    std::vector<std::thread> pool;
    for (long t = 0; t < nthr; ++t)
      pool.emplace_back(fill, NE * t / nthr, NE * (t + 1) / nthr);
    for (auto& th : pool) th.join();
  }
  return SDG_OK;
}

}  // namespace

extern "C" {

int sdg_init_fields(int ic_kind, unsigned long long seed, int vel_kind,
                    double vx, double vy, double vz, const double* pos_en,
                    int Np, int Ne, double* q, double* u, double* v,
                    double* w) {
  if (!pos_en || !q || !u || !v || !w || Np < 1 || Ne < 1)
    return fail(SDG_ERR_ARG, "sdg_init_fields: bad argument");
  const long NE = static_cast<long>(Np) * Ne;
  return fill_fields(ic_kind, seed, vel_kind, vx, vy, vz, NE,
                     [&](long x, double* px, double* py, double* pz) {
                       *px = pos_en[x];
                       *py = pos_en[x + NE];
                       *pz = pos_en[x + 2 * NE];
                     },
                     q, u, v, w);
}

int sdg_box_fields(int NeX, int NeY, int NeZ, int p, const double* x1D, int ic_kind,
                   unsigned long long seed, int vel_kind, double vx, double vy, double vz,
                   double* q, double* u, double* v, double* w) {
  int sz[6];
  int rc = sdg_mesh_sizes(NeX, NeY, NeZ, p, sz);
  if (rc) return rc;
  if (!x1D || !q || !u || !v || !w) return fail(SDG_ERR_ARG, "sdg_box_fields: null array");
  const int Ne = sz[0], Np = sz[4];
  const int Nq = p + 1, Nfp = Nq * Nq;
  const double h[3] = {1.0 / static_cast<double>(NeX), 1.0 / static_cast<double>(NeY),
                       1.0 / static_cast<double>(NeZ)};
  const long NE = static_cast<long>(Np) * Ne;
  // The node positions of sdg_mesh_setup on the unit box, computed where
  // they are used: element centre (i - 1/2) h (1-based i) plus h/2 x1D.
  return fill_fields(ic_kind, seed, vel_kind, vx, vy, vz, NE,
                     [&](long x, double* px, double* py, double* pz) {
                       const long e = x / Np;
                       const int n = static_cast<int>(x - e * Np);
                       const long ej = e / NeX;
                       const int el[3] = {static_cast<int>(e - ej * NeX) + 1,
                                          static_cast<int>(ej % NeY) + 1,
                                          static_cast<int>(ej / NeY) + 1};
                       const int ix[3] = {n % Nq, (n / Nq) % Nq, n / Nfp};
                       double r3[3];
                       for (int d = 0; d < 3; ++d)
                         r3[d] = (static_cast<double>(el[d]) - 0.5) * h[d] +
                                 0.5 * h[d] * x1D[ix[d]];
                       *px = r3[0];
                       *py = r3[1];
                       *pz = r3[2];
                     },
                     q, u, v, w);
}



}  // extern "C"
