// Command-line twin of the reference driver (main.f90) over the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY: it prints the same "istep min max" lines
// (main.f90:76-79, format (I8,2ES24.15)) and timer report (main.f90:169-181,
// mod_advect3d_eq.f90:31-37) as the reference program, so that the product
// driver's output can be compared line by line.  It reads the
// &PARAM_ADVECT3D namelist of main.f90:103-107 plus the additive keys
// IC_kind, IC_seed and Vel_kind (seeded initial condition and velocity).
//
// Usage: sdg_oracle input.conf [operator_data_dir]

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "sdg_oracle.h"

namespace {

std::string upper(std::string s) {
  for (auto& c : s) c = static_cast<char>(std::toupper(c));
  return s;
}

// Minimal namelist reader for one group: key = value pairs separated by
// commas or newlines, '!' comments, quoted strings, D/E exponents.
bool read_namelist(const std::string& path, const std::string& group,
                   std::map<std::string, std::string>* kv) {
  std::ifstream in(path);
  if (!in) return false;
  std::stringstream ss;
  ss << in.rdbuf();
  std::string text = ss.str(), clean;
  bool inq = false, comment = false;
  char qc = 0;
  for (char c : text) {
    if (comment) {
      if (c == '\n') { comment = false; clean += '\n'; }
      continue;
    }
    if (inq) {
      clean += c;
      if (c == qc) inq = false;
      continue;
    }
    if (c == '\'' || c == '"') { inq = true; qc = c; clean += c; continue; }
    if (c == '!') { comment = true; continue; }
    clean += c;
  }
  const std::string tag = "&" + upper(group);
  size_t pos = upper(clean).find(tag);
  if (pos == std::string::npos) return false;
  pos += tag.size();
  // Split into tokens at commas/newlines outside quotes, stop at '/'.
  std::string cur;
  inq = false;
  auto flush = [&]() {
    size_t eq = cur.find('=');
    if (eq != std::string::npos) {
      std::string k = cur.substr(0, eq), v = cur.substr(eq + 1);
      auto trim = [](std::string s) {
        size_t a = s.find_first_not_of(" \t\r\n");
        size_t b = s.find_last_not_of(" \t\r\n");
        return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
      };
      k = upper(trim(k));
      v = trim(v);
      if (v.size() >= 2 && (v[0] == '"' || v[0] == '\''))
        v = v.substr(1, v.size() - 2);
      (*kv)[k] = v;
    }
    cur.clear();
  };
  for (size_t i = pos; i < clean.size(); ++i) {
    char c = clean[i];
    if (inq) { cur += c; if (c == qc) inq = false; continue; }
    if (c == '\'' || c == '"') { inq = true; qc = c; cur += c; continue; }
    if (c == '/') { flush(); return true; }
    if (c == ',' || c == '\n') { flush(); continue; }
    cur += c;
  }
  return false;
}

double to_real(std::string v) {
  for (auto& c : v)
    if (c == 'D' || c == 'd') c = 'E';
  return std::strtod(v.c_str(), nullptr);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr,
                 "Error: configuration file argument is required.\n"
                 "Usage: sdg_oracle input.conf [operator_data_dir]\n");
    return 1;
  }
  std::map<std::string, std::string> kv;
  if (!read_namelist(argv[1], "PARAM_ADVECT3D", &kv)) {
    std::fprintf(stderr, "Error: cannot read &PARAM_ADVECT3D from %s\n",
                 argv[1]);
    return 1;
  }
  const std::string opdir = argc > 2 ? argv[2] : "operator_data";
  // Defaults, main.f90:94-101,113-115.
  int NeX = 4, NeY = 4, NeZ = 4, p = 3, nstep = 100, out_int = 10;
  double vx = 1.0, vy = 1.0, vz = 1.0, dt = 1.0e-3;
  std::string opt = "OPT1";
  int ic_kind = 0, vel_kind = 0;
  unsigned long long seed = 0;
  for (auto& it : kv) {
    const std::string& k = it.first;
    const std::string& v = it.second;
    if (k == "NEX") NeX = std::atoi(v.c_str());
    else if (k == "NEY") NeY = std::atoi(v.c_str());
    else if (k == "NEZ") NeZ = std::atoi(v.c_str());
    else if (k == "POLYORDER") p = std::atoi(v.c_str());
    else if (k == "DT") dt = to_real(v);
    else if (k == "NSTEP") nstep = std::atoi(v.c_str());
    else if (k == "OUTPUT_INTERVAL") out_int = std::atoi(v.c_str());
    else if (k == "VEL_X") vx = to_real(v);
    else if (k == "VEL_Y") vy = to_real(v);
    else if (k == "VEL_Z") vz = to_real(v);
    else if (k == "DGOPTRKERNEL_OPTTYPE") opt = upper(v);
    else if (k == "IC_KIND") ic_kind = std::atoi(v.c_str());
    else if (k == "IC_SEED") seed = std::strtoull(v.c_str(), nullptr, 10);
    else if (k == "VEL_KIND") vel_kind = std::atoi(v.c_str());
    // Keys that only the GPU driver uses are accepted and ignored here.
  }
  int evaltype = 0;
  if (opt == "GENERAL") evaltype = ORC_GENERAL;
  else if (opt == "OPT1") evaltype = ORC_OPT1;
  else {
    std::fprintf(stderr, "Unsupported dgoptr_evaltype: %s\n", opt.c_str());
    return 2;
  }
  int sz[6];
  orc_mesh_sizes(NeX, NeY, NeZ, p, sz);
  const int Ne = sz[0], NeA = sz[2], NhaloNode = sz[3], Np = sz[4],
            NfpTot = sz[5], Nq = p + 1;
  std::vector<double> x1D(Nq), D1D(Nq * Nq), Lift(6L * Np);
  if (orc_read_operators(opdir.c_str(), p, x1D.data(), D1D.data(),
                         Lift.data())) {
    std::fprintf(stderr, "Error: cannot read %s/p%d.dat\n", opdir.c_str(), p);
    return 3;
  }
  const size_t NA = static_cast<size_t>(Np) * NeA;
  std::vector<int> VMapM(static_cast<size_t>(NfpTot) * Ne),
      VMapP(static_cast<size_t>(NfpTot) * Ne), hmap(NhaloNode);
  std::vector<double> nfn(3 * static_cast<size_t>(NfpTot) * Ne),
      Esc(3 * static_cast<size_t>(Np) * Ne),
      Fsc(static_cast<size_t>(NfpTot) * Ne),
      pos(3 * static_cast<size_t>(Np) * Ne);
  orc_mesh_setup(NeX, NeY, NeZ, p, 1.0, 1.0, 1.0, x1D.data(), VMapM.data(),
                 VMapP.data(), hmap.data(), nfn.data(), Esc.data(), Fsc.data(),
                 pos.data());
  std::vector<double> q(NA, 0.0), u(NA, 0.0), v(NA, 0.0), w(NA, 0.0);
  orc_init_fields(ic_kind, seed, vel_kind, vx, vy, vz, pos.data(), Np, Ne, NeA,
                  q.data(), u.data(), v.data(), w.data());
  orc_update_halo(q.data(), Np, Ne, NhaloNode, hmap.data());
  orc_update_halo(u.data(), Np, Ne, NhaloNode, hmap.data());
  orc_update_halo(v.data(), Np, Ne, NhaloNode, hmap.data());
  orc_update_halo(w.data(), Np, Ne, NhaloNode, hmap.data());
  const int ndiag = out_int > 0 ? nstep / out_int : 0;
  std::vector<double> diag(3 * (ndiag + 1)), times(4);
  int rc = orc_run_rk3(evaltype, q.data(), u.data(), v.data(), w.data(),
                       D1D.data(), Lift.data(), VMapM.data(), VMapP.data(),
                       hmap.data(), nfn.data(), Esc.data(), Fsc.data(), Nq, Ne,
                       NeA, NhaloNode, dt, nstep, out_int, diag.data(),
                       times.data());
  if (rc) {
    std::fprintf(stderr, "Error: oracle run failed (%d)\n", rc);
    return 4;
  }
  for (int i = 0; i < ndiag; ++i)
    std::printf("%8d%24.15E%24.15E\n", static_cast<int>(diag[3 * i]),
                diag[3 * i + 1], diag[3 * i + 2]);
  std::printf("= Report of execution time [sec]\n");
  std::printf("%30s%24.5E\n", "Main:", times[0]);
  std::printf("%30s%24.5E\n", "Cal_tend:", times[1]);
  std::printf("%30s%24.5E\n", "Element boundary flux:", times[2]);
  std::printf("%30s%24.5E\n", "Volume derivate + surface lift:", times[3]);
  return 0;
}
