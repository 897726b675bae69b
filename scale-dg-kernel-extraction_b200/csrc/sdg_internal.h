// Internal helpers shared by the host set-up and the GPU core.
#pragma once

#include <string>
#include <vector>

namespace sdg {

// Records a formatted message as the calling thread's last error and
// returns `code`.
int fail(int code, const char* fmt, ...);
const std::string& last_error();

// Reference faces 1..6 as 0..5: normal axis (0 x, 1 y, 2 z), sign and the
// opposite face (mod_mesh.f90:266-276, 420-480).
extern const int kFaceAxis[6];
extern const double kFaceSign[6];
extern const int kOppFace[6];

// Fmask(fp+1, f+1) - 1: the 0-based element node of face node fp on face f.
int face_node(int Nq, int f, int fp);

// Relative tolerance of the factored lift: the largest tangential spread
// of a Lift_mat column, relative to max|Lift_mat|, that the fast kernels
// accept.  The reference's operator files spread by at most 2.4e-14
// (p = 15) and 3.4e-15 (p = 7).
constexpr double kLiftFactorTol = 1e-13;

// Tensor-product factorisation of Lift_mat(Np, 6).  On a hexahedron with
// tensor-product nodes, Lift(i,j,k,f) depends only on the node index
// along face f's normal; `expanded` receives the table rebuilt from the
// first tangential row of each face (entry (i,j,k,f) = Lift at normal
// index n, tangential indices 0) and `lift_z` the z-face factors as
// lift_z[k] (face -z) and lift_z[Nq + k] (face +z).  Returns false (and
// leaves the outputs empty) when some entry differs from its factor by
// more than kLiftFactorTol * max|Lift_mat|.
bool lift_factor(const double* Lift, int Nq, std::vector<double>* expanded,
                 std::vector<double>* lift_z);

}  // namespace sdg
