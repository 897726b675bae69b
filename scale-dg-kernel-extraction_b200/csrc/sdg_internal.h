// Internal helpers shared by the host set-up and the GPU core.
#pragma once

#include <string>

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

}  // namespace sdg
