/*
 * CPU oracle for the SCALE-DG 3D DG advection right-hand side.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a C++/OpenMP restatement of the
 * reference Fortran (seiya/scale-dg-kernel-extraction), written loop for loop
 * with the same summation order, built with -ffp-contract=off so that every
 * product and sum rounds exactly as an x86-64 gfortran -O3 build of the
 * reference does (no FMA contraction on the baseline x86-64 ISA).  Only the
 * test-suite, the smoke check and the bench's CPU-baseline leg may load it;
 * the product library never does.
 *
 * Parity status: the reference ships no golden vectors and no Fortran
 * compiler exists in this image, so the oracle cannot be checked against a
 * reference binary.  It is pinned instead (a) against golden vectors made by
 * evaluating the reference's own Fortran source text through a mechanical
 * translator (tests/golden/make_golden.py), and (b) by analytic known-answer
 * tests (free-stream preservation, discrete mass conservation, spectral
 * accuracy, periodic return).
 *
 * All arrays follow the reference's Fortran layout: column-major, and the
 * integer maps (VMapM, VMapP, halo_src_map, Fmask) hold 1-based indices.
 */
#ifndef SDG_ORACLE_H
#define SDG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Evaluation types, as DGOPTR_EVALTYPEID_* in mod_dg_optr_kernel.f90:39-42. */
#define ORC_GENERAL 1
#define ORC_OPT1 2

/* element_init file read (mod_mesh.f90:253-263): x1D(Nq), D1D(Nq,Nq),
 * Lift_mat(Nq,Nq,Nq,6).  Returns 0 on success, nonzero on a missing or
 * short file. */
int orc_read_operators(const char* dir, int p, double* x1D, double* D1D,
                       double* Lift_mat);

/* Sizes from mesh_setup (mod_mesh.f90:96-100): out[0..5] =
 * Ne, Nhalo, NeA, NhaloNode, Np, NfpTot. */
int orc_mesh_sizes(int NeX, int NeY, int NeZ, int p, int* out);

/* Fmask(Nfp,6) from element_init (mod_mesh.f90:278-324), 1-based. */
void orc_fmask(int Nq, int* Fmask);

/* mesh_setup (mod_mesh.f90:74-193) with the helpers set_element_position
 * (332-353), set_face_geometry (356-397), eval_neighbor_element (407-483) and
 * elem_id (486-493). */
int orc_mesh_setup(int NeX, int NeY, int NeZ, int p, double domx,
                   double domy, double domz, const double* x1D, int* VMapM,
                   int* VMapP, int* halo_src_map, double* normal_fn,
                   double* Escale, double* Fscale, double* pos_en);

/* update_halo (mod_mesh.f90:209-221). */
void orc_update_halo(double* f, int Np, int Ne, int NhaloNode,
                     const int* halo_src_map);

/* advect3d_eq_cal_tend (mod_advect3d_eq.f90:41-85) with the operator
 * dispatch of mod_dg_optr_kernel.f90:62-190.  t_flux / t_dqdt receive the
 * seconds spent in the two phases (may be NULL). */
int orc_cal_tend(int evaltype, double* dqdt, const double* q, const double* u,
                 const double* v, const double* w, const double* D1D,
                 const double* D1D_tr, const double* Lift_mat,
                 const int* VMapM, const int* VMapP, const double* normal_fn,
                 const double* Escale, const double* Fscale, int Nq, int Np,
                 int NfpTot, int Ne, int NeA, double* t_flux, double* t_dqdt);

/* The SSP-RK3 time loop of main.f90:51-80 (coefficients mod_common.f90:28-30)
 * on caller-owned q,u,v,w (Np,NeA) whose halos are already filled.  Every
 * output_interval steps the (istep, min, max) triple is appended to `diag`
 * (capacity 3*(nstep/output_interval)).  times[0..3] receive the Main,
 * Cal_tend, Element-boundary-flux and Volume-derivative timers (seconds). */
int orc_run_rk3(int evaltype, double* q, const double* u, const double* v,
                const double* w, const double* D1D, const double* Lift_mat,
                const int* VMapM, const int* VMapP, const int* halo_src_map,
                const double* normal_fn, const double* Escale,
                const double* Fscale, int Nq, int Ne, int NeA, int NhaloNode,
                double dt, int nstep, int output_interval, double* diag,
                double* times);

/* Initial fields.  kind 0: the reference's sine product (main.f90:146-157);
 * kind 1: Gaussian bump (sigma 0.1 at the cube centre) plus 8 seeded Fourier
 * modes.  Velocity kind 0: constant (vx,vy,vz); kind 1: divergence-free
 * (sin 2*pi*y, sin 2*pi*z, sin 2*pi*x).  Writes q,u,v,w(:,1:Ne) from pos_en;
 * the caller fills the halos. */
int orc_init_fields(int ic_kind, unsigned long long seed, int vel_kind,
                    double vx, double vy, double vz, const double* pos_en,
                    int Np, int Ne, int NeA, double* q, double* u, double* v,
                    double* w);

/* Random constant velocity drawn from U[-1,1]^3 with the given seed. */
void orc_random_velocity(unsigned long long seed, double* vel3);

/* Number of OpenMP threads the oracle will use. */
int orc_num_threads(void);

/* element_operation_kernel_matvec_divlike_dirXYZ_var5_P<p>
 * (mod_dg_optr_kernel_opt1.F90.erb:347-465) over Ne elements of nvar fields:
 * for each (element, field) unit of Np nodes at offset Np*(v + nvar*e),
 * ox/oy/oz = the x/y/z contraction of ix/iy/iz with D1D, in the OPT1 order
 * (the same per-direction sums as divlike_dirXYZ_P<p>, erb:228-344) or the
 * GENERAL order (mod_dg_optr_kernel.f90:197-258).  With ix = iy = iz and
 * nvar = 1 this is element_operation_kernel_matvec_gradlike_dirXYZ_P<p>
 * (erb:166-219).  It computes what those routines are written for: the var5
 * y output index of erb:400 and the gradlike z first term of erb:209 are
 * index slips in the reference text (out-of-range and transposed indices),
 * not reproduced.  Returns 0, or 1 on bad sizes or evaltype. */
int orc_divlike_fields(int evaltype, int Nq, int nvar, long long Ne,
                       const double* D1D, const double* ix, const double* iy,
                       const double* iz, double* ox, double* oy, double* oz);

#ifdef __cplusplus
}
#endif
#endif
