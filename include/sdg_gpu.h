/*
 * sdg_gpu.h - C ABI of the B200 (sm_100a) SCALE-DG 3D DG advection library.
 *
 * The library replaces, at whole-mesh granularity, the hot path of
 * seiya/scale-dg-kernel-extraction:
 *
 *   advect3d_eq_cal_tend      mod_advect3d_eq.f90:41-85   (flux + dqdt)
 *   update_halo               mod_mesh.f90:209-221
 *   SSP-RK3 stage update      main.f90:51-80, mod_common.f90:28-30
 *
 * and mirrors the host-side set-up the Fortran driver performs
 * (element_init mod_mesh.f90:226-327, mesh_setup mod_mesh.f90:74-193) so a
 * host program in any language can drive it.  Every symbol is extern "C"
 * and Fortran bind(C)-compatible: scalars are passed by value (int32 or
 * double), arrays as plain pointers in the reference's Fortran layout
 * (column-major; VMapM, VMapP and halo_src_map hold 1-based indices), and
 * every call returns an int status (SDG_OK = 0).  sdg_last_error() gives the
 * message of the last failure on the calling thread.
 *
 * Ownership: host arrays passed in are only read (or written, for outputs)
 * during the call and stay owned by the caller.  Device buffers belong to
 * the handle.  Threading: one host thread at a time per handle; each handle
 * owns one CUDA stream; separate handles are independent.
 *
 * There is no CPU fallback: without a usable CUDA device, sdg_init fails
 * with SDG_ERR_CUDA.
 */
#ifndef SDG_GPU_H
#define SDG_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define SDG_OK 0
#define SDG_ERR_ARG 1     /* invalid argument or size                    */
#define SDG_ERR_CUDA 2    /* CUDA runtime error, or no device            */
#define SDG_ERR_IO 3      /* operator file missing or malformed          */
#define SDG_ERR_MESH 4    /* mesh tables not in the supported form       */
#define SDG_ERR_STATE 5   /* call out of order (e.g. no state uploaded)  */

/* sdg_init flags. */
#define SDG_FLAG_EXACT 1          /* no FMA: every product and sum rounded
                                     separately in the reference's order,
                                     bit-for-bit the x86-64 reference      */
#define SDG_FLAG_ORDER_GENERAL 2  /* GENERAL summation order (mod_dg_optr_
                                     kernel.f90:221-257) instead of OPT1's
                                     three partial sums for p > 7 (erb:242) */
#define SDG_FLAG_MIXED 4          /* resident RK path in mixed precision:
                                     FP32 velocity, tendency and stage
                                     intermediates, FP64 RK accumulation   */
#define SDG_FLAG_EXTERNAL_HALO 8  /* resident path for a subdomain: every
                                     boundary face reads its plus side from
                                     the halo region of the stage input, and
                                     the caller fills that halo before each
                                     sdg_rk3_stage (sdg_update_halo_stage plus
                                     its own exchange, e.g. of z-slabs);
                                     sdg_rk3_steps is then unavailable       */

/* Fields for sdg_set_field / sdg_get_field. */
#define SDG_FIELD_Q 0
#define SDG_FIELD_U 1
#define SDG_FIELD_V 2
#define SDG_FIELD_W 3
/* Further resident arrays for sdg_resident_array: the inputs of RK stages 2
 * and 3 (stage 1 reads SDG_FIELD_Q). */
#define SDG_ARRAY_STAGE2 4
#define SDG_ARRAY_STAGE3 5

typedef struct sdg_handle sdg_handle;

/* Copies the last error message of this thread into buf (NUL-terminated,
 * truncated to buflen); returns the message length. */
int sdg_last_error(char* buf, int buflen);

/* Library version string "major.minor.patch". */
const char* sdg_version(void);

/* ---------------------------------------------------------------------
 * Host-side set-up (mirrors of the reference's Fortran set-up routines)
 * --------------------------------------------------------------------- */

/* element_init operator read (mod_mesh.f90:253-263): reads
 * <dir>/p<p>.dat into x1D(Nq), D1D(Nq,Nq), Lift_mat(Nq,Nq,Nq,6).
 * p must be 1..15.  SDG_ERR_IO on a missing or short file. */
int sdg_read_operators(const char* dir, int p, double* x1D, double* D1D,
                       double* Lift_mat);

/* Mesh sizes of mesh_setup (mod_mesh.f90:96-100):
 * sizes[0..5] = Ne, Nhalo, NeA, NhaloNode, Np, NfpTot.  Fails when
 * Np*NeA would overflow the int32 index space of VMapM/VMapP. */
int sdg_mesh_sizes(int NeX, int NeY, int NeZ, int p, int* sizes);

/* Fmask(Nfp,6) of element_init (mod_mesh.f90:278-324), 1-based. */
int sdg_fmask(int p, int* Fmask);

/* mesh_setup (mod_mesh.f90:74-193) for the periodic box
 * [0,domx]x[0,domy]x[0,domz]: VMapM, VMapP (NfpTot,Ne), halo_src_map
 * (NhaloNode), normal_fn (NfpTot,Ne,3), Escale (Np,Ne,3), Fscale (NfpTot,Ne)
 * and pos_en (Np,Ne,3), bit-identical to the reference's tables.  Any
 * output pointer may be NULL to skip that table. */
int sdg_mesh_setup(int NeX, int NeY, int NeZ, int p, double domx, double domy,
                   double domz, const double* x1D, int* VMapM, int* VMapP,
                   int* halo_src_map, double* normal_fn, double* Escale,
                   double* Fscale, double* pos_en);

/* update_halo (mod_mesh.f90:209-221) on a host array f(Np*NeA). */
int sdg_update_halo_host(double* f, int Np, int Ne, int NhaloNode,
                         const int* halo_src_map);

/* Initial fields (main.f90:146-157 and the seeded workloads):
 *   ic_kind 0: q = sin(2 pi x) sin(2 pi y) sin(2 pi z)   (main.f90:149-151)
 *   ic_kind 1: Gaussian bump (sigma 0.1, cube centre) + 8 Fourier modes
 *              (integer wavenumbers 1..4 per axis, amplitude N(0,0.01),
 *              phase U[0,2 pi)) from a splitmix64 stream seeded by `seed`
 *   vel_kind 0: constant (vx,vy,vz);  1: (sin 2 pi y, sin 2 pi z, sin 2 pi x)
 * Writes q,u,v,w(:,1:Ne); halos are left to update_halo. */
int sdg_init_fields(int ic_kind, unsigned long long seed, int vel_kind,
                    double vx, double vy, double vz, const double* pos_en,
                    int Np, int Ne, double* q, double* u, double* v,
                    double* w);

/* sdg_init_fields on the periodic unit box NeX x NeY x NeZ of order p
 * without the mesh tables: the node positions of sdg_mesh_setup are formed
 * where they are used (the same values bit for bit).  For callers that need
 * many instances' fields quickly (batched and served workloads). */
int sdg_box_fields(int NeX, int NeY, int NeZ, int p, const double* x1D,
                   int ic_kind, unsigned long long seed, int vel_kind,
                   double vx, double vy, double vz, double* q, double* u,
                   double* v, double* w);

/* A constant velocity drawn from U[-1,1]^3 by a splitmix64 stream. */
int sdg_random_velocity(unsigned long long seed, double* vel3);

/* ---------------------------------------------------------------------
 * Handle: operators and mesh resident on the GPU
 * --------------------------------------------------------------------- */

/* Uploads the operators and mesh tables that advect3d_eq_cal_tend receives
 * (mod_advect3d_eq.f90:41-65) plus halo_src_map (mod_mesh.f90:68), once.
 * The verbatim tables are validated and compressed on the host: per-element
 * Escale, per-face Fscale, axis-aligned normals and a per-face neighbour
 * table equivalent node-for-node to VMapM/VMapP.  Tables that do not have
 * that structure are rejected with SDG_ERR_MESH.  Replaces the selection
 * of dg_optr_kernel_setup (mod_dg_optr_kernel.f90:45-58) for the "GPU"
 * evaluation type; flags pick the arithmetic (SDG_FLAG_*). */
int sdg_init(sdg_handle** h, int Nq, int Np, int NfpTot, int Ne, int NeA,
             int NhaloNode, const double* D1D, const double* Lift_mat,
             const int* VMapM, const int* VMapP, const int* halo_src_map,
             const double* normal_fn, const double* Escale,
             const double* Fscale, int flags);

/* Releases the handle and its device memory. */
int sdg_finalize(sdg_handle* h);

/* Drop-in for advect3d_eq_cal_tend (mod_advect3d_eq.f90:41-85) on host
 * arrays q,u,v,w(Np,NeA) (halo filled by the caller, as the reference
 * reads it through VMapP) -> dqdt(Np,NeA), of which (:,1:Ne) is written.
 * Copies in, runs the fused kernel, copies out; synchronous.  Meshes of
 * 2,048+ elements go by element chunks (the halo parts first), each
 * chunk's kernel starting once the chunks it reads are up and its dqdt
 * going back at once, so the copies overlap (host arrays pinned for that);
 * the result equals sdg_cal_tend_dev on the same arrays. */
int sdg_cal_tend(sdg_handle* h, double* dqdt, const double* q,
                 const double* u, const double* v, const double* w);

/* The same on device arrays, asynchronously on `stream` (a cudaStream_t;
 * NULL = the handle's stream). */
int sdg_cal_tend_dev(sdg_handle* h, double* dqdt, const double* q,
                     const double* u, const double* v, const double* w,
                     void* stream);

/* update_halo (mod_mesh.f90:209-221) on a device array f(Np*NeA). */
int sdg_update_halo_dev(sdg_handle* h, double* f, void* stream);

/* ---------------------------------------------------------------------
 * Resident RK3 path (main.f90:51-80 with the state kept in HBM)
 * --------------------------------------------------------------------- */

/* Uploads field `which` (SDG_FIELD_*) from a host array (Np,NeA) or
 * (Np,Ne); only (:,1:Ne) is read, halos are rebuilt on the device. */
int sdg_set_field(sdg_handle* h, int which, const double* host);

/* Downloads the current state q(:,1:Ne) (FP64) into host (Np,Ne). */
int sdg_get_field(sdg_handle* h, int which, double* host);

/* Advances nsteps SSP-RK3 steps of size dt: each stage fuses the halo read,
 * the tendency and the stage update in one kernel; steps replay a CUDA
 * graph.  Asynchronous on the handle's stream. */
int sdg_rk3_steps(sdg_handle* h, double dt, int nsteps);

/* sdg_set_field(SDG_FIELD_Q, q) + sdg_rk3_steps(dt, nsteps) +
 * sdg_get_field(SDG_FIELD_Q, q) in one call, with the same result bit for
 * bit: q (Np,Ne) FP64 on the host in, the state after nsteps steps back in
 * q.  The element range is cut into chunks (runs of z-layers in a box;
 * one layer thin at both ends) and the first step's stages run chunk by
 * chunk as soon as the chunks they read are uploaded, the last step's as
 * the state's chunks go back, so the two copies and the stages overlap
 * (host memory pinned with cudaHostAlloc / cudaHostRegister for the copies
 * to run asynchronously).  Calls of up to three steps run as one chunked
 * plan, so that the first chunks' results go back while the last chunks go
 * up, and on pinned memory replay a CUDA graph captured for that array, dt
 * and step count; longer calls run the first and last steps by chunks and
 * the ones between through the step graph.  Meshes of fewer than 2,048
 * elements (fewer than 4 chunks of 512 elements or 2^18 nodes), or whose
 * boundary faces read the halo buffer, take the three calls in order.
 * Velocities must be set (sdg_set_field).  Synchronises the handle. */
int sdg_rk3_steps_host(sdg_handle* h, double* q, double dt, int nsteps);

/* min/max of q(:,1:Ne) (main.f90:76-79); synchronises the handle. */
int sdg_minmax(sdg_handle* h, double* qmin, double* qmax);

/* FP64 global diagnostics with the tensor LGL weights w(Nq) and the element
 * Jacobian jac (= dx*dy*dz/8): mass = sum W*jac*q, l2 = sqrt(sum W*jac*q^2).
 * Synchronises the handle. */
int sdg_diagnostics(sdg_handle* h, const double* lgl_w, double jac,
                    double* mass, double* l2);

/* Enqueues stage `stage` (1..3) of one SSP-RK3 step (main.f90:58-74) on the
 * handle's stream without a graph: stage 1 reads q0 and writes q1, stage 2
 * reads q1 and q0 and writes q2, stage 3 reads q2 and q0 and overwrites q0.
 * For timing and profiling single stage kernels. */
int sdg_rk3_stage(sdg_handle* h, int stage, double dt);

/* The handle's CUDA stream (a cudaStream_t) for event timing by callers. */
int sdg_get_stream(sdg_handle* h, void** stream);

/* Waits for all work queued on the handle's stream. */
int sdg_synchronize(sdg_handle* h);

/* Device pointer of a resident field (SDG_FIELD_Q gives the FP64 state). */
int sdg_field_dev_ptr(sdg_handle* h, int which, void** ptr);

/* A resident (Np, NeA) device array as the kernels read it: SDG_FIELD_Q
 * (FP64 state, the input of RK stage 1), SDG_FIELD_U/V/W (velocity at the
 * compute precision) or SDG_ARRAY_STAGE2/3 (inputs of stages 2 and 3);
 * *elem_bytes receives 8 (FP64) or 4 (FP32).  For callers that fill halos
 * themselves (SDG_FLAG_EXTERNAL_HALO): the halo region of each array starts
 * at element Np*Ne.  Replaces the halo buffer of mod_mesh.f90:119-130 as the
 * landing zone of a domain-decomposition exchange. */
int sdg_resident_array(sdg_handle* h, int which, void** ptr, int* elem_bytes);

/* update_halo (mod_mesh.f90:209-221) of the input array of RK stage
 * `stage` (1..3) from this subdomain's own halo_src_map, on the handle's
 * stream.  With SDG_FLAG_EXTERNAL_HALO the caller then overwrites the slots
 * that belong to other subdomains and calls sdg_rk3_stage. */
int sdg_update_halo_stage(sdg_handle* h, int stage);

/* Accumulated device time in seconds: t[0] = tendency/stage kernels of
 * sdg_cal_tend*, t[1] = sdg_rk3_steps, t[2] = halo updates, t[3] = copies
 * of sdg_cal_tend (host<->device). */
int sdg_timers(sdg_handle* h, double* t4);

/* Number of fused-kernel launches issued so far by the handle. */
long long sdg_launch_count(sdg_handle* h);

/* Selects the fused-kernel variant: 0 = automatic (default; also set by the
 * environment variable SDG_KERNEL=block|pipe|blockocc|split at sdg_init),
 * 1 = one element tile per block, 2 = persistent blocks with a bulk-copy
 * (TMA) ring, 3 = one tile per block built for 8 resident blocks (p = 3..7),
 * 4 = the bulk-copy ring with each z-column split over two threads (p >= 8;
 * other orders run variant 2).  All compute identical results; the choice
 * only affects speed. */
int sdg_set_kernel_variant(sdg_handle* h, int variant);

/* Test hook for the failure path of the bounded waits (no reference
 * counterpart: the reference has no device waits; its only error handling
 * is the file-open check of main.f90:117-122).  With tile >= 0, the
 * persistent bulk-copy kernel of this handle never issues the copies of
 * element tile `tile`, so the wait for them runs out after `spins` polls
 * (0: the default limit); the kernel then records a timeout in the
 * handle's status word and returns, and the next synchronising call
 * (sdg_synchronize, sdg_get_field, sdg_minmax) fails with SDG_ERR_CUDA and
 * clears the word.  tile < 0 restores normal operation; the handle stays
 * usable throughout.  Only the pipelined kernel variant has waits. */
int sdg_debug_inject_wait_timeout(sdg_handle* h, int tile, int spins);

/* Host logic of sdg_rk3_steps_host and the chunked sdg_cal_tend, exposed
 * for tests (no device needed).  sdg_debug_chunk_bounds: the chunk
 * boundaries e0[0..S] (S + 1 values, at most cap) that Ne elements of Np
 * nodes get when face neighbours lie within cyclic index distance `reach`
 * (NeX * NeY in a periodic box); *nchunks = S, 0 when the mesh is too small
 * to pipeline.  sdg_debug_step_plan: the launches of `steps` (1..64)
 * chunked RK steps over S chunks whose neighbour lists (each holding the
 * chunk itself; symmetric) are nbr_idx[nbr_ptr[j] .. nbr_ptr[j+1]-1], with
 * or without the chunk uploads: *nops launches as (stage 0 .. 3*steps-1,
 * first chunk, last chunk, upload to wait for or -1) in ops[4 * nops], at
 * most cap ints. */
int sdg_debug_chunk_bounds(int Ne, int Np, int reach, int* e0, int cap, int* nchunks);
int sdg_debug_step_plan(int S, const int* nbr_ptr, const int* nbr_idx, int steps, int uploads,
                        int* ops, int cap, int* nops);

/* ---------------------------------------------------------------------
 * Batched ensembles: many independent periodic-box instances of uneven
 * size and order advanced together (the reference runs one mesh per
 * process, main.f90:51-80; this is its ensemble form).
 * --------------------------------------------------------------------- */
typedef struct sdg_batch sdg_batch;

/* flags: 0 (FMA FP64), SDG_FLAG_EXACT (+ SDG_FLAG_ORDER_GENERAL), or
 * SDG_FLAG_MIXED.  Errors with SDG_ERR_CUDA when no device exists. */
int sdg_batch_create(sdg_batch** b, int flags);

/* Adds a periodic unit box of NeX x NeY x NeZ elements of order p with its
 * operators (D1D, Lift_mat as read by sdg_read_operators; every instance of
 * one order must pass the same operators), initial state q and velocity
 * u, v, w (host arrays of at least Np*Ne values, (Np, Ne) layout) and time
 * step dt.  The mesh tables are those of sdg_mesh_setup on that box.
 * Returns the instance id in *id. */
int sdg_batch_add(sdg_batch* b, int NeX, int NeY, int NeZ, int p,
                  const double* D1D, const double* Lift_mat, const double* q,
                  const double* u, const double* v, const double* w, double dt,
                  int* id);

/* Freezes membership.  Instances of one order form a group whose RK stage
 * is one persistent launch over a tile table; with autotune != 0 each
 * group's tile shape (kernel variant: elements per block x nodes per
 * thread) is chosen by timing the candidates on the group's instances.
 * The environment variable SDG_KERNEL=block|pipe|blockocc|split, when set,
 * overrides the choice for every group whose order supports that variant.
 * One RK step of all groups is captured as a CUDA graph; its groups run one
 * after another. */
int sdg_batch_commit(sdg_batch* b, int autotune);

/* Advances every instance by nsteps SSP-RK3 steps (graph replays);
 * synchronous. */
int sdg_batch_run(sdg_batch* b, int nsteps);

/* Copies instance `id`'s state q (Np, Ne) to the host. */
int sdg_batch_get(sdg_batch* b, int id, double* q);

/* Up to n values: instances, total DOF, run seconds, DOF x steps run,
 * groups, then per group p, mixed, tiles, chosen variant and the tuned
 * stage times (ms) of the pipelined, block, 8-blocks-per-SM and
 * split-column variants (0 where not a candidate).
 * Returns the number of values available. */
int sdg_batch_info(sdg_batch* b, double* out, int n);

/* The batch's form of sdg_debug_inject_wait_timeout: tile `tile` of every
 * group's tile table is skipped; sdg_batch_run then fails with
 * SDG_ERR_CUDA.  A committed batch re-captures its step graph. */
int sdg_batch_debug_inject_wait_timeout(sdg_batch* b, int tile, int spins);

int sdg_batch_destroy(sdg_batch* b);

/* ---------------------------------------------------------------------
 * Serving loop: solve requests admitted as device memory frees up, all
 * admitted requests advanced together one RK step at a time.
 * --------------------------------------------------------------------- */
typedef struct sdg_server sdg_server;

/* Starts a server whose requests may use at most max_bytes of device memory
 * (<= 0: 85% of the memory free now).  A worker thread drives the GPU. */
int sdg_serve_create(sdg_server** s, double max_bytes);

/* Queues a request: the box, operators and host arrays as sdg_batch_add,
 * nsteps RK3 steps, flags 0 (FMA FP64) or SDG_FLAG_MIXED.  The arrays are
 * copied; the call returns at once with the request id.  A request larger
 * than the server's memory cap is rejected with SDG_ERR_ARG. */
int sdg_serve_submit(sdg_server* s, int NeX, int NeY, int NeZ, int p,
                     const double* D1D, const double* Lift_mat, const double* q,
                     const double* u, const double* v, const double* w,
                     double dt, int nsteps, int flags, int* id);

/* State of a request: 0 queued, 1 running, 2 done, 3 failed.  times[0] =
 * queue wait (s, -1 until admitted), times[1] = time to solution (s, -1
 * until done). */
int sdg_serve_poll(sdg_server* s, int id, int* state, double* times2);

/* Copies a done request's final q (Np, Ne) to the host and forgets it. */
int sdg_serve_result(sdg_server* s, int id, double* q);

/* Blocks until no request is queued or running (timeout_s <= 0: no
 * limit); reports the first request failure, if any. */
int sdg_serve_wait(sdg_server* s, double timeout_s);

/* out4: device-busy seconds, DOF x RK steps done, RK iterations run, device
 * bytes held by admitted requests. */
int sdg_serve_stats(sdg_server* s, double* out4);

/* Stops the worker and frees everything. */
int sdg_serve_destroy(sdg_server* s);

/* Sum-factorised x-, y- and z-derivatives of nvar fields per element, on
 * device arrays, asynchronously on `stream` (a cudaStream_t; NULL = the
 * legacy default stream).  Replaces
 * element_operation_kernel_matvec_divlike_dirXYZ_var5_P<p>
 * (mod_dg_optr_kernel_opt1.F90.erb:347-465; nvar = 5 there, any nvar >= 1
 * here): out_x(i,j,k) = sum_l D(i,l) in_x(l,j,k), out_y(i,j,k) =
 * sum_l in_y(i,l,k) D(j,l), out_z(i,j,k) = sum_l in_z(i,j,l) D(k,l), per
 * element and field.  Arrays hold element e, field v, node
 * n = i + Nq*j + Nq^2*k at n + Np*(v + nvar*e) (the reference's per-element
 * vec_in_x(np, np^2*5) stacked over elements); D1D is the host (Nq,Nq)
 * column-major matrix of operator_data.  flags: 0 (FMA, OPT1 order),
 * SDG_FLAG_EXACT (every product and sum rounded, OPT1 order: bit-exact with
 * the reference routine), SDG_FLAG_EXACT | SDG_FLAG_ORDER_GENERAL
 * (mod_dg_optr_kernel.f90:197-258 order).  Outputs must not overlap the
 * inputs.  The reference's y output index (erb:400) overruns its array for
 * kv >= 3; this computes the derivative that routine is written for.
 * Nq = 2..16; SDG_ERR_ARG on bad sizes, flags or null arrays. */
int sdg_divlike_dev(int Nq, int nvar, long long Ne, const double* D1D,
                    const double* in_x, const double* in_y, const double* in_z,
                    double* out_x, double* out_y, double* out_z, int flags,
                    void* stream);

/* The x-, y- and z-derivatives of one field per element (layout as above with
 * nvar = 1), reading the input once.  Replaces
 * element_operation_kernel_matvec_gradlike_dirXYZ_P<p>
 * (mod_dg_optr_kernel_opt1.F90.erb:166-219); the z-derivative's first term
 * reads vec_in(i,j,1)*Mat_tr(1,k) like its other terms (the reference text
 * has vec_in(i,1,k)*Mat_tr(1,j) there, erb:209).  Flags and errors as
 * sdg_divlike_dev. */
int sdg_gradlike_dev(int Nq, long long Ne, const double* D1D, const double* in,
                     double* out_x, double* out_y, double* out_z, int flags,
                     void* stream);

/* min and max of n doubles at device pointer q, written to the device
 * pointer out2 (out2[0] = min, out2[1] = max), asynchronously on `stream`
 * (a cudaStream_t; NULL = the legacy default stream).  No counterpart in the
 * reference: this is sdg_minmax's reduction for callers that cannot
 * allocate device memory (a time loop under a fixed device-memory budget,
 * or a caller with a raw device array and no handle).  It allocates
 * nothing: its scratch is a fixed 64 KB file-scope device array that every
 * GPU loading the library holds until exit, so n may be at most 33,554,432
 * (larger n returns SDG_ERR_ARG).  All calls share that scratch: calls that
 * overlap on the GPU race, so serialise them.  The first call on a device
 * looks up the scratch's address; make it before any stream capture. */
int sdg_minmax_dev_noalloc(const double* q, long long n, double* out2,
                           void* stream);

#ifdef __cplusplus
}
#endif
#endif
