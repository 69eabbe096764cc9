/*
 * mxm_dg.h -- C ABI of the B200 nodal-DG right-hand-side library.
 *
 * Drop-in for mojoxm's hot path: the 3D `Solver[PhysT, P]` stage kernel,
 * SSPRK3 stepping and Barth-Jespersen/Venkatakrishnan cell limiter on
 * periodic/bounded Kuhn tetrahedral meshes, and the 2D per-physics stage
 * kernels on Kuhn triangle meshes.  Conventions follow the reference's only
 * native shim, src/mpi_shim.c: plain C functions, `int` return codes (0 = OK,
 * negative = MXM_DG_E*), opaque `void*` handles, caller-owned host arrays, no
 * structs with implementation-defined layout.  A Mojo binding wraps each call
 * as `external_call["mxm_dg_...", c_int](...)` and raises on rc != 0, as
 * src/mpi.mojo:33-43 does for the MPI shim.
 *
 * State layout (identical to the reference, src/solver.mojo:17-22):
 *   q[(e * NP + i) * NC + c]   element-major, node, then component,
 * elements numbered cell * 6 + tet (3D, cell = i + Nx*(j + Ny*k)) or
 * cell * 2 + tri (2D, cell = j*Nx + i), nodes in the reference's equispaced
 * Lagrange order (src/reference.mojo:136-200, src/reference.mojo:203-237).
 *
 * Threading: one host thread per handle (MPI_THREAD_FUNNELED model of
 * src/mpi_shim.c:44).  All work is enqueued on the handle's own CUDA stream;
 * mxm_dg_synchronize() blocks.  Errors raised asynchronously on the device
 * are reported by the next call that synchronizes.
 */
#ifndef MXM_DG_H
#define MXM_DG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MXM_DG_VERSION 20100 /* 2.1.0: z-slab decomposition; 2.0.0: physics descriptor p[32] */

/* Return codes (mpi_shim.c returns the MPI error code; we use negatives). */
#define MXM_DG_OK 0
#define MXM_DG_EINVAL (-1)     /* bad argument, unsupported P/physics/flux   */
#define MXM_DG_ENOMEM (-2)     /* device allocation failed / over budget     */
#define MXM_DG_ECUDA (-3)      /* CUDA runtime error (message in last_error) */
#define MXM_DG_ENONFINITE (-4) /* non-finite value detected in a reduction   */
#define MXM_DG_ETIMEDOUT (-5)  /* bounded device wait gave up                */
#define MXM_DG_ENOTREADY (-6)  /* request not finished yet (serving poll)    */

/* Physics kinds: src/advection.mojo, src/euler.mojo, src/maxwell.mojo,
 * src/shallow_water.mojo, src/mhd.mojo.  MHD in 3D is IdealMHD (9
 * components); in 2D it is the GLM stack of src/local_mesh_2d_gpu_mhd_glm.mojo
 * (7 components: rho, mx, my, Bx, By, E, psi; psi *= exp(-alpha_d dt) after
 * every SSPRK3 step).  MHD_PLAIN is the 2D stack without cleaning,
 * src/local_mesh_2d_gpu_mhd.mojo (6 components, 2D only). */
#define MXM_DG_PHYS_ADVECTION 0
#define MXM_DG_PHYS_EULER 1
#define MXM_DG_PHYS_MAXWELL 2
#define MXM_DG_PHYS_SHALLOW_WATER 3
#define MXM_DG_PHYS_MHD 4
#define MXM_DG_PHYS_MHD_PLAIN 5
#define MXM_DG_PHYS_TWO_FLUID 6 /* src/two_fluid.mojo, 3D, 17 components */

/* Numerical fluxes.  3D Euler: FLUX_RUSANOV..FLUX_HLLEC (euler.mojo:33-36).
 * 2D Euler: RUSANOV (|v|+c speed, local_mesh_2d_gpu_euler.mojo:220-337),
 * HLLC (:392-545) or HLLE (3D HLLE on the w=0, n_z=0 embedding).
 * 2D shallow water: RUSANOV or HLL (local_mesh_2d_gpu_sw.mojo:178,308).
 * Maxwell and advection have a single flux each and ignore this field. */
#define MXM_DG_FLUX_RUSANOV 0
#define MXM_DG_FLUX_ROE 1
#define MXM_DG_FLUX_HLLE 2
#define MXM_DG_FLUX_HLLEC 3
#define MXM_DG_FLUX_HLLC 4
#define MXM_DG_FLUX_HLL 5

/* Boundary-condition codes, src/boundary.mojo:310-313.  BC_INTERIOR on an
 * axis means periodic. */
#define MXM_DG_BC_INTERIOR 0
#define MXM_DG_BC_WALL 1
#define MXM_DG_BC_OUTFLOW 2
#define MXM_DG_BC_INFLOW 3

/* Arithmetic of a handle. */
#define MXM_DG_PREC_F64 0   /* state, geometry and all arithmetic in FP64       */
#define MXM_DG_PREC_F32 1   /* FP32 state and arithmetic (the reference's path) */
#define MXM_DG_PREC_MIXED 2 /* FP32 state/flux, split-BF16 tensor-core contractions */
/* FP32 state/flux, split-TF32 tensor-core contractions (tcgen05 kind::tf32,
 * hi + lo of 11 significant bits each: the operator carries ~22 bits
 * against 16 for split-BF16, for long linear runs).  3D P = 2..4; where no
 * TF32 tile fits (P = 5, P = 1, 2D, two-fluid) the FP32 kernel runs. */
#define MXM_DG_PREC_MIXED_TF32 3

/* Physics parameters, `p[]` in the field order of the Mojo structs:
 *  ADVECTION (advection.mojo:192-199): p = {vx, vy, vz, inflow_q}
 *  EULER (euler.mojo:534-554): p = {gamma, min_density, min_pressure, gx, gy,
 *        gz, inflow_rho, inflow_rhou, inflow_rhov, inflow_rhow, inflow_E};
 *        flux_type and entropy_fix are the integer fields below.  In 2D the
 *        inflow state is {rho, rhou, rhov, E} = p[6], p[7], p[8], p[10].
 *  MAXWELL (maxwell.mojo:55-74): p = {c, Jx, Jy, Jz, Mx, My, Mz, inflow_Ex,
 *        inflow_Ey, inflow_Ez, inflow_Bx, inflow_By, inflow_Bz}
 *  SHALLOW_WATER (shallow_water.mojo:34-40): p = {g, h_min, inflow_h,
 *        inflow_hu, inflow_hv}
 *  MHD (mhd.mojo:202-254): p = {gamma, min_density, min_pressure, c_h,
 *        alpha_d, inflow_rho, inflow_rhou, inflow_rhov, inflow_rhow,
 *        inflow_E, inflow_Bx, inflow_By, inflow_Bz, inflow_psi}; 9 components
 *        [rho, rho u, rho v, rho w, E, Bx, By, Bz, psi].  2D MHD and
 *        MHD_PLAIN use the same layout (rhow and Bz unused; c_h, alpha_d and
 *        psi only with GLM).
 *  TWO_FLUID (two_fluid.mojo:141-206): p = {gamma_e, gamma_i, q_e, m_e, q_i,
 *        m_i, eps0, c_light, c_h, alpha_d, min_density, min_pressure,
 *        inflow[17]}; 17 components [electrons rho, m, E | ions rho, m, E |
 *        Ex, Ey, Ez, Bx, By, Bz | psi].  MIXED runs it on the FP32 kernel (a
 *        128-row tensor-core tile holds fewer than 8 elements of 17
 *        components); FP64 at P5 exceeds the stage tile's shared memory
 *        (mxm_dg_create returns MXM_DG_EINVAL). */
typedef struct mxm_dg_physics_desc {
  int32_t kind;
  int32_t flux_type;
  int32_t entropy_fix;
  int32_t reserved;
  double p[32];
} mxm_dg_physics_desc;

/* Mesh: dim 3 -> Nx*Ny*Nz cubes x 6 Kuhn tets on [0,Lx]x[0,Ly]x[0,Lz]
 * (src/local_mesh.mojo:1241-1485); dim 2 -> Nx*Ny cells x 2 triangles
 * (src/local_mesh_2d.mojo:106-395, nz/Lz ignored).  bc[] = {x_lo, x_hi,
 * y_lo, y_hi, z_lo, z_hi} (boundary.mojo:328-333; 2D uses the first four). */
typedef struct mxm_dg_mesh_desc {
  int32_t dim;
  int32_t nx, ny, nz;
  double lx, ly, lz;
  int32_t bc[6];
} mxm_dg_mesh_desc;

/* ---- lifetime ----------------------------------------------------------- */
int mxm_dg_version(void);
/* Replaces Solver.__init__(ctx, mesh, halo, physics, D_ref, Lift_ref,
 * node_weights) (src/solver.mojo:595-643) and Mesh[P](...) (mesh.mojo:362):
 * builds operators (host FP64) and mesh tables for order P (1..5), allocates
 * q/q1/q2 zero-filled on the current CUDA device. */
int mxm_dg_create(const mxm_dg_mesh_desc* mesh, const mxm_dg_physics_desc* phys, int P, int precision, void** handle);
int mxm_dg_destroy(void* handle);
/* num_elements, NP, NFP (nodes per face), NC, bytes per state value. */
int mxm_dg_sizes(void* handle, int64_t* num_elements, int32_t* np, int32_t* nfp, int32_t* nc, int32_t* real_bytes);
/* Solver.dof_count (solver.mojo:757-763): num_elements * NP * NC. */
int mxm_dg_dof_count(void* handle, int64_t* dof);
/* Solver.state_bytes_per_step (solver.mojo:804-824): 8 buffer touches per step. */
int mxm_dg_state_bytes_per_step(void* handle, int64_t* bytes);

/* ---- state access ------------------------------------------------------- */
/* Device pointer to d_q (which=0), d_q1 (1) or d_q2 (2), for caller IC
 * kernels (the reference's drivers write solver.d_q directly). */
int mxm_dg_state_ptr(void* handle, int which, void** dptr);
/* Device pointer to node coordinates, float32 [Ne*NP*dim], the reference's
 * elem_node_xyz (local_mesh.mojo:777-845; 2D: local_mesh_2d.mojo:163-180). */
int mxm_dg_node_xyz_ptr(void* handle, void** dptr);
/* Host copies of node coordinates in FP64 [Ne*NP*dim]. */
int mxm_dg_node_xyz(void* handle, double* host);
/* The Float32 coordinates of mxm_dg_node_xyz_ptr on the host (the values
 * the reference's VTU frames store as points). */
int mxm_dg_node_xyz_f32(void* handle, float* host);
/* Copy a whole state buffer from/to caller-owned host memory; `nbytes` must
 * equal Ne*NP*NC*real_bytes.  Synchronous. */
int mxm_dg_upload_state(void* handle, int which, const void* host, size_t nbytes);
int mxm_dg_download_state(void* handle, int which, void* host, size_t nbytes);
/* Solver.download_owned_component (solver.mojo:711-729): component c of d_q
 * for all elements, Float32 [Ne*NP] (as the reference) or FP64. */
int mxm_dg_download_component(void* handle, int c, float* host);
int mxm_dg_download_component_f64(void* handle, int c, double* host);

/* ---- stepping ------------------------------------------------------------ */
/* Solver.enable_cell_limiter (solver.mojo:741-755).  3D: theta over all
 * components; 2D: theta from component 0, BC self-neighbours excluded
 * (local_mesh_2d_gpu_limiter.mojo:74-133).  Default off, eps 0.1. */
int mxm_dg_enable_limiter(void* handle, int on, double venkat_eps);
/* Solver.step_ssprk3 (solver.mojo:1071-1092) / ssprk3_stage_plans. */
int mxm_dg_step_ssprk3(void* handle, double dt);
/* Advance `nsteps` SSPRK3 steps (one enqueue, no host sync). */
int mxm_dg_step_n(void* handle, double dt, int nsteps);
/* One Shu-Osher stage s in {0,1,2} (q->q1, (q,q1)->q2, (q,q2)->q) incl. the
 * limiter when enabled. */
int mxm_dg_rk_stage(void* handle, int stage, double dt);
/* Semi-discrete RHS L(q) of device buffer q_dev into rhs_dev (both
 * Ne*NP*NC values of the handle's real type); no RK combine, no floors. */
int mxm_dg_eval_rhs(void* handle, const void* q_dev, void* rhs_dev);
/* Apply the cell limiter once to state buffer `which`. */
int mxm_dg_limit(void* handle, int which);
/* Host-buffer entry: upload q_host into d_q, take `nsteps` SSPRK3 steps and
 * download d_q into q_out_host (the same layout).  Pinned host memory gives
 * asynchronous copies; pageable memory works too. */
int mxm_dg_advance_host(void* handle, const void* q_host, void* q_out_host, int nsteps, double dt);
/* The same, returning once enqueued: q_out_host holds the result after
 * mxm_dg_synchronize.  Successive calls pipeline (one call's download runs
 * beside the next call's upload and steps); the host buffers must stay
 * valid until the synchronize and should be pinned (mxm_dg_host_alloc).
 * The first call allocates four device staging buffers of one state each
 * (two per direction, used by alternate calls); they live until destroy. */
int mxm_dg_advance_host_async(void* handle, const void* q_host, void* q_out_host, int nsteps, double dt);

/* ---- diagnostics (FP64 device reductions) -------------------------------- */
/* Max over all face nodes of the signal speed numerical_flux/boundary_flux
 * return (discarded by the reference, solver.mojo:266-268), on d_q. */
int mxm_dg_max_wavespeed(void* handle, double* out);
/* kind 0: integral of q_c over the domain (sum_e V_e sum_i w_i q);
 * kind 1: integral of q_c^2 (nodal quadrature); kind 2: max |q_c|;
 * kinds 3 and 4: the reference's DiagnosticsWriter "linear" and "squared"
 * rows (src/diagnostics.mojo:162-229), sum over all nodes of q_c (q_c^2)
 * times domain volume / (elements x nodes per element), without the
 * per-component download.  Reductions accumulate in FP64 on the device in a
 * fixed order. */
int mxm_dg_reduce_conserved(void* handle, int which, int c, int kind, double* out);
/* The same reduction without any device allocation; it has no counterpart
 * in the reference.  Its scratch is a static device array of the library
 * (4096 first-pass partials plus the result slot), so `nblocks`, an upper
 * bound on the first-pass blocks, must lie in 0..4096; the count launched is
 * min(nblocks, ceil(owned elements / 256)) (0 picks the same count as
 * mxm_dg_reduce_conserved, min(ceil(owned elements / 256), 1024), which
 * makes the two results bit-identical); larger values return MXM_DG_EINVAL
 * with a message.  The first call on a device looks the scratch's address
 * up (one-time set-up) and caches it for the life of the library, which
 * assumes the device's primary context lives as long as the library does
 * (no cudaDeviceReset in between); make that first call before any stream
 * capture.  Nothing in the scratch needs to start at zero.  The scratch is
 * shared by all handles on a device: calls whose work overlaps on one
 * device (other host threads, other streams) race on it. */
int mxm_dg_reduce_conserved_noalloc(void* handle, int which, int c, int kind, int nblocks, double* out);

/* ---- misc ---------------------------------------------------------------- */
/* Make `device` the current CUDA device of the calling thread; handles are
 * created on the thread's current device (one process per GPU). */
int mxm_dg_set_device(int device);
/* Page-locked host buffers for asynchronous state transfers. */
int mxm_dg_host_alloc(size_t nbytes, void** host);
int mxm_dg_host_free(void* host);
int mxm_dg_synchronize(void* handle);
/* Time `nsteps` SSPRK3 steps with CUDA events on the handle's stream; the
 * device time in milliseconds goes to *ms. */
int mxm_dg_time_steps(void* handle, double dt, int nsteps, double* ms);
/* Number of kernel launches the handle issues per SSPRK3 step. */
int mxm_dg_launches_per_step(void* handle, int32_t* n);
/* Copies the handle's last error message (NUL-terminated). handle may be NULL
 * for errors raised by mxm_dg_create. */
int mxm_dg_last_error(void* handle, char* buf, int len);
/* Device operator blocks for inspection: the per-tet-type fused
 * [Dx|Dy|Dz|-Lift] matrices in FP64, type-major [ntypes][NP][K]
 * (K = 3*NP + 4*NFP in 3D, 2*NP + 3*(P+1) in 2D).  `count` in/out. */
int mxm_dg_operator(void* handle, double* host, int64_t* count);
/* Reference operators the library built (host FP64): D [dim*NP*NP],
 * Lift [nfaces*NP*NFP] in the reference's face-local order, w [NP]. */
int mxm_dg_reference_operators(int dim, int P, double* D, double* Lift, double* w);

/* Self-test of the bounded device waits the stage kernels use (no
 * reference counterpart): a kernel waits on a barrier that nothing
 * completes, with a `limit_ms` limit (1..2000); it must give up by itself
 * (*gave_up = 1) after about limit_ms (*waited_ms) and leave the context
 * usable.  Runs on the calling thread's current device. */
int mxm_dg_selftest_wait_timeout(double limit_ms, int32_t* gave_up, double* waited_ms);

/* ---- initial conditions on the device ------------------------------------
 * Fill state buffer `which` from node coordinates computed on the device
 * (the role of the reference's IC kernels, e.g. examples/euler_vortex.mojo:
 * 87-129).  params (nparams <= 32):
 *   CONSTANT    NC state values
 *   SINE_WAVE   Euler: rho0, amp, u, v, w, p, kx, ky, kz:
 *               rho = rho0 + amp sin(2 pi (kx x + ky y + kz z)), uniform u, p
 *   VORTEX      Euler isentropic vortex: beta, x0, y0, u, v, w, periodic(0/1)
 *               (nearest periodic image when 1); gamma from the physics
 *   SOD         Euler tanh-smoothed tube along x: rhoL, pL, rhoR, pR, x0, width
 *   DAM_BREAK   shallow water at rest: hL, hR, x0, width
 *   CAVITY      Maxwell: mx, my, amp: E_z = amp sin(mx pi x/Lx) sin(my pi y/Ly)
 *   PLANE_WAVE  Maxwell: amp, k: E_z = amp sin(2 pi k x/Lx), B_y = -E_z/c
 *   ALFVEN      MHD (3D and 2D): rho0, B0, p0, amp, k: right-going Alfven
 *               wave along x, v = amp sin(2 pi k x/Lx), B = (B0, -amp sqrt(rho0)
 *               sin(.), 0), psi = 0 (benchmarks/bench_mhd_alfven_3d_p3.mojo:68-102) */
#define MXM_DG_IC_CONSTANT 0
#define MXM_DG_IC_SINE_WAVE 1
#define MXM_DG_IC_VORTEX 2
#define MXM_DG_IC_SOD 3
#define MXM_DG_IC_DAM_BREAK 4
#define MXM_DG_IC_CAVITY 5
#define MXM_DG_IC_PLANE_WAVE 6
#define MXM_DG_IC_ALFVEN 7
int mxm_dg_fill_ic(void* handle, int which, int kind, const double* params, int nparams);

/* ---- z-slab domain decomposition (np > 1) ---------------------------------
 * Replaces Partition/build_partition (src/partition.mojo:26-228) and
 * HaloExchange (src/halo_exchange.mojo:187-395): one 3D mesh split into
 * `nparts` slabs of whole z layers of cubes, part r owning global layers
 * [r*Nz/nparts, (r+1)*Nz/nparts).  A part's state buffers hold its owned
 * layers between one ghost layer below and one above (where a neighbouring
 * part exists: z periodic, or not the first/last part); the ghost layers are
 * refilled from the neighbours before every stage, and before the limiter.
 * Owned results are bit-identical to the undecomposed solve.  The z
 * boundaries must be both periodic or both bounded.  Reductions,
 * max_wavespeed and download_component cover the owned elements only (sum
 * or max them over the parts for the global value); node coordinates and
 * fill_ic use global positions. */
/* Host-only plan of part `part`: out8 = {cz0, cz1 (owned global z layers),
 * ghost_lo, ghost_hi (0/1), local bc_z_lo, local bc_z_hi, lo neighbour part,
 * hi neighbour part (-1 = none)}.  Needs no GPU. */
int mxm_dg_slab_plan(int nz, int bc_z_lo, int bc_z_hi, int nparts, int part, int32_t* out8);
/* Host-only: the point-to-point operations of part `part`'s ghost exchange
 * in the order the NCCL transport issues them (sends up then down, receives
 * from below then from above; the counterpart of HaloExchange.exchange's
 * message schedule, src/halo_exchange.mojo:313-395).  out12 holds *nops
 * triples {0 send / 1 receive, peer part, local z layer (0 = ghost below
 * when there is one)}.  Needs no GPU. */
int mxm_dg_slab_exchange_ops(int nz, int bc_z_lo, int bc_z_hi, int nparts, int part, int32_t* out12, int* nops);
/* As mxm_dg_create, for part `part` of an nparts-slab decomposition of the
 * global mesh `mesh` (nparts = 1: a plain handle). */
int mxm_dg_create_slab(const mxm_dg_mesh_desc* mesh, const mxm_dg_physics_desc* phys, int P, int precision,
                       int nparts, int part, void** handle);
/* out8 = {nparts, part, cz0, cz1, ghost_lo, ghost_hi, first owned element,
 * owned element count}. */
int mxm_dg_slab_info(void* handle, int64_t* out8);
/* For a caller-driven exchange: out5 = {values per z layer, offset of the
 * bottom owned layer, of the top owned layer, of the ghost layer below, of
 * the ghost layer above (-1 = none)}, offsets in values from the start of a
 * state buffer.  Ghost below <- the lo neighbour's top owned layer; ghost
 * above <- the hi neighbour's bottom owned layer. */
int mxm_dg_slab_layout(void* handle, int64_t* out5);
/* Stage kernel of Shu-Osher stage s over the owned cells only (no exchange,
 * no limiter; the caller refills the ghost layers of the stage's input
 * first and runs mxm_dg_limit on its output after refilling those). */
int mxm_dg_slab_stage(void* handle, int s, double dt);
/* Multi-process transport: rank 0 makes a 128-byte NCCL id and sends it to
 * every part (MPI_Bcast or any other channel); each part then connects
 * (collective: all parts call it) and afterwards steps by itself
 * (mxm_dg_step_ssprk3 / step_n / rk_stage exchange over NCCL point-to-point
 * on the handle's stream).  NCCL is loaded at run time (libnccl.so.2). */
int mxm_dg_nccl_unique_id(unsigned char* id128);
int mxm_dg_slab_connect_nccl(void* handle, const unsigned char* id128);
/* In-process transport: the parts 0..n-1 (on one or several devices of this
 * process) stepped in lock-step by one host thread; ghost layers are copied
 * with cudaMemcpyPeerAsync, ordered by events.  The group does not own the
 * handles; destroy it before them. */
int mxm_dg_group_create(void* const* handles, int n, void** group);
int mxm_dg_group_step_n(void* group, double dt, int nsteps);
int mxm_dg_group_synchronize(void* group);
/* `nsteps` group steps timed with CUDA events that bracket every part's work. */
int mxm_dg_group_time_steps(void* group, double dt, int nsteps, double* ms);
int mxm_dg_group_last_error(void* group, char* buf, int len);
int mxm_dg_group_destroy(void* group);

/* ---- batched engine (no reference counterpart: the reference runs each
 * 2D solve through its own driver loop, examples/euler_sod_2d_gpu.mojo +
 * src/ssprk3.mojo:56-78) ----------------------------------------------------
 * A batch advances many independent 2D solves of uneven mesh size, order P
 * and physics together: per SSPRK3 stage one persistent stage launch per
 * physics group (solves whose physics descriptors are identical) plus the
 * two limiter passes for groups with limited solves, the whole step captured
 * once in a CUDA graph and replayed.  Members are ordinary solver handles
 * (2D, one precision per batch); their state stays in their own buffers and
 * each advances with its own dt.  Enable limiters and upload states before
 * the first batch step; adding a solve re-plans the batch.  Synchronize the
 * batch before reading a member's state; destroy the batch before its
 * members. */
int mxm_dg_batch_create(void** batch);
int mxm_dg_batch_destroy(void* batch);
int mxm_dg_batch_add(void* batch, void* solver, double dt, int32_t* index);
/* Pick the cells per tile of every (physics group, P) by timing the batched
 * stage kernel on the batch's own solves; runs by itself on the first step
 * when not called. */
int mxm_dg_batch_autotune(void* batch);
/* The tuned cells per tile used for member `member`. */
int mxm_dg_batch_tile_cells(void* batch, int member, int32_t* cells);
/* `nsteps` SSPRK3 steps of every member (one graph replay per step). */
int mxm_dg_batch_step(void* batch, int nsteps);
/* As mxm_dg_batch_step, timed with CUDA events on the batch stream. */
int mxm_dg_batch_time_steps(void* batch, int nsteps, double* ms);
int mxm_dg_batch_synchronize(void* batch);
/* Sum over members of Ne*NP*NC. */
int mxm_dg_batch_dof_count(void* batch, int64_t* dof);
/* Kernel launches per batched SSPRK3 step. */
int mxm_dg_batch_launches_per_step(void* batch, int32_t* n);
/* Last error message of the batch (batch may be NULL for create errors). */
int mxm_dg_batch_last_error(void* batch, char* buf, int len);

/* ---- serving loop (no reference counterpart) -----------------------------
 * Continuous batching of independent solves on the calling thread's device:
 * a scheduler thread admits submitted requests in arrival order while their
 * device footprint (three state buffers, limiter means and nodal extrema,
 * operator) fits `hbm_budget_bytes` and fewer than `max_active` are
 * running, builds each on
 * its own stream (handle + device IC fill, see mxm_dg_fill_ic) and feeds
 * every running solve chunks of `steps_per_chunk` SSPRK3 steps, so requests
 * that arrive while others run are admitted as memory frees up and their
 * kernels overlap.  A finished solve's state (buffer q, Ne*NP*NC values of
 * its real type) is copied to `out_host` (caller-owned, may be NULL) and its
 * memory released; latency = submit -> result on the host.  Each solve's
 * arithmetic is that of a single solve on its own buffers.  All calls are
 * thread-safe. */
int mxm_dg_server_create(double hbm_budget_bytes, int max_active, int steps_per_chunk, void** server);
/* Stops the scheduler: queued requests fail, running ones are drained. */
int mxm_dg_server_destroy(void* server);
int mxm_dg_server_submit(void* server, const mxm_dg_mesh_desc* mesh, const mxm_dg_physics_desc* phys, int P,
                         int precision, int ic_kind, const double* ic_params, int nparams, int limiter,
                         double venkat_eps, double dt, int nsteps, void* out_host, int64_t* request_id);
/* MXM_DG_OK when finished, MXM_DG_ENOTREADY while queued or running. */
int mxm_dg_server_poll(void* server, int64_t request_id, double* latency_ms);
/* Block until finished or `timeout_s` passes (MXM_DG_ETIMEDOUT). */
int mxm_dg_server_wait(void* server, int64_t request_id, double timeout_s, double* latency_ms);
/* out[0] completed, [1] failed, [2] p50 ms, [3] p99 ms, [4] mean ms,
 * [5] solves/s and [6] DOF·stage/s from the first submit to the last
 * completion, [7] peak admitted bytes, [8] peak concurrent solves,
 * [9] queued now, [10] running now, [11] admitted bytes now. */
int mxm_dg_server_stats(void* server, double* out, int n);
int mxm_dg_server_last_error(void* server, char* buf, int len);

#ifdef __cplusplus
}
#endif
#endif /* MXM_DG_H */
