/* cfdb.h -- C ABI of the B200-native cfdARCO finite-volume time step.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status (CFDB_OK = 0) and never aborts the process; the message of the
 * last failure is read with cfdb_last_error().  Device work is enqueued on the
 * context's stream (cfdb_ctx_set_stream) and is asynchronous unless the
 * comment says otherwise.  Field pointers are DEVICE pointers holding n cells
 * in the reference's cell order (id = Z*Y*x + Z*y + z, z fastest;
 * src/mesh3d.cpp:387-389); multi-field states are stored field after field
 * ([p|u|v|w] for the wave system, [rho|mx|my|mz|E] for Euler).
 *
 * The comment above each function names the reference interface it replaces
 * (paths inside int0vrt/cfdARCOV2).
 */
#ifndef CFDB_H
#define CFDB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFDB_ABI_VERSION 1

/* Status codes.  Replaces gpuAssert() -> exit(code)
 * (include/cuda_operators.hpp:29-36) and the std::runtime_error throws of
 * src/fvm3d.cpp:475-476. */
enum {
  CFDB_OK = 0,
  CFDB_EINVAL = 1,       /* bad argument (null pointer, size, dtype, mask) */
  CFDB_ENOMEM = 2,       /* device or host allocation failed / over budget */
  CFDB_ECUDA = 3,        /* a CUDA runtime call failed */
  CFDB_ETIMEOUT = 4,     /* a bounded device-side wait gave up */
  CFDB_ENUMERIC = 5,     /* non-finite values detected */
  CFDB_EUNSUPPORTED = 6, /* valid request this build or mesh kind cannot serve */
  CFDB_EIO = 7           /* a file could not be written */
};

/* Arithmetic type of a field (the reference computes in float only,
 * include/decls.hpp:25-29). */
enum { CFDB_F32 = 0, CFDB_F64 = 1 };

/* Execution path of a time step. */
enum {
  CFDB_PATH_PLAIN = 0, /* per-operator kernels over the reference's N x 6 geometry arrays */
  CFDB_PATH_FUSED = 1  /* one kernel per step: TMA-staged tiles (uniform mesh) or the
                          compact area-vector gather (vertex mesh) */
};

/* Binary / scalar operator codes of cfdb_op_binary / cfdb_op_scalar. */
enum { CFDB_OP_ADD = 0, CFDB_OP_SUB = 1, CFDB_OP_MUL = 2, CFDB_OP_DIV = 3,
       CFDB_OP_RSUB = 4, /* scalar - a */
       CFDB_OP_RDIV = 5  /* scalar / a */ };

/* Host copies of the reference's flattened geometry (cfdb_mesh_geometry). */
enum { CFDB_GEOM_NORMAL = 0,     /* 3 x 6N  (_normal_x/_y/_z)          */
       CFDB_GEOM_NORMAL_ALT = 1, /* 3 x 6N  (_normal_alt_x/_y/_z)      */
       CFDB_GEOM_AREA = 2,       /* 6N      (_face_areas)              */
       CFDB_GEOM_ALPHA_D = 3,    /* 6N      (_alpha_d)                 */
       CFDB_GEOM_LEN_C2F = 4,    /* 6N      (_len_node_center_to_face) */
       CFDB_GEOM_VOLUME = 5,     /* N       (_volumes)                 */
       CFDB_GEOM_CENTER = 6,     /* 3 x N   cell centres               */
       CFDB_GEOM_IS_BOUNDARY = 7 /* N       (_node_is_boundary)        */ };

/* cfdb_mesh_create_from_vertices flags. */
enum { CFDB_MESH_COMPAT_AREA = 1 /* reference geometry formulas verbatim, src/mesh3d.cpp:43-105 */ };

typedef struct cfdb_ctx cfdb_ctx;
typedef struct cfdb_mesh cfdb_mesh;
typedef struct cfdb_euler cfdb_euler;
typedef struct cfdb_batch cfdb_batch;

/* ---- context, errors, memory ------------------------------------------ */

int cfdb_abi_version(void);

/* CFDArcoGlobalInit::initialize + enable_cuda (src/cfdarcho_main_3d.cpp:276-347;
 * include/cfdarcho_main_3d.hpp:33-79): binds a device; no memory pool. */
int cfdb_ctx_create(int device, cfdb_ctx** out);

/* CFDArcoGlobalInit::finalize (src/cfdarcho_main_3d.cpp:53-62). */
int cfdb_ctx_destroy(cfdb_ctx* ctx);

/* Message of the last failure on ctx (ctx may be NULL for failures that had no
 * context); replaces gpuAssert's stderr print (include/cuda_operators.hpp:29-36). */
const char* cfdb_last_error(const cfdb_ctx* ctx);

/* The reference runs everything on the default stream with a device sync
 * after each kernel (src/cuda_operators.cu:184,303,463,484,567); here the
 * caller picks the stream (a cudaStream_t passed as void*, NULL = default). */
int cfdb_ctx_set_stream(cfdb_ctx* ctx, void* stream);

/* sync_device() (include/cuda_operators.hpp:93-96, src/fvm3d.cpp:1391-1393). */
int cfdb_sync(cfdb_ctx* ctx);

/* Caps the device bytes this context may allocate (0 = no cap); allocations
 * beyond it fail with CFDB_ENOMEM.  Host-side fault injection in place of the
 * RMM pool exhaustion the reference hit (rmm_log.txt:2). */
int cfdb_ctx_set_alloc_budget(cfdb_ctx* ctx, int64_t bytes);
int cfdb_ctx_allocated_bytes(const cfdb_ctx* ctx, int64_t* out);

/* Per-call workspaces (cfdb_wave_gradient's checkpoint slots, adjoint and
 * objective buffers) come from a stream-ordered pool owned by the context;
 * freed workspace stays cached there, so repeated calls of one size do not
 * allocate.  Returns the cached, unused blocks to the device (synchronises
 * the context's stream).  No reference counterpart: the reference's RMM pool
 * (src/pool_allocator.cpp:20, sized at src/cfdarcho_main_3d.cpp:335-341) is
 * never trimmed. */
int cfdb_ctx_trim(cfdb_ctx* ctx);

/* Bound of every device-side wait of the TMA sweep kernels, in SM clock
 * cycles (default 4e9, about 2 s), after which a launch gives up, lets the
 * copies it issued land, and reports CFDB_ETIMEOUT through cfdb_sync; its
 * results are then invalid and the context stays usable.  missing_plane >= 0
 * is a test hook: the first CTA of every later sweep arms that plane's
 * barrier without issuing its copy, and the second cluster of the
 * cluster-resident heat solver (cfdb_heat_run) does not publish its edge
 * planes of that step, so a wait runs out without any fault (-1 turns it
 * off).  The resident solver's waits (for a neighbouring cluster's planes)
 * have the same bound.  Drops the context's cached step graphs.  No reference
 * counterpart: the reference's kernels have no waits, and gpuAssert exits
 * the process on any CUDA error (include/cuda_operators.hpp:29-36). */
int cfdb_ctx_set_wait_limit(cfdb_ctx* ctx, int64_t cycles, int32_t missing_plane);

/* Kernels this context has launched so far, those run by CUDA-graph replays
 * included (each replay adds the kernels it runs).  No reference
 * counterpart; benchmarks read it around a timed region. */
int cfdb_ctx_launch_count(const cfdb_ctx* ctx, int64_t* out);

/* CudaDataMatrix<T> allocation and from_eigen / to_eigen
 * (include/cuda_data_matrix.hpp:60-188).  upload/download are synchronous
 * with respect to the host buffer. */
int cfdb_alloc(cfdb_ctx* ctx, int64_t bytes, void** out);
int cfdb_free(cfdb_ctx* ctx, void* ptr);
int cfdb_upload(cfdb_ctx* ctx, void* dst_device, const void* src_host, int64_t bytes);
int cfdb_download(cfdb_ctx* ctx, void* dst_host, const void* src_device, int64_t bytes);
/* The same copies queued on the context's stream without waiting: the host
 * buffer must stay valid (and, for a download, unread) until the stream has
 * passed the copy (cfdb_sync, or a later stream event).  With page-locked
 * host memory the copy runs on a copy engine, overlapping kernels of other
 * streams.  A caller that streams solves puts the copies on a second
 * context bound to its own stream.  No reference counterpart: from_eigen /
 * to_eigen are synchronous. */
int cfdb_upload_async(cfdb_ctx* ctx, void* dst_device, const void* src_host, int64_t bytes);
int cfdb_download_async(cfdb_ctx* ctx, void* dst_host, const void* src_device, int64_t bytes);

/* ---- mesh ------------------------------------------------------------- */

/* Mesh3D(x, y, z, dx, dy, dz) + init_basic_internals() + compute() +
 * CudaMesh3D::host_to_device() (include/mesh3d.hpp:120-125,209-236;
 * src/mesh3d.cpp:151-385).  The device's face arrays are computed on the
 * device on first use (in double, rounded to the storage type); the host
 * copies (cfdb_mesh_geometry) are computed on the host, from the same
 * formulas, when first asked for.  ctx may be NULL for a host-only mesh (the
 * geometry queries work; device calls fail with CFDB_EINVAL). */
int cfdb_mesh_create_structured(cfdb_ctx* ctx, int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
                                double dz, cfdb_mesh** out);

/* Mesh3D::compute over caller-supplied vertex coordinates (src/mesh3d.cpp:43-105):
 * vertices holds (nx+1)(ny+1)(nz+1) x 3 doubles in vertex-id order
 * (src/mesh3d.cpp:405-416).  By default every face gets its exact vector
 * area S = (C - A) x (D - B) / 2 (n = S/|S|, A = |S|) and cell volumes are
 * taken about the cell centre, so jittered cells stay closed and positive;
 * CFDB_MESH_COMPAT_AREA keeps the reference formulas verbatim (one-triangle
 * normal, component-sum area).  Tangled cells (volume <= 0) are rejected.
 * dx/dy/dz are the nominal spacings used for CFL conventions. */
int cfdb_mesh_create_from_vertices(cfdb_ctx* ctx, int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
                                   double dz, const double* vertices, int flags, cfdb_mesh** out);

int cfdb_mesh_destroy(cfdb_mesh* mesh);

/* Mesh3D::_num_nodes, _x/_y/_z, _dx/_dy/_dz (include/mesh3d.hpp:137-151);
 * *is_uniform = 1 for cfdb_mesh_create_structured meshes. */
int cfdb_mesh_info(const cfdb_mesh* mesh, int64_t dims[3], double spacing[3], int* is_uniform);

/* Host copy of one flattened geometry array (Mesh3D::_normal_x ... _volumes,
 * include/mesh3d.hpp:155-173), in double. */
int cfdb_mesh_geometry(const cfdb_mesh* mesh, int which, double* out);

/* Mesh3D::_ids and _ids_bound_free (include/mesh3d.hpp:165-166), 6N each. */
int cfdb_mesh_ids(const cfdb_mesh* mesh, int64_t* ids, int64_t* ids_bound_free);

/* ---- operator layer (include/cuda_operators.hpp:38-96) ------------------
 * dims_mask bit 0/1/2 = x/y/z, the clc_x/clc_y/clc_z flags of
 * d1dx/d1dy/d1dz, d2dx..., lapl, stab* (include/fvm3d.hpp:421-511). */

/* GradVar::evaluate_cu -> eval_grad (src/fvm3d.cpp:825-829; src/cuda_operators.cu:237-305). */
int cfdb_op_grad(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, const void* phi, void* out, int dims_mask);

/* Grad2Var::evaluate_cu -> eval_grad2 (src/fvm3d.cpp:902-905; src/cuda_operators.cu:490-569). */
int cfdb_op_lapl(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, const void* phi, void* out, int dims_mask);

/* StabVar::evaluate_cu -> eval_stab (src/fvm3d.cpp:938-941; src/cuda_operators.cu:307-487).
 * Uses a mesh-owned 18N temporary allocated on first call. */
int cfdb_op_stab(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, const void* phi, void* out, int dims_mask);

/* add_mtrx / sub_mtrx / mul_mtrx / div_mtrx (src/cuda_operators.cu:27-106);
 * Variable::operator+ - * / (src/fvm3d.cpp:378-405). */
int cfdb_op_binary(cfdb_ctx* ctx, int dtype, int op, const void* a, const void* b, void* out, int64_t n);

/* mul_mtrx(a, float), div_const (src/cuda_operators.cu:62-120) and the
 * float-operand overloads (src/fvm3d.cpp:434-470): out = a op s, or s op a for
 * CFDB_OP_RSUB / CFDB_OP_RDIV. */
int cfdb_op_scalar(cfdb_ctx* ctx, int dtype, int op, const void* a, double s, void* out, int64_t n);

/* neg_mtrx (src/cuda_operators.cu:122-136). */
int cfdb_op_neg(cfdb_ctx* ctx, int dtype, const void* a, void* out, int64_t n);

/* Constant Variable / DT::evaluate_cu / PointerVariable::evaluate_cu
 * (src/fvm3d.cpp:122-148, 670-672, 570-583). */
int cfdb_op_fill(cfdb_ctx* ctx, int dtype, void* out, double value, int64_t n);

/* DtVar::extract_cu: next = dt * rhs + cur (src/fvm3d.cpp:694-697). */
int cfdb_op_d1t(cfdb_ctx* ctx, int dtype, const void* rhs, const void* cur, double dt, void* next, int64_t n);

/* D2tVar::extract_cu: next = dt*dt*rhs + 2*cur - prev, or dt*rhs + cur when
 * second_order == 0 (first step) (src/fvm3d.cpp:742-751). */
int cfdb_op_d2t(cfdb_ctx* ctx, int dtype, const void* rhs, const void* cur, const void* prev, double dt,
                int second_order, void* next, int64_t n);

/* _boundary_copy_cu: out = arr * (1 - is_boundary) + copy * is_boundary
 * (examples/main_3d_heat.cpp:41-46). */
int cfdb_op_boundary_copy(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, const void* arr, const void* copy,
                          void* out);

/* The boundary copy in place, touching the boundary cells only: field[i] =
 * values[i] for every cell on the box surface (the cells whose
 * _node_is_boundary is 1), all other cells untouched.  Equals
 * cfdb_op_boundary_copy(arr = out = field) for finite states up to the sign
 * of interior zeros (the reference's blend turns -0 into +0), and reads and
 * writes 2 x 6N^2 cells of an N^3 mesh instead of streaming all N^3 three
 * times. */
int cfdb_op_boundary_set(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, void* field, const void* values);
/* cfdb_op_boundary_set for `count` fields at once (fields[k] from values[k]),
 * one launch per 16 fields: the boundary copies of a system's variables
 * after a step (src/fvm3d.cpp:1008-1049 applies them one variable at a
 * time). */
int cfdb_op_boundary_set_many(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, int32_t count, void* const* fields,
                              const void* const* values);

/* UpdatePolicies::CourantFriedrichsLewy3DCu / 1DCu + cfl_cu
 * (src/fvm3d.cpp:528-567; src/cuda_operators.cu:138-235):
 * *dt_out = cfl * min_P dl / (sqrt(gamma p / rho) + |u|), dl = min spacing.
 * v and w may be NULL (1-D form).  Synchronous: waits for the result. */
int cfdb_cfl_dt(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, double cfl, double gamma, const void* p,
                const void* rho, const void* u, const void* v, const void* w, double* dt_out);

/* Neumaier-compensated FP64 total sum_P field_P * V_P, returned to the host
 * (synchronous).  No counterpart in the reference (it prints float sums,
 * src/fvm3d.cpp:1060-1066). */
int cfdb_total_fp64(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, const void* field, double* out);

/* The same compensated FP64 total, sum_P field_P * V_P, for callers that may
 * not allocate device memory (a plugin whose host application owns every
 * device allocation, a step recorded into another framework's CUDA graph, a
 * loop that cannot pay for cudaMalloc's implicit synchronisation).  It needs
 * no context and calls no cudaMalloc, cudaFree or allocating routine: its
 * reduction scratch is a fixed 1 MiB array inside the library, held by every
 * GPU that loads the library until exit.  No counterpart in the reference.
 * field: n values of dtype on the current device; volumes: n per-cell
 * volumes of dtype, or NULL to use `volume` for every cell; out_device: one
 * double in device memory receiving the total; stream: a cudaStream_t (NULL =
 * default).  Asynchronous.  n may be at most 268,435,456 cells (larger n
 * returns CFDB_EINVAL without launching).  Every call overwrites the scratch
 * it uses, so nothing needs clearing, but all calls share it: calls that
 * overlap on the GPU race and must be serialised by the caller.  The first
 * call on a device looks up the scratch's device address; make it before any
 * stream capture.  That address is kept for the life of the process: after a
 * cudaDeviceReset, reload the library before calling this again on that
 * device.  Errors are read with cfdb_last_error(NULL). */
int cfdb_total_fp64_noalloc(int dtype, const void* field, const void* volumes, double volume, int64_t n,
                            void* stream, double* out_device);

/* ---- fused time steps (KernelBuilder replacement, src/fvm3d.cpp:1219-1394) */

/* Heat equation d1t(T) = k * lapl(T) with zero-gradient walls
 * (examples/main_3d_heat.cpp:89-91): T_next = T + dt * k * lapl(T).
 * PLAIN = lapl kernel + update kernel; FUSED = one TMA-tiled kernel
 * (uniform meshes, CFDB_F32 or CFDB_F64). */
int cfdb_heat_step(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, int path, const void* T, void* T_next, double k,
                   double dt);

/* The fused heat step followed by the examples' boundary copy
 * (examples/main_3d_heat.cpp:41-60: the cells of the box surface reset to
 * fixed values after each step) in the same pass: T_next = the heat update
 * inside, fixed[i] on the surface cells.  The same values as cfdb_heat_step
 * followed by cfdb_op_boundary_set.  CFDB_F32, uniform meshes with
 * nz % 4 == 0, 16-byte aligned T and T_next. */
int cfdb_heat_step_fixed(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, const void* T, void* T_next, double k, double dt,
                         const void* fixed);

/* Leapfrog step of d2t(u) = k * (L_m1(u) + L_m2(u) + ...) with L_m the
 * Laplacian over the directions of mask m (1 = d2dx, 2 = d2dy, 4 = d2dz,
 * 7 = lapl) -- the equation examples/main_3d_wave.cu builds, whose
 * KernelBuilder kernel (src/fvm3d.cpp:1219-1394, update src/fvm3d.cpp:710-765)
 * this replaces with one TMA-tiled pass.  first_step != 0: u_next = dt R + u
 * (u_prev unused, may be NULL); else u_next = (dt dt R + 2 u) - u_prev.
 * Rounds like the operator kernels and the generated ones, operation by
 * operation, so all give the same bits.  CFDB_F32 on an exact lattice
 * (cfdb_mesh_lattice_geometry) with nz % 4 == 0 and 16-byte aligned fields;
 * CFDB_EUNSUPPORTED otherwise. */
int cfdb_d2t_step(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, const void* u, const void* u_prev, void* u_next,
                  double k, const int32_t* masks, int32_t n_terms, double dt, int first_step);

/* First-order acoustic system (p,u,v,w), rho = 1: p_t = -c^2 div u,
 * u_t = -grad p, Rusanov face flux, reflective walls, forward Euler.
 * c_field (n values, same dtype) may be NULL for the constant c_const.
 * speed_mode 0: face speed max(c_P, c_N); 1: (c_P + c_N)/2 (differentiable).
 * No reference counterpart (first-order form of examples/main_3d_wave.cu). */
int cfdb_wave_step(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, int path, const void* q, void* q_next,
                   const void* c_field, double c_const, int speed_mode, double dt);

/* The time loop of Equation::evaluate (src/fvm3d.cpp:1008-1058) for a single
 * equation: `steps` steps alternating a -> b -> a ...; *final_in_b = 1 when
 * the last state is in b.  use_graph captures the step launches into a CUDA
 * graph (after two eager steps that perform any one-time setup) and replays
 * it, so host launch latency never gaps the device.  Asynchronous.
 * cfdb_heat_run, fused FP32: a uniform mesh whose field fits twice into the
 * shared memory of one thread-block cluster (e.g. 64^3), or else of four
 * co-resident clusters (e.g. 128 x 64 x 64), runs all steps in one launch
 * instead, field resident on chip; same arithmetic, same result.  Only the
 * buffer *final_in_b names is defined afterwards. */
int cfdb_heat_run(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, int path, void* T_a, void* T_b, double k, double dt,
                  int32_t steps, int use_graph, int* final_in_b);
int cfdb_wave_run(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, int path, void* q_a, void* q_b, const void* c_field,
                  double c_const, int speed_mode, double dt, int32_t steps, int use_graph, int* final_in_b);

/* Stable step for cfdb_wave_step: cfl * min_P 2 V_P / sum_f c_P A_f
 * (= cfl / sum_d c/dx_d on a uniform mesh).  c_host (n doubles) may be NULL. */
int cfdb_wave_dt(const cfdb_mesh* mesh, const double* c_host, double c_const, double cfl, double* dt_out);

/* ---- compressible Euler (first-order Rusanov) ---------------------------
 * Replaces the Equation::evaluate loop of the Euler examples
 * (src/fvm3d.cpp:969-1069; examples/main_3d_sod_shock.cpp) with device-side
 * dt: each step reads the previous step's per-direction max signal speeds,
 * sets dt = cfl / sum_d(lam_d / dx_d), clips the last step onto t_end, and
 * writes FP64 Neumaier totals (sum rho V, sum E V) per step.  Faces in
 * slots 4/5 (x ends) are zero-gradient, the others reflective walls. */
int cfdb_euler_create(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, int path, double gamma, double cfl,
                      double t_end, int64_t max_steps, cfdb_euler** out);
int cfdb_euler_destroy(cfdb_euler* e);
/* Resets the clock to t = 0 and derives the first dt and totals from U0. */
int cfdb_euler_begin(cfdb_euler* e, const void* U0);
/* One step U -> U_next (a no-op once t_end is reached; then U_next is not written). */
int cfdb_euler_step(cfdb_euler* e, const void* U, void* U_next);
/* Synchronous: simulated time, steps taken and whether t_end was reached. */
int cfdb_euler_status(cfdb_euler* e, double* t, int64_t* steps_done, int* finished);
/* Synchronous: totals rows (2 doubles each: sum rho V, sum E V), row 0 = initial state. */
int cfdb_euler_totals(cfdb_euler* e, double* out, int64_t max_rows, int64_t* rows);
/* Runs to t_end alternating U_a -> U_b -> U_a ..., checking the clock every
 * check_every steps; *final_in_b = 1 when the last state is in U_b.  At each
 * check a non-finite conservation total (a NaN or Inf in the state) stops
 * the run with CFDB_ENUMERIC. */
int cfdb_euler_run(cfdb_euler* e, void* U_a, void* U_b, int64_t check_every, int64_t* steps_done,
                   int* final_in_b);

/* ---- batched ensemble of independent small problems ---------------------
 * No reference counterpart (one mesh per process there).  Each problem is a
 * cube of n^3 uniform cells on [0,1]^3: kind 0 = heat (param = k), kind 1 =
 * wave system (param = c, reflective walls); dt per problem.  All problems
 * advance together in one persistent launch per step; cfdb_batch_run replays
 * the step from a CUDA graph. */
typedef struct {
  int32_t n;      /* cells per edge */
  int32_t kind;   /* 0 heat, 1 wave */
  double param;   /* k (heat) or c (wave) */
  double dt;      /* time step */
  int64_t offset; /* first element of this problem in the state pool (set by the library) */
} cfdb_problem;

/* probs[i].offset is filled in on return; *pool_elems = elements (of dtype
 * F32) one state pool must hold: the problems' cells plus 4 spare floats
 * before the first problem and 4 after the last (the kernels read, and
 * discard, one float beyond a column's end and the staged kernel's 16-byte
 * copies may reach past the last problem). */
int cfdb_batch_create(cfdb_ctx* ctx, cfdb_problem* probs, int32_t count, int64_t* pool_elems, cfdb_batch** out);
int cfdb_batch_destroy(cfdb_batch* b);
/* cells_per_item: cells one CTA work item covers (threads (y, z) columns x
 * cells_per_item / threads x planes); threads: CTA size; ctas_per_sm:
 * persistent grid = SMs x ctas_per_sm. */
int cfdb_batch_set_config(cfdb_batch* b, int32_t cells_per_item, int32_t threads, int32_t ctas_per_sm);
int cfdb_batch_get_config(const cfdb_batch* b, int32_t* cells_per_item, int32_t* threads, int32_t* ctas_per_sm);
/* Kernel form: 0 (the default) = the column march (one (y, z) column per
 * thread, neighbours through L1); 2 = the same compiled to 48 registers
 * (blocks of up to 256 threads: more resident warps); 1 = the staged form,
 * which streams each work item's plane rows into a shared-memory ring with
 * bulk copies (a producer warp and `threads` consumer threads per CTA; needs
 * 16-byte aligned pools and a ring that fits shared memory, otherwise the
 * column march runs).  All give the same bits.  cfdb_batch_tune times every
 * form and keeps the fastest (its cache entries record the form). */
int cfdb_batch_set_staged(cfdb_batch* b, int staged);
/* Autotuner: times candidate configurations on the given pools (contents are
 * advanced and must be re-initialised afterwards) and keeps the fastest;
 * results are cached in cache_path (JSON, may be NULL) keyed by device and
 * problem set. */
int cfdb_batch_tune(cfdb_batch* b, void* pool_a, void* pool_b, const char* cache_path);
/* One step a -> b (one persistent launch). */
int cfdb_batch_step(cfdb_batch* b, const void* pool_a, void* pool_b);
/* steps steps alternating a -> b -> a ...; use_graph replays a captured
 * two-step CUDA graph.  The final state is in a when steps is even. */
int cfdb_batch_run(cfdb_batch* b, void* pool_a, void* pool_b, int32_t steps, int use_graph);
/* Kernel launches the last cfdb_batch_run enqueued (graph replays count their nodes). */
int cfdb_batch_launch_count(const cfdb_batch* b, int64_t* out);

/* ---- discrete adjoint of the wave step (speed_mode 1) -------------------
 * No reference counterpart.  lam_n = lam_next + dt A(c)^T lam_next and
 * grad_c += dt (d(A(c) q_n)/dc)^T lam_next, applied as a gather over the six
 * neighbours (transpose of the flux scatter). */
int cfdb_wave_adjoint_step(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, int path, const void* q_n,
                           const void* lam_next, void* lam_n, const void* c_field, void* grad_c, double dt);

/* Statistics of a cfdb_wave_gradient run. */
typedef struct {
  int64_t forward_steps;  /* forward steps taken including recomputation */
  int64_t adjoint_steps;  /* reverse steps */
  int32_t snapshots_used; /* checkpoint slots used */
  int32_t reserved;
  double forward_ms;      /* device time of the forward sweep (first pass) */
  double reverse_ms;      /* device time of the reverse sweep incl. recomputation */
} cfdb_gradient_stats;

/* J = 0.5 |p_T - p_target|^2 after `steps` wave steps (speed_mode 1) from q0,
 * and its gradient with respect to c (grad_c, n values) and p0 (grad_p0, n
 * values).  snapshots = checkpoint slots (>= steps stores every state;
 * fewer uses binomial checkpointing after Griewank and Walther, ACM TOMS
 * 26(1) 2000, Alg. 799 "revolve").  Synchronous; *J_out on the host. */
int cfdb_wave_gradient(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, int path, const void* q0,
                       const void* c_field, const void* p_target, int32_t steps, double dt, int32_t snapshots,
                       double* J_out, void* grad_c, void* grad_p0, cfdb_gradient_stats* stats);

/* J only (forward run, no storage); synchronous. */
int cfdb_wave_objective(cfdb_ctx* ctx, cfdb_mesh* mesh, int dtype, int path, const void* q0,
                        const void* c_field, const void* p_target, int32_t steps, double dt, double* J_out);

/* Action codes of a checkpointing schedule (host only, no device needed). */
enum { CFDB_RV_ADVANCE = 1,  /* arg = steps to advance from the current state  */
       CFDB_RV_TAKESHOT = 2, /* arg = slot: store the current state            */
       CFDB_RV_RESTORE = 3,  /* arg = slot: load the current state from a slot */
       CFDB_RV_FIRSTURN = 4, /* first adjoint step (current state = step T-1)  */
       CFDB_RV_YOUTURN = 5   /* adjoint step of the current state              */ };

/* Binomial checkpointing schedule for `steps` steps with `snapshots` slots.
 * Writes up to capacity (action, arg, step) triples; *count = actions needed
 * (call with capacity 0 to size the buffers); *forward_steps = total
 * forward steps the schedule performs. */
int cfdb_revolve_plan(int32_t steps, int32_t snapshots, int32_t* actions, int32_t* args, int32_t* at_step,
                      int64_t capacity, int64_t* count, int64_t* forward_steps);

/* ---- run-time compiled kernels (the KernelBuilder of src/fvm3d.cpp:1071-1394)
 * The reference turns each use_jit equation into CUDA source and compiles
 * it with OCCA (KernelBuilder::build, src/fvm3d.cpp:1219-1316); here NVRTC
 * compiles for sm_100a and the CUDA runtime loads the cubin.  Generated
 * sources may #include "cfdb_jit.cuh": struct CfdbGeom (the mesh's plain
 * FP32 geometry, see cfdb_mesh_plain_geometry) and the device helpers
 * cfdb_grad / cfdb_lapl / cfdb_stab of the operator layer's formulas.
 * Compiled with --fmad=false and IEEE division, so a generated kernel
 * rounds like the plain operator kernels it fuses. */
typedef struct cfdb_kernel cfdb_kernel;

/* Compiles `source` (once per context and source text: later calls return
 * the cached module) and looks up the extern "C" __global__ `name`.  A
 * compile error returns CFDB_EINVAL with the compiler log in
 * cfdb_last_error. */
int cfdb_kernel_build(cfdb_ctx* ctx, const char* source, const char* name, cfdb_kernel** out);
/* KernelBuilder::build for a whole equation system at once: compiles the
 * `count` sources (the distinct ones not yet loaded in ctx) on several host
 * threads, or loads them from the on-disk kernel cache (the role of OCCA's
 * cache: $CFDB_KERNEL_CACHE, else $XDG_CACHE_HOME/cfdb_kernels, else
 * $HOME/.cache/cfdb_kernels; CFDB_KERNEL_CACHE=off disables it), then looks
 * up names[k] in sources[k] into out[k].  On failure no kernel is
 * returned. */
int cfdb_kernel_build_many(cfdb_ctx* ctx, int count, const char* const* sources, const char* const* names,
                           cfdb_kernel** out);
/* KernelBuilder::run (src/fvm3d.cpp:1318-1394) without its two device
 * syncs: launches ceil(n_threads / block) CTAs of `block` threads on the
 * context's stream; args points to the kernel's argument values in order
 * (the cudaLaunchKernel convention).  Asynchronous. */
int cfdb_kernel_launch(cfdb_kernel* k, int64_t n_threads, int block, void** args);
int cfdb_kernel_destroy(cfdb_kernel* k);
/* Resources of a built kernel as the device reports them: registers per
 * thread, local (spill and stack) bytes per thread, the largest CTA it can
 * be launched with.  No reference counterpart (OCCA reports nothing). */
int cfdb_kernel_info(const cfdb_kernel* k, int* registers, int64_t* local_bytes, int* max_threads);

/* The plain FP32 geometry of a mesh as device pointers (uploaded on first
 * use, owned by the mesh): the inputs KernelBuilder wires into generated
 * kernels (GradVar / Grad2Var::reset_input_pointers, src/fvm3d.cpp:1147-1216),
 * N x 6 arrays column-major (entry (i, f) at f*n + i), per-dimension arrays
 * stacked (d*6n + f*n + i), ids int32 with the cell itself on boundary faces. */
typedef struct {
  const int32_t* ids;
  const float* normal;
  const float* normal_alt;
  const float* area;
  const float* alpha;
  const float* len;
  const float* volume;
  int64_t n;
} cfdb_plain_geometry;
int cfdb_mesh_plain_geometry(cfdb_mesh* mesh, cfdb_plain_geometry* out);

/* The same geometry as per-slot constants when the mesh is a lattice whose
 * FP32 face values are identical in every cell (axis-aligned cells with
 * exactly representable coordinates, e.g. unit cells): then a generated
 * kernel may take the constants and compute the neighbour ids from the cell
 * index instead of reading ~250 bytes of geometry per cell, and still round
 * exactly like the array kernels.  exact = 0 otherwise (vertex meshes,
 * spacings whose multiples round).  Per-slot arrays: normal / normal_alt
 * entry d*6 + f, alpha / len entry wall*6 + f (wall = 1 for a boundary face).
 * Checked once per mesh on the device, without building the arrays. */
typedef struct {
  int64_t nx, ny, nz;
  int32_t exact;
  int32_t reserved;
  float normal[18];
  float normal_alt[18];
  float area[6];
  float alpha[12];
  float len[12];
  float volume;
} cfdb_lattice_geometry;
int cfdb_mesh_lattice_geometry(cfdb_mesh* mesh, cfdb_lattice_geometry* out);

/* ---- output files (host side, no GPU needed) ------------------------------
 * store_history's .vti writer (include/io_operators_tmpl.hpp:44-100) without
 * VTK: a VTK XML ImageData file with dimensions nx x ny x nz carrying one
 * Float32 point array `name`, point (x, y, z) = values[Z*Y*x + Z*y + z]
 * (host memory, reference cell order), written x-fastest as VTK orders image
 * points, appended raw with UInt64 size headers.  Origin 0 and spacing 1 as
 * the reference's vtkImageData (it never sets them), so its readers see the
 * same grid.  Error messages go to cfdb_last_error(NULL). */
int cfdb_write_vti(const char* path, const char* name, int64_t nx, int64_t ny, int64_t nz, const float* values);

/* store_mesh (include/io_operators_tmpl.hpp:161-212) without nlohmann::json:
 * mesh.json with "vertexes" [[x,y,z],...], "face" [{"vertexes_id": [4],
 * "nodes_id": [...]}, ...], "nodes" [{"vertexes": [8], "face": [6]}, ...],
 * "x", "y", "z", "lx", "ly", "lz", numbered as Mesh3D::init_basic_internals
 * (src/mesh3d.cpp:323-416).  vertices: (nx+1)(ny+1)(nz+1) x 3 doubles in
 * the vertex numbering, or NULL for the uniform lattice of spacing dx, dy, dz. */
int cfdb_write_mesh_json(const char* path, int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                         const double* vertices);

/* Checkpoint and resume of a solver state (host memory).  No counterpart in
 * the reference, which keeps history in RAM and whose raw stepping writer
 * (include/io_operators_tmpl.hpp:131-159) has no header and no reader: here
 * the file carries a 64-byte header (magic, version, dtype, nx/ny/nz, field
 * count, step, t) and then the `fields` x n values in field order and the
 * reference's cell order.  save writes a temporary file and renames it, so
 * an interrupted save leaves no truncated checkpoint; load fails with
 * CFDB_EINVAL when dtype, dimensions or field count differ from the file's
 * and with CFDB_EIO for a missing, foreign or truncated file.  Errors go to
 * cfdb_last_error(NULL). */
int cfdb_state_save(const char* path, int dtype, int64_t nx, int64_t ny, int64_t nz, int32_t fields, int64_t step,
                    double t, const void* host_data);
int cfdb_state_load(const char* path, int dtype, int64_t nx, int64_t ny, int64_t nz, int32_t fields, int64_t* step,
                    double* t, void* host_data);

#ifdef __cplusplus
}
#endif

#endif /* CFDB_H */
