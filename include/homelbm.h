/*
 * homelbm.h - C ABI of the B200 (sm_100a) HOME-LBM library, libhomelbm.so.
 *
 * Each entry point replaces one NVIDIA Warp kernel (or one solver method) of
 * kuiwuchn/OpenHOMELBM; the comment above it names the reference it replaces. The reference
 * binds its kernels from Python through Warp; this library is bound from Python through
 * ctypes (openhomelbm_b200/_lib.py), and any other host language can bind the same symbols.
 *
 * Conventions
 *  - All pointers are device pointers unless the name ends in _host. The caller owns every
 *    buffer (fields live in PyTorch tensors); the library allocates nothing in step calls.
 *  - Every call takes the CUDA stream to run on and performs no host synchronisation and no
 *    allocation. hl_d3q27_stream_collide, hl_d3q27_solid_links, hl_d3q27_apply_bc, the
 *    hl_d2q9_step* calls, the hl_couple* calls and the init calls can be captured into a
 *    CUDA graph.
 *  - Return value: HL_OK (0) or a negative hl_status. hl_last_error() gives a message.
 *    Nothing throws across the ABI.
 *
 * Field layout (the reference's (nx, ny[, nz]) C-order per field, stored as SoA planes in
 * one allocation per buffer):
 *   D2Q9  moments [6][nx][ny]      planes rho, ux, uy, Sxx, Syy, Sxy
 *   D3Q27 moments [10][nx][ny][nz] planes rho, ux, uy, uz, Sxx, Syy, Szz, Sxy, Sxz, Syz
 * S is the reference's second moment Pi/rho - cs^2 I (it includes u u).
 * Flags are the reference's ML_FLUID = 0, ML_SOLID = 1, ML_WALL = 2, ML_INVALID = 6;
 * only ML_FLUID cells are updated, as in stream_and_collide.
 */
#ifndef HOMELBM_H
#define HOMELBM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HL_API __attribute__((visibility("default")))
#else
#define HL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  HL_OK = 0,
  HL_ERR_ARG = -1,          /* invalid argument (maps to ValueError) */
  HL_ERR_UNSUPPORTED = -2,  /* valid but not supported by this build */
  HL_ERR_CUDA = -3,         /* a CUDA runtime error */
  HL_ERR_TIMEOUT = -4       /* a bounded device-side wait gave up */
} hl_status;

/* Storage type of the moment fields. Arithmetic is binary32 for all but HL_F64. */
typedef enum { HL_F32 = 0, HL_F16 = 1, HL_BF16 = 2, HL_F64 = 3 } hl_dtype;

typedef void* hl_stream; /* a cudaStream_t */

HL_API const char* hl_last_error(void);
HL_API const char* hl_version(void);

/* Process-wide tuning knobs (no reference counterpart; for benchmarking and tests):
 *   "d3q27_kernel": 0 automatic, 1 the asynchronous-copy kernel, 2 the TMA-staged kernel
 *   "d3q27_chunks": 0 automatic, k > 0 splits x into k chunks per tile column (read by
 *     hl_d3q27_stream_collide at launch and by hl_d3q27_batch_prepare)
 *   "d3q27_stages": 0 automatic (4), 3..5 planes staged by the TMA kernel
 *   "d3q27_link_blocks": 0 automatic, k > 0 blocks of the cut-link kernel over the listed
 *     cells (fewer leave SMs free for other domains' kernels on other streams): blocks of 16
 *     warps for hl_d3q27_solid_links (automatic: one per SM), of 4 warps for
 *     hl_d3q27_solid_links_batch (automatic: four per SM)
 * Returns HL_ERR_ARG for an unknown key. A CUDA graph keeps the choice it was captured with. */
HL_API int hl_set_tuning(const char* key, int value);

/* ------------------------------------------------------------------ encoding */
/* Reduced-precision storage (HL_F16 / HL_BF16): a cell stores rho-1, u/u_scale and the
 * non-equilibrium second moment (S - u u)/s_scale; every kernel decodes to binary32 on load
 * and encodes on store. HL_F32 / HL_F64 store the moments as they are (scales ignored). */
typedef struct {
  hl_dtype dtype;
  float u_scale; /* velocity scale, e.g. the domain's reference speed */
  float s_scale; /* scale of S - u u */
} hl_storage;

/* Round already-encoded binary32 moments into a storage type exactly as the stream-collide
 * kernels store them. values and out are [n_moments][n_cells] (plane order); cell c's moment
 * k is stored as moment k of cell first_cell + c. HL_F16 / HL_BF16 round stochastically (a
 * value goes to the upper neighbour with probability equal to its distance from the lower
 * one, the random bits a hash of the value, the cell and k); paired != 0 rounds cells 2j and
 * 2j + 1 in one two-lane conversion, as the TMA kernel does, with the same results. HL_F32
 * copies, HL_F64 widens. An extension: the reference stores binary32 only (HomeFlow3D's
 * fields are wp.float32, envs/lbm3d/lbm_core_3d.py:66-82). */
HL_API int hl_round_to_storage(const float* values, long long n_cells, int n_moments, hl_dtype dtype,
                               long long first_cell, int paired, void* out, hl_stream stream);

/* ------------------------------------------------------------------ D3Q27 */
/* One D3Q27 world. cur/post are the two moment buffers (the reference's fields and their
 * *_post twins); the step reads cur and writes post, and the caller swaps them afterwards
 * (Swap_Mom_3D, envs/lbm3d/lbm_func_3d.py:689-727). */
typedef struct {
  int nx, ny, nz;
  hl_storage storage;
  const void* cur;
  void* post;
  const int32_t* flag;   /* [nx][ny][nz], or NULL: border cells are ML_WALL (InitBoundary3D) */
  const float* force;    /* [3][nx][ny][nz] forcex, forcey, forcez, or NULL (zero) */
  int periodic;          /* 1: periodic in x, y, z, every cell fluid, no apply_bc_3d
                            (an extension: the reference has only walls) */
} hl_world3d;

/* Outer-boundary conditions of apply_bc_3d (envs/lbm3d/lbm_func_3d.py:607-648), faces in
 * the reference's order 0 left x=0, 1 right x=nx-1, 2 top y=ny-1, 3 bottom y=0,
 * 4 front z=nz-1, 5 back z=0; type 0 = fixed velocity bc_value, 1 = zero gradient. */
typedef struct {
  int bc_type[6];
  float bc_value[6][3];
} hl_bc3d;

/* Scratch for the diagnostics of one step: per-CTA partial sums and a completion counter.
 * Size it with hl_d3q27_scratch_bytes(); zero it once before first use. */
typedef struct {
  void* scratch;
  size_t scratch_bytes;
  double* mass;          /* out: sum of rho over updated cells (binary64), or NULL */
  int32_t* health;       /* out: number of updated cells with non-finite or rho <= 0 moments */
} hl_diag;

/* Replaces stream_and_collide_3d (envs/lbm3d/lbm_func_3d.py:364-604) for worlds without
 * immersed solids: pull streaming from the neighbours' moments with the reference's
 * second-order reconstruction (mlCalEquilibrium3D_s, 224-251), clamped at zero, then the
 * regularised collision (564-604) with relaxation omega = 1/(3 vis_shear + 0.5), evaluated
 * in the storage precision (binary32, or binary64 for HL_F64). diag may be NULL. */
HL_API int hl_d3q27_stream_collide(const hl_world3d* w, double vis_shear, const hl_diag* diag,
                            hl_stream stream);

/* Replaces apply_bc_3d (envs/lbm3d/lbm_func_3d.py:607-624) on post, with the reference's
 * sequential thread order reproduced at edges and corners. scratch: hl_d3q27_bc_scratch_bytes()
 * bytes. No-op for periodic worlds. */
HL_API int hl_d3q27_apply_bc(const hl_world3d* w, const hl_bc3d* bc, void* scratch, hl_stream stream);

HL_API size_t hl_d3q27_scratch_bytes(const hl_world3d* w);

/* hl_d3q27_stream_collide with its diagnostics, for callers that cannot allocate device
 * memory. No counterpart in the reference.
 *
 * Some callers cannot call cudaMalloc: a host that has handed the whole HBM budget to a
 * caching allocator or to resident fluid domains (a serving loop admits domains against a
 * fixed budget), a real-time control loop that must not take allocation latency, or a
 * plugin whose host owns all device memory. This entry point needs no scratch from them:
 * the per-CTA partial sums and the completion counter live in a 16 KiB file-scope device
 * array of the library, which every GPU that loads the library keeps until the process exits.
 *  - Computes what hl_d3q27_stream_collide computes with a non-NULL diag: post <- step(cur),
 *    *mass (binary64 sum of rho over updated cells) and *health (count of updated cells with
 *    non-finite moments or rho <= 0); mass and health may be NULL. Storage float32 or
 *    float64 (other storages return HL_ERR_ARG); it always runs the general kernel, never
 *    the TMA-staged one, so its results can differ from hl_d3q27_stream_collide in rounding.
 *  - Limit: 16 + 12 bytes per CTA of scratch, i.e. devices with up to 1364 SMs (a B200 has
 *    148); larger needs are rejected with HL_ERR_ARG.
 *  - The first call on a device resolves the array's device address (cudaGetSymbolAddress,
 *    with that device current); make that first call before any stream capture.
 *  - Every call shares the one array and leaves its last contents there; each call clears the
 *    counter it needs first (stream-ordered). Calls that overlap on the GPU (other streams,
 *    other host threads) race on the array: serialise them. */
HL_API int hl_d3q27_stream_collide_noalloc(const hl_world3d* w, double vis_shear, double* mass, int32_t* health,
                                           hl_stream stream);

/* Batched domains (the serving form; no reference counterpart: the reference launches each
 * LBM_Solver3D's step on its own, envs/lbm3d/lbm_solver_3d.py:88-127). One stream-collide
 * launch steps many walled domains of different sizes: the tiles of all of them form one item
 * sequence that the CTAs share, so small domains do not leave SMs idle.
 *  - hl_d3q27_batch_bytes: device bytes of the descriptors of n domains.
 *  - hl_d3q27_batch_prepare: writes the descriptors of worlds[0 .. n) into desc (device
 *    memory, 64-byte aligned): buffers (parity 0 reads cur, parity 1 reads post), sizes, x
 *    split and tensor maps. Every world walled, without force or flag fields, TMA-eligible
 *    (ny % 16 == 0, nz % 32 == 0, 16-byte aligned buffers), float32/float16/bfloat16, one
 *    storage type and scale for all. Sets *n_items. Synchronises the stream (not for stream
 *    capture); prepare again after any domain's buffers change.
 *  - hl_d3q27_stream_collide_batch: one stream-collide of every domain of desc at parity p
 *    (reads buffer p, writes buffer p ^ 1); per cell the same result as
 *    hl_d3q27_stream_collide. n_domains and n_items must be those of the prepare call.
 *    Capturable. status (or NULL) is set to HL_ERR_TIMEOUT if a bounded wait gave up. */
HL_API size_t hl_d3q27_batch_bytes(int n_domains);
HL_API int hl_d3q27_batch_prepare(const hl_world3d* worlds, int n_domains, void* desc, size_t desc_bytes,
                                  int* n_items, hl_stream stream);
HL_API int hl_d3q27_stream_collide_batch(const void* desc, int n_domains, int n_items, double vis_shear,
                                         const hl_storage* storage, int parity, int* status, hl_stream stream);
HL_API size_t hl_d3q27_bc_scratch_bytes(const hl_world3d* w);

/* Batched boundaries (the serving form's batched substep; no reference counterpart: the
 * reference runs apply_bc_3d per world, envs/lbm3d/lbm_solver_3d.py:88-127). The three waves
 * of hl_d3q27_apply_bc run as three launches over all domains of a set instead of three per
 * domain; per cell the same result as hl_d3q27_apply_bc on each domain.
 *  - hl_d3q27_bc_batch_bytes: device bytes of the descriptors of n domains.
 *  - hl_d3q27_bc_batch_prepare: writes the descriptors of worlds[0 .. n) (given at parity 0:
 *    the step reads cur and writes post), their conditions bcs[i] and boundary scratch
 *    scratch[i] (hl_d3q27_bc_scratch_bytes each, one per domain) into desc (device memory,
 *    16-byte aligned). Every world walled with sides >= 3, one storage type. Synchronises the
 *    stream (not for stream capture); prepare again after a domain's buffers change.
 *  - hl_d3q27_apply_bc_batch: the boundary pass of every domain at parity p (parity 0 writes
 *    each world's post, parity 1 its cur buffer). n_domains must be the prepared one.
 *    Capturable. */
HL_API size_t hl_d3q27_bc_batch_bytes(int n_domains);
HL_API int hl_d3q27_bc_batch_prepare(const hl_world3d* worlds, const hl_bc3d* bcs, void* const* scratch,
                                     int n_domains, void* desc, size_t desc_bytes, hl_stream stream);
HL_API int hl_d3q27_apply_bc_batch(const void* desc, int n_domains, int parity, hl_stream stream);

/* Replaces InitFlow3D (envs/lbm3d/lbm_func_3d.py:22-83) and set_uniform_flow_3d_kernel
 * (envs/lbm3d/karman/karman_lbm_env_3d.py:15-64): rho = 1, u = (ux, uy, uz), S from the
 * equilibrium populations with the reference's cs2_local quirk, forces zeroed, written to
 * both buffers. force may be NULL. */
HL_API int hl_d3q27_init_uniform(int nx, int ny, int nz, hl_storage storage, void* m_a, void* m_b,
                          float* force, float ux, float uy, float uz, hl_stream stream);

/* Taylor-Green vortex initial state on the periodic box [0, 2 pi)^3 sampled at 2 pi i/n:
 * u = u0 (sin x cos y cos z, -cos x sin y cos z, 0), rho = 1 + 3 (u0^2/16)(cos 2x + cos 2y)
 * (cos 2z + 2), S = u u. (No reference counterpart: the reference has no periodic case.) */
HL_API int hl_d3q27_init_tgv(int nx, int ny, int nz, hl_storage storage, void* m_a, void* m_b,
                      float u0, hl_stream stream);

/* Replaces InitBoundary3D (envs/lbm3d/lbm_func_3d.py:13-19). */
HL_API int hl_d3q27_init_boundary(int nx, int ny, int nz, int32_t* flag, hl_stream stream);

/* ------------------------------------------------------------------ masked world resets
 * The reference's flows_wp (a device array of HomeFlow / HomeFlow3D structs,
 * envs/lbm3d/lbm_solver_3d.py:68, envs/lbm/lbm_solver.py:80) is here a device array of the
 * descriptors below, one per world; reset kernels read it and a device int32 mask with one entry
 * per world (non-zero: reset that world), as the reference's kernels do. Parts (what):
 *   HL_RESET_FLOW            ResetSingleWorldFlow(3D) (envs/lbm/lbm_func.py:66-114,
 *                            envs/lbm3d/lbm_func_3d.py:86-150): rho = 1, u = 0, S = 0 in both
 *                            buffers (the reference's rest state, its cs2_local quirk giving
 *                            S = +0), body force zeroed
 *   HL_RESET_SOLID_TRANSFORM ResetSingleWorldSolidTransform3D (lbm_func_3d.py:153-175): mesh
 *                            transforms and last transforms = identity, initialized = 0; in 2D
 *                            ResetSingleWorldSolidTransform (lbm_func.py:117-140): the first
 *                            solid_line_num[s] points of both transformed outlines = (0, 0)
 *   HL_RESET_FORCES          ResetSingleWorldForces(3D) (lbm_func.py:143-160,
 *                            lbm_func_3d.py:178-196): per-solid force and torque = 0
 *   HL_RESET_INITIALIZED     3D only: initialized = 0 alone (LBM_Solver3D.reset_world(s),
 *                            envs/lbm3d/lbm_solver_3d.py:348-385)
 * One launch does every requested part of every masked world; max_cells is at least the largest
 * cell count of any world (2D: and its n_objects * max_segments); n_objects <= 256. Pointers
 * that are NULL are skipped. Stream-ordered, allocation-free, capturable. */
#define HL_RESET_FLOW 1
#define HL_RESET_SOLID_TRANSFORM 2
#define HL_RESET_FORCES 4
#define HL_RESET_INITIALIZED 8

typedef struct {
  int nx, ny, nz;
  hl_storage storage;
  void* m0;                  /* moment buffer 0 [10][nx][ny][nz] */
  void* m1;                  /* moment buffer 1 */
  float* force;              /* [3][nx][ny][nz] forcex, forcey, forcez, or NULL */
  int n_objects;
  float* transforms;         /* [n][7] mesh_transforms (p, q x y z w) */
  float* transforms_last;    /* [n][7] mesh_transforms_last */
  int32_t* initialized;      /* [n] mesh_transforms_initialized */
  float* solid_force;        /* [n][3] */
  float* solid_torque;       /* [n][3] */
} hl_flow3d;

HL_API int hl_d3q27_reset_worlds(const hl_flow3d* flows, int nworld, hl_dtype dtype, const int32_t* reset_mask,
                                 int what, long long max_cells, hl_stream stream);

/* Immersed triangle-mesh solids of one 3D world (HomeFlow3D's per-solid fields,
 * envs/lbm3d/lbm_core_3d.py:91-119). Solid k's mesh is the triangles
 * tris[tri_offset[k] .. tri_offset[k+1]) in its body frame, vertices already scaled by
 * lbm_scale * nx (create_solid_from_mesh, lbm_solver_3d.py:166-196); a solid with no
 * triangles is an unset mesh id and is skipped. Transforms are p (3) then q (x, y, z, w). */
typedef struct {
  int n_objects;             /* <= 64 */
  float max_bound_radius;    /* host copy of max(bound_radius): sizes the band launch */
  const int32_t* tri_offset; /* [n+1] */
  const float* tris;         /* [total][3][3] */
  const float* transforms;   /* [n][7] mesh_transforms */
  const float* transforms_last; /* [n][7] mesh_transforms_last */
  const int32_t* initialized;   /* [n] mesh_transforms_initialized */
  const float* scale_sizes;  /* [n][3] mesh_scale_sizes */
  const float* position;     /* [n][3] solid_position */
  const float* bound_radius; /* [n] solid_bound_radius */
  const float* linear_v;     /* [n][3] */
  const float* angle_v;      /* [n][3] */
  double* loads64;           /* [n][6] scratch: force then torque summed in binary64 */
  float* force;              /* [n][3] solid_force (out) */
  float* torque;             /* [n][3] solid_torque (out) */
  /* Optional triangle bins (NULL: every link ray tests all triangles of the solid). Per solid
   * a uniform grid in its body frame; bin (i, j, k) lists the triangles whose bounding box,
   * widened by at least sqrt(3) (the longest link), meets the bin, so a ray starting in the
   * bin finds every hit with t <= 1 among them (same closest hit as testing all). Used where
   * mesh_scale_sizes is (1, 1, 1); other solids fall back to all triangles. */
  const float* bin_box;      /* [n][4] grid origin x, y, z and bin edge */
  const int32_t* bin_dims;   /* [n][4] bins along x, y, z (0: no grid) and the solid's first bin */
  const int32_t* bin_start;  /* [bins + n] start of each bin's list in bin_tris (CSR per solid) */
  const int32_t* bin_tris;   /* triangle indices, relative to the solid's first triangle */
  /* Scratch of hl_d3q27_solid_links_work_ints() int32 (NULL: the single-pass kernel): the
   * list of cells that can have a cut link, so that the cut-cell work is spread evenly over
   * the GPU instead of staying with the warps whose cells happen to lie near the surface. */
  int32_t* work;
} hl_solids3d;

/* The solid part of one stream_and_collide_3d step (envs/lbm3d/lbm_func_3d.py:364-604) and
 * init_force_3d_batch (736-747). Call it after hl_d3q27_stream_collide and before
 * hl_d3q27_apply_bc of the same step, on the same world. It zeroes the loads, then recomputes
 * post for every fluid cell within bound_radius + 2 of a solid (the narrow band, 387-393):
 * links whose backward ray hits a mesh within one lattice step (get_cutcell_multi_3d,
 * 254-316; Moller-Trumbore, double-sided, closest hit) take the wall population rebuilt with
 * the wall velocity (452-489, not clamped), the others the clamped neighbour population
 * (525-526); the momentum exchange and its torque about solid_position (490-511) are summed
 * per solid in binary64 and copied to force / torque in binary32. */
HL_API int hl_d3q27_solid_links(const hl_world3d* w, double vis_shear, const hl_solids3d* s, hl_stream stream);

/* int32 entries of the work scratch of hl_solids3d for n_objects solids whose bound_radius is
 * at most max_bound_radius. */
HL_API size_t hl_d3q27_solid_links_work_ints(int n_objects, float max_bound_radius);

/* The cut links of many domains in one classify and one process launch (the serving form;
 * the reference runs each world's step on its own). Per cell the same computation as
 * hl_d3q27_solid_links; each domain's loads are its binary64 sums and binary32 force/torque.
 *  - hl_d3q27_links_batch_bytes(n, total solids): device bytes of the descriptors.
 *  - hl_d3q27_links_batch_prepare: writes the descriptors of worlds[k] / solids[k] (parity 0
 *    reads cur, parity 1 reads post; the solids' force / torque pointers are where this
 *    descriptor set writes the loads) into desc (64-byte aligned device memory) and sets
 *    *work_ints, the int32 work list the launches need. One storage type for all domains.
 *    Synchronises the stream; prepare again when any pointer changes.
 *  - hl_d3q27_solid_links_batch: one pass at `parity`, after the domains' stream-collide
 *    (batched or not). Capturable. */
HL_API size_t hl_d3q27_links_batch_bytes(int n_domains, int n_solids_total);
HL_API int hl_d3q27_links_batch_prepare(const hl_world3d* worlds, const hl_solids3d* solids, int n_domains,
                                        double vis_shear, void* desc, size_t desc_bytes, size_t* work_ints,
                                        hl_stream stream);
HL_API int hl_d3q27_solid_links_batch(const void* desc, int n_domains, int parity, int32_t* work, size_t work_ints,
                                      hl_stream stream);

/* ------------------------------------------------------------------ coupling
 * The MuJoCo-Warp coupling kernels of the environments, over batched per-world arrays:
 * a per-solid array of nworld worlds is [nworld][n_objects][...] with world stride
 * n_objects * components. MuJoCo buffers are borrowed as they are: xipos [nworld][nbody][3],
 * xquat [nworld][nbody][4] (w, x, y, z), xfrc [nworld][nbody][6] (force then torque). */

/* extract_body_states(_3d) (envs/lbm/lbm_fluid_env_func.py:8-24,
 * envs/lbm3d/lbm_fluid_env_3d_func.py:11-36): pos_out [nworld][nsel][3] and quat_out
 * [nworld][nsel][4] from the bodies body_ids[nsel]. */
HL_API int hl_couple_body_states(int nworld, int nbody, int nsel, const float* xipos, const float* xquat,
                                 const int32_t* body_ids, float* pos_out, float* quat_out, hl_stream stream);

/* convert_and_update_solid_batch_3d (lbm_fluid_env_3d_func.py:42-100): for each world and
 * selected solid, solid_position = (pos - mujoco_origin) * scale + lbm_origin, the
 * quaternion copied, mesh_transforms_last <- mesh_transforms (once initialised) and the new
 * transform (p, q(x, y, z, w)); the first call sets last = current and initialized = 1.
 * position [nworld][n][3], quaternion [nworld][n][4], transforms / transforms_last
 * [nworld][n][7], initialized [nworld][n]; origins [nsel][3], scales [nsel]. */
HL_API int hl_couple3d_update_solids(int nworld, int n_objects, int nsel, const int32_t* solid_ids,
                                     const float* mj_pos, const float* mj_quat, const float* mujoco_origins,
                                     const float* lbm_origins, const float* scales, float* position,
                                     float* quaternion, float* transforms, float* transforms_last,
                                     int32_t* initialized, hl_stream stream);

/* convert_and_update_solid_batch_2d (lbm_fluid_env_func.py:72-105): solid_position
 * [nworld][n][2] = (pos.xy - origin) * scale + lbm_origin, solid_angle [nworld][n] = the yaw
 * atan2(2 (w z + x y), 1 - 2 (y^2 + z^2)); origins [nsel][2]. */
HL_API int hl_couple2d_update_solids(int nworld, int n_objects, int nsel, const int32_t* solid_ids,
                                     const float* mj_pos, const float* mj_quat, const float* mujoco_origins,
                                     const float* lbm_origins, const float* scales, float* position, float* angle,
                                     hl_stream stream);

/* Loads of the selected solids for MuJoCo, [nworld][nsel][3] each:
 *   mode 0, extract_forces_torques_physical_3d (lbm_fluid_env_3d_func.py:138-178):
 *          force * force_conv, torque * torque_conv (force / torque [nworld][n][3]);
 *   mode 1, extract_forces_torques_batch_3d (104-135): force / scale, torque / scale^2;
 *   mode 2, extract_forces_torques_batch (lbm_fluid_env_func.py:51-69), 2D: force is
 *          (solid_forcex, solid_forcey, 0) / scale and torque (0, 0, torque / scale), read from
 *          force = per world the three planes [nworld][3][n] solid_forcex, solid_forcey,
 *          torque (the torque argument is unused and may be NULL).
 * scales [nsel] (modes 1, 2). */
HL_API int hl_couple_loads(int mode, int nworld, int n_objects, int nsel, const int32_t* solid_ids,
                           const float* force, const float* torque, const float* scales, float force_conv,
                           float torque_conv, float* forces_out, float* torques_out, hl_stream stream);

/* fill_xfrc_kernel / fill_xfrc_3d_kernel (lbm_fluid_env_func.py:27-48,
 * lbm_fluid_env_3d_func.py:181-210): xfrc[w][body_ids[i]] = (forces[w][i], torques[w][i]). */
HL_API int hl_couple_fill_xfrc(int nworld, int nbody, int nsel, const int32_t* body_ids, const float* forces,
                               const float* torques, float* xfrc, hl_stream stream);

/* ------------------------------------------------------------------ D2Q9 */
/* One D2Q9 world (HomeFlow, envs/lbm/lbm_core.py:17-88); cur/post as for D3Q27. */
typedef struct {
  int nx, ny;
  hl_storage storage;
  const void* cur;
  void* post;
  const int32_t* flag;   /* [nx][ny], or NULL: border cells are ML_WALL (InitBoundary) */
  const float* forcex;   /* [nx][ny] or NULL */
  const float* forcey;   /* [nx][ny] or NULL */
  int periodic;          /* extension: periodic in x and y, every cell fluid, no apply_bc */
} hl_world2d;

/* Scalar parameters of HomeFlow used by the step (lbm_core.py:103-135). */
typedef struct {
  double vis_shear;      /* kinematic viscosity; omega = 1/(3 vis_shear + 0.5) in the storage precision */
  float grid_length;     /* torque scale, the reference's 1/nx; <= 0 selects 1/nx */
  float time_step;       /* wall velocity = displacement / time_step; <= 0 selects 1 */
} hl_step2d;

/* apply_bc faces in the reference's order 0 left, 1 top, 2 right, 3 bottom
 * (envs/lbm/lbm_func.py:610-631); type 0 fixed velocity, 1 zero gradient. */
typedef struct {
  int bc_type[4];
  float bc_value[4][2];
} hl_bc2d;

/* Polygon solids of one world (HomeFlow solid fields, lbm_core.py:57-79), device pointers.
 * loads64 and band_box are library scratch owned by the caller. */
typedef struct {
  int n_objects;           /* <= 64 */
  int max_segments;
  const float* line;       /* [n][max_segments][2] local polygon (solid_line) */
  const int32_t* line_num; /* [n] solid_line_num */
  float* line_tf;          /* [n][max_segments][2] solid_line_transformed (in/out) */
  float* line_tf_last;     /* [n][max_segments][2] solid_line_transformed_last (out) */
  const float* position;   /* [n][2] */
  const float* angle;      /* [n] */
  const float* scale;      /* [n] */
  const float* mass_center;/* [n][2] */
  const float* max_radius; /* [n] squared normalised radius bound (configure_solid) */
  double* loads64;         /* [n][3] binary64 force x, force y, torque accumulators */
  float* force_x;          /* [n] solid_forcex, or NULL */
  float* force_y;          /* [n] solid_forcey, or NULL */
  float* torque;           /* [n] torque, or NULL */
  int32_t* band_box;       /* [4] scratch */
} hl_solids2d;

/* Phases of a 2D step (hl_d2q9_step_phases): */
#define HL_PHASE_SEGMENTS 1 /* precompute_transformed_segments + load reset (lbm_func.py:503-542) */
#define HL_PHASE_STREAM 2   /* stream_and_collide (lbm_func.py:322-467) incl. cut links and loads */
#define HL_PHASE_BC 4       /* apply_bc (lbm_func.py:610-682) + binary32 load copies */
#define HL_PHASE_ALL 7

/* Replaces one LBM_Solver.step (envs/lbm/lbm_solver.py:97-141) of one world: segments,
 * stream_and_collide with polygon cut cells and momentum exchange, apply_bc. solids may be
 * NULL. The caller swaps cur/post afterwards (Swap_Mom, lbm_func.py:475-500). */
HL_API int hl_d2q9_step(const hl_world2d* w, const hl_step2d* p, const hl_bc2d* bc, const hl_solids2d* solids,
                 hl_stream stream);
/* The same, restricted to a subset of HL_PHASE_* (each phase is one reference kernel). */
HL_API int hl_d2q9_step_phases(const hl_world2d* w, const hl_step2d* p, const hl_bc2d* bc,
                        const hl_solids2d* solids, int phases, hl_stream stream);

/* Batched worlds of different sizes (the reference batches only same-size worlds,
 * lbm_solver.py:117-139): hl_d2q9_pack writes one descriptor of hl_d2q9_desc_bytes() bytes
 * on the host; the caller copies n descriptors to device memory once, then each step runs
 * hl_d2q9_step_batch with parity 0 (cur = the world's cur) or 1 (buffers swapped). */
HL_API size_t hl_d2q9_desc_bytes(void);
HL_API int hl_d2q9_pack(const hl_world2d* w, const hl_step2d* p, const hl_bc2d* bc, const hl_solids2d* solids,
                 void* desc_host);
HL_API int hl_d2q9_step_batch(const void* desc_dev, int n_worlds, int parity, hl_dtype dtype, int max_nx,
                       int max_ny, int any_solid, int phases, hl_stream stream);

/* Batching form: the stream phase of batched worlds of different sizes as ONE persistent
 * launch over a tile work-list (no reference counterpart; it replaces the per-world
 * stream_and_collide launches of LBM_Solver.step, lbm_solver.py:117-139, for uneven worlds).
 * hl_d2q9_tile_shapes writes the supported tile shapes (tile_x, tile_y pairs, at most cap)
 * and returns their number. Shapes with tile_y = 30 are strips: one warp per tile marches its
 * 30 rows along x and exchanges populations by warp shuffles (ctas counts blocks of 8 warps);
 * the others stage a tile in shared memory (ctas counts CTAs of 256 threads). hl_d2q9_tile_list (host only, no GPU) writes the tiles of n_worlds
 * worlds of nx[w] x ny[w] cells, world-major, 4 int32 per tile (world, x0, y0, 0), into out
 * (NULL: count only) and their number into *n_tiles; HL_ERR_ARG if they do not fit in
 * cap_tiles. hl_d2q9_step_tiles runs hl_d2q9_step_batch's phases with the stream phase taken
 * by min(n_tiles, ctas) CTAs that take the tiles in turn; tiles_dev (device, 16-byte aligned)
 * holds the list for the same tile shape. Results are identical to hl_d2q9_step_batch. */
HL_API int hl_d2q9_tile_shapes(int32_t* out, int cap);
HL_API int hl_d2q9_tile_list(const int32_t* nx, const int32_t* ny, int n_worlds, int tile_x, int tile_y, int32_t* out,
                             size_t cap_tiles, size_t* n_tiles);
HL_API int hl_d2q9_step_tiles(const void* desc_dev, int n_worlds, int parity, hl_dtype dtype, const int32_t* tiles_dev,
                              int n_tiles, int tile_x, int tile_y, int ctas, int any_solid, int phases,
                              hl_stream stream);

/* Replaces InitFlow (envs/lbm/lbm_func.py:26-63) and set_uniform_flow_kernel
 * (envs/lbm/karman/karman_lbm_env.py:15-53), both buffers. fx/fy may be NULL. */
HL_API int hl_d2q9_init_uniform(int nx, int ny, hl_storage storage, void* m_a, void* m_b, float* fx, float* fy,
                         float ux, float uy, hl_stream stream);
/* Replaces InitBoundary (envs/lbm/lbm_func.py:17-23). */
HL_API int hl_d2q9_init_boundary(int nx, int ny, int32_t* flag, hl_stream stream);

/* One world of the 2D flows_wp for hl_d2q9_reset_worlds (see hl_d3q27_reset_worlds). */
typedef struct {
  int nx, ny;
  hl_storage storage;
  void* m0;                  /* moment buffer 0 [6][nx][ny] */
  void* m1;                  /* moment buffer 1 */
  float* forcex;             /* [nx][ny] or NULL */
  float* forcey;             /* [nx][ny] or NULL */
  int n_objects, max_segments;
  const int32_t* line_num;   /* [n] solid_line_num */
  float* line_tf;            /* [n][max_segments][2] solid_line_transformed */
  float* line_tf_last;       /* [n][max_segments][2] solid_line_transformed_last */
  float* solid_forcex;       /* [n] */
  float* solid_forcey;       /* [n] */
  float* torque;             /* [n] */
} hl_flow2d;

/* ResetSingleWorldFlow, ResetSingleWorldSolidTransform and ResetSingleWorldForces
 * (envs/lbm/lbm_func.py:66-160) over the worlds whose reset_mask entry is non-zero; parts as for
 * hl_d3q27_reset_worlds (HL_RESET_INITIALIZED is 3D only). */
HL_API int hl_d2q9_reset_worlds(const hl_flow2d* flows, int nworld, hl_dtype dtype, const int32_t* reset_mask,
                                int what, long long max_cells, hl_stream stream);

/* Field diagnostics: headless images of a world's current moments (cur), the arithmetic of the
 * reference's display kernels, into a caller-owned binary32 device buffer (no GL texture).
 *
 * hl_d2q9_image, out [nx][ny] (kind 1: [nx][ny][3]):
 *   kind 0  |u|                                   get_u_img (envs/lbm/lbm_func.py:163-166)
 *   kind 1  (|u|, ux, uy) / param mapped to [0, 1]  get_velocity_rgb (169-193), param = max_velocity
 *   kind 2  dv/dx - du/dy, one-sided on the border  get_vorticity_img (196-233); with solids,
 *           pixels inside a polygon or within `thickness` of one are 1000
 *           (get_vorticity_with_solid_img, 236-319)
 *   kind 3  1 inside or within `thickness` of a polygon, else 0  get_solid_boundary_img (804-866)
 * grid_length <= 0 selects 1/nx (HomeFlow.grid_length). solids (kinds 2, 3) use line_tf,
 * line_num, position, scale and max_radius; NULL or no objects: no overlay.
 *
 * hl_d3q27_image (envs/lbm3d/lbm_func_3d.py:753-1313), out [na][nb] over the two axes other than
 * `axis` in increasing order (axis 2: (x, y); axis 0: (y, z); axis 1: (x, z)):
 *   mode 0, slice at coordinate `index` along `axis`:
 *     kind 0  |u|                               get_u_img_xy_3d / get_u_img_yz_3d
 *     kind 1  the vorticity component along `axis` (z: dv/dx - du/dy, x: dw/dy - dv/dz,
 *             y: du/dz - dw/dx)               get_vorticity_xy_3d / _yz_3d; with solids, voxels
 *             flagged ML_SOLID, inside a mesh or within `thickness` of it are 1000 (_with_solid_3d)
 *   mode 1, projection seen from beyond the high end of `axis`, looking down it:
 *     kind 0  max |u| over the column, walls skipped  get_u_projection_max_topdown_3d,
 *             get_u_projection_side_3d (axis 0), get_u_projection_front_3d (axis 1)
 *     kind 1  |u| of the first moving cell from the viewer  get_u_projection_topdown_3d
 *     kind 2  the vorticity component along `axis` of largest magnitude, sign kept
 *             get_vorticity_projection_topdown_3d / _side_3d / _front_3d
 *     with solids, a column whose ray from the viewer hits a mesh is 1000
 *     (any_mesh_hit_along_ray_3d, 320-362).
 * solids uses tri_offset, tris, transforms and scale_sizes. Calls are stream-ordered, allocate
 * nothing and can be captured in a CUDA graph. */
HL_API int hl_d2q9_image(const hl_world2d* w, int kind, float param, float grid_length, const hl_solids2d* solids,
                         float thickness, float* out, hl_stream stream);
HL_API int hl_d3q27_image(const hl_world3d* w, int mode, int axis, int index, int kind, float grid_length,
                          const hl_solids3d* solids, float thickness, float* out, hl_stream stream);

/* The live view's slice stack (tools/lbm3d_realtime_control.py:68-148, 157-182; a device
 * RGBA buffer replaces the GL atlas):
 *  - hl_d3q27_live_slices: values[(slice * plane_height + q) * plane_width + p] is the
 *    vorticity component color_axis (0 x, 1 y, 2 z) at the cell of plane p, q of slice
 *    slice_positions[slice] along slice_axis, the in-plane coordinates p * stride and
 *    q * stride clamped to the grid; central differences clamped at the border, divided by the
 *    clamped span; zero within boundary_margin of a face. With collect_histogram, every
 *    |value| > 1e-8 adds one to histogram[bin], bin = floor(256 * clamp((log|value| - log 1e-8)
 *    / -log 1e-8, 0, 0.999999)) (the caller zeroes the 256 int32 bins first). slice_positions
 *    is device memory; a position outside the grid gives zeros and no count.
 *  - hl_live_rgba: rgba[4 i ..] = the blue-white-red map of values[i] / vmax (clamped) and
 *    255 alpha (clamped to [0, 1]), each channel truncated to a byte.
 * Stream-ordered, allocation-free, capturable. */
HL_API int hl_d3q27_live_slices(const hl_world3d* w, const int32_t* slice_positions, int n_slices, int plane_width,
                                int plane_height, int stride, int slice_axis, int color_axis, int boundary_margin,
                                int collect_histogram, float* values, int32_t* histogram, hl_stream stream);
HL_API int hl_live_rgba(const float* values, long long n, float vmax, float alpha, uint8_t* rgba, hl_stream stream);

/* The 2D realtime tool's GPU kernels (tools/lbm2d_realtime_control.py), headless:
 *  - hl_d2q9_uimg_rgba (lbm_uimg_to_rgba_kernel 417-464): an (nx, ny) image, e.g. u_img, to
 *    RGBA bytes laid out (ny, nx, 4); render_mode 0 velocity magnitude over vmax, 1 vorticity
 *    over +-vmax (values >= 999 grey), 2 solid boundary.
 *  - hl_d2q9_local_force (set_local_force_kernel 144-157): forcex/forcey (nx, ny) =
 *    (fx, fy) * max(0, 1 - ((x - cx)/rx)^2 - ((y - cy)/ry)^2).
 * Stream-ordered, allocation-free, capturable. */
HL_API int hl_d2q9_uimg_rgba(const float* u_img, int nx, int ny, int render_mode, float vmax, uint8_t* rgba,
                             hl_stream stream);
HL_API int hl_d2q9_local_force(float* forcex, float* forcey, int nx, int ny, float cx, float cy, float rx, float ry,
                               float fx, float fy, hl_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* HOMELBM_H */
