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
 *    allocation. hl_d3q27_stream_collide, hl_d3q27_apply_bc, the hl_d2q9_step* calls and the
 *    init calls can be captured into a CUDA graph.
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
 *   "d3q27_chunks": 0 automatic, k > 0 splits x into k chunks per tile column
 *   "d3q27_stages": 0 automatic (4), 3..5 planes staged by the TMA kernel
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
HL_API size_t hl_d3q27_bc_scratch_bytes(const hl_world3d* w);

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

/* Replaces InitFlow (envs/lbm/lbm_func.py:26-63) and set_uniform_flow_kernel
 * (envs/lbm/karman/karman_lbm_env.py:15-53), both buffers. fx/fy may be NULL. */
HL_API int hl_d2q9_init_uniform(int nx, int ny, hl_storage storage, void* m_a, void* m_b, float* fx, float* fy,
                         float ux, float uy, hl_stream stream);
/* Replaces InitBoundary (envs/lbm/lbm_func.py:17-23). */
HL_API int hl_d2q9_init_boundary(int nx, int ny, int32_t* flag, hl_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* HOMELBM_H */
