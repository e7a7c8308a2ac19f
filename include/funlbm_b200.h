/*
 * funlbm_b200 -- C ABI of the B200 (sm_100a) lattice-Boltzmann step path.
 *
 * Every entry point replaces one function (or a fused sequence of functions)
 * of funlbm 1.2.0; the reference function is cited beside each declaration as
 * file:line inside the funlbm source tree (src/funlbm/...).
 *
 * Conventions
 *  - All buffers are device pointers allocated and owned by the caller; the
 *    library never allocates or frees them.  Sizes are element counts.
 *  - Populations are stored structure-of-arrays, f[q][x][y][z] (z fastest),
 *    in the storage type named by lbm_lattice.storage.  Node counts are the
 *    reference's size + 1 per axis.  Velocity, force: [x][y][z][3] float32;
 *    density: [x][y][z] float32 -- the reference's own [X,Y,Z,3] / [X,Y,Z,1].
 *  - `stream` is a cudaStream_t (NULL = the legacy default stream).  Calls are
 *    asynchronous on that stream; results are ready when the stream is.
 *  - Every call returns LBM_OK (0) or an error code; lbm_last_error() returns a
 *    message for the calling thread.  Nothing is thrown across the ABI.
 *  - Calls on different lattices are independent.  Calls on one lattice must
 *    be ordered by the caller (same stream, or events).
 */
#ifndef FUNLBM_B200_H
#define FUNLBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define LBM_OK 0
#define LBM_ERR_INVALID 1     /* bad argument: the reference raises ValueError   */
#define LBM_ERR_UNSUPPORTED 2 /* face code / velocity set: NotImplementedError   */
#define LBM_ERR_CUDA 3        /* CUDA launch or runtime error                    */

/* ---- device status word bits (written by kernels with atomicOr) --------- */
#define LBM_STATUS_RHO_BAD 0x1u      /* density <= 0 or not finite at some node  */
#define LBM_STATUS_U_BAD 0x2u        /* velocity not finite at some node         */
#define LBM_STATUS_STENCIL_EMPTY 0x4u /* a marker's normalised weight sum != 1   */
                                      /* after step 100 (lbm/lbm3d.py:84-86)     */
#define LBM_STATUS_WAIT_TIMEOUT 0x8u  /* a bounded device-side wait gave up      */
#define LBM_STATUS_DRAIN_FAILED 0x10u /* after such a timeout, a kernel could not */
                                      /* confirm that its own bulk copies ended:  */
                                      /* treat the lattice buffers as lost        */

/* ---- boundary codes: values of funlbm's BoundaryCondition (config/base.py:17-23) */
#define LBM_BC_PERIODICAL 11000
#define LBM_BC_WALL 1200
#define LBM_BC_WALL_WITH_SPEED 1201
#define LBM_BC_NON_EQUILIBRIUM 1400

/* face order: input (x=0), output (x=X-1), back (y=0), forward (y=Y-1),
 * bottom (z=0), top (z=Z-1) -- the order of FlowD3.f_stream_bound
 * (flow/d3/base.py:183-196); a later face overrides an earlier one. */
#define LBM_NFACES 6

/* ---- population storage ------------------------------------------------ */
#define LBM_STORAGE_FP32 0  /* float32 of (f_i - w_i), collided in float32: the */
                            /* reference's type, stored as the deviation so a   */
                            /* low-Mach flow keeps its velocity bits            */
#define LBM_STORAGE_FP16S 1 /* float16 of 4096 (f_i - w_i), collided in float32 */
#define LBM_STORAGE_BF16S 2 /* bfloat16 of (f_i - w_i), collided in float32      */
#define LBM_STORAGE_FP64 3  /* float64 populations and float64 arithmetic: the  */
                            /* comparison run of the storage error figures (the */
                            /* reference itself is float32 only).  Every float  */
                            /* buffer of a call on such a lattice -- initial    */
                            /* field, force fields, face densities, observed    */
                            /* f / rho / u, particle arrays -- holds float64.   */

#define LBM_STEP_ROWS (-1)

/* One lattice: velocity set, shape, faces and relaxation.  Mirrors the
 * reference's FlowConfig + Param (flow/base.py:15-114, flow/d3/base.py:72-101). */
typedef struct lbm_lattice {
  int32_t q;              /* 13, 15, 19 or 27 (create_flow, flow/__init__.py:16-41) */
  int32_t nx, ny, nz;     /* node counts = size + 1 (flow/d3/base.py:81-82)         */
  int32_t face[LBM_NFACES];        /* LBM_BC_* per face                             */
  float face_uw[LBM_NFACES][3];    /* wall velocity of WALL_WITH_SPEED faces         */
  float tau;              /* float32(3 mu + 0.5) (flow/d3/base.py:96)               */
  float cs2;              /* float32(sqrt(1/3))^2 (flow/base.py:37-39)              */
  int32_t storage;        /* LBM_STORAGE_*                                          */
  float re_mu;            /* Re * mu, NON_EQUILIBRIUM inlet scale (flow/d3/base.py:137-143) */
  const double *neq_profile; /* device [ny*nz] duct profile init_u / u_max (float64, */
                             /* as cul_u returns it); NULL unless face[0] is NEQ    */
  int32_t step_nodes;     /* launch shape of lbm_flow_step: consecutive z-nodes per  */
                          /* thread (1, 2, 4, 8; nz a multiple of it, except 2 for  */
                          /* 16-bit rows of odd length: pairs within rows),         */
                          /* LBM_STEP_ROWS (whole z-rows staged in shared memory by */
                          /* TMA bulk copies), 0 = default (measured best per Q /   */
                          /* storage / forcing)                                     */
  int32_t step_threads;   /* threads per block (128 or 256; 0 = 128 with the        */
                          /* default shape, else 256)                               */
  int32_t pz;             /* row pitch of the population buffers in elements: a     */
                          /* node (x, y, z) of direction i sits at                  */
                          /* i*nx*ny*pz + (x*ny + y)*pz + z; pz >= nz, 0 = nz.      */
                          /* Padding elements are never read as a source.  A pitch  */
                          /* that is a multiple of the vector width lets rows of    */
                          /* any length use the vectorised step.  Every other array */
                          /* (fields, face planes, observation) stays dense.  The   */
                          /* single-function calls (lbm_collide, lbm_stream,        */
                          /* lbm_moments, lbm_add_force) take dense arrays only.    */
} lbm_lattice;

/* Forcing seen by one step: FOL = uniform + field.  `uniform` is a body force
 * applied at every node; `field` is the spread IBM force ([x][y][z][3], zero
 * outside the 32-node chunks flagged in `chunks`; NULL = no field).
 * "old" is the FOL of the previous step (used by the first moment pass,
 * update_u_rou after f_stream, lbm/base.py:159-163); "new" the FOL of this
 * step (cul_equ2 and the second update_u_rou, lbm/base.py:173-175). */
typedef struct lbm_force {
  float old_uniform[3];
  float new_uniform[3];
  const float *old_field;
  const float *new_field;
  const uint8_t *old_chunks; /* [ceil(n/32)] flags, NULL = all chunks */
  const uint8_t *new_chunks;
} lbm_force;

/* Optional per-step outputs: the reference's state at the end of the step
 * (flow.f after cul_equ2, rou / u after the second update_u_rou). */
typedef struct lbm_observe {
  float *f;   /* float32 SoA [q][x][y][z] or NULL */
  float *rho; /* [x][y][z] or NULL */
  float *u;   /* [x][y][z][3] or NULL */
} lbm_observe;

/* Bytes of the caller-allocated face-density plane buffer for a lattice
 * (2*ny*nz + 2*nx*nz + 2*nx*ny floats; needed when a face is WALL_WITH_SPEED
 * or NON_EQUILIBRIUM, else may be NULL). */
size_t lbm_face_plane_floats(const lbm_lattice *lat);

/* Validate a lattice description.  Returns LBM_ERR_UNSUPPORTED for a face code
 * the reference cannot stream (flow/d3/base.py:218-219, 242-243, 262-263, ...)
 * and LBM_ERR_INVALID for a bad shape, velocity set or tau. */
int lbm_lattice_check(const lbm_lattice *lat);

/* FlowD3.init + the first LBMD3._init collision (flow/d3/base.py:72-101,
 * lbm/lbm3d.py:23-27), followed by step 1's collision, which the reference
 * applies with the init-time moments: writes post-collision populations
 * `fa` (storage type).  `f0` is an optional float32 SoA initial field
 * (NULL = rho*w with rho = 1).  `face_rho` receives the density on the six
 * face planes (may be NULL when no face needs it). */
int lbm_flow_init(const lbm_lattice *lat, const float *f0, void *fa, float *face_rho,
                  void *stream);

/* One fused time step: f_stream + update_u_rou + cul_equ2 + update_u_rou of
 * step k and the cul_equ of step k+1 (lbm/base.py:159-175,
 * flow/d3/base.py:103-181) in one sweep.  Reads post-collision populations
 * `fa`, writes post-collision populations `fb` (fb may be NULL: observation
 * only, nothing but `obs` is written).  face_rho_in / face_rho_out hold the
 * face-plane densities before / after the step (WALL_WITH_SPEED, NEQ).
 * `status` (may be NULL) receives LBM_STATUS_* bits. */
int lbm_flow_step(const lbm_lattice *lat, const void *fa, void *fb, const lbm_force *force,
                  const float *face_rho_in, float *face_rho_out, const lbm_observe *obs,
                  uint32_t *status, void *stream);

/* Statistics of the state at the end of the step that streams from `fa`
 * (the reference's f after cul_equ2, rou / u after the second update_u_rou)
 * without materialising it: FlowD3.to_json (flow/base.py:183-206) as
 * LBMBase._log_step_info logs it (lbm/base.py:105-144).  Reads the
 * populations once and writes `out`, a device buffer of 9 doubles (8-byte
 * aligned): min, mean, max of f (over all nodes and directions), of u (all
 * components) and of rho.  Arguments as lbm_flow_step with fb = NULL. */
int lbm_flow_stats(const lbm_lattice *lat, const void *fa, const lbm_force *force,
                   const float *face_rho_in, double *out, uint32_t *status, void *stream);

/* ---- many lattices per launch (serving) ---------------------------------
 * One fused step (as lbm_flow_step) for up to thousands of independent
 * lattices of one velocity set and storage in a single launch -- the form
 * LBMBase.run_step (lbm/base.py:146-157) takes when many simulations are
 * served together.  The caller packs one entry per lattice on the host
 * (lbm_batch_pack, lbm_batch_entry_bytes() bytes each; the entry records the
 * buffer addresses, so it is valid while they are), copies the entries and
 * the exclusive prefix sum of their block counts to device memory, and
 * launches.  A lattice's result is the same in a batch as alone. */
size_t lbm_batch_entry_bytes(void);
/* nodes: 1 (one node per thread), 2 or 4 (that many z-nodes per thread; rows
 * of a multiple of that many nodes, at least twice as many).  *blocks
 * receives the lattice's block count. */
int lbm_batch_pack(const lbm_lattice *lat, const void *fa, void *fb, const lbm_force *force,
                   const float *face_rho_in, float *face_rho_out, uint32_t *status, int32_t nodes,
                   void *entry, uint32_t *blocks);
/* entries / block_begin: device arrays of `count` packed entries (all with
 * the same q, storage and nodes) and their first-block indices;
 * total_blocks = sum of the block counts; force != 0 if any entry has a
 * force. */
int lbm_flow_step_batch(int32_t q, int32_t storage, int32_t nodes, int32_t force,
                        const void *entries, const uint32_t *block_begin, int32_t count,
                        uint32_t total_blocks, void *stream);

/* Single reference functions on float32 SoA populations, for callers that
 * invoke FlowD3's methods one at a time. */
/* FlowD3.cul_equ (flow/d3/base.py:150-159): f <- f - (f - feq)/tau in place;
 * feq (may be NULL) receives the equilibrium. */
int lbm_collide(const lbm_lattice *lat, float *f, const float *rho, const float *u, float *feq,
                void *stream);
/* FlowD3.f_stream + f_stream_bound* (flow/d3/base.py:161-323): f_out from
 * f_in (the reference's fcopy).  rho: densities for WALL_WITH_SPEED faces;
 * feq: equilibrium of the last cul_equ for NON_EQUILIBRIUM faces. */
int lbm_stream(const lbm_lattice *lat, const float *f_in, float *f_out, const float *rho,
               const float *feq, void *stream);
/* FlowD3.update_u_rou + update_u_rou_boundary (flow/d3/base.py:116-148):
 * rho, u, p from f and FOL (fol may be NULL = zero).  `scratch` is one
 * caller-allocated float used for the inlet's global density maximum when
 * the input face is NON_EQUILIBRIUM (else may be NULL). */
int lbm_moments(const lbm_lattice *lat, const float *f, const float *fol, float *rho, float *u,
                float *p, float *scratch, void *stream);
/* FlowD3.cul_equ2 (flow/d3/base.py:103-114): f += forcing(u, FOL) in place. */
int lbm_add_force(const lbm_lattice *lat, float *f, const float *u, const float *fol,
                  void *stream);

/* ---- immersed boundary and rigid particles ------------------------------ */

/* Marker / particle state of all particles of one lattice, concatenated in
 * the reference's (particle, marker) loop order.  Float32 like the reference,
 * except the particle state that is integrated in float64. */
typedef struct lbm_particles {
  int32_t n_particles;
  int32_t n_markers;             /* total over all particles                  */
  const int32_t *marker_offset;  /* [n_particles + 1] first marker of each    */
  const int32_t *marker_owner;   /* [n_markers] particle index of each marker */
  const float *lagrange;         /* [n_markers][3] body-frame marker points   */
  float *lx;                     /* [n_markers][3] marker positions           */
  float *lu;                     /* [n_markers][3] rigid velocity at markers  */
  float *lF;                     /* [n_markers][3] marker force               */
  float *lrou;                   /* [n_markers] interpolated density          */
  const float *lm;               /* [n_markers] marker area weight            */
  float *cx, *cu, *cw, *cF, *cT; /* [n_particles][3] float32 mirrors          */
  float *angle;                  /* [n_particles][3] rotation vector          */
  const float *mass;             /* [n_particles]                             */
  const float *inertia;          /* [n_particles][3]                          */
  const float *rou;              /* [n_particles] particle density            */
  int32_t fp64;                  /* 1: every float array above holds float64  */
                                 /* (particles of an LBM_STORAGE_FP64 lattice) */
  int32_t *extreme;              /* [n_particles][6] markers of least x, y, z */
                                 /* and greatest x, y, z (first on ties), the  */
                                 /* wall spring's markers; kept by rigid_step  */
                                 /* / rigid_extremes, read by                  */
                                 /* ibm_interpolate_wall (NULL otherwise)      */
} lbm_particles;

/* LBMD3.flow_to_lagrange (lbm/lbm3d.py:66-100) fused with the moment pass
 * it reads: for every marker, streams the 4x4x4 stencil nodes from the
 * post-collision populations `fa`, takes the first update_u_rou moments there
 * (with the previous step's force), interpolates with the normalised cosine
 * delta, and writes lu (rigid velocity), lF and lrou.  With fa == NULL the
 * moments are read from `u_field` ([x][y][z][3]) and `rho_field` ([x][y][z])
 * instead (the reference's flow.u / flow.rou).  `step` is the reference's
 * step counter (the weight-sum sentinel is active after step 100). */
int ibm_interpolate(const lbm_lattice *lat, const void *fa, const lbm_force *force,
                    const float *face_rho_in, const float *u_field, const float *rho_field,
                    const lbm_particles *pt, float dt, int32_t step, uint32_t *status,
                    void *stream);

/* LBMD3.particle_to_wall (lbm/lbm3d.py:121-167) and
 * Particle.update_from_lar (particle/base/base.py:120-151) for all particles:
 * the spring force on the six extreme markers (what & 1), then force / torque
 * sums over markers in float64 and the explicit Euler update of cu, cx, cw
 * (what & 2).  `lat` (the wall bounds) may be NULL when what == RIGID_UPDATE. */
#define RIGID_WALL 1
#define RIGID_UPDATE 2
int rigid_wall_and_update(const lbm_lattice *lat, const lbm_particles *pt, int32_t what, float dt,
                          float dx, float gl, float rouf, void *stream);

/* LBMD3.lagrange_to_flow (lbm/lbm3d.py:102-119): FOL := 0, then each
 * marker's stencil box receives w * lF * lm.  mode 0 = the reference's
 * assignment, the last (particle, marker) in loop order wins; mode 1 =
 * accumulation (the physical spreading sum).  `field` is [x][y][z][3];
 * `chunks` flags the 32-node chunks written (and, on entry, those written
 * last time, which are cleared first); `owner` is an int32 scratch array of
 * n nodes that must hold -1 everywhere on entry and holds -1 again on exit. */
int ibm_spread(const lbm_lattice *lat, const lbm_particles *pt, int32_t mode, float *field,
               uint8_t *chunks, int32_t *owner, void *stream);

/* LBMD3.lagrange_to_flow (lbm/lbm3d.py:102-119) as ibm_spread, resolved in
 * 8 x 8 x 8-node tiles in shared memory: one pass lists each marker under the
 * tiles its stencil touches; one block per tile then takes the last writer of
 * every node (mode 0) or sums the contributions (mode 1) in shared memory and
 * writes each node once.  Mode 0 gives ibm_spread's field bit for bit.
 * `scratch`: caller-owned device memory of at least
 * ibm_spread_tiled_scratch_bytes(lat, pt->n_markers) bytes, zero before its
 * first use (every call leaves the part that must start at zero at zero). */
size_t ibm_spread_tiled_scratch_bytes(const lbm_lattice *lat, int32_t n_markers);
int ibm_spread_tiled(const lbm_lattice *lat, const lbm_particles *pt, int32_t mode, float *field,
                     uint8_t *chunks, void *scratch, size_t scratch_bytes, void *stream);

/* Allocation-free ibm_spread.  No counterpart in the reference.  For callers
 * that cannot allocate device memory themselves -- a host program that only
 * has the lattice's own buffers (a solver coupled in through this C ABI from
 * another language, or a loop with a fixed device-memory budget where a
 * cudaMalloc would fail or synchronise the device) -- the per-node claim
 * array that ibm_spread takes from the caller is here a static array inside
 * the library: LBM_SPREAD_NOALLOC_MAX_NODES int32 (16 MiB), held on every GPU
 * that loads the library until the process exits.  Lattices with more nodes
 * are rejected with LBM_ERR_INVALID.  The call allocates nothing.  Its first
 * call on a device looks up the array's device address, and its first
 * reference-mode call (mode 0) on a device also sets the whole array to -1
 * (every later call leaves it at -1 again); make those first calls before any
 * stream capture.  The looked-up address belongs to the device's primary
 * context: after cudaDeviceReset it is stale, so do not call this entry point
 * again in that process.  All calls share the one array: calls whose work
 * overlaps on the GPU race, so issue them in order on one stream.  Arguments
 * and results are those of ibm_spread without `owner`. */
#define LBM_SPREAD_NOALLOC_MAX_NODES (1 << 22)
int ibm_spread_noalloc(const lbm_lattice *lat, const lbm_particles *pt, int32_t mode, float *field,
                       uint8_t *chunks, void *stream);

/* LBMD3.flow_to_lagrange fused with LBMD3.particle_to_wall
 * (lbm/lbm3d.py:66-167): the interpolation of ibm_interpolate from the
 * post-collision populations `fa`, and the wall spring of
 * rigid_wall_and_update(RIGID_WALL) applied to the six extreme markers of each
 * particle as their forces are written (pt->extreme must hold the extremes of
 * the current positions: rigid_step keeps it, rigid_extremes recomputes it).
 * `dx` is the spring's length scale.  Same results as the two calls. */
int ibm_interpolate_wall(const lbm_lattice *lat, const void *fa, const lbm_force *force,
                         const float *face_rho_in, const lbm_particles *pt, float dt, float dx,
                         int32_t step, uint32_t *status, void *stream);

/* LBMD3.flow_to_lagrange + particle_to_wall + the first half of
 * lagrange_to_flow in reference mode (lbm/lbm3d.py:66-119): ibm_interpolate_wall,
 * and in the same launch the claims of ibm_spread's reference mode (every
 * in-box stencil node of every marker gets the largest marker index in
 * `owner`, which must hold -1 there) and the clearing of the chunks of `field`
 * flagged in `chunks` (those written the last time this buffer was used).
 * ibm_spread_claimed finishes the spreading; the pair gives the results of
 * ibm_interpolate_wall followed by ibm_spread(mode 0) in two launches fewer.
 * With no markers only the clearing runs. */
int ibm_interpolate_wall_claim(const lbm_lattice *lat, const void *fa, const lbm_force *force,
                               const float *face_rho_in, const lbm_particles *pt, float dt,
                               float dx, int32_t step, uint32_t *status, float *field,
                               uint8_t *chunks, int32_t *owner, void *stream);

/* The second half of reference-mode LBMD3.lagrange_to_flow
 * (lbm/lbm3d.py:102-119) after ibm_interpolate_wall_claim, in one launch: the
 * owner of each claimed node writes w lF lm there, flags its chunk and
 * releases the claim (`owner` holds -1 again afterwards). */
int ibm_spread_claimed(const lbm_lattice *lat, const lbm_particles *pt, float *field,
                       uint8_t *chunks, int32_t *owner, void *stream);

/* Particle.update_from_lar then Particle.update (particle/base/base.py:120-156,
 * particle/coord.py:87-108) for all particles in one launch -- the rigid
 * update of rigid_wall_and_update(RIGID_UPDATE) followed by the marker
 * transform of rigid_update_markers -- and the six extreme markers of the new
 * positions into pt->extreme (when not NULL) for the next step's wall spring.
 * The spring itself is not applied here (ibm_interpolate_wall does it).
 * Same results as the two calls. */
int rigid_step(const lbm_particles *pt, float dt, float gl, float rouf, void *stream);

/* The six extreme markers of the current positions into pt->extreme
 * (the argmin / argmax of lbm/lbm3d.py:121-167). */
int rigid_extremes(const lbm_particles *pt, void *stream);

/* Particle.update + Coordinate.update/cul_point (particle/base/base.py:153-156,
 * particle/coord.py:87-108): angle += cw; lx = R(angle) lagrange + cx, with the
 * rotation built in float64 from the rotation vector. */
int rigid_update_markers(const lbm_particles *pt, void *stream);

/* Test hook, no counterpart in the reference: poll limit of the consumer-side
 * mbarrier waits of the row-staged step (lattices with step_nodes =
 * LBM_STEP_ROWS) for the launches that follow, process-wide.  A negative
 * value restores the default (2^24 polls, also the maximum); 0 makes every
 * such wait give up before its first poll, so that the timeout path --
 * LBM_STATUS_WAIT_TIMEOUT in the status word, the kernel's own bulk copies
 * drained under the default limit, an orderly return -- can be exercised
 * without a fault.  Populations of a step that timed out are incomplete. */
void lbm_debug_set_wait_limit(int64_t polls);

/* Bounds-checked builds (liblbm_b200_checked.so, compiled with
 * -DLBM_BOUNDS_CHECK; no counterpart in the reference): the number of index
 * violations the kernels caught since the last reset (each one skipped or
 * clamped its access), over all translation units; reset != 0 zeroes the
 * counts.  -1 in a normal build, -2 if a count could not be read. */
int64_t lbm_debug_bounds_faults(int32_t reset);

/* Thread-local message of the last failed call. */
const char *lbm_last_error(void);

/* Library version string. */
const char *lbm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FUNLBM_B200_H */
