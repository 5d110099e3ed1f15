/*
 * tlbm.h - C ABI of the B200 lattice-Boltzmann step library (libtlbm.so).
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * (passed as void*), enqueues its kernels on that stream and returns a
 * tlbm_status without synchronising.  The caller owns every buffer.
 *
 * Population layout (all lattices): structure of arrays, shape (Q, nz, ny, nx)
 * with x fastest; 2-D lattices use nz = 1, i.e. (Q, ny, nx).  Element q of
 * cell (z, y, x) sits at  q*N + (z*ny + y)*nx + x,  N = nx*ny*nz.  Direction
 * numbering is TensorLBM's (tensorlbm/d2q9.py:8-26, tensorlbm/d3q19.py:6-67,
 * tensorlbm/d3q27.py:32-84).
 *
 * Each declaration names the TensorLBM function (file:line, paths inside the
 * TensorLBM source tree) whose behaviour it reproduces.
 */
#ifndef TLBM_H
#define TLBM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TLBM_API __attribute__((visibility("default")))
#define TLBM_ABI_VERSION 3

typedef enum tlbm_status {
  TLBM_OK = 0,
  TLBM_ERR_SHAPE = 1,       /* bad sizes / plane too small */
  TLBM_ERR_DTYPE = 2,       /* unsupported dtype or dtype combination */
  TLBM_ERR_ALIAS = 3,       /* f_in == f_out where the kernel pulls from neighbours */
  TLBM_ERR_LAUNCH = 4,      /* a CUDA launch or runtime call failed */
  TLBM_ERR_TIMEOUT = 5,     /* a bounded device-side wait expired */
  TLBM_ERR_NONFINITE = 6,   /* reported by callers that read the status word */
  TLBM_ERR_ARG = 7,         /* null pointer or invalid parameter */
  TLBM_ERR_UNSUPPORTED = 8, /* lattice / collision / boundary combination not built */
  TLBM_ERR_TOO_LARGE = 9    /* input larger than a fixed-size static scratch array or an index width */
} tlbm_status;

typedef enum tlbm_lattice { TLBM_D2Q9 = 9, TLBM_D3Q19 = 19, TLBM_D3Q27 = 27 } tlbm_lattice;

/* Storage / arithmetic formats.  The shifted half formats store the deviation
 * f_q - w_q (times 2^14 for float16, which keeps it out of the subnormal
 * range), stochastically rounded (unbiased; the random bits hash the cell and
 * the new value), and compute in float32. */
typedef enum tlbm_dtype {
  TLBM_F32 = 0,
  TLBM_F64 = 1,
  TLBM_F16_SHIFTED = 2,
  TLBM_BF16_SHIFTED = 3,
  TLBM_F16 = 4,        /* plain float16 f, round-to-nearest on store: the storage of
                          triton_fused.py:440-522 (D3Q19 stream and BGK only) */
  TLBM_BF16 = 5        /* plain bfloat16 f, round-to-nearest (D3Q19 stream and BGK only) */
} tlbm_dtype;

typedef enum tlbm_collision {
  TLBM_COLL_NONE = 0,             /* no collision (stream / boundary only, or a format conversion) */
  TLBM_COLL_BGK = 1,              /* solver.py:67, solver3d.py:100, d3q27.py:423 */
  TLBM_COLL_MRT = 2,              /* solver.py:249, solver3d.py:107, d3q27.py:643 */
  TLBM_COLL_CUMULANT = 3,         /* D3Q27 legacy, cumulant.py:935 */
  TLBM_COLL_CUMULANT_GEIER = 4,   /* D3Q27 Geier 2015, cumulant.py:1050 */
  TLBM_COLL_CUMULANT_D3Q19 = 5,   /* cumulant.py:1159 (Smagorinsky via c_smag) */
  TLBM_COLL_SMAGORINSKY = 6,      /* turbulence.py:245 (D3Q19), :216 (D2Q9), :472 (D3Q27) */
  TLBM_COLL_TRT = 7,              /* solver.py:440, solver3d.py:303, d3q27.py:438 (tau = tau_plus > 1/2) */
  TLBM_COLL_CASCADED = 8,         /* cascaded_collision.py:445 (D3Q19), :512 (D3Q27); rates: omega_b = s_bulk,
                                     omega_odd = s_3, omega_even = s_4, cm_s5 / cm_s6 (D3Q27) */
  TLBM_COLL_RLBM = 9              /* regularised BGK: solver.py:338 (D2Q9), solver3d.py:342 (D3Q19),
                                     d3q27.py:481 (D3Q27); a tau field is ignored */
} tlbm_collision;

/* Boundary conditions applied by tlbm_step after the pull, in this order:
 *   obstacle force sample -> Zou/He inlet (x=0) -> Zou/He outlet (x=nx-1)
 *   -> far field -> full-way bounce-back on TLBM_FLAG_SOLID cells -> moving lid (y=ny-1).
 * This is the order of tensorlbm/d3q27_sphere_flow.py:246-256 and
 * benchmarks/verified/cavity_3d_full (collide, stream, walls, lid). */
typedef enum tlbm_bc_bits {
  TLBM_BC_LID = 1u,        /* boundaries3d.py:324 / lid_driven_cavity.py:431 */
  TLBM_BC_ZH_INLET = 2u,   /* boundaries.py:50, boundaries3d.py:205, boundaries_d3q27.py:107 */
  TLBM_BC_ZH_OUTLET = 4u,  /* boundaries.py:102, boundaries3d.py:269, boundaries_d3q27.py:179 */
  /* free-stream far field (boundaries.py:199 far_field_bc_2d, boundaries3d.py:446
   * far_field_bc_3d, boundaries_d3q27.py:63 far_field_bc_27): the x = 0 plane and
   * the y = 0, y = ny-1 planes take feq(1, u_in); the x = nx-1 plane takes the
   * post-stream populations of x = nx-2 (zero gradient; the lateral planes win on
   * their edges).  Not with the Zou/He bits. */
  TLBM_BC_FAR_FIELD = 8u,
  TLBM_BC_FAR_FIELD_Z = 16u /* with TLBM_BC_FAR_FIELD, 3-D: the z = 0, z = nz-1 planes too */
} tlbm_bc_bits;

/* Per-cell flag byte. */
typedef enum tlbm_flag_bits {
  TLBM_FLAG_SOLID = 1u,     /* post-stream full-way bounce-back (wall XOR obstacle, as two
                               successive swaps cancel): bounce_back_cells* after stream */
  TLBM_FLAG_OBSTACLE = 2u,  /* summed into the momentum-exchange force */
  TLBM_FLAG_HALFWAY = 4u,   /* pre-stream half-way wall: the cell is not collided, its
                               populations are stored reversed (where(wall, f_pre[opp], f)
                               before stream: cases/base.py:270-289 pre-boundaries,
                               lbm_step_correct.py:62 "bb" mode) */
  TLBM_FLAG_MOVING = 8u,    /* Ladd moving wall (with SOLID): swap plus 2 w rho (c.u_w)/c_s^2,
                               u_w from tlbm_desc.wall_velocity (propeller_benchmark.py:221) */
  TLBM_FLAG_CURVED = 16u    /* fluid cell with Bouzidi (BFL) interpolated links to a curved wall
                               (bfl_common.py:106): after the pull, in place of the bounce-back,
                               f[opp_d] = 2q P_d + (1-2q) P_d(x-c_d) (q < 1/2) or
                               P_d/(2q) + (2q-1)/(2q) P_opp (q >= 1/2) on every link d of the cell;
                               tables tlbm_desc.link_row / link_q.  With a force buffer the step
                               adds the BFL ledger sum_links c_d (P_d + f_bc) (bfl_d3q19.py:339) */
} tlbm_flag_bits;

typedef struct tlbm_desc {
  int32_t lattice;     /* tlbm_lattice */
  int32_t dtype;       /* tlbm_dtype of the population buffers */
  int32_t collision;   /* tlbm_collision */
  int32_t nx, ny, nz;  /* nz = 1 for D2Q9 */
  uint32_t bc;         /* tlbm_bc_bits */
  double tau;          /* shear relaxation time */
  double s_e, s_eps, s_q, s_pi;          /* MRT rates; s_pi < 0 means s_pi = s_e */
  double omega_b, omega_odd, omega_even; /* cumulant rates */
  double c_smag;       /* Smagorinsky constant (TLBM_COLL_SMAGORINSKY, CUMULANT_D3Q19) */
  double u_lid;        /* lid x-velocity */
  double u_in[3];      /* Zou/He inlet velocity */
  double rho_out;      /* Zou/He outlet density */
  const void* wall_velocity; /* (DIM, N) wall velocity of TLBM_FLAG_MOVING cells in the compute
                                type (float32; float64 for TLBM_F64), x-component first; may be NULL */
  double force_lin;    /* linear body force F = force_lin * rho * u (Lundgren forcing of forced
                          isotropic turbulence), exact-difference scheme: after the collision
                          f += feq(rho, (1 + A) u) - feq(rho, u); 0 = none.  BGK, MRT and
                          Smagorinsky collisions (else TLBM_ERR_UNSUPPORTED) on float32
                          populations (else TLBM_ERR_DTYPE); |A| < 1.  New in this library. */
  double lambda_trt;   /* TRT magic parameter: tau_minus = 1/2 + lambda_trt / (tau - 1/2)
                          (TLBM_COLL_TRT; TensorLBM's default is 3/16) */
  const int32_t* link_row; /* TLBM_FLAG_CURVED cells: row of the cell in link_q (may be NULL: no links) */
  const float* link_q;     /* (rows, Q) wall fraction of each link of the row, in (0, 1]; 0 = no link */
  double cm_s5, cm_s6;     /* cascaded D3Q27 5th / 6th-order rates; negative = omega_even (TensorLBM's
                              defaults) */
  double ff_inlet_du[3];   /* TLBM_BC_FAR_FIELD: the x = 0 plane takes feq(1, u_in + ff_inlet_du) (a
                              perturbation seeded at the inlet, benchmarks/verified/cylinder); 0 = none.
                              New in ABI version 3. */
} tlbm_desc;

/* ---- fused time step ------------------------------------------------------
 * One kernel pass: periodic pull f_in[q, x - c_q] -> boundary conditions ->
 * collision -> store at x in f_out.  The stored state is post-collision, so
 * repeated calls advance the TensorLBM chain collide -> stream -> boundaries
 * by one step each with the phase shifted by half a step (a collision-only
 * call with tlbm_collide turns a TensorLBM state into this phase, and a call
 * with collision = TLBM_COLL_NONE turns it back).
 * f_in must not alias f_out.  force (3 doubles, may be NULL) accumulates
 * 2*sum_{obstacle} sum_q c_q f_q (post-stream, pre-bounce-back; obstacles.py:91,
 * :197, boundaries.py:162) - zero it before the first step you want summed.
 * status (may be NULL) gets bit 0 set if a non-finite density was seen, and
 * bit 3 if the row-staged kernel (tlbm_set_row_staging) gave up waiting for
 * its shared-memory copies (the step is then incomplete).
 * tau_field (may be NULL) gives a per-cell tau for BGK / MRT shear rates.
 * Replaces: cases/base.py:270-289 make_step() closures, triton_fused.py:804
 * TritonFusedSolver3D.step, triton_fused_obstacle.py:1695. */
TLBM_API int tlbm_step(const tlbm_desc* d, const void* f_in, void* f_out, const uint8_t* flags,
                       const float* tau_field, double* force, unsigned int* status, void* stream);

/* tlbm_step on the planes z_begin .. z_begin + z_count - 1 only (the others of
 * f_out are not written); neighbours still wrap periodically over d->nz.  With
 * one ghost plane on each side of a slab (planes 0 and nz - 1 hold the
 * neighbouring slabs' boundary planes) and z_begin = 1, z_count = nz - 2, the
 * owned planes get exactly the values of the undivided domain: the slab step
 * of the z-decomposed solver (triton_fused_distributed.py:564 runs its kernel
 * over the ghost planes as well).  force and status cover the updated planes. */
TLBM_API int tlbm_step_planes(const tlbm_desc* d, const void* f_in, void* f_out, const uint8_t* flags,
                              const float* tau_field, double* force, unsigned int* status, int32_t z_begin,
                              int32_t z_count, void* stream);

/* Local collision only (no streaming, no boundaries); f_in may equal f_out.
 * dtype_out may differ from d->dtype only for TLBM_COLL_NONE (format
 * conversion).  flags (may be NULL): TLBM_FLAG_HALFWAY cells are stored
 * reversed instead of collided.
 * Replaces: collide_bgk (solver.py:67), collide_mrt (solver.py:249),
 * collide_bgk3d (solver3d.py:100), collide_mrt3d (solver3d.py:107),
 * collide_bgk27 (d3q27.py:423), collide_mrt27 (d3q27.py:643),
 * collide_cumulant_d3q27 (cumulant.py:935), collide_cumulant_geier_d3q27
 * (cumulant.py:1050), collide_cumulant_d3q19 (cumulant.py:1159),
 * collide_smagorinsky_bgk3d (turbulence.py:245). */
TLBM_API int tlbm_collide(const tlbm_desc* d, int32_t dtype_out, const void* f_in, void* f_out,
                          const uint8_t* flags, const float* tau_field, void* stream);

/* Periodic pull streaming.  Replaces stream (solver.py:396), stream3d
 * (solver3d.py:210), stream3d_roll (solver3d.py:266), stream27 (d3q27.py:766). */
TLBM_API int tlbm_stream(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz,
                         const void* f_in, void* f_out, void* stream);

/* f_eq from (rho, ux, uy[, uz]); uz ignored for D2Q9.  F32/F64 only.
 * Replaces equilibrium (d2q9.py:39), equilibrium3d (d3q19.py:83),
 * equilibrium27 (d3q27.py:353). */
TLBM_API int tlbm_equilibrium(int32_t lattice, int32_t dtype, int64_t ncells, const void* rho,
                              const void* ux, const void* uy, const void* uz, void* f_out,
                              void* stream);

/* (rho, ux, uy[, uz]) from f; uz may be NULL for D2Q9.  F32/F64 only.
 * Replaces macroscopic (d2q9.py:61), macroscopic3d (d3q19.py:165),
 * macroscopic27 (d3q27.py:395). */
TLBM_API int tlbm_macroscopic(int32_t lattice, int32_t dtype, int64_t ncells, const void* f,
                              void* rho, void* ux, void* uy, void* uz, void* stream);

/* f_out = where(mask, f_in[opp], f_in); mask is one byte per cell.
 * Replaces bounce_back_cells (boundaries.py:39), bounce_back_cells_3d
 * (boundaries3d.py:112), bounce_back_cells_27 (boundaries_d3q27.py:45). */
TLBM_API int tlbm_bounce_back(int32_t lattice, int32_t dtype, int64_t ncells, const void* f_in,
                              const uint8_t* mask, void* f_out, void* stream);

/* Ladd moving-wall bounce-back: f_out = where(mask, bounce_back(f_in) +
 * 2 w rho (c.u_w) / c_s^2, f_in) with rho = sum f_in and u_w given per cell as
 * DIM consecutive arrays of ncells (x first).  D2Q9 / D3Q19, F32/F64.
 * Replaces moving_wall_bounce_back (rotating_cylinder.py:140) and
 * moving_wall_bounce_back_3d (propeller_benchmark.py:221). */
TLBM_API int tlbm_moving_wall_bounce_back(int32_t lattice, int32_t dtype, int64_t ncells, const void* f_in,
                                          const uint8_t* mask, const void* wall_velocity, void* f_out,
                                          void* stream);

/* Zou/He velocity inlet on the x = 0 plane, in place.  ux_profile / uy_profile
 * (D2Q9 only, length ny, may be NULL) override u_in / uy_in per row.
 * Replaces zou_he_inlet_velocity (boundaries.py:50), zou_he_inlet_velocity_3d
 * (boundaries3d.py:205), zou_he_inlet_velocity_27 (boundaries_d3q27.py:107). */
TLBM_API int tlbm_zou_he_inlet(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz,
                               void* f, double u_in, double uy_in, double uz_in,
                               const void* ux_profile, const void* uy_profile, void* stream);

/* Zou/He pressure outlet on the x = nx-1 plane, in place.
 * Replaces zou_he_outlet_pressure (boundaries.py:102), zou_he_outlet_pressure_3d
 * (boundaries3d.py:269), zou_he_outlet_pressure_27 (boundaries_d3q27.py:179). */
TLBM_API int tlbm_zou_he_outlet(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz,
                                void* f, double rho_out, void* stream);

/* Free-stream far field, in place: the x = 0 plane and the y = 0 / y = ny-1
 * planes (and with z_faces != 0 in 3-D the z = 0 / z = nz-1 planes) take
 * feq(1, (ux, uy, uz)), after the x = nx-1 plane took the values of x = nx-2.
 * The obstacle bounce-back of the reference functions is tlbm_bounce_back.
 * Replaces far_field_bc_2d (boundaries.py:199), far_field_bc_3d
 * (boundaries3d.py:446) and far_field_bc_27 (boundaries_d3q27.py:63). */
TLBM_API int tlbm_far_field(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz, void* f,
                            double ux, double uy, double uz, int32_t z_faces, void* stream);

/* Zou/He moving lid on the y = ny-1 plane (all cells, corners included), in place.
 * Replaces zou_he_moving_lid (lid_driven_cavity.py:431) and zou_he_moving_lid_3d
 * (boundaries3d.py:324).  D2Q9 / D3Q19 only. */
TLBM_API int tlbm_moving_lid(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz,
                             void* f, double u_lid, void* stream);

/* Momentum-exchange force 2*sum_{mask} sum_q c_q f_q into out[0..2] (float64,
 * overwritten).  Replaces compute_obstacle_forces (boundaries.py:162),
 * compute_obstacle_forces_3d (obstacles.py:91), compute_obstacle_forces_27
 * (obstacles.py:197). */
TLBM_API int tlbm_obstacle_force(int32_t lattice, int32_t dtype, int64_t ncells, const void* f,
                                 const uint8_t* mask, double* out, void* stream);

/* f_out = f_in * (target_mass / sum(f_in)), unless |sum| < 1e-30 (then a copy).
 * The sum is accumulated in float64 in scratch[0] (one double the caller
 * provides).  Replaces correct_mass (solver.py:420), correct_mass3d
 * (solver3d.py:287), correct_mass27 (d3q27.py:729). */
TLBM_API int tlbm_correct_mass(int32_t dtype, int64_t count, const void* f_in, void* f_out,
                               double target_mass, double* scratch, void* stream);

/* float64 sums over cells: out[0] = sum rho, out[1..3] = sum j (momentum).
 * out overwritten.  Diagnostic counterpart of the mass / momentum checks in
 * tensorlbm/reporters.py and utils.DiagnosticPoint. */
TLBM_API int tlbm_moment_sums(int32_t lattice, int32_t dtype, int64_t ncells, const void* f,
                              double* out, void* stream);

/* Obstacle masks, one byte per cell, evaluated in float32 exactly as
 * sphere_mask (boundaries3d.py:29) and cylinder_mask (boundaries.py:8). */
TLBM_API int tlbm_sphere_mask(int32_t nx, int32_t ny, int32_t nz, double cx, double cy, double cz,
                              double radius, uint8_t* out, void* stream);
TLBM_API int tlbm_cylinder_mask(int32_t nx, int32_t ny, double cx, double cy, double radius,
                                uint8_t* out, void* stream);

/* With wall_flag = TLBM_FLAG_SOLID:
 *   flags = (wall XOR obstacle ? SOLID : 0) | (obstacle ? OBSTACLE : 0),
 * which encodes the successive bounce_back_cells(wall),
 * bounce_back_cells(obstacle) calls of apply_zou_he_channel_boundaries_3d
 * (boundaries3d.py:707).  With wall_flag = TLBM_FLAG_HALFWAY, wall cells get
 * HALFWAY (pre-stream walls) and obstacle cells SOLID | OBSTACLE.
 * wall or obstacle may be NULL. */
TLBM_API int tlbm_build_flags(int64_t ncells, const uint8_t* wall, const uint8_t* obstacle,
                              uint32_t wall_flag, uint8_t* flags, void* stream);

/* missing[q, cell] = 1 where the pull source cell - c_q is solid or outside a
 * non-periodic face.  periodic_bits: 1 = x, 2 = y, 4 = z periodic.
 * Replaces derive_missing_mask (boundary_registry.py:488). */
TLBM_API int tlbm_missing_mask(int32_t lattice, int32_t nx, int32_t ny, int32_t nz,
                               const uint8_t* solid, int32_t periodic_bits, uint8_t* missing,
                               void* stream);

/* Link list of a byte mask: the flat indices of its non-zero entries in
 * increasing order (torch.nonzero order of the (q, z, y, x) mask).
 * tlbm_link_count writes the count to *count_out (device int64);
 * block_counts must hold tlbm_link_blocks(count) int64 values.
 * tlbm_link_list writes the indices (int64) using the same block_counts. */
TLBM_API int64_t tlbm_link_blocks(int64_t count);
TLBM_API int tlbm_link_count(const uint8_t* mask, int64_t count, int64_t* block_counts,
                             int64_t* count_out, void* stream);
TLBM_API int tlbm_link_list(const uint8_t* mask, int64_t count, const int64_t* block_counts,
                            int64_t* out, void* stream);

/* Allocation-free link list.  No counterpart in TensorLBM: it exists for host
 * programs that reserve all device memory up front and may not call
 * cudaMalloc/cudaFree (or any allocating library) while they run - a fixed
 * memory budget owned by a solver framework or a caching allocator, where a
 * new allocation can fail or stall the device mid-pipeline.
 * Same result as tlbm_link_count + tlbm_link_list in one call, but the
 * per-block scratch is a static device array inside the library (1 MiB on every
 * device that loads it, kept until the process exits), so the mask may hold at
 * most tlbm_link_list_static_capacity() bytes (128 Mi); larger masks return
 * TLBM_ERR_TOO_LARGE before any work.  *count_out (device int64) receives the
 * number of non-zero entries; the first min(count, out_capacity) indices are
 * written to out (out may be NULL when out_capacity is 0: a count-only
 * query).  The first call on each device looks the array up with
 * cudaGetSymbolAddress (make it before any stream capture).  All calls share
 * the array: calls whose kernels overlap on the GPU (different streams or
 * devices sharing nothing but the array - it is per device) race and must be
 * ordered by the caller.  Nothing in the array needs clearing between calls:
 * each call writes every entry it reads. */
TLBM_API int tlbm_link_list_noalloc(const uint8_t* mask, int64_t count, int64_t* out, int64_t out_capacity,
                                    int64_t* count_out, void* stream);
TLBM_API int64_t tlbm_link_list_static_capacity(void);

/* ---- batched runner: many independent small domains --------------------------
 * Replaces the sequential per-point loop of the scan runner
 * (scan_runner.py:697 run_scan_point, :979 ScanExecutor): D2Q9 for the
 * cylinder-flow chain of cylinder_flow.py:854-899 (collide -> stream -> force
 * -> Zou/He inlet -> outlet -> bounce-back), D3Q19 for the case chain of
 * cases/base.py:270-289 (collide -> pre-streaming half-way walls -> stream ->
 * lid), the lid-driven cavity of cases/cavity.py:25-110.  Each domain is a
 * (Q, nz, ny, nx) block at f_offset (elements) in one packed population
 * buffer, with its nz*ny*nx flag bytes at cell_offset in one packed flag
 * buffer.  tiles holds ntiles triplets (domain, x0, r0) of tile_x x tile_y
 * cells, where r0 counts the domain's nz*ny rows (row r is y = r % ny,
 * z = r / ny); every cell of every domain must be in exactly one tile.  Every
 * domain evolves bit for bit as tlbm_step would advance it alone. */
typedef struct tlbm_batch_domain {
  int64_t f_offset;
  int64_t cell_offset;
  int32_t nx, ny;
  double tau;
  double u_in;      /* Zou/He inlet x-velocity (TLBM_BC_ZH_INLET) */
  double rho_out;   /* Zou/He outlet density (TLBM_BC_ZH_OUTLET) */
  uint32_t bc;
  int32_t nz;       /* planes (D3Q19); 0 or 1 for D2Q9 */
  double u_lid;     /* lid x-velocity at y = ny - 1 (TLBM_BC_LID) */
} tlbm_batch_domain;

typedef struct tlbm_batch_desc {
  int32_t lattice;      /* TLBM_D2Q9 or TLBM_D3Q19 */
  int32_t dtype;        /* TLBM_F32 */
  int32_t collision;    /* TLBM_COLL_BGK or TLBM_COLL_MRT */
  int32_t ndomains;
  int32_t tile_x;       /* cells: a multiple of 32 * cells_per_thread */
  int32_t tile_y;       /* rows; (tile_x / cells_per_thread) * tile_y <= 256 threads */
  int32_t ctas_per_sm;  /* persistent mode: CTAs per SM (0 = occupancy limit) */
  int32_t cells_per_thread; /* 0 or 1: one cell per thread; 2: two cells of a
                             * row per thread (the pair update in domains of
                             * even nx), same results bit for bit */
  uint32_t* domain_status; /* device, ndomains words, or NULL.  When given, a
                            * domain's non-finite density sets its own word
                            * (bit 0) instead of the status word, and a domain
                            * whose word is non-zero is retired: later tiles
                            * and steps skip it, its state stays as it was. */
} tlbm_batch_desc;

/* One step of every domain, one launch (grid = tiles).  domains and tiles are
 * device arrays.  forces (may be NULL): ndomains x 3 doubles, accumulated
 * (zero before the step).  force_slot (device int, may be NULL): when given,
 * the forces go to forces + 3 * ndomains * (*force_slot), so that a captured
 * CUDA graph can record into a history whose slot tlbm_batch_advance_slot
 * moves on.  status bit 0: non-finite density. */
TLBM_API int tlbm_batch_step(const tlbm_batch_desc* b, const tlbm_batch_domain* domains, const int32_t* tiles,
                             int64_t ntiles, const void* f_in, void* f_out, const uint8_t* flags, double* forces,
                             const int32_t* force_slot, unsigned int* status, void* stream);

/* *slot += 1 on the stream (one thread).  No reference counterpart. */
TLBM_API int tlbm_batch_advance_slot(int32_t* slot, void* stream);

/* nsteps steps in one persistent cooperative launch; the state ping-pongs
 * f_a -> f_b -> f_a ..., so it ends in f_a when nsteps is even.  Step s with
 * s % record_every == 0 accumulates its forces into
 * force_history[(s / record_every) * ndomains * 3 ...] (zeroed by the caller).
 * sync: 3 device words, zero before the first call (and after a timeout).
 * The grid barrier between steps gives up after max_spins polls: status gets
 * bit 1 and every CTA returns (no hang). */
TLBM_API int tlbm_batch_run(const tlbm_batch_desc* b, const tlbm_batch_domain* domains, const int32_t* tiles,
                            int64_t ntiles, void* f_a, void* f_b, const uint8_t* flags, int32_t nsteps,
                            double* force_history, int32_t record_every, unsigned int* sync, unsigned int* status,
                            int64_t max_spins, void* stream);

/* ---- learned LES closure (D3Q19) ---------------------------------------------
 * TensorLBM's closure is 2-D (ai/model.py:40-92 EddyViscosityMLP, 3 strain
 * inputs -> 2x16 tanh -> softplus nu_t; ai/inference.py:68-92
 * collide_ai_les_bgk, tau + 3 nu_t; ai/train.py:310 Adam/MSE).  These entry
 * points are its 3-D replacement: 9 invariants of Pi_neq -> 3 x 64 SiLU ->
 * nu_t = nu_scale softplus(y); tau_eff = tau0 + 3 nu_t, Smagorinsky tau_s
 * (turbulence.py:183-208) outside the training range of any feature.
 *
 * Training vector theta (float32, tlbm_mlp_param_count() entries):
 * W1 (64x9, row = output), b1, W2 (64x64), b2, W3, b3, w4 (64), b4.
 * Features are normalised as (x - mean) * istd before the first layer. */

/* Block means over factor^3 cells of rho, u, u_iu_j from D3Q19 float32
 * populations (Q, nz, ny, nx); out: (10, nz/f, ny/f, nx/f) float32 in the order
 * rho, ux, uy, uz, uxux, uyuy, uzuz, uxuy, uxuz, uyuz.  u includes half the
 * linear force, m / rho (1 + A/2).  Extends ai/pipeline.py:93 (_coarsen_mean)
 * to 3-D and to the velocity products. */
TLBM_API int tlbm_les_filter_moments(const float* f, int32_t nx, int32_t ny, int32_t nz, int32_t factor,
                                     double a_lin, float* out, void* stream);

/* Training samples of one filtered field (nx, ny, nz are the filtered sizes):
 * features (N, 9) of Pi = -(2/3) rho tau_eff S (S by periodic central
 * differences; tau_eff = tau0 + 3 nu_hat if nu_hat != NULL, else the
 * Smagorinsky tau of c_s), target nu* = -(tau_sgs_dev : S) / (2 S:S),
 * weight S:S.  No reference counterpart. */
TLBM_API int tlbm_les_samples(const float* moments, int32_t nx, int32_t ny, int32_t nz, double tau0, double c_s,
                              const float* nu_hat, float* features, float* target, float* weight, void* stream);

TLBM_API int32_t tlbm_mlp_param_count(void);
TLBM_API int32_t tlbm_mlp_blob_bytes(void);
/* number of gradient partial blocks (rows of N_PARAMS + 1 floats) for a batch */
TLBM_API int64_t tlbm_mlp_grad_blocks(int64_t batch);

/* Gradient of L = sum_s w_s (softplus(y_s) - t_s)^2 / count over the rows
 * idx[0..count) (idx NULL: rows 0..count-1) of x (.., 9), t, w (w NULL: 1).
 * Writes per-block partial gradients and block losses to
 * partial[tlbm_mlp_grad_blocks(count)][N_PARAMS + 1].  Replaces the autograd
 * backward of ai/train.py:310 (train_eddy_viscosity_model). */
TLBM_API int tlbm_mlp_grad(const float* theta, const float* mean, const float* istd, const float* x,
                           const float* target, const float* weight, const int64_t* idx, int64_t count,
                           float* partial, void* stream);

/* Sum the partials in block order; Adam step number `step` (from 1) on theta
 * with moments m, v (lr = 0: no update).  grad_out (N_PARAMS) and loss_out
 * (1 float) may be NULL. */
TLBM_API int tlbm_mlp_adam(float* theta, float* m, float* v, const float* partial, int64_t nblocks, double lr,
                           double beta1, double beta2, double eps, int64_t step, float* grad_out, float* loss_out,
                           void* stream);

/* float32 forward: y (count) of raw features x (count, 9). */
TLBM_API int tlbm_mlp_eval(const float* theta, const float* mean, const float* istd, const float* x, int64_t count,
                           float* y, void* stream);

/* Pack theta, the feature statistics (mean, std) and the training range
 * (lo, hi) into the inference blob (tlbm_mlp_blob_bytes(), 16-byte aligned):
 * bf16 weight tiles in the tensor cores' 128-byte-swizzled K-major layout. */
TLBM_API int tlbm_mlp_pack(const float* theta, const float* mean, const float* std, const float* lo, const float* hi,
                           double nu_scale, void* blob, void* stream);

/* Tensor-core inference (tcgen05, bf16 weights and layer inputs, fp32
 * accumulation): y (count) of raw features x (count, 9).  status bit 2: a
 * bounded tensor-core wait expired. */
TLBM_API int tlbm_mlp_infer(const void* blob, const float* x, int64_t count, float* y, unsigned int* status,
                            void* stream);

/* One fused D3Q19 LES step on a periodic box (float32 populations, pull):
 * BGK with the learned tau_eff and exact-difference linear forcing
 * F = force_lin rho u.  tau_out (per cell), fallback_count (cells that used the
 * Smagorinsky tau of c_s) and status may be NULL.  nx ny nz + 1024 must stay
 * below 2^31 (32-bit cell offsets; else TLBM_ERR_TOO_LARGE).  Replaces
 * collide_ai_les_bgk (ai/inference.py:68-92) + stream for 3-D. */
TLBM_API int tlbm_les_step(int32_t nx, int32_t ny, int32_t nz, double tau0, double c_s, double force_lin,
                           const void* blob, const float* f_in, float* f_out, float* tau_out,
                           unsigned int* fallback_count, unsigned int* status, void* stream);

TLBM_API const char* tlbm_status_string(int status);
TLBM_API int tlbm_abi_version(void);
/* Kernel choice of the fused pull step: with enable != 0 the unforced D3Q19
 * BGK / MRT and D3Q27 cumulant steps on float32 or shifted half storage run
 * the row-staged kernel (bulk asynchronous copies of whole x-rows into
 * shared memory) where the layout allows it (nx a multiple of 64 up to 512,
 * 16-byte aligned buffers); enable == 0 (the default) keeps them on the
 * two-cells-per-thread kernel, which measured faster on B200.  Both give the
 * same results bit for bit.  Returns the previous setting; process-wide.  No
 * reference counterpart (a tuning switch of this library's kernels). */
TLBM_API int tlbm_set_row_staging(int32_t enable);
/* sizeof of the structs a binding mirrors: 0 tlbm_desc, 1 tlbm_batch_domain,
 * 2 tlbm_batch_desc (-1 otherwise), so that a binding can check its layout.
 * No reference counterpart. */
TLBM_API int64_t tlbm_struct_size(int32_t which);

/* ---- AA pattern: the step in place, one population buffer -------------------
 * Between steps the buffer holds one of three layouts: TLBM_AA_LOADED (slot q
 * of x holds S_0 as loaded), TLBM_AA_SWAPPED (slot opp(q) of x holds x's
 * post-collision population q) or TLBM_AA_NATURAL (slot q of x holds what
 * streamed into x, not yet bounded).  tlbm_step_aa advances one step in place
 * (loaded -> swapped -> natural -> swapped ...) with the boundaries,
 * collision, forcing and status of tlbm_step.  The pipeline runs one collision
 * behind the two-buffer step (one buffer cannot keep P_{n-1}): the first
 * launch collides S_0 without boundaries (the two-buffer load pass), launch n
 * >= 2 is the regular step, and tlbm_aa_populations after n launches returns
 * S_n, equal to the two-buffer field bit for bit (float32).  Launch n samples
 * the obstacle force of step n - 1; the readout samples step n.
 * Not supported here: Bouzidi links, moving walls (TLBM_ERR_UNSUPPORTED).
 * dtype F32, F16_SHIFTED, BF16_SHIFTED; collisions BGK, MRT, TRT, Smagorinsky,
 * cumulant (D3Q27), cascaded.
 * Replaces the second buffer of the two-buffer step (half the memory: D3Q19
 * float32 fits about 2.3 G cells in 180 GB instead of 1.2 G). */
typedef enum tlbm_aa_layout { TLBM_AA_SWAPPED = 0, TLBM_AA_NATURAL = 1, TLBM_AA_LOADED = 2 } tlbm_aa_layout;

/* f0: the TensorLBM-phase populations in the compute type (float32); f: the
 * AA buffer in d->dtype (f0 == f allowed for float32).  Writes the loaded
 * layout. */
TLBM_API int tlbm_aa_load(const tlbm_desc* d, const void* f0, void* f, const uint8_t* flags, const float* tau_field,
                          void* stream);
/* One step in place from the given layout; the buffer then holds the other. */
TLBM_API int tlbm_step_aa(const tlbm_desc* d, void* f, int32_t layout, const uint8_t* flags, const float* tau_field,
                          double* force, unsigned int* status, void* stream);
/* The TensorLBM-phase populations (boundaries applied, float32) of an AA
 * buffer in the given layout, into out (out != f); force (may be NULL) gets
 * the obstacle force sample of that state added. */
TLBM_API int tlbm_aa_populations(const tlbm_desc* d, const void* f, int32_t layout, const uint8_t* flags,
                                 void* out, double* force, void* stream);

/* ---- curved walls (Bouzidi / BFL interpolated bounce-back) -------------------
 * tlbm_sphere_links: the boundary links of a sphere and their wall fractions,
 * the outputs of compute_q_sphere_common (bfl_common.py:384) / compute_q_sphere_27
 * (interpolated_bc_common.py:136): link_mask (Q, nz, ny, nx) bytes (1 = link
 * (x, d): x outside, x + c_d inside, float64 squared distances against r^2) and
 * q_field (Q, nz, ny, nx) float32 (ray-sphere fraction along c_d in float64,
 * clamped to [1e-6, 1]; 0.5 off the links).  solid (nz, ny, nx, may be NULL)
 * receives the cells inside the sphere by the same test.  D3Q19 / D3Q27. */
TLBM_API int tlbm_sphere_links(int32_t lattice, int32_t nx, int32_t ny, int32_t nz, double cx, double cy, double cz,
                               double radius, uint8_t* link_mask, float* q_field, uint8_t* solid, void* stream);

/* tlbm_bfl_bounce_back: the link update of bfl_bounce_back_common (bfl_common.py:106)
 * on whole fields: f_out = f except f_out[opp_d](x) = BFL value of link (x, d),
 * from the post-stream f and the pre-stream f_prev (d->lattice D3Q19 / D3Q27,
 * d->dtype F32 / F64, d->nx/ny/nz).  force (may be NULL) receives, added in
 * float64, sum over links of c_d (f_prev_d + value) (bfl_d3q19.py:339-377).
 * Replaces: bfl_bounce_back_common, bouzidi_bounce_back_d3q19 (stationary wall). */
TLBM_API int tlbm_bfl_bounce_back(const tlbm_desc* d, const void* f, const void* f_prev, const uint8_t* link_mask,
                                  const float* q_field, void* f_out, double* force, void* stream);

/* ---- link-wise momentum exchange (MEM drag variants) -----------------------
 * tlbm_link_momentum_sums: for every cell x with near[x] != 0 and every
 * direction q >= 1 whose periodic neighbour x + c_q has solid != 0,
 *   sums[q]     += (f_q(x) + f_opp(q)(x + c_q)) * w   (in d->dtype, summed in float64)
 *   sums[Q + q] += 1
 * with w = 1 when q_wall is NULL, else w = 1 / max(q_wall, 1e-6) in float32,
 * q_wall (nz, ny, nx) or, with q_wall_per_direction != 0, (Q, nz, ny, nx).
 * sums (2Q float64) is zeroed first.  f is (Q, nz, ny, nx), post-streaming;
 * d->lattice, d->dtype (F32 / F64) and d->nx/ny/nz are read.  The forces of
 * momentum_exchange_standard (momentum_exchange.py:75), _galilean (:138),
 * _background_subtracted (:206) and _bfl (:285) are sum_q c_q times sums[q]
 * (times 1 + 1/(2 tau); minus the background per link times sums[Q + q]). */
TLBM_API int tlbm_link_momentum_sums(const tlbm_desc* d, const void* f, const uint8_t* solid, const uint8_t* near,
                                     const float* q_wall, int32_t q_wall_per_direction, double* sums, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TLBM_H */
