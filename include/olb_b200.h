/* openlb_b200 — C ABI of the B200-native collide-and-stream step.
 *
 * This is the seam an OpenLB platform specialisation binds to.  In the
 * reference the same seam is the platform tag: `enum struct Platform`
 * (src/core/platform/platform.h:35-39), the dispatch switches
 * (src/core/platform/dispatch.h:40-132) and the per-platform specialisations
 * of ConcreteBlockLattice (src/core/blockLattice.h:458-701), its population
 * columns (src/core/platform/gpu/cuda/column.h:100-188) and collision
 * operators (src/core/platform/gpu/cuda/operator.h:47-126).  Each entry point
 * below names the reference interface it replaces.
 *
 * Conventions
 *   - Every call returns an olb_b200_status; OLB_B200_OK is 0.  The message of
 *     the last failure on the calling thread is olb_b200_last_error().  A C++
 *     host shim turns non-OK into std::runtime_error(olb_b200_last_error()),
 *     as OpenLB's gpu::cuda::device::check() does (gpu/cuda/device.hh:48-62).
 *   - Populations cross the ABI in OpenLB's LOGICAL layout: shifted values
 *     f_i - w_i (src/dynamics/lbm.h:57-63,267-275), structure of arrays
 *     pops[i*n + cell], cell = (x*ny + y)*nz + z over the core cells (z fastest,
 *     no overlap/padding; src/core/blockStructure.h:65-75,150), the state after
 *     the last stream.  The element type is the compute type: double for
 *     OLB_B200_STORAGE_F64, float otherwise.  How the library keeps them in
 *     device memory (AA pattern, 16-bit storage) is internal.
 *   - Host pointers are borrowed for the duration of the call.  Device
 *     memory, the CUDA stream and any CUDA graphs are owned by the handle.
 *   - One host thread drives one lattice handle; distinct handles may be used
 *     from distinct threads.  All device work of a handle is ordered on its
 *     own non-blocking stream.
 */
#ifndef OLB_B200_H
#define OLB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OLB_B200_ABI_VERSION 3

typedef struct olb_b200_lattice olb_b200_lattice;

typedef enum {
  OLB_B200_OK = 0,
  OLB_B200_ERR_CUDA = 1,        /* a CUDA runtime call failed */
  OLB_B200_ERR_OOM = 2,         /* device allocation failed */
  OLB_B200_ERR_ARG = 3,         /* invalid argument */
  OLB_B200_ERR_DIVERGED = 4,    /* non-finite density/velocity detected */
  OLB_B200_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
  OLB_B200_ERR_UNSUPPORTED = 6  /* valid request this build cannot serve */
} olb_b200_status;

typedef enum {
  OLB_B200_STORAGE_F32 = 0,     /* populations stored as float */
  OLB_B200_STORAGE_F64 = 1,     /* populations stored and collided in double */
  OLB_B200_STORAGE_F16 = 2,     /* (f_i - w_i)*2^k_i stored as IEEE half, FP32 math */
  OLB_B200_STORAGE_BF16 = 3     /* (f_i - w_i)*2^k_i stored as bfloat16, FP32 math */
} olb_b200_storage;

/* Dynamics kinds; one per reference alias. */
typedef enum {
  OLB_B200_DYN_NONE = 0,                 /* NoDynamics              src/dynamics/dynamics.h:51-62 */
  OLB_B200_DYN_BGK = 1,                  /* BGKdynamics             src/dynamics/dynamics.h:89-98 */
  OLB_B200_DYN_TRT = 2,                  /* TRTdynamics             src/dynamics/dynamics.h:445-451 */
  OLB_B200_DYN_SMAGORINSKY = 3,          /* SmagorinskyBGKdynamics  src/dynamics/smagorinskyBGKdynamics.h:37-44 */
  OLB_B200_DYN_BOUNCE_BACK = 4,          /* BounceBack              src/dynamics/dynamics.h:472-483 */
  OLB_B200_DYN_BOUNCE_BACK_VELOCITY = 5, /* BounceBackVelocity      src/dynamics/dynamics.h:549-555 */
  OLB_B200_DYN_FORCED_BGK = 6,           /* ForcedBGKdynamics       src/dynamics/dynamics.h:214 */
  OLB_B200_DYN_FORCED_TRT = 7,           /* ForcedTRTdynamics       src/dynamics/dynamics.h:457-464 */
  /* Interpolated boundaries on a flat face (discrete normal type Flat): the
   * mixin dynamics with exchanged momenta, plus PlaneFdBoundaryProcessor3D in
   * the PostStream stage (src/boundary/boundaryPostProcessors3D.hh:39-92). */
  OLB_B200_DYN_INTERPOLATED_VELOCITY = 8, /* boundary::InterpolatedVelocity  src/boundary/interpolatedVelocity3D.h:44-81 */
  OLB_B200_DYN_INTERPOLATED_PRESSURE = 9, /* boundary::InterpolatedPressure  src/boundary/interpolatedPressure3D.h:47-90 */
  /* Local velocity boundary on a flat face: CombinedRLBdynamics<MIXIN,
   * momenta::RegularizedVelocityBoundaryTuple<direction,orientation>>
   * (src/dynamics/dynamics.h:394-437), no post-processor. */
  OLB_B200_DYN_LOCAL_VELOCITY = 10,       /* boundary::LocalVelocity (flat)  src/boundary/localVelocity3D.h:47-80 */
  /* External edges and corners of velocity boundaries (local and
   * interpolated): MIXIN::exchange_momenta<momenta::FixedVelocityBoundaryTuple>
   * plus OuterVelocityEdgeProcessor3D / OuterVelocityCornerProcessor3D in the
   * PostStream stage (src/boundary/boundaryPostProcessors3D.hh:164-292);
   * `normal` holds the discrete normal. */
  OLB_B200_DYN_VELOCITY_EDGE = 11,        /* src/boundary/localVelocity3D.h:90-93,113-114 */
  OLB_B200_DYN_VELOCITY_CORNER = 12,      /* src/boundary/localVelocity3D.h:82-85,111-112 */
  /* Internal edges and corners of velocity boundaries (local and
   * interpolated): CombinedRLBdynamics<MIXIN, momenta::InnerEdgeVelocityTuple3D
   * / InnerCornerVelocityTuple3D> (src/dynamics/momenta/aliases.h:203-217), no
   * post-processor; `normal` holds the discrete normal; BGK or TRT mixin. */
  OLB_B200_DYN_VELOCITY_INNER_EDGE = 13,   /* src/boundary/localVelocity3D.h:98-101 */
  OLB_B200_DYN_VELOCITY_INNER_CORNER = 14, /* src/boundary/localVelocity3D.h:88-91 */
  /* Local pressure boundary on a flat face: CombinedRLBdynamics<MIXIN,
   * momenta::RegularizedPressureBoundaryTuple<direction,orientation>>
   * (src/dynamics/momenta/aliases.h:136-141), no post-processor; BGK or TRT
   * mixin.  The reference defines pressure boundaries on flat faces only
   * (src/boundary/localPressure3D.h:47-57, interpolatedPressure3D.h:47-75). */
  OLB_B200_DYN_LOCAL_PRESSURE = 15         /* boundary::LocalPressure (flat)  src/boundary/localPressure3D.h:47-57 */
} olb_b200_dyn_kind;

typedef struct {
  int32_t q;            /* 19 (D3Q19) or 27 (D3Q27) */
  int32_t nx, ny, nz;   /* core extent in cells */
  int32_t periodic[3];  /* CuboidDecomposition::setPeriodicity */
  int32_t storage;      /* olb_b200_storage */
  int32_t device;       /* CUDA device ordinal */
  int32_t reserved[3];  /* must be 0 */
} olb_b200_desc;

/* One entry of the per-cell dynamics table.  Parameters mirror the
 * reference's per-dynamics parameters and fields:
 *   omega        descriptors::OMEGA             (setParameter<OMEGA>)
 *   magic        collision::TRT::MAGIC          (src/dynamics/collision.h:210)
 *   smagorinsky  collision::LES::SMAGORINSKY    (src/dynamics/collisionLES.h:70)
 *   force        descriptors::FORCE field value (Guo forcing, forcing.h:38-74)
 *   wall_u       descriptors::VELOCITY field of BounceBackVelocity (defineU)
 *   wall_rho     FixedDensity RHO field (1 unless defineRho)
 * Boundary entries (interpolated, local velocity or pressure, edges, corners) also carry
 *   mixin        the MixinDynamics template argument of the boundary setter
 *                (BGK, TRT or SMAGORINSKY; must be the lattice's fluid
 *                collision; local faces, internal edges and corners take BGK or TRT)
 *   direction,   flat faces: the discrete normal as the boundary setter derives
 *   orientation  it (src/boundary/setBoundary3D.h:204-227): axis 0..2 and the
 *                sign of the outward normal, -1 or +1
 *   normal       edges and corners: the discrete normal (each component -1, 0
 *                or +1; two nonzero for an edge, three for a corner), as
 *                promiseForNormalSpecial maps it (setBoundary3D.h:586-627)
 * The boundary values of an entry's cells are stored over the bounding box of
 * those cells: keep each entry's cells in one plane (one line for an edge). */
typedef struct {
  int32_t kind;         /* olb_b200_dyn_kind */
  int32_t mixin;        /* olb_b200_dyn_kind of the mixin (interpolated boundaries), else 0 */
  double omega;
  double magic;
  double smagorinsky;
  double force[3];
  double wall_u[3];
  double wall_rho;
  int32_t direction;    /* flat boundaries: normal axis */
  int32_t orientation;  /* flat boundaries: normal sign */
  int32_t normal[3];    /* edges and corners: discrete normal */
  int32_t reserved;     /* must be 0 */
} olb_b200_dyn_params;

/* Statistics of one step as OpenLB's LatticeStatistics reports them
 * (src/core/latticeStatistics.h:49-71, SuperLattice::collectStatistics
 * src/core/superLattice.hh:61-106), reduced in FP64 on the device. */
typedef struct {
  double sum_rho;       /* over cells whose collision reports a statistic */
  double sum_usqr;
  double max_usqr;
  int64_t n_cells;
  double average_rho;   /* sum_rho / n_cells              (getAverageRho)    */
  double average_energy;/* 0.5 * sum_usqr / n_cells       (getAverageEnergy) */
  double max_u;         /* sqrt(max_usqr)                 (getMaxU)          */
  int64_t n_nonfinite;  /* cells with non-finite rho or |u|^2 */
} olb_b200_stats;

/* Lifecycle — replaces constructUsingConcretePlatform + ConcreteBlockLattice
 * ctor (src/core/platform/dispatch.h:106-132, src/core/blockLattice.hh:393-416).
 * Allocates the population columns; all cells start as NoDynamics with zero
 * (equilibrium at rest) populations. */
olb_b200_status olb_b200_create(const olb_b200_desc* desc, olb_b200_lattice** out);
void olb_b200_destroy(olb_b200_lattice* lattice);

/* Per-cell dynamics — replaces BlockDynamicsMap::set + the per-dynamics masks
 * and DynamicsPromise (src/core/blockDynamicsMap.h:72-171,266-278) and
 * setParameter (src/core/blockLattice.h:562-572).  ids[cell] indexes table;
 * ids == NULL assigns table[0] to every cell.  At most 256 entries; every
 * fluid entry must use the same collision kind (walls and NoDynamics may be
 * mixed in freely). */
olb_b200_status olb_b200_set_dynamics(olb_b200_lattice* lattice, const uint8_t* ids,
                                      const olb_b200_dyn_params* table, int32_t n_entries);

/* Boundary values of the velocity and pressure boundary cells — replaces defineRho /
 * defineU on their cells (src/core/cell.h:194-198; FixedDensity RHO of
 * pressure cells, the VELOCITY field of FixedVelocityMomentumGeneric /
 * FixedPressureMomentum).  values[4*j .. 4*j+3] = RHO, VELOCITY x, y, z of
 * cells[j] (logical cell index).  RHO is unused by velocity cells and the
 * normal VELOCITY component by pressure cells.  Until set, RHO = 1 and
 * VELOCITY = 0.  Synchronous. */
olb_b200_status olb_b200_set_boundary_values(olb_b200_lattice* lattice, const int64_t* cells, int64_t count,
                                             const double* values);

/* A FORCE value per cell for the Guo-forced dynamics (FORCED_BGK,
 * FORCED_TRT) in place of their entry's constant force — replaces OpenLB's
 * per-cell FORCE field (defineField<descriptors::FORCE>, cell.setField;
 * read by forcing::Guo, src/dynamics/forcing.h:53-69, and by the forced
 * momenta, src/dynamics/momenta/elements.h:1480-1488).  force holds 3 x cells
 * values of the ABI element type (double for OLB_B200_STORAGE_F64, float
 * otherwise), component-major (x of every cell, then y, then z), cells in the
 * populations' order.  Other dynamics ignore the field.  force == NULL removes
 * it (the entries' forces apply again).  The step then reads 3 more values per
 * cell.  Synchronous. */
olb_b200_status olb_b200_set_force_field(olb_b200_lattice* lattice, const void* force);

/* Per-step fluctuations of the interpolated velocity inlets — what an OpenLB
 * example does by calling defineU with a random field before every step.  No
 * counterpart in the reference's library.  Before step t (t = steps done so
 * far) every interpolated-velocity cell gets
 *   VELOCITY_d = U_d + amplitude * |U| * (2 r - 1),
 * U the values set by olb_b200_set_boundary_values and r the top 53 bits of
 * splitmix64(seed + (t * cells + cell) * 3 + d) over 2^53 (splitmix64 as in
 * Steele, Lea, Flood, OOPSLA 2014: x += 0x9E3779B97F4A7C15;
 * x = (x ^ x>>30) * 0xBF58476D1CE4E5B9; x = (x ^ x>>27) * 0x94D049BB133111EB;
 * x ^ x>>31).  amplitude 0 turns it off and restores U.  Synchronous. */
olb_b200_status olb_b200_set_boundary_noise(olb_b200_lattice* lattice, double amplitude, uint64_t seed);

/* SuperLattice::initialize (src/core/superLattice.hh:191-204,
 * src/core/blockLattice.hh:56-67): applies the PostStream post-processors
 * (the interpolated boundaries) once to the current state.  The first
 * collide_and_stream does it implicitly when it has not been done; later
 * calls do nothing.  Synchronous. */
olb_b200_status olb_b200_initialize(olb_b200_lattice* lattice);

/* Every cell's populations set to the second-order equilibrium of its density
 * and velocity — replaces SuperLattice::iniEquilibrium over the whole lattice
 * (src/core/superLattice.hh:542-577; Cell::iniEquilibrium with
 * equilibrium::secondOrder, src/dynamics/lbm.h:50-64), with the expansion done
 * on the device: 4 values per cell cross PCIe instead of q.  rho holds one
 * value per cell, u three columns (x of every cell, then y, then z), both of
 * the ABI element type, cells in the populations' order.  Synchronous. */
olb_b200_status olb_b200_ini_equilibrium(olb_b200_lattice* lattice, const void* rho, const void* u);

/* Full population state, host <-> device — replaces
 * setProcessingContext(Simulation/Evaluation) for POPULATION
 * (src/core/platform/gpu/cuda/column.hh:157-187,285-296).  Logical layout. */
olb_b200_status olb_b200_set_populations(olb_b200_lattice* lattice, const void* host_pops);
olb_b200_status olb_b200_get_populations(olb_b200_lattice* lattice, void* host_pops);

/* The hot path — replaces SuperLattice::collideAndStream
 * (src/core/superLattice.hh:601-663): collide (gpu/cuda/operator.hh:311-318)
 * fused with streaming (column.h:144-154, blockLattice.hh:317-339) in one
 * kernel per step, then the PostStream stage when the lattice has
 * interpolated boundary cells (two small kernels over those cells).  Runs
 * `steps` steps.  With stats == NULL the call only
 * enqueues work on the lattice's stream and returns; with stats != NULL the
 * last step also reduces the statistics, the call waits for them and returns
 * OLB_B200_ERR_DIVERGED if any cell was non-finite. */
olb_b200_status olb_b200_collide_and_stream(olb_b200_lattice* lattice, int32_t steps,
                                            olb_b200_stats* stats);

/* Density and velocity per cell as SuperLatticeDensity3D / Velocity3D report
 * them (src/functors/lattice/latticeVelocity3D.hh:65-71,
 * latticeDensity3D.hh:67), computed on the device: only 4 values per cell
 * cross PCIe instead of q.  rho: n values, u: 3*n values (component-major).
 * Element type as for populations. */
olb_b200_status olb_b200_get_moments(olb_b200_lattice* lattice, void* host_rho, void* host_u);

/* Waits for all work enqueued on the lattice. */
olb_b200_status olb_b200_synchronize(olb_b200_lattice* lattice);

/* Bounds the pipeline of olb_b200_collide_and_stream calls without
 * statistics: with calls = n > 0, a call first waits until the device work of
 * the call issued n calls earlier has finished, so at most n calls are
 * pending on the device when it returns; 0 (the default) leaves the queue
 * unbounded.  A host that times steps with a wall clock, as OpenLB's
 * util::Timer does (src/utilities/timer.hh:36-76), then measures device time
 * to within n steps, while the device is never left idle between steps.  The
 * reference's GPU platform instead synchronises the device three times per
 * step (src/core/superLattice.hh:669-671).  Waits for pending work first. */
olb_b200_status olb_b200_set_max_steps_in_flight(olb_b200_lattice* lattice, int32_t calls);

/* Device time of `steps` collide-and-stream steps, measured with CUDA events
 * on the lattice's stream (synchronous). */
olb_b200_status olb_b200_time_steps(olb_b200_lattice* lattice, int32_t steps, float* milliseconds);

/* Introspection: the lattice's cudaStream_t, the number of steps done, the
 * bytes of device memory the handle holds, and the launch shape in use. */
olb_b200_status olb_b200_get_stream(olb_b200_lattice* lattice, void** stream);
olb_b200_status olb_b200_get_info(olb_b200_lattice* lattice, int64_t* steps_done,
                                  int64_t* device_bytes, int32_t* block_z, int32_t* block_y);

/* Launch shape of the step kernel (threads along z and y, product <= 256,
 * block_z a multiple of 32).  0,0 selects the built-in default. */
olb_b200_status olb_b200_set_launch_shape(olb_b200_lattice* lattice, int32_t block_z, int32_t block_y);

/* Step-kernel tuning.  The library compiles a few variants of the step kernel
 * (cells per thread x register cap) that compute identical results and differ
 * only in speed; it picks a default per lattice class.  The reference has no
 * counterpart (its kernels launch 32-thread blocks, gpu/cuda/operator.hh:424-427). */
typedef struct {
  int32_t variant;            /* index of the step-kernel variant */
  int32_t cells_per_thread;
  int32_t min_blocks_per_sm;  /* register cap = 65536 / (256 * min_blocks_per_sm) */
  int32_t block_z, block_y;
  int32_t tuned;              /* 1 if chosen by olb_b200_autotune */
  int32_t candidates;         /* (variant, shape) pairs timed by the last autotune */
  float ms_per_step;          /* best time per step measured by autotune, else 0 */
} olb_b200_tuning;

/* Times every (variant, launch shape) pair on this lattice for trial_steps
 * steps each (0: 4) and keeps the fastest.  The lattice state is copied to a
 * temporary device buffer first and restored afterwards, so the simulation does
 * not advance.  Synchronous. */
olb_b200_status olb_b200_autotune(olb_b200_lattice* lattice, int32_t trial_steps, olb_b200_tuning* out);
olb_b200_status olb_b200_get_tuning(olb_b200_lattice* lattice, olb_b200_tuning* out);
/* Selects a variant explicitly (-1: the library's default for this lattice). */
olb_b200_status olb_b200_set_step_variant(olb_b200_lattice* lattice, int32_t variant);

/* Collide-and-stream on caller-owned device memory, allocating nothing.  This
 * entry point has no counterpart in the reference.
 *
 * It is for callers that cannot let a plug-in allocate device memory: a host
 * application that owns a fixed device-memory pool and forbids cudaMalloc /
 * cudaFree outside it, or a service that sizes its memory once at start-up and
 * must not allocate on the request path.  No lattice handle is involved (the
 * handle allocates); the caller owns the populations:
 *   desc         periodic must be {1,1,1}: every axis wraps (a lattice with
 *                walls needs a handle); reserved must be 0; nx <= 65535.
 *   device_pops  q columns of stride = round_up(nx*ny*nz, 64) elements of the
 *                storage type, in this library's in-place (AA) order: after an
 *                even number of steps it is the logical post-stream layout,
 *                after an odd number each f_i(x) sits in column opp(i) at
 *                x - c_i.  steps_done tells the call which of the two it is.
 *                One cell per element in every storage (the natural layout;
 *                a handle's paired 16-bit layout is not used here).  F32 and
 *                F64 hold f_i - w_i.  F16 and BF16 hold (f_i - w_i) * s_i
 *                rounded to the 16-bit type, s_i the power of two nearest
 *                1/w_i (s/sqrt2 < 1/w_i <= s*sqrt2): D3Q19 s = 4 (rest), 16
 *                (axis), 32 (diagonal); D3Q27 s = 4, 16, 64 (edge), 256
 *                (corner).
 *   bulk         one fluid dynamics applied to every cell (no walls).
 *   stats        NULL, or receives the last step's statistics (the call then
 *                waits for the stream).
 *   stream       a cudaStream_t, or NULL for the default stream.
 * The statistics reduction uses a fixed 2.5 MiB __device__ scratch array that
 * every GPU loading this library holds until exit.  With stats requested the
 * call needs ceil(nz/bz) * ceil(ny/by) * nx reduction blocks, (bz, by) =
 * (128, 2) if nz >= 128, (64, 4) if nz >= 64, else (32, 8); more than 65536
 * (e.g. any lattice above 256^3 cells) is rejected with OLB_B200_ERR_ARG.
 * The first call on each device looks up the scratch address and keeps it:
 * it should come before any stream capture, and the kept address is stale
 * after cudaDeviceReset on that device.  Calls whose device work overlaps
 * (two threads, two streams) race on the shared scratch: the caller
 * serialises them. */
olb_b200_status olb_b200_collide_and_stream_noalloc(const olb_b200_desc* desc, void* device_pops,
                                                    int64_t steps_done,
                                                    const olb_b200_dyn_params* bulk, int32_t steps,
                                                    olb_b200_stats* stats, void* stream);

/* Velocity-change residual ||u - u_prev||_2 / ||u||_2 over the fluid cells,
 * u_prev being the velocity at the previous call (0 before the first), as the
 * steady-state criterion of a converging solve; the velocity is kept on the
 * device.  The reference tracks convergence on the host with
 * util::ValueTracer over the average energy (src/utilities/benchmarkUtil.h:49-79);
 * this is the residual the ensemble server below uses as well.  Synchronous. */
olb_b200_status olb_b200_velocity_residual(olb_b200_lattice* lattice, double* residual);

/* ------------------------------------------------------------------------
 * Ensemble of independent lattices (the serving layer's device side).  No
 * counterpart in the reference, which runs one SuperLattice per program.
 * Instances of different sizes share one device pool and advance together in
 * one kernel launch per step over a flattened cell index; a chunk of steps is
 * a replayed CUDA graph.  Instances are admitted while slots and pool memory
 * last and leave when the host removes them.
 * ------------------------------------------------------------------------ */
typedef struct olb_b200_ensemble olb_b200_ensemble;

typedef enum {
  OLB_B200_ENSEMBLE_CAVITY = 1,   /* lid-driven cavity: bounce-back box, lid wall_u on y = ny-1,
                                     BGK fluid (cavity3dBenchmark geometry) */
  OLB_B200_ENSEMBLE_CHANNEL = 2,  /* x-periodic channel, bounce-back walls at y and z faces,
                                     Guo-forced BGK fluid with body force `force` */
  OLB_B200_ENSEMBLE_GEOMETRY = 3  /* the instance's own geometry table `cells`: one byte per
                                     cell (z fastest), 0 fluid, 1 bounce-back wall, 2 moving wall
                                     with velocity wall_u; BGK fluid, Guo-forced BGK when `force`
                                     is nonzero; every axis wraps (a face is closed by wall cells) */
} olb_b200_instance_kind;

typedef struct {
  int32_t q;              /* 19 */
  int32_t storage;        /* OLB_B200_STORAGE_F32 */
  int32_t device;
  int32_t max_instances;  /* slots */
  uint64_t pool_bytes;    /* device memory for all instances (admission budget) */
} olb_b200_ensemble_desc;

typedef struct {
  int32_t kind;           /* olb_b200_instance_kind */
  int32_t nx, ny, nz;
  double omega;
  double wall_u[3];       /* lid velocity (cavity), moving-wall velocity (geometry) */
  double force[3];        /* body force (channel, geometry) */
  const uint8_t* cells;   /* OLB_B200_ENSEMBLE_GEOMETRY: nx*ny*nz cell classes, copied by
                             olb_b200_ensemble_add; NULL otherwise */
} olb_b200_instance_desc;

olb_b200_status olb_b200_ensemble_create(const olb_b200_ensemble_desc* desc, olb_b200_ensemble** out);
void olb_b200_ensemble_destroy(olb_b200_ensemble* ensemble);
/* Admits an instance at rest (rho = 1, u = 0); OLB_B200_ERR_OOM when no slot
 * or not enough pool memory is free (the caller queues the request). */
olb_b200_status olb_b200_ensemble_add(olb_b200_ensemble* ensemble, const olb_b200_instance_desc* desc,
                                      int32_t* slot);
olb_b200_status olb_b200_ensemble_remove(olb_b200_ensemble* ensemble, int32_t slot);
/* Advances every active instance by `steps` steps.  With check != 0 a pass
 * after the last step computes each instance's velocity-change residual
 * against the previous check (as olb_b200_velocity_residual does).
 * residual / steps_done (max_instances entries each, may be NULL) receive the
 * per-slot values.  Synchronous. */
olb_b200_status olb_b200_ensemble_run(olb_b200_ensemble* ensemble, int32_t steps, int32_t check,
                                      double* residual, uint32_t* steps_done);
/* Density / velocity of one instance (n and 3n floats, z fastest). */
olb_b200_status olb_b200_ensemble_get_moments(olb_b200_ensemble* ensemble, int32_t slot, float* rho, float* u);
olb_b200_status olb_b200_ensemble_info(olb_b200_ensemble* ensemble, int64_t* pool_free_bytes,
                                       int32_t* active, int32_t* tiles);
/* Resident blocks per SM of the batched kernel (2, 3 or 4); the grid is that
 * many blocks per SM. */
olb_b200_status olb_b200_ensemble_set_occupancy(olb_b200_ensemble* ensemble, int32_t blocks_per_sm);
/* Pool bytes one instance of this extent occupies (a geometry instance adds
 * its table: the cell count rounded up to 256 bytes). */
uint64_t olb_b200_ensemble_bytes_per_instance(int32_t nx, int32_t ny, int32_t nz);

/* Thread-local message of the last failed call on this thread ("" if none). */
const char* olb_b200_last_error(void);

/* ABI version and a build description (compiler, architecture, flags). */
int32_t olb_b200_abi_version(void);
const char* olb_b200_build_info(void);

#ifdef __cplusplus
}
#endif

#endif /* OLB_B200_H */
