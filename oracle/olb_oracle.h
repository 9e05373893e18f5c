/* CPU oracle for OpenLB's collide-and-stream — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's per-cell collision templates and of
 * its periodic-shift (PS) streaming, operating on the reference's LOGICAL
 * layout: shifted populations f_i - w_i, structure of arrays pops[i*n + cell],
 * cell = (x*ny + y)*nz + z (z fastest), core cells only.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker.  The product (openlb_b200) never
 * links or calls it.
 *
 * Parity pin: every arithmetic expression follows the generic (non-CSE)
 * template it cites, operand by operand and with the same C++ type promotions,
 * so that built with -ffp-contract=off it reproduces OpenLB's CPU_SISD build
 * with -DDISABLE_CSE bit for bit (checked against golden fixtures made by the
 * compiled reference in tests/golden/).  Against the default (CSE) reference
 * build it agrees to rounding.
 */
#ifndef OLB_ORACLE_H
#define OLB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* dynamics kinds (one per reference dynamics alias) */
enum {
  ORACLE_NONE = 0,                 /* NoDynamics                dynamics/dynamics.h:51-62 */
  ORACLE_BGK = 1,                  /* BGKdynamics               dynamics/dynamics.h:89-98 */
  ORACLE_TRT = 2,                  /* TRTdynamics               dynamics/dynamics.h:445-451 */
  ORACLE_SMAGORINSKY = 3,          /* SmagorinskyBGKdynamics    dynamics/smagorinskyBGKdynamics.h:37-44 */
  ORACLE_BOUNCE_BACK = 4,          /* BounceBack                dynamics/dynamics.h:472-483 */
  ORACLE_BOUNCE_BACK_VELOCITY = 5, /* BounceBackVelocity        dynamics/dynamics.h:549-555 */
  ORACLE_FORCED_BGK = 6,           /* ForcedBGKdynamics         dynamics/dynamics.h:214 */
  ORACLE_FORCED_TRT = 7,           /* ForcedTRTdynamics         dynamics/dynamics.h:457-464 */
  /* flat-face interpolated boundaries: the mixin collision with exchanged
   * momenta, plus PlaneFdBoundaryProcessor3D after every stream */
  ORACLE_INTERP_VELOCITY = 8,      /* boundary::InterpolatedVelocity  boundary/interpolatedVelocity3D.h:44-50,78-81 */
  ORACLE_INTERP_PRESSURE = 9,      /* boundary::InterpolatedPressure  boundary/interpolatedPressure3D.h:47-90 */
  /* flat-face local velocity boundary: CombinedRLBdynamics<MIXIN,
   * RegularizedVelocityBoundaryTuple<direction,orientation>>, no post-processor */
  ORACLE_LOCAL_VELOCITY = 10,      /* boundary::LocalVelocity (Flat)  boundary/localVelocity3D.h:47-80 */
  /* external edges and corners of velocity boundaries (local and
   * interpolated): MIXIN::exchange_momenta<FixedVelocityBoundaryTuple> plus
   * OuterVelocityEdgeProcessor3D (priority 0) / OuterVelocityCornerProcessor3D
   * (priority 1) after every stream; normal[] is the discrete normal */
  ORACLE_VELOCITY_EDGE = 11,       /* boundary/localVelocity3D.h:90-93,113-114; interpolatedVelocity3D.h:62-63,85-87 */
  ORACLE_VELOCITY_CORNER = 12,     /* boundary/localVelocity3D.h:82-85,111-112; interpolatedVelocity3D.h:54-55,81-83 */
  /* internal edges and corners of velocity boundaries (local and
   * interpolated): CombinedRLBdynamics<MIXIN, InnerEdgeVelocityTuple3D<plane,n1,n2>
   * / InnerCornerVelocityTuple3D<nx,ny,nz>> (momenta/aliases.h:203-217), no
   * post-processor; normal[] is the discrete normal */
  ORACLE_VELOCITY_INNER_EDGE = 13,   /* boundary/localVelocity3D.h:98-101; interpolatedVelocity3D.h:64-67 */
  ORACLE_VELOCITY_INNER_CORNER = 14, /* boundary/localVelocity3D.h:88-91; interpolatedVelocity3D.h:56-59 */
  /* flat-face local pressure boundary: CombinedRLBdynamics<MIXIN,
   * RegularizedPressureBoundaryTuple<direction,orientation>> (momenta/aliases.h:136-141),
   * no post-processor */
  ORACLE_LOCAL_PRESSURE = 15         /* boundary::LocalPressure (Flat)  boundary/localPressure3D.h:47-57 */
};

typedef struct {
  int32_t kind;
  int32_t mixin;       /* interpolated boundaries: collision of the mixin dynamics (BGK, TRT, SMAGORINSKY) */
  double omega;        /* OMEGA */
  double magic;        /* collision::TRT::MAGIC */
  double smagorinsky;  /* collision::LES::SMAGORINSKY */
  double force[3];     /* FORCE field value (Guo forcing) */
  double wall_u[3];    /* VELOCITY field of moving-wall bounce-back */
  double wall_rho;     /* FixedDensity RHO field (1 after initialize) */
  int32_t direction;   /* flat boundaries: axis of the outward normal */
  int32_t orientation; /* flat boundaries: its sign, -1 or +1 */
  int32_t normal[3];   /* edges and corners: the discrete normal (components -1, 0, +1) */
  int32_t reserved;
} oracle_dyn;

typedef struct {
  int32_t q;             /* 19 or 27 */
  int32_t nx, ny, nz;
  int32_t periodic[3];
  int32_t n_dyn;
  const uint8_t* dyn_id; /* per cell index into table, or NULL = all 0 */
  const oracle_dyn* table;
  /* boundary values of interpolated cells, [4][cells]: RHO (fixed density of
   * pressure cells), then the VELOCITY field x, y, z; NULL if none */
  const double* bc_values;
  /* the FORCE field per cell, [3][cells], read by the Guo-forced dynamics in
   * place of their entry's force (forcing::Guo, dynamics/forcing.h:53-69,
   * momenta::ForcedMomentum, momenta/elements.h:1480-1488); NULL: the entry's */
  const double* force_field;
} oracle_lattice;

typedef struct {
  double sum_rho;       /* sum over cells whose collision reports statistics */
  double sum_usqr;
  double max_usqr;
  int64_t n_cells;
} oracle_stats;

/* One or more collideAndStream steps in place on the logical layout.
 * Populations streamed in from outside a non-periodic face get `ghost`
 * (NaN marks every slot whose value depends on OpenLB's unspecified padding).
 * stats may be NULL; if given it receives the statistics of the LAST step. */
int oracle_step_f32(const oracle_lattice* lat, float* pops, int steps, float ghost,
                    oracle_stats* stats);
int oracle_step_f64(const oracle_lattice* lat, double* pops, int steps, double ghost,
                    oracle_stats* stats);

/* The PostStream post-processors alone (PlaneFdBoundaryProcessor3D on every
 * interpolated cell, then the outer edge and corner processors), as
 * BlockLattice::initialize() runs them once on the initial state
 * (core/blockLattice.hh:56-67) before the first collision. */
int oracle_post_process_f32(const oracle_lattice* lat, float* pops);
int oracle_post_process_f64(const oracle_lattice* lat, double* pops);

/* Density / velocity as OpenLB's Density3D/Velocity3D functors report them
 * (per-dynamics momenta: bulk, forced, fixed density, wall velocity, none). */
int oracle_moments_f32(const oracle_lattice* lat, const float* pops, float* rho, float* u);
int oracle_moments_f64(const oracle_lattice* lat, const double* pops, double* rho, double* u);

/* Equilibrium populations (equilibrium::secondOrder, dynamics/lbm.h:50-64)
 * for per-cell rho/u, as Cell::iniEquilibrium writes them for bulk dynamics. */
int oracle_equilibrium_f32(int q, int64_t n, const float* rho, const float* u, float* pops);
int oracle_equilibrium_f64(int q, int64_t n, const double* rho, const double* u, double* pops);

/* descriptor tables (descriptor/definition/common.h:120-168, 313-366) */
int oracle_descriptor(int q, int32_t* c /* q*3 */, int32_t* opposite /* q */, double* w /* q */);

#ifdef __cplusplus
}
#endif

#endif
