/* Platform::GPU_B200 — which OpenLB dynamics the device step implements.
 *
 * The second half of olb_b200_platform.h: it names dynamics aliases that
 * OpenLB declares after src/core/blockLattice.h (smagorinskyBGKdynamics.h,
 * the boundary dynamics), so patch_openlb.py includes it at the end of
 * src/olb3D.h when PLATFORM_GPU_B200 is defined.  Each specialisation of
 * gpu::b200::Describe maps one dynamics type to an entry of the device's
 * dynamics table (olb_b200_dyn_params): its kind, the operator-wide
 * parameters (OMEGA, MAGIC, SMAGORINSKY) and the per-cell fields the
 * reference reads (FORCE, the wall's VELOCITY and FixedDensity RHO).
 * Dynamics without a specialisation are rejected when a cell uses them.
 */
#ifndef OLB_B200_DYNAMICS_H
#define OLB_B200_DYNAMICS_H

#include "olb_b200_platform.h"

namespace olb {

namespace gpu {

namespace b200 {

// --- the dynamics the device implements (src/dynamics/dynamics.h) -----------

template <typename T, typename DESCRIPTOR>
struct Describe<T,DESCRIPTOR,NoDynamics<T,DESCRIPTOR>> {
  static constexpr int kind = OLB_B200_DYN_NONE;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS&, olb_b200_dyn_params&) { }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR>
struct Describe<T,DESCRIPTOR,BGKdynamics<T,DESCRIPTOR>> {
  static constexpr int kind = OLB_B200_DYN_BGK;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    p.omega = parameter<descriptors::OMEGA>(parameters);
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR>
struct Describe<T,DESCRIPTOR,TRTdynamics<T,DESCRIPTOR>> {
  static constexpr int kind = OLB_B200_DYN_TRT;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    p.omega = parameter<descriptors::OMEGA>(parameters);
    p.magic = parameter<collision::TRT::MAGIC>(parameters);
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR>
struct Describe<T,DESCRIPTOR,SmagorinskyBGKdynamics<T,DESCRIPTOR>> {
  static constexpr int kind = OLB_B200_DYN_SMAGORINSKY;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    p.omega = parameter<descriptors::OMEGA>(parameters);
    p.smagorinsky = parameter<collision::LES::SMAGORINSKY>(parameters);
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

/// Guo-forced BGK / TRT read the FORCE field per cell (src/dynamics/forcing.h:59-69)
template <typename T, typename DESCRIPTOR>
struct Describe<T,DESCRIPTOR,ForcedBGKdynamics<T,DESCRIPTOR>> {
  static constexpr int kind = OLB_B200_DYN_FORCED_BGK;
  static constexpr bool perCell = true;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    p.omega = parameter<descriptors::OMEGA>(parameters);
  }
  template <typename BLOCK>
  static void cell(BLOCK& block, CellID iCell, olb_b200_dyn_params& p)
  {
    const auto g = cellField<descriptors::FORCE>(block, iCell, 0.0);
    for (int iD = 0; iD < 3; ++iD) {
      p.force[iD] = g[iD];
    }
  }
};

template <typename T, typename DESCRIPTOR>
struct Describe<T,DESCRIPTOR,ForcedTRTdynamics<T,DESCRIPTOR>> {
  static constexpr int kind = OLB_B200_DYN_FORCED_TRT;
  static constexpr bool perCell = true;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    p.omega = parameter<descriptors::OMEGA>(parameters);
    p.magic = parameter<collision::TRT::MAGIC>(parameters);
  }
  template <typename BLOCK>
  static void cell(BLOCK& block, CellID iCell, olb_b200_dyn_params& p)
  {
    Describe<T,DESCRIPTOR,ForcedBGKdynamics<T,DESCRIPTOR>>::cell(block, iCell, p);
  }
};

/// Full-way bounce-back (src/dynamics/dynamics.h:472-483); its FixedDensity
/// RHO only enters the moments reported for the cell
template <typename T, typename DESCRIPTOR>
struct Describe<T,DESCRIPTOR,BounceBack<T,DESCRIPTOR>> {
  static constexpr int kind = OLB_B200_DYN_BOUNCE_BACK;
  static constexpr bool perCell = true;
  template <typename PARAMETERS>
  static void shared(PARAMETERS&, olb_b200_dyn_params&) { }
  template <typename BLOCK>
  static void cell(BLOCK& block, CellID iCell, olb_b200_dyn_params& p)
  {
    p.wall_rho = cellField<momenta::FixedDensity::RHO>(block, iCell, 1.0)[0];
  }
};

/// Moving-wall bounce-back (src/dynamics/dynamics.h:549-555): VELOCITY and
/// FixedDensity RHO per cell (NguyenLaddCorrection, collision.h:322-348)
template <typename T, typename DESCRIPTOR>
struct Describe<T,DESCRIPTOR,BounceBackVelocity<T,DESCRIPTOR>> {
  static constexpr int kind = OLB_B200_DYN_BOUNCE_BACK_VELOCITY;
  static constexpr bool perCell = true;
  template <typename PARAMETERS>
  static void shared(PARAMETERS&, olb_b200_dyn_params&) { }
  template <typename BLOCK>
  static void cell(BLOCK& block, CellID iCell, olb_b200_dyn_params& p)
  {
    p.wall_rho = cellField<momenta::FixedDensity::RHO>(block, iCell, 1.0)[0];
    const auto u = cellField<descriptors::VELOCITY>(block, iCell, 0.0);
    for (int iD = 0; iD < 3; ++iD) {
      p.wall_u[iD] = u[iD];
    }
  }
};

// --- boundaries (src/boundary/) ----------------------------------------------

/// The mixin collision of a boundary dynamics MIX::exchange_momenta<...>
template <typename COLLISION>
struct MixinKind {
  static constexpr int kind = -1;
};

template <>
struct MixinKind<collision::BGK> {
  static constexpr int kind = OLB_B200_DYN_BGK;
};

template <>
struct MixinKind<collision::TRT> {
  static constexpr int kind = OLB_B200_DYN_TRT;
};

template <>
struct MixinKind<collision::SmagorinskyEffectiveOmega<collision::BGK>> {
  static constexpr int kind = OLB_B200_DYN_SMAGORINSKY;
};

/// Operator-wide parameters of a boundary's mixin collision, read from the
/// parameters of the boundary dynamics (which are the mixin's)
template <typename PARAMETERS_LIST, typename PARAMETERS>
void mixinParameters(PARAMETERS& parameters, olb_b200_dyn_params& p)
{
  p.omega = parameter<descriptors::OMEGA>(parameters);
  if constexpr (PARAMETERS_LIST::template contains<collision::TRT::MAGIC>()) {
    p.magic = parameter<collision::TRT::MAGIC>(parameters);
  }
  if constexpr (PARAMETERS_LIST::template contains<collision::LES::SMAGORINSKY>()) {
    p.smagorinsky = parameter<collision::LES::SMAGORINSKY>(parameters);
  }
}

/// VELOCITY of FixedVelocityMomentumGeneric (what Cell::defineU sets on
/// velocity boundary cells, momenta/elements.h:528-560)
template <typename BLOCK>
void fixedVelocity(BLOCK& block, CellID iCell, double (&v)[4])
{
  const auto u = cellField<momenta::FixedVelocityMomentumGeneric::VELOCITY>(block, iCell, 0.0);
  v[0] = 1.0;
  v[1] = u[0];
  v[2] = u[1];
  v[3] = u[2];
}

/// boundary::LocalVelocity on a flat face (src/boundary/localVelocity3D.h:47-80):
/// CombinedRLBdynamics<MIX, RegularizedVelocityBoundaryTuple<d,o>>
template <typename T, typename DESCRIPTOR, typename MIX, int d, int o>
struct Describe<T,DESCRIPTOR,CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::RegularizedVelocityBoundaryTuple<d,o>>> {
  using DYN = CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::RegularizedVelocityBoundaryTuple<d,o>>;
  static constexpr int kind = Describe<T,DESCRIPTOR,MIX>::kind >= 0 ? OLB_B200_DYN_LOCAL_VELOCITY : -1;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    mixinParameters<typename DYN::parameters>(parameters, p);
    p.mixin = Describe<T,DESCRIPTOR,MIX>::kind;
    p.direction = d;
    p.orientation = o;
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR, typename MIX, int d, int o>
struct BoundaryValues<T,DESCRIPTOR,CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::RegularizedVelocityBoundaryTuple<d,o>>> {
  static constexpr bool valued = true;
  template <typename BLOCK>
  static void get(BLOCK& block, CellID iCell, double (&v)[4])
  {
    fixedVelocity(block, iCell, v);
  }
};

/// boundary::LocalPressure on a flat face (src/boundary/localPressure3D.h:47-57):
/// CombinedRLBdynamics<MIX, RegularizedPressureBoundaryTuple<d,o>>
template <typename T, typename DESCRIPTOR, typename MIX, int d, int o>
struct Describe<T,DESCRIPTOR,CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::RegularizedPressureBoundaryTuple<d,o>>> {
  using DYN = CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::RegularizedPressureBoundaryTuple<d,o>>;
  static constexpr int kind = Describe<T,DESCRIPTOR,MIX>::kind >= 0 ? OLB_B200_DYN_LOCAL_PRESSURE : -1;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    mixinParameters<typename DYN::parameters>(parameters, p);
    p.mixin = Describe<T,DESCRIPTOR,MIX>::kind;
    p.direction = d;
    p.orientation = o;
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR, typename MIX, int d, int o>
struct BoundaryValues<T,DESCRIPTOR,CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::RegularizedPressureBoundaryTuple<d,o>>> {
  static constexpr bool valued = true;
  template <typename BLOCK>
  static void get(BLOCK& block, CellID iCell, double (&v)[4])
  {
    // FixedDensity RHO and the tangential velocity of FixedPressureMomentum<d,o>
    v[0] = cellField<momenta::FixedDensity::RHO>(block, iCell, 1.0)[0];
    const auto u = cellField<typename momenta::FixedPressureMomentum<d,o>::VELOCITY>(block, iCell, 0.0);
    v[1] = u[0];
    v[2] = u[1];
    v[3] = u[2];
  }
};

/// Internal edge of a local or interpolated velocity boundary
/// (src/boundary/localVelocity3D.h:98-101, interpolatedVelocity3D.h:64-67):
/// CombinedRLBdynamics<MIX, InnerEdgeVelocityTuple3D<plane,n1,n2>>; the discrete
/// normal has n1 on axis (plane+1)%3 and n2 on axis (plane+2)%3
/// (src/boundary/setBoundary3D.h:156-197)
template <typename T, typename DESCRIPTOR, typename MIX, int plane, int n1, int n2>
struct Describe<T,DESCRIPTOR,CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::InnerEdgeVelocityTuple3D<plane,n1,n2>>> {
  using DYN = CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::InnerEdgeVelocityTuple3D<plane,n1,n2>>;
  static constexpr int kind = Describe<T,DESCRIPTOR,MIX>::kind >= 0 ? OLB_B200_DYN_VELOCITY_INNER_EDGE : -1;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    mixinParameters<typename DYN::parameters>(parameters, p);
    p.mixin = Describe<T,DESCRIPTOR,MIX>::kind;
    p.normal[plane] = 0;
    p.normal[(plane + 1) % 3] = n1;
    p.normal[(plane + 2) % 3] = n2;
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR, typename MIX, int plane, int n1, int n2>
struct BoundaryValues<T,DESCRIPTOR,CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::InnerEdgeVelocityTuple3D<plane,n1,n2>>> {
  static constexpr bool valued = true;
  template <typename BLOCK>
  static void get(BLOCK& block, CellID iCell, double (&v)[4])
  {
    fixedVelocity(block, iCell, v);
  }
};

/// Internal corner of a local or interpolated velocity boundary
/// (src/boundary/localVelocity3D.h:88-91, interpolatedVelocity3D.h:56-59):
/// CombinedRLBdynamics<MIX, InnerCornerVelocityTuple3D<nx,ny,nz>>
template <typename T, typename DESCRIPTOR, typename MIX, int nx, int ny, int nz>
struct Describe<T,DESCRIPTOR,CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::InnerCornerVelocityTuple3D<nx,ny,nz>>> {
  using DYN = CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::InnerCornerVelocityTuple3D<nx,ny,nz>>;
  static constexpr int kind = Describe<T,DESCRIPTOR,MIX>::kind >= 0 ? OLB_B200_DYN_VELOCITY_INNER_CORNER : -1;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    mixinParameters<typename DYN::parameters>(parameters, p);
    p.mixin = Describe<T,DESCRIPTOR,MIX>::kind;
    p.normal[0] = nx;
    p.normal[1] = ny;
    p.normal[2] = nz;
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR, typename MIX, int nx, int ny, int nz>
struct BoundaryValues<T,DESCRIPTOR,CombinedRLBdynamics<T,DESCRIPTOR,MIX,momenta::InnerCornerVelocityTuple3D<nx,ny,nz>>> {
  static constexpr bool valued = true;
  template <typename BLOCK>
  static void get(BLOCK& block, CellID iCell, double (&v)[4])
  {
    fixedVelocity(block, iCell, v);
  }
};

/// Interpolated velocity on a flat face (src/boundary/interpolatedVelocity3D.h:47-50):
/// MIX::exchange_momenta<BasicDirichletVelocityBoundaryTuple<d,o>>
template <typename T, typename DESCRIPTOR, typename EQ, typename COLL, typename COMB, int d, int o>
struct Describe<T,DESCRIPTOR,dynamics::Tuple<T,DESCRIPTOR,momenta::BasicDirichletVelocityBoundaryTuple<d,o>,EQ,COLL,COMB>> {
  using DYN = dynamics::Tuple<T,DESCRIPTOR,momenta::BasicDirichletVelocityBoundaryTuple<d,o>,EQ,COLL,COMB>;
  static constexpr int kind = MixinKind<COLL>::kind >= 0 ? OLB_B200_DYN_INTERPOLATED_VELOCITY : -1;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    mixinParameters<typename DYN::parameters>(parameters, p);
    p.mixin = MixinKind<COLL>::kind;
    p.direction = d;
    p.orientation = o;
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR, typename EQ, typename COLL, typename COMB, int d, int o>
struct BoundaryValues<T,DESCRIPTOR,dynamics::Tuple<T,DESCRIPTOR,momenta::BasicDirichletVelocityBoundaryTuple<d,o>,EQ,COLL,COMB>> {
  static constexpr bool valued = true;
  template <typename BLOCK>
  static void get(BLOCK& block, CellID iCell, double (&v)[4])
  {
    fixedVelocity(block, iCell, v);
  }
};

/// Interpolated pressure on a flat face (src/boundary/interpolatedPressure3D.h:47-90):
/// MIX::exchange_momenta<BasicDirichletPressureBoundaryTuple<d,o>>
template <typename T, typename DESCRIPTOR, typename EQ, typename COLL, typename COMB, int d, int o>
struct Describe<T,DESCRIPTOR,dynamics::Tuple<T,DESCRIPTOR,momenta::BasicDirichletPressureBoundaryTuple<d,o>,EQ,COLL,COMB>> {
  using DYN = dynamics::Tuple<T,DESCRIPTOR,momenta::BasicDirichletPressureBoundaryTuple<d,o>,EQ,COLL,COMB>;
  static constexpr int kind = MixinKind<COLL>::kind >= 0 ? OLB_B200_DYN_INTERPOLATED_PRESSURE : -1;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    mixinParameters<typename DYN::parameters>(parameters, p);
    p.mixin = MixinKind<COLL>::kind;
    p.direction = d;
    p.orientation = o;
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR, typename EQ, typename COLL, typename COMB, int d, int o>
struct BoundaryValues<T,DESCRIPTOR,dynamics::Tuple<T,DESCRIPTOR,momenta::BasicDirichletPressureBoundaryTuple<d,o>,EQ,COLL,COMB>> {
  static constexpr bool valued = true;
  template <typename BLOCK>
  static void get(BLOCK& block, CellID iCell, double (&v)[4])
  {
    // FixedDensity RHO and the tangential velocity of FixedPressureMomentum<d,o>
    v[0] = cellField<momenta::FixedDensity::RHO>(block, iCell, 1.0)[0];
    const auto u = cellField<typename momenta::FixedPressureMomentum<d,o>::VELOCITY>(block, iCell, 0.0);
    v[1] = u[0];
    v[2] = u[1];
    v[3] = u[2];
  }
};

/// External edges and corners of velocity boundaries (local and
/// interpolated): MIX::exchange_momenta<FixedVelocityBoundaryTuple>; which of
/// the two, and the normal, come from the cell's outer post-processor
template <typename T, typename DESCRIPTOR, typename EQ, typename COLL, typename COMB>
struct Describe<T,DESCRIPTOR,dynamics::Tuple<T,DESCRIPTOR,momenta::FixedVelocityBoundaryTuple,EQ,COLL,COMB>> {
  using DYN = dynamics::Tuple<T,DESCRIPTOR,momenta::FixedVelocityBoundaryTuple,EQ,COLL,COMB>;
  static constexpr int kind = MixinKind<COLL>::kind >= 0 ? kOuterPlaceholder : -1;
  static constexpr bool perCell = true;
  template <typename PARAMETERS>
  static void shared(PARAMETERS& parameters, olb_b200_dyn_params& p)
  {
    mixinParameters<typename DYN::parameters>(parameters, p);
    p.mixin = MixinKind<COLL>::kind;
  }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

template <typename T, typename DESCRIPTOR, typename EQ, typename COLL, typename COMB>
struct BoundaryValues<T,DESCRIPTOR,dynamics::Tuple<T,DESCRIPTOR,momenta::FixedVelocityBoundaryTuple,EQ,COLL,COMB>> {
  static constexpr bool valued = true;
  template <typename BLOCK>
  static void get(BLOCK& block, CellID iCell, double (&v)[4])
  {
    fixedVelocity(block, iCell, v);
  }
};

/// The boundaries' post-processors, performed by the device step
template <typename T, typename DESCRIPTOR, int d, int o>
struct RunsInDeviceStep<PlaneFdBoundaryProcessor3D<T,DESCRIPTOR,d,o>> : std::true_type { };

template <typename T, typename DESCRIPTOR, int plane, int n1, int n2>
struct RunsInDeviceStep<OuterVelocityEdgeProcessor3D<T,DESCRIPTOR,plane,n1,n2>> : std::true_type { };

template <typename T, typename DESCRIPTOR, int xN, int yN, int zN>
struct RunsInDeviceStep<OuterVelocityCornerProcessor3D<T,DESCRIPTOR,xN,yN,zN>> : std::true_type { };

/// OuterVelocityEdgeProcessor3D<plane,normal1,normal2>: normal1 along
/// (plane+1)%3, normal2 along (plane+2)%3 (src/boundary/setBoundary3D.h:586-627)
template <typename T, typename DESCRIPTOR, int plane, int n1, int n2>
struct OuterNormal<OuterVelocityEdgeProcessor3D<T,DESCRIPTOR,plane,n1,n2>> {
  static constexpr int kind = OLB_B200_DYN_VELOCITY_EDGE;
  static constexpr int normal[3] = {plane == 0 ? 0 : (plane == 1 ? n2 : n1),
                                    plane == 1 ? 0 : (plane == 2 ? n2 : n1),
                                    plane == 2 ? 0 : (plane == 0 ? n2 : n1)};
};

template <typename T, typename DESCRIPTOR, int xN, int yN, int zN>
struct OuterNormal<OuterVelocityCornerProcessor3D<T,DESCRIPTOR,xN,yN,zN>> {
  static constexpr int kind = OLB_B200_DYN_VELOCITY_CORNER;
  static constexpr int normal[3] = {xN, yN, zN};
};

}

}

}

#endif
