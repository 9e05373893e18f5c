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

}

}

}

#endif
