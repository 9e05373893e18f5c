// Host launchers of the step / gather / scatter / moments kernels.  Included
// by one translation unit per (lattice, storage) pair, which instantiates
// them explicitly (see OLB_B200_INSTANTIATE) so the kernel variants compile
// in parallel.
#pragma once

#include <type_traits>

#include "aa_kernels.cuh"

namespace olb_b200 {

template <int Q, class S, class R, int KIND, int CPT, int MINB>
static cudaError_t launch_step_variant(const StepLaunch& a, bool odd, bool masked, bool stats)
{
  const dim3 block(a.block_z, a.block_y);
  const dim3 grid = step_grid(a.g, a.block_z, a.block_y, CPT);
  S* pops = static_cast<S*>(a.pops);
  const DynDevice<R>* table = static_cast<const DynDevice<R>*>(a.table);
  const DynDevice<R>& bulk = *static_cast<const DynDevice<R>*>(a.bulk);
  constexpr bool kHalf = std::is_same_v<S, __half> || std::is_same_v<S, __nv_bfloat16>;
  if (masked) {
#define OLB_LAUNCH(O, ST)                                                                          \
  do {                                                                                             \
    if constexpr (kHalf) {                                                                         \
      if (a.g.paired) {                                                                            \
        aa_step_masked_paired_kernel<Q, S, KIND, O, ST, CPT, MINB><<<grid, block, 0, a.stream>>>(  \
          pops, a.g, a.ids, table, bulk, a.partials);                                              \
        break;                                                                                     \
      }                                                                                            \
    }                                                                                              \
    aa_step_masked_kernel<Q, S, R, KIND, O, ST, CPT, MINB><<<grid, block, 0, a.stream>>>(          \
      pops, a.g, a.ids, table, bulk, a.partials);                                                  \
  } while (0)
    if (odd) {
      if (stats) OLB_LAUNCH(true, true); else OLB_LAUNCH(true, false);
    } else {
      if (stats) OLB_LAUNCH(false, true); else OLB_LAUNCH(false, false);
    }
#undef OLB_LAUNCH
  } else {
#define OLB_LAUNCH(O, ST)                                                                          \
  do {                                                                                             \
    if constexpr (kHalf) {                                                                         \
      if (a.g.paired) {                                                                            \
        aa_step_paired_kernel<Q, S, KIND, O, ST, CPT, MINB><<<grid, block, 0, a.stream>>>(         \
          pops, a.g, bulk, a.partials);                                                            \
        break;                                                                                     \
      }                                                                                            \
    }                                                                                              \
    aa_step_kernel<Q, S, R, KIND, O, ST, CPT, MINB><<<grid, block, 0, a.stream>>>(pops, a.g, bulk, a.partials); \
  } while (0)
    if (odd) {
      if (stats) OLB_LAUNCH(true, true); else OLB_LAUNCH(true, false);
    } else {
      if (stats) OLB_LAUNCH(false, true); else OLB_LAUNCH(false, false);
    }
#undef OLB_LAUNCH
  }
  return cudaGetLastError();
}

template <int Q, class S, class R, int KIND>
static cudaError_t launch_step_kind(const StepLaunch& a, bool odd, bool masked, bool stats)
{
#define OLB_VARIANT(V)                                                                             \
  launch_step_variant<Q, S, R, KIND, kStepVariants[V].cells_per_thread, kStepVariants[V].min_blocks>( \
    a, odd, masked, stats)
  switch (a.variant) {
  case 0: return OLB_VARIANT(0);
  case 1: return OLB_VARIANT(1);
  case 2: return OLB_VARIANT(2);
  case 3: return OLB_VARIANT(3);
  default: return cudaErrorInvalidValue;
  }
#undef OLB_VARIANT
}

template <int Q, class S, class R>
cudaError_t launch_step(const StepLaunch& a, int kind, bool odd, bool masked, bool stats)
{
  switch (kind) {
  case K_BGK: return launch_step_kind<Q, S, R, K_BGK>(a, odd, masked, stats);
  case K_TRT: return launch_step_kind<Q, S, R, K_TRT>(a, odd, masked, stats);
  case K_SMAGORINSKY: return launch_step_kind<Q, S, R, K_SMAGORINSKY>(a, odd, masked, stats);
  case K_FORCED_BGK: return launch_step_kind<Q, S, R, K_FORCED_BGK>(a, odd, masked, stats);
  case K_FORCED_TRT: return launch_step_kind<Q, S, R, K_FORCED_TRT>(a, odd, masked, stats);
  default: return cudaErrorInvalidValue;
  }
}

template <int Q, class S, class R>
cudaError_t launch_gather(const void* pops, const Geometry& g, bool shifted, void* out, int i_begin,
                          int i_end, cudaStream_t stream)
{
  const dim3 block(32, 8);
  const dim3 grid = cell_grid(g, 32, 8);
  gather_logical_kernel<Q, S, R><<<grid, block, 0, stream>>>(static_cast<const S*>(pops), g, shifted,
                                                              static_cast<R*>(out), i_begin, i_end);
  return cudaGetLastError();
}

template <int Q, class S, class R>
cudaError_t launch_scatter(void* pops, const Geometry& g, const void* in, int i_begin, int i_end,
                           cudaStream_t stream)
{
  const dim3 block(32, 8);
  const dim3 grid = cell_grid(g, 32, 8);
  scatter_natural_kernel<Q, S, R><<<grid, block, 0, stream>>>(static_cast<S*>(pops), g,
                                                              static_cast<const R*>(in), i_begin, i_end);
  return cudaGetLastError();
}

template <int Q, class S, class R>
cudaError_t launch_equilibrium(void* pops, const Geometry& g, const void* rho_u, cudaStream_t stream)
{
  const dim3 block(32, 8);
  const dim3 grid = cell_grid(g, 32, 8);
  equilibrium_kernel<Q, S, R><<<grid, block, 0, stream>>>(static_cast<S*>(pops), g, static_cast<const R*>(rho_u));
  return cudaGetLastError();
}

template <int Q, class S, class R>
cudaError_t launch_moments(const void* pops, const Geometry& g, bool shifted, const uint8_t* ids,
                           const void* table, void* rho, void* u, cudaStream_t stream)
{
  const dim3 block(32, 8);
  const dim3 grid = cell_grid(g, 32, 8);
  moments_kernel<Q, S, R><<<grid, block, 0, stream>>>(static_cast<const S*>(pops), g, shifted, ids,
                                                       static_cast<const DynDevice<R>*>(table),
                                                       static_cast<R*>(rho), static_cast<R*>(u));
  return cudaGetLastError();
}

template <int Q, class S, class R>
cudaError_t launch_boundary_collide(void* pops, const Geometry& g, bool shifted, const uint8_t* ids,
                                    const void* table, int kind, const uint32_t* cells, uint32_t count,
                                    StatPartial* partials, cudaStream_t stream)
{
  if (count == 0) return cudaSuccess;
  const unsigned blocks = (count + kBoundaryThreads - 1) / kBoundaryThreads;
  S* p = static_cast<S*>(pops);
  const auto* t = static_cast<const DynDevice<R>*>(table);
#define OLB_BC_LAUNCH(K)                                                                             \
  do {                                                                                               \
    if (partials)                                                                                    \
      boundary_collide_kernel<Q, S, R, K, true><<<blocks, kBoundaryThreads, 0, stream>>>(            \
        p, g, shifted, ids, t, cells, count, partials);                                              \
    else                                                                                             \
      boundary_collide_kernel<Q, S, R, K, false><<<blocks, kBoundaryThreads, 0, stream>>>(           \
        p, g, shifted, ids, t, cells, count, partials);                                              \
  } while (0)
  switch (kind) {
  case K_TRT: OLB_BC_LAUNCH(K_TRT); break;
  case K_SMAGORINSKY: OLB_BC_LAUNCH(K_SMAGORINSKY); break;
  default: OLB_BC_LAUNCH(K_BGK); break;
  }
#undef OLB_BC_LAUNCH
  return cudaGetLastError();
}

template <int Q, class S, class R>
cudaError_t launch_boundary(void* pops, const Geometry& g, bool shifted, const uint8_t* ids, const void* table,
                            int periodic, const uint32_t* cells, uint32_t n_flat, uint32_t n_edge,
                            uint32_t n_corner, cudaStream_t stream)
{
  const int threads = 128;
  const auto* t = static_cast<const DynDevice<R>*>(table);
  cudaError_t e = cudaSuccess;
  if (n_flat) {
    const unsigned blocks = (n_flat + threads - 1) / threads;
    bc_velocity_kernel<Q, S, R><<<blocks, threads, 0, stream>>>(static_cast<const S*>(pops), g, shifted, ids, t,
                                                                cells, n_flat);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    plane_fd_kernel<Q, S, R><<<blocks, threads, 0, stream>>>(static_cast<S*>(pops), g, shifted, ids, t, periodic,
                                                             cells, n_flat);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (n_edge) {
    const unsigned blocks = (n_edge + threads - 1) / threads;
    outer_velocity_kernel<Q, S, R, false><<<blocks, threads, 0, stream>>>(
      static_cast<S*>(pops), g, shifted, ids, t, periodic, cells + n_flat, n_edge);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (n_corner) {
    const unsigned blocks = (n_corner + threads - 1) / threads;
    outer_velocity_kernel<Q, S, R, true><<<blocks, threads, 0, stream>>>(
      static_cast<S*>(pops), g, shifted, ids, t, periodic, cells + n_flat + n_edge, n_corner);
    e = cudaGetLastError();
  }
  return e;
}

} // namespace olb_b200

#define OLB_B200_INSTANTIATE(Q, S, R)                                                              \
  namespace olb_b200 {                                                                             \
  template cudaError_t launch_step<Q, S, R>(const StepLaunch&, int, bool, bool, bool);             \
  template cudaError_t launch_gather<Q, S, R>(const void*, const Geometry&, bool, void*, int, int, \
                                              cudaStream_t);                                       \
  template cudaError_t launch_scatter<Q, S, R>(void*, const Geometry&, const void*, int, int,      \
                                               cudaStream_t);                                      \
  template cudaError_t launch_equilibrium<Q, S, R>(void*, const Geometry&, const void*, cudaStream_t); \
  template cudaError_t launch_moments<Q, S, R>(const void*, const Geometry&, bool, const uint8_t*, \
                                               const void*, void*, void*, cudaStream_t);           \
  template cudaError_t launch_boundary_collide<Q, S, R>(void*, const Geometry&, bool, const uint8_t*, \
                                                        const void*, int, const uint32_t*, uint32_t, \
                                                        StatPartial*, cudaStream_t);               \
  template cudaError_t launch_boundary<Q, S, R>(void*, const Geometry&, bool, const uint8_t*,      \
                                                const void*, int, const uint32_t*, uint32_t,       \
                                                uint32_t, uint32_t, cudaStream_t);                 \
  }
