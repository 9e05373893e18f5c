// Batched collide-and-stream over many independent lattices (the serving
// layer's device side).
//
// All admitted instances live in one device pool.  Each instance owns a region
// holding its q population columns (AA layout, as a single lattice) and three
// columns with the velocity of its last convergence check.  One kernel launch
// advances every active instance by one step: one block per tile of a tile
// list, each tile being 256 x kTileCells consecutive cells of one instance's
// flattened cell index (z fastest).  Cell coordinates come from the
// flat index by multiply-shift division (Granlund & Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994) with per-instance
// constants, so instances of any size share the launch without idle lanes.
// An instance's geometry is its own table (one class byte per cell in its
// pool region: fluid, bounce-back wall, moving wall; read with the cell's
// populations) or procedural: a lid-driven cavity (bounce-back box, moving lid
// on the y = ny-1 face) or a channel (x periodic, bounce-back walls at the y
// and z faces, Guo body force along x).  Per-instance relaxation, lid velocity and
// force come from the instance table.  A chunk can end with the
// velocity-change residual of every instance (FP64 sums per tile, reduced per
// instance in a fixed order, so results do not depend on the mix), in a pass
// over the logical post-stream state after the chunk.
//
// The kernel arguments never change while instances come and go (the host
// rewrites the tables in device memory) and the step grid is the tile count
// rounded up by at most 25 %, so a chunk of steps is captured once as a CUDA
// graph and replayed until the load changes notably.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/olb_b200.h"
#include "aa_kernels.cuh"

namespace olb_b200 {
namespace detail {
void set_last_error(const std::string& message);
} // namespace detail
} // namespace olb_b200

using namespace olb_b200;

namespace {

constexpr int kQ = 19;
using L19 = Lattice<19>;
constexpr int kEnsembleThreads = 256;
constexpr int kTileCells = 1;  // cells per thread in a tile
constexpr int kTile = kEnsembleThreads * kTileCells;

// q = floor(n / d) for n < 2^31 by one multiply-high, an add and a shift
struct FastDiv {
  uint32_t m;
  uint32_t s;
  static FastDiv make(uint32_t d)
  {
    uint32_t s = 0;
    while ((uint64_t(1) << s) < d) ++s;
    const uint64_t m = ((uint64_t(1) << 32) * ((uint64_t(1) << s) - d)) / d + 1;
    return FastDiv{uint32_t(m), s};
  }
  OLB_HD uint32_t div(uint32_t n) const
  {
#ifdef __CUDA_ARCH__
    return (__umulhi(n, m) + n) >> s;
#else
    return uint32_t(((uint64_t(n) * m >> 32) + n) >> s);
#endif
  }
};

struct InstanceDevice {
  uint64_t pops;       // element offset of population column 0 in the pool
  uint64_t uprev;      // element offset of the stored velocity (3 columns)
  uint64_t geom;       // element offset of the cell-class bytes (geometry instances), 0: procedural
  uint32_t stride;     // column length in elements
  uint32_t cells;
  int32_t nx, ny, nz;
  uint32_t nz_u, nynz;
  FastDiv div_nynz, div_nz;
  int32_t kind;        // OLB_B200_ENSEMBLE_CAVITY / _CHANNEL / _GEOMETRY
  int32_t forced;      // fluid cells collide with Guo-forced BGK
  int32_t active;
  uint32_t steps_done; // steps completed before the current chunk
  float omega;
  float force[3];
  float force_relax;
  float lid_term[kQ][3];
  float lid_u[3];
};

struct Tile {
  uint32_t inst;
  uint32_t start;
};

struct ResidualPartial {
  double du2;
  double u2;
};

enum : int32_t { CELL_FLUID = 0, CELL_WALL = 1, CELL_LID = 2 };

// flat-index offset of lattice vector (CX, CY, CZ) in a box with ny*nz = nynz
// (modulo 2^32: negative components wrap, and n + offset is exact whenever the
// neighbour lies inside the box)
template <int CX, int CY, int CZ>
OLB_DEV uint32_t flat_offset(uint32_t nynz, uint32_t nz)
{
  return uint32_t(CX) * nynz + uint32_t(CY) * nz + uint32_t(CZ);
}

// the cell's class: the instance's geometry table, else its procedural geometry
OLB_DEV int cell_kind(const float* __restrict__ pool, const InstanceDevice& I, uint32_t n, int x, int y, int z)
{
  if (I.geom) {
    return int(__ldg(reinterpret_cast<const uint8_t*>(pool + I.geom) + n));
  }
  if (I.kind == OLB_B200_ENSEMBLE_CAVITY) {
    if (x == 0 || x == I.nx - 1 || y == 0 || z == 0 || z == I.nz - 1) return CELL_WALL;
    return y == I.ny - 1 ? CELL_LID : CELL_FLUID;
  }
  // channel: periodic in x
  if (y == 0 || y == I.ny - 1 || z == 0 || z == I.nz - 1) return CELL_WALL;
  return CELL_FLUID;
}

template <int MINB>
__global__ void __launch_bounds__(kEnsembleThreads, MINB)
ensemble_step_kernel(float* __restrict__ pool, const InstanceDevice* __restrict__ table,
                     const Tile* __restrict__ tiles, const int* __restrict__ ntiles_ptr, int k_in_chunk)
{
  using L = L19;
  const int ntiles = *ntiles_ptr;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tile = tiles[t];
    const InstanceDevice& I = table[tile.inst];
    if (!I.active) continue;
    const bool odd = ((I.steps_done + uint32_t(k_in_chunk)) & 1u) != 0u;
    // 32-bit element indices within the instance (ensemble_add keeps an
    // instance's columns below 2^32 elements)
    float* __restrict__ pops = pool + I.pops;
    const uint32_t stride = I.stride;
    const Geometry g{I.nx, I.ny, I.nz, stride, 0};
#pragma unroll 1
    for (int k = 0; k < kTileCells; ++k) {
      const uint32_t n = tile.start + threadIdx.x + uint32_t(k) * kEnsembleThreads;
      if (n >= I.cells) break;
      const uint32_t x = I.div_nynz.div(n);
      const uint32_t r = n - x * I.nynz;
      const uint32_t y = I.div_nz.div(r);
      const uint32_t z = r - y * I.nz_u;
      const int kind = cell_kind(pool, I, n, int(x), int(y), int(z));
      if (kind == CELL_WALL) continue;  // full-way bounce-back: AA no-op
      // Odd steps address neighbours.  A cell off every face of its box reaches
      // them without wrap-around: neighbour (x+cx, y+cy, z+cz) is the flat index
      // n + cx*ny*nz + cy*nz + cz, so each population's address is n plus a
      // per-instance constant.  Cells on a face (the lid row, the periodic x
      // ends of a channel) take the wrap-around offsets.
      const bool inner = (x - 1u < uint32_t(I.nx - 2)) && (y - 1u < uint32_t(I.ny - 2)) &&
                         (z - 1u < uint32_t(I.nz - 2));
      const uint32_t nynz = I.nynz, nzu = I.nz_u;
      float f[kQ];
      if (!odd) {
        static_for<0, kQ>([&](auto i) { f[i] = pops[uint32_t(i.value) * stride + n]; });
      } else if (inner) {
        static_for<0, kQ>([&](auto i) {
          constexpr int o = L::opp(i);
          f[i] = pops[n + (uint32_t(o) * stride +
                           flat_offset<-L::c(i, 0), -L::c(i, 1), -L::c(i, 2)>(nynz, nzu))];
        });
      } else {
        Neighbours nb(g, int(x), int(y), int(z));
        static_for<0, kQ>([&](auto i) {
          constexpr int o = L::opp(i);
          f[i] = pops[uint32_t(o) * stride + nb.template at<-L::c(i, 0), -L::c(i, 1), -L::c(i, 2)>()];
        });
      }
      if (kind == CELL_FLUID) {
        float rho, u[3];
        if (I.forced) {
          const float gg[3] = {I.force[0], I.force[1], I.force[2]};
          float delta;
          compute_rho_delta_u_forced<L>(f, gg, rho, delta, u);
          relax_bgk<L>(f, rho, delta, u, I.omega);
          add_force<L>(f, rho, u, I.force_relax, gg);
        } else {
          float delta;
          compute_rho_delta_u<L>(f, rho, delta, u);
          relax_bgk<L>(f, rho, delta, u, I.omega);
        }
      } else {
        // moving lid: collision::NguyenLaddCorrection<Revert>
        revert<L>(f);
        static_for<1, kQ>([&](auto i) {
          f[i] += I.lid_term[i][0];
          f[i] += I.lid_term[i][1];
          f[i] += I.lid_term[i][2];
        });
      }
      const uint32_t st = opaque(stride);
      if (!odd) {
        static_for<0, kQ>([&](auto i) {
          constexpr int o = L::opp(i);
          pops[uint32_t(o) * st + n] = f[i];
        });
      } else if (inner) {
        static_for<0, kQ>([&](auto i) {
          pops[n + (uint32_t(i.value) * st + flat_offset<L::c(i, 0), L::c(i, 1), L::c(i, 2)>(nynz, nzu))] = f[i];
        });
      } else {
        Neighbours nb(g, int(x), int(y), int(z));
        static_for<0, kQ>([&](auto i) {
          pops[uint32_t(i.value) * st + nb.template at<L::c(i, 0), L::c(i, 1), L::c(i, 2)>()] = f[i];
        });
      }
    }
  }
}

// Velocity-change residual after `steps_in_chunk` steps: the velocity of the
// logical post-stream state of every fluid cell against the stored one (then
// stored), summed per tile in FP64 with a fixed-order block reduction.  The
// same quantity as olb_b200_velocity_residual on a single lattice.
__global__ void __launch_bounds__(kEnsembleThreads)
ensemble_check_kernel(float* __restrict__ pool, const InstanceDevice* __restrict__ table,
                      const Tile* __restrict__ tiles, const int* __restrict__ ntiles_ptr, int steps_in_chunk,
                      ResidualPartial* __restrict__ partials)
{
  using L = L19;
  const int ntiles = *ntiles_ptr;
  __shared__ double sh[2][kEnsembleThreads / 32];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tile = tiles[t];
    const InstanceDevice& I = table[tile.inst];
    double du2 = 0., u2 = 0.;
    if (I.active) {
      const bool shifted = ((I.steps_done + uint32_t(steps_in_chunk)) & 1u) != 0u;
      const float* __restrict__ pops = pool + I.pops;
      float* __restrict__ up = pool + I.uprev;
      const Geometry g{I.nx, I.ny, I.nz, I.stride, 0};
      for (int k = 0; k < kTileCells; ++k) {
        const uint32_t n = tile.start + threadIdx.x + uint32_t(k) * kEnsembleThreads;
        if (n >= I.cells) break;
        const uint32_t x = I.div_nynz.div(n);
        const uint32_t r = n - x * I.nynz;
        const uint32_t y = I.div_nz.div(r);
        const uint32_t z = r - y * I.nz_u;
        if (cell_kind(pool, I, n, int(x), int(y), int(z)) != CELL_FLUID) continue;
        float f[kQ];
        static_for<0, kQ>([&](auto i) {
          f[i] = logical_pop<kQ, float, float, i.value>(pops, g, int(x), int(y), int(z), shifted);
        });
        float rho, u[3];
        if (I.forced) {
          const float gg[3] = {I.force[0], I.force[1], I.force[2]};
          compute_rho_u_forced<L>(f, gg, rho, u);
        } else {
          compute_rho_u<L>(f, rho, u);
        }
        for (int d = 0; d < 3; ++d) {
          const double du = double(u[d]) - double(up[size_t(d) * I.stride + n]);
          du2 += du * du;
          u2 += double(u[d]) * double(u[d]);
          up[size_t(d) * I.stride + n] = u[d];
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      du2 += __shfl_down_sync(0xffffffffu, du2, o);
      u2 += __shfl_down_sync(0xffffffffu, u2, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
      sh[0][warp] = du2;
      sh[1][warp] = u2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0., b = 0.;
      for (int w = 0; w < kEnsembleThreads / 32; ++w) {
        a += sh[0][w];
        b += sh[1][w];
      }
      partials[t] = ResidualPartial{a, b};
    }
    __syncthreads();
  }
}

// per instance: reduce its contiguous tile range in order; advance steps_done
__global__ void ensemble_finish_kernel(InstanceDevice* __restrict__ table, const int* __restrict__ tile_begin,
                                       const int* __restrict__ tile_end, const int* __restrict__ ninst_ptr,
                                       int steps, int check, const ResidualPartial* __restrict__ partials,
                                       double* __restrict__ residual_out, uint32_t* __restrict__ steps_out)
{
  const int ninst = *ninst_ptr;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ninst) return;
  InstanceDevice& I = table[s];
  if (!I.active) return;
  I.steps_done += uint32_t(steps);
  steps_out[s] = I.steps_done;
  if (check) {
    double a = 0., b = 0.;
    for (int t = tile_begin[s]; t < tile_end[s]; ++t) {
      a += partials[t].du2;
      b += partials[t].u2;
    }
    residual_out[s] = b > 0. ? sqrt(a / b) : (a > 0. ? INFINITY : 0.);
  }
}

// density / velocity of one instance (Density3D / Velocity3D semantics)
__global__ void ensemble_moments_kernel(const float* __restrict__ pool, InstanceDevice I, float* __restrict__ rho_out,
                                        float* __restrict__ u_out)
{
  using L = L19;
  const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= I.cells) return;
  const uint32_t x = I.div_nynz.div(n);
  const uint32_t r = n - x * I.nynz;
  const uint32_t y = I.div_nz.div(r);
  const uint32_t z = r - y * I.nz_u;
  const int kind = cell_kind(pool, I, n, int(x), int(y), int(z));
  float rho = 1.f, u[3] = {0.f, 0.f, 0.f};
  if (kind == CELL_LID) {
    u[0] = I.lid_u[0]; u[1] = I.lid_u[1]; u[2] = I.lid_u[2];
  } else if (kind == CELL_FLUID) {
    const bool shifted = (I.steps_done & 1u) != 0u;
    const Geometry g{I.nx, I.ny, I.nz, I.stride, 0};
    const float* pops = pool + I.pops;
    float f[kQ];
    static_for<0, kQ>([&](auto i) {
      f[i] = logical_pop<kQ, float, float, i.value>(pops, g, int(x), int(y), int(z), shifted);
    });
    if (I.forced) {
      const float gg[3] = {I.force[0], I.force[1], I.force[2]};
      compute_rho_u_forced<L>(f, gg, rho, u);
    } else {
      compute_rho_u<L>(f, rho, u);
    }
  }
  rho_out[n] = rho;
  u_out[n] = u[0];
  u_out[I.cells + n] = u[1];
  u_out[2 * size_t(I.cells) + n] = u[2];
}

struct Region {
  uint64_t offset;
  uint64_t size;
};

} // namespace

struct olb_b200_ensemble {
  int device = 0;
  int max_instances = 0;
  uint64_t pool_elems = 0;
  float* pool = nullptr;
  InstanceDevice* table_dev = nullptr;
  std::vector<InstanceDevice> table;          // host mirror
  std::vector<Region> regions;                 // per slot
  std::vector<char> used;                      // slot in use
  std::vector<Region> free_list;               // sorted by offset
  Tile* tiles_dev = nullptr;
  int max_tiles = 0;
  int* counts_dev = nullptr;                   // [0] ntiles, [1] ninst
  int* tile_begin_dev = nullptr;
  int* tile_end_dev = nullptr;
  ResidualPartial* partials = nullptr;
  double* residual_dev = nullptr;
  uint32_t* steps_dev = nullptr;
  double* residual_host = nullptr;             // pinned
  uint32_t* steps_host = nullptr;              // pinned
  float* moments_dev = nullptr;                // staging for get_moments
  size_t moments_cap = 0;
  bool dirty = true;                           // tables changed since upload
  int grid = 0;                                // persistent grid of the check kernel
  int step_grid = 0;                           // blocks of the step kernel: ntiles rounded up
  int min_blocks = 4;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  int graph_check = -1;
  int graph_minb = 0;
};

namespace {

olb_b200_status efail(olb_b200_status code, const std::string& msg)
{
  detail::set_last_error(msg);
  return code;
}

olb_b200_status ecuda(cudaError_t e, const char* what)
{
  return efail(e == cudaErrorMemoryAllocation ? OLB_B200_ERR_OOM : OLB_B200_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}

#define OLB_ECUDA(call)                                                                            \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return ecuda(e_, #call);                                                \
  } while (0)

uint64_t round_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

uint64_t instance_elems(uint64_t cells)
{
  const uint64_t stride = round_up(cells, 64);
  return stride * (kQ + 3);
}

bool pool_alloc(olb_b200_ensemble* E, uint64_t size, uint64_t& offset)
{
  for (size_t k = 0; k < E->free_list.size(); ++k) {
    Region& r = E->free_list[k];
    if (r.size >= size) {
      offset = r.offset;
      r.offset += size;
      r.size -= size;
      if (r.size == 0) E->free_list.erase(E->free_list.begin() + long(k));
      return true;
    }
  }
  return false;
}

void pool_free(olb_b200_ensemble* E, Region reg)
{
  auto it = std::lower_bound(E->free_list.begin(), E->free_list.end(), reg,
                             [](const Region& a, const Region& b) { return a.offset < b.offset; });
  it = E->free_list.insert(it, reg);
  size_t k = size_t(it - E->free_list.begin());
  if (k + 1 < E->free_list.size() && E->free_list[k].offset + E->free_list[k].size == E->free_list[k + 1].offset) {
    E->free_list[k].size += E->free_list[k + 1].size;
    E->free_list.erase(E->free_list.begin() + long(k + 1));
  }
  if (k > 0 && E->free_list[k - 1].offset + E->free_list[k - 1].size == E->free_list[k].offset) {
    E->free_list[k - 1].size += E->free_list[k].size;
    E->free_list.erase(E->free_list.begin() + long(k));
  }
}

// tile list of the active instances, in slot order; per-slot tile ranges
olb_b200_status upload_tables(olb_b200_ensemble* E)
{
  std::vector<Tile> tiles;
  std::vector<int> begin(E->max_instances, 0), end(E->max_instances, 0);
  for (int s = 0; s < E->max_instances; ++s) {
    begin[s] = int(tiles.size());
    if (E->used[s] && E->table[s].active) {
      for (uint32_t c = 0; c < E->table[s].cells; c += kTile) tiles.push_back(Tile{uint32_t(s), c});
    }
    end[s] = int(tiles.size());
  }
  if (int(tiles.size()) > E->max_tiles) {
    // the captured graph holds the old pointers
    if (E->graph) {
      cudaGraphExecDestroy(E->graph);
      E->graph = nullptr;
    }
    OLB_ECUDA(cudaStreamSynchronize(E->stream));
    if (E->tiles_dev) cudaFree(E->tiles_dev);
    if (E->partials) cudaFree(E->partials);
    E->tiles_dev = nullptr;
    E->partials = nullptr;
    E->max_tiles = 0;
    const int cap = int(tiles.size()) * 2 + 1024;
    OLB_ECUDA(cudaMalloc(&E->tiles_dev, size_t(cap) * sizeof(Tile)));
    OLB_ECUDA(cudaMalloc(&E->partials, size_t(cap) * sizeof(ResidualPartial)));
    E->max_tiles = cap;
  }
  // one block per tile, the grid rounded up (at most 25 %) so that it, and
  // with it the captured graph, only changes when the load changes notably;
  // blocks past the tile count return at once
  {
    const int n = std::max(1, int(tiles.size()));
    int p = 1;
    while (p * 2 <= n) p *= 2;
    const int quantum = std::max(1, p / 4);
    const int bucket = (n + quantum - 1) / quantum * quantum;
    if (bucket != E->step_grid) {
      if (E->graph) {
        OLB_ECUDA(cudaStreamSynchronize(E->stream));
        cudaGraphExecDestroy(E->graph);
        E->graph = nullptr;
      }
      E->step_grid = bucket;
    }
  }
  const int counts[2] = {int(tiles.size()), E->max_instances};
  if (!tiles.empty()) {
    OLB_ECUDA(cudaMemcpyAsync(E->tiles_dev, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice, E->stream));
  }
  OLB_ECUDA(cudaMemcpyAsync(E->counts_dev, counts, sizeof counts, cudaMemcpyHostToDevice, E->stream));
  OLB_ECUDA(cudaMemcpyAsync(E->tile_begin_dev, begin.data(), begin.size() * sizeof(int), cudaMemcpyHostToDevice, E->stream));
  OLB_ECUDA(cudaMemcpyAsync(E->tile_end_dev, end.data(), end.size() * sizeof(int), cudaMemcpyHostToDevice, E->stream));
  OLB_ECUDA(cudaMemcpyAsync(E->table_dev, E->table.data(), E->table.size() * sizeof(InstanceDevice),
                            cudaMemcpyHostToDevice, E->stream));
  // the staged host vectors die here: make the copies complete first
  OLB_ECUDA(cudaStreamSynchronize(E->stream));
  E->dirty = false;
  return OLB_B200_OK;
}

olb_b200_status enqueue_chunk(olb_b200_ensemble* E, int steps, int check)
{
  for (int k = 0; k < steps; ++k) {
    switch (E->min_blocks) {
    case 2:
      ensemble_step_kernel<2><<<E->step_grid, kEnsembleThreads, 0, E->stream>>>(
        E->pool, E->table_dev, E->tiles_dev, E->counts_dev, k);
      break;
    case 4:
      ensemble_step_kernel<4><<<E->step_grid, kEnsembleThreads, 0, E->stream>>>(
        E->pool, E->table_dev, E->tiles_dev, E->counts_dev, k);
      break;
    default:
      ensemble_step_kernel<3><<<E->step_grid, kEnsembleThreads, 0, E->stream>>>(
        E->pool, E->table_dev, E->tiles_dev, E->counts_dev, k);
      break;
    }
    OLB_ECUDA(cudaGetLastError());
  }
  if (check) {
    ensemble_check_kernel<<<E->grid, kEnsembleThreads, 0, E->stream>>>(E->pool, E->table_dev, E->tiles_dev,
                                                                       E->counts_dev, steps, E->partials);
    OLB_ECUDA(cudaGetLastError());
  }
  const int threads = 128;
  const int blocks = (E->max_instances + threads - 1) / threads;
  ensemble_finish_kernel<<<blocks, threads, 0, E->stream>>>(E->table_dev, E->tile_begin_dev, E->tile_end_dev,
                                                             E->counts_dev + 1, steps, check, E->partials,
                                                             E->residual_dev, E->steps_dev);
  OLB_ECUDA(cudaGetLastError());
  OLB_ECUDA(cudaMemcpyAsync(E->residual_host, E->residual_dev, size_t(E->max_instances) * sizeof(double),
                            cudaMemcpyDeviceToHost, E->stream));
  OLB_ECUDA(cudaMemcpyAsync(E->steps_host, E->steps_dev, size_t(E->max_instances) * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, E->stream));
  return OLB_B200_OK;
}

} // namespace

extern "C" {

olb_b200_status olb_b200_ensemble_create(const olb_b200_ensemble_desc* desc, olb_b200_ensemble** out)
{
  detail::set_last_error("");
  if (!desc || !out) return efail(OLB_B200_ERR_ARG, "ensemble_create: null argument");
  *out = nullptr;
  if (desc->q != 19 || desc->storage != OLB_B200_STORAGE_F32)
    return efail(OLB_B200_ERR_UNSUPPORTED, "ensemble_create: D3Q19 with FP32 storage only");
  if (desc->max_instances < 1 || desc->max_instances > 65536)
    return efail(OLB_B200_ERR_ARG, "ensemble_create: max_instances must be in [1, 65536]");
  if (desc->pool_bytes < (1u << 20)) return efail(OLB_B200_ERR_ARG, "ensemble_create: pool_bytes below 1 MiB");
  auto* E = new olb_b200_ensemble;
  E->device = desc->device;
  E->max_instances = desc->max_instances;
  E->pool_elems = uint64_t(desc->pool_bytes) / sizeof(float) / 64 * 64;
  E->table.assign(size_t(E->max_instances), InstanceDevice{});
  E->regions.assign(size_t(E->max_instances), Region{0, 0});
  E->used.assign(size_t(E->max_instances), 0);
  E->free_list.push_back(Region{0, E->pool_elems});
  auto cleanup = [&](olb_b200_status st) {
    olb_b200_ensemble_destroy(E);
    return st;
  };
#define OLB_ECUDA_C(call)                                                                          \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return cleanup(ecuda(e_, #call));                                       \
  } while (0)
  OLB_ECUDA_C(cudaSetDevice(E->device));
  OLB_ECUDA_C(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking));
  OLB_ECUDA_C(cudaMalloc(&E->pool, E->pool_elems * sizeof(float)));
  OLB_ECUDA_C(cudaMalloc(&E->table_dev, size_t(E->max_instances) * sizeof(InstanceDevice)));
  OLB_ECUDA_C(cudaMalloc(&E->counts_dev, 2 * sizeof(int)));
  OLB_ECUDA_C(cudaMalloc(&E->tile_begin_dev, size_t(E->max_instances) * sizeof(int)));
  OLB_ECUDA_C(cudaMalloc(&E->tile_end_dev, size_t(E->max_instances) * sizeof(int)));
  OLB_ECUDA_C(cudaMalloc(&E->residual_dev, size_t(E->max_instances) * sizeof(double)));
  OLB_ECUDA_C(cudaMalloc(&E->steps_dev, size_t(E->max_instances) * sizeof(uint32_t)));
  OLB_ECUDA_C(cudaMallocHost(&E->residual_host, size_t(E->max_instances) * sizeof(double)));
  OLB_ECUDA_C(cudaMallocHost(&E->steps_host, size_t(E->max_instances) * sizeof(uint32_t)));
  OLB_ECUDA_C(cudaMemsetAsync(E->residual_dev, 0, size_t(E->max_instances) * sizeof(double), E->stream));
  OLB_ECUDA_C(cudaMemsetAsync(E->steps_dev, 0, size_t(E->max_instances) * sizeof(uint32_t), E->stream));
  int sms = 0;
  OLB_ECUDA_C(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E->device));
  E->min_blocks = 4;
  E->grid = sms * E->min_blocks;
  olb_b200_status st = upload_tables(E);
  if (st != OLB_B200_OK) return cleanup(st);
#undef OLB_ECUDA_C
  *out = E;
  return OLB_B200_OK;
}

void olb_b200_ensemble_destroy(olb_b200_ensemble* E)
{
  if (!E) return;
  cudaSetDevice(E->device);
  if (E->stream) cudaStreamSynchronize(E->stream);
  if (E->graph) cudaGraphExecDestroy(E->graph);
  cudaFree(E->pool);
  cudaFree(E->table_dev);
  cudaFree(E->tiles_dev);
  cudaFree(E->counts_dev);
  cudaFree(E->tile_begin_dev);
  cudaFree(E->tile_end_dev);
  cudaFree(E->partials);
  cudaFree(E->residual_dev);
  cudaFree(E->steps_dev);
  cudaFree(E->moments_dev);
  if (E->residual_host) cudaFreeHost(E->residual_host);
  if (E->steps_host) cudaFreeHost(E->steps_host);
  if (E->stream) cudaStreamDestroy(E->stream);
  delete E;
}

olb_b200_status olb_b200_ensemble_add(olb_b200_ensemble* E, const olb_b200_instance_desc* d, int32_t* slot_out)
{
  detail::set_last_error("");
  if (!E || !d || !slot_out) return efail(OLB_B200_ERR_ARG, "ensemble_add: null argument");
  if (d->kind != OLB_B200_ENSEMBLE_CAVITY && d->kind != OLB_B200_ENSEMBLE_CHANNEL &&
      d->kind != OLB_B200_ENSEMBLE_GEOMETRY)
    return efail(OLB_B200_ERR_ARG, "ensemble_add: unknown instance kind");
  const bool table = d->kind == OLB_B200_ENSEMBLE_GEOMETRY;
  if (table != (d->cells != nullptr))
    return efail(OLB_B200_ERR_ARG, "ensemble_add: a geometry table is given exactly for geometry instances");
  if (d->nx < 3 || d->ny < 3 || d->nz < 3) return efail(OLB_B200_ERR_ARG, "ensemble_add: extent below 3");
  if (!(d->omega > 0.0 && d->omega < 2.0)) return efail(OLB_B200_ERR_ARG, "ensemble_add: omega outside (0,2)");
  const uint64_t cells = uint64_t(d->nx) * d->ny * d->nz;
  if (table) {
    for (uint64_t c = 0; c < cells; ++c) {
      if (d->cells[c] > 2)
        return efail(OLB_B200_ERR_ARG, "ensemble_add: cell " + std::to_string(c) + " has class " +
                                         std::to_string(unsigned(d->cells[c])) +
                                         " (0 fluid, 1 wall, 2 moving wall)");
    }
  }
  // the step kernel indexes an instance's populations with 32 bits
  if (instance_elems(cells) >= (uint64_t(1) << 32))
    return efail(OLB_B200_ERR_ARG, "ensemble_add: instance too large (q x cells must stay below 2^32)");
  int slot = -1;
  for (int s = 0; s < E->max_instances; ++s) {
    if (!E->used[s]) {
      slot = s;
      break;
    }
  }
  if (slot < 0) return efail(OLB_B200_ERR_OOM, "ensemble_add: no free instance slot");
  // populations and stored velocity, then the geometry table (bytes, in
  // whole 256-byte units)
  const uint64_t table_elems = table ? round_up(cells, 256) / sizeof(float) : 0;
  const uint64_t need = instance_elems(cells) + table_elems;
  uint64_t offset = 0;
  if (!pool_alloc(E, need, offset)) return efail(OLB_B200_ERR_OOM, "ensemble_add: HBM pool budget exhausted");
  OLB_ECUDA(cudaSetDevice(E->device));
  // rest state: shifted populations 0 = equilibrium at rho 1, u 0; stored velocity 0
  OLB_ECUDA(cudaMemsetAsync(E->pool + offset, 0, need * sizeof(float), E->stream));
  InstanceDevice I{};
  if (table) {
    I.geom = offset + instance_elems(cells);
    OLB_ECUDA(cudaMemcpyAsync(E->pool + I.geom, d->cells, cells, cudaMemcpyHostToDevice, E->stream));
    OLB_ECUDA(cudaStreamSynchronize(E->stream));  // the caller's table may go away after this call
  }
  const uint32_t stride = uint32_t(round_up(cells, 64));
  I.pops = offset;
  I.uprev = offset + uint64_t(stride) * kQ;
  I.stride = stride;
  I.cells = uint32_t(cells);
  I.nx = d->nx;
  I.ny = d->ny;
  I.nz = d->nz;
  I.nz_u = uint32_t(d->nz);
  I.nynz = uint32_t(d->ny) * uint32_t(d->nz);
  I.div_nynz = FastDiv::make(I.nynz);
  I.div_nz = FastDiv::make(I.nz_u);
  I.kind = d->kind;
  I.forced = d->kind == OLB_B200_ENSEMBLE_CHANNEL ||
             (table && (d->force[0] != 0.0 || d->force[1] != 0.0 || d->force[2] != 0.0));
  I.active = 1;
  I.steps_done = 0;
  I.omega = float(d->omega);
  for (int e = 0; e < 3; ++e) {
    I.force[e] = float(d->force[e]);
    I.lid_u[e] = float(d->wall_u[e]);
  }
  I.force_relax = 1.f - I.omega * 0.5f;
  // Nguyen-Ladd terms 2 rho u_d c_id w_i cs^-2 with rho = 1, in the order of
  // the single-lattice table (collision.h:341-343)
  for (int i = 0; i < kQ; ++i) {
    const float w = float(L19::wnum(i)) / float(L19::wden(i));
    for (int e = 0; e < 3; ++e) {
      float t = 2.f * 1.f;
      t = t * I.lid_u[e];
      t = t * float(L19::c(i, e));
      t = t * w;
      t = t * 3.f;
      I.lid_term[i][e] = t;
    }
  }
  E->table[slot] = I;
  E->regions[slot] = Region{offset, need};
  E->used[slot] = 1;
  E->residual_host[slot] = INFINITY;
  E->dirty = true;
  *slot_out = slot;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_ensemble_remove(olb_b200_ensemble* E, int32_t slot)
{
  detail::set_last_error("");
  if (!E || slot < 0 || slot >= E->max_instances || !E->used[slot])
    return efail(OLB_B200_ERR_ARG, "ensemble_remove: no instance in this slot");
  OLB_ECUDA(cudaSetDevice(E->device));
  OLB_ECUDA(cudaStreamSynchronize(E->stream));
  pool_free(E, E->regions[slot]);
  E->table[slot] = InstanceDevice{};
  E->regions[slot] = Region{0, 0};
  E->used[slot] = 0;
  E->dirty = true;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_ensemble_run(olb_b200_ensemble* E, int32_t steps, int32_t check,
                                      double* residual, uint32_t* steps_done)
{
  detail::set_last_error("");
  if (!E || steps < 1) return efail(OLB_B200_ERR_ARG, "ensemble_run: bad argument");
  OLB_ECUDA(cudaSetDevice(E->device));
  if (E->dirty) {
    const olb_b200_status st = upload_tables(E);
    if (st != OLB_B200_OK) return st;
  }
  const int chk = check ? 1 : 0;
  if (!E->graph || E->graph_steps != steps || E->graph_check != chk || E->graph_minb != E->min_blocks) {
    if (E->graph) {
      cudaGraphExecDestroy(E->graph);
      E->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    OLB_ECUDA(cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal));
    const olb_b200_status st = enqueue_chunk(E, steps, chk);
    const cudaError_t e = cudaStreamEndCapture(E->stream, &g);
    if (st != OLB_B200_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return ecuda(e, "cudaStreamEndCapture");
    const cudaError_t e2 = cudaGraphInstantiate(&E->graph, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) return ecuda(e2, "cudaGraphInstantiate");
    E->graph_steps = steps;
    E->graph_check = chk;
    E->graph_minb = E->min_blocks;
  }
  OLB_ECUDA(cudaGraphLaunch(E->graph, E->stream));
  OLB_ECUDA(cudaStreamSynchronize(E->stream));
  for (int s = 0; s < E->max_instances; ++s) {
    if (E->used[s]) E->table[s].steps_done = E->steps_host[s];
  }
  if (residual) std::memcpy(residual, E->residual_host, size_t(E->max_instances) * sizeof(double));
  if (steps_done) std::memcpy(steps_done, E->steps_host, size_t(E->max_instances) * sizeof(uint32_t));
  return OLB_B200_OK;
}

olb_b200_status olb_b200_ensemble_get_moments(olb_b200_ensemble* E, int32_t slot, float* host_rho, float* host_u)
{
  detail::set_last_error("");
  if (!E || slot < 0 || slot >= E->max_instances || !E->used[slot] || !host_rho || !host_u)
    return efail(OLB_B200_ERR_ARG, "ensemble_get_moments: bad argument");
  OLB_ECUDA(cudaSetDevice(E->device));
  const InstanceDevice& I = E->table[slot];
  const size_t need = size_t(I.cells) * 4;
  if (need > E->moments_cap) {
    OLB_ECUDA(cudaStreamSynchronize(E->stream));
    cudaFree(E->moments_dev);
    E->moments_dev = nullptr;
    E->moments_cap = 0;
    OLB_ECUDA(cudaMalloc(&E->moments_dev, need * sizeof(float)));
    E->moments_cap = need;
  }
  float* dev = E->moments_dev;
  ensemble_moments_kernel<<<(I.cells + 255) / 256, 256, 0, E->stream>>>(E->pool, I, dev, dev + I.cells);
  OLB_ECUDA(cudaGetLastError());
  OLB_ECUDA(cudaMemcpyAsync(host_rho, dev, size_t(I.cells) * sizeof(float), cudaMemcpyDeviceToHost, E->stream));
  OLB_ECUDA(cudaMemcpyAsync(host_u, dev + I.cells, size_t(I.cells) * 3 * sizeof(float), cudaMemcpyDeviceToHost,
                            E->stream));
  OLB_ECUDA(cudaStreamSynchronize(E->stream));
  return OLB_B200_OK;
}

olb_b200_status olb_b200_ensemble_info(olb_b200_ensemble* E, int64_t* pool_free_bytes, int32_t* active,
                                       int32_t* tiles)
{
  if (!E) return efail(OLB_B200_ERR_ARG, "ensemble_info: null ensemble");
  uint64_t free_elems = 0;
  for (const Region& r : E->free_list) free_elems += r.size;
  int n = 0, t = 0;
  for (int s = 0; s < E->max_instances; ++s) {
    if (E->used[s] && E->table[s].active) {
      ++n;
      t += int((E->table[s].cells + kTile - 1) / kTile);
    }
  }
  if (pool_free_bytes) *pool_free_bytes = int64_t(free_elems * sizeof(float));
  if (active) *active = n;
  if (tiles) *tiles = t;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_ensemble_set_occupancy(olb_b200_ensemble* E, int32_t blocks_per_sm)
{
  detail::set_last_error("");
  if (!E || (blocks_per_sm != 2 && blocks_per_sm != 3 && blocks_per_sm != 4))
    return efail(OLB_B200_ERR_ARG, "ensemble_set_occupancy: blocks_per_sm must be 2, 3 or 4");
  int sms = 0;
  OLB_ECUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E->device));
  E->min_blocks = blocks_per_sm;
  E->grid = sms * blocks_per_sm;
  if (E->graph) {
    cudaGraphExecDestroy(E->graph);
    E->graph = nullptr;
  }
  return OLB_B200_OK;
}

uint64_t olb_b200_ensemble_bytes_per_instance(int32_t nx, int32_t ny, int32_t nz)
{
  return instance_elems(uint64_t(nx) * ny * nz) * sizeof(float);
}

} // extern "C"
