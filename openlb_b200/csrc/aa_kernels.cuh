// Fused collide-and-stream for sm_100a on the in-place AA pattern.
//
// Memory layout in HBM: one column per population i, `stride` elements long
// (the cell count rounded up to 64 elements, so every column starts on a 256 B
// boundary), cell = (x*ny + y)*nz + z with z fastest — OpenLB's order
// (src/core/blockStructure.h:65-75) without the overlap layers.  Periodic and
// non-periodic faces alike wrap per axis; at non-periodic faces the wrapped
// values only ever reach wall cells, exactly as OpenLB's unspecified padding
// values only reach its wall cells.
//
// AA pattern (one array, in place):
//   even step t: cell x reads f_i from column i at x, collides, writes f*_i to
//                column opp(i) at x.
//   odd step   : cell x reads f_i from column opp(i) at x - c_i, collides,
//                writes f*_i to column i at x + c_i.
// After an odd step the array holds the post-stream state in natural order
// (f_i(x) in column i at x); after an even step f_i(x) sits in column opp(i)
// at x - c_i.  Every cell reads and writes exactly the same q slots, so no two
// cells touch the same slot.  This is equivalent to OpenLB's collide followed
// by the periodic-shift stream (src/core/blockLattice.hh:317-339,
// src/core/platform/cpu/sisd/column.h:193-204).
//
// Full-way bounce-back (collision::Revert) writes f*_i = f_opp(i) to exactly
// the slot f_opp(i) was read from, so wall cells need no memory access at
// all; moving walls add their Nguyen-Ladd term in place.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lbm_device.cuh"

namespace olb_b200 {

struct Geometry {
  int32_t nx, ny, nz;
  uint32_t stride;  // column length in storage elements
  int32_t paired;   // 1: 16-bit storage with cells x and x + nx/2 in one 4-byte element
  // masked lattices: a box [lo, hi) whose cells all use the bulk entry, so the
  // step kernel skips their dynamics id (empty when lo == hi)
  int32_t bulk_lo[3], bulk_hi[3];
  // FORCE per cell for the Guo-forced dynamics (3 columns of `stride` values
  // of the compute type, natural cell order), or nullptr: the entries' forces
  const void* force;
  // masked lattices: 1 when every entry of the bulk entry's collision kind has
  // the bulk entry's constants, so the step kernel takes them from the kernel
  // argument instead of loading them from the cell's table entry
  int32_t uniform;
};

// the entry index the masked kernels give a cell of the bulk box (the table
// holds at most 256 entries): it collides with the bulk entry, the kernel
// argument, and loads nothing from the table
constexpr int kBoxCell = 256;

OLB_HD bool in_bulk_box(const Geometry& g, int x, int y, int z)
{
  return x >= g.bulk_lo[0] && x < g.bulk_hi[0] && y >= g.bulk_lo[1] && y < g.bulk_hi[1] && z >= g.bulk_lo[2] &&
         z < g.bulk_hi[2];
}

// Scalar slot of a cell within a population column.
//   natural layout: (x*ny + y)*nz + z
//   paired layout (16-bit storage, nx even): element ((x mod nx/2)*ny + y)*nz + z
//   holds cell x in its low half and cell x + nx/2 in its high half, so the
//   slot is 2*element + (x >= nx/2).  Shifts along y and z keep elements
//   aligned; only the x seam swaps the halves.
OLB_HD uint32_t cell_slot(const Geometry& g, int x, int y, int z)
{
  if (!g.paired) {
    return (uint32_t(x) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z);
  }
  const int nxh = g.nx >> 1;
  const int hi = x >= nxh;
  const uint32_t e = (uint32_t(hi ? x - nxh : x) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z);
  return 2u * e + uint32_t(hi);
}

OLB_HD int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// A copy of v the compiler cannot see through: store addresses computed from
// it are recomputed after the collision (one multiply-add each) instead of
// being kept live in registers from the load phase.
OLB_DEV uint32_t opaque(uint32_t v)
{
  uint32_t r;
  asm volatile("mov.b32 %0, %1;" : "=r"(r) : "r"(v));
  return r;
}

// per-block partial of the fused statistics reduction (FP64)
struct StatPartial {
  double sum_rho;
  double sum_usqr;
  double max_usqr;
  unsigned long long n_cells;
  unsigned long long n_nonfinite;
};

// ---------------------------------------------------------------------------
// storage element conversions (plain loads: the array is read and written in
// place by the same kernel, so the read-only data path is not used)

template <class S, class R> struct Store;

template <class R> struct Store<float, R> {
  template <class L, int I> OLB_DEV static R load(const float* p) { return R(*p); }
  template <class L, int I> OLB_DEV static void store(float* p, R v) { *p = float(v); }
};
template <class R> struct Store<double, R> {
  template <class L, int I> OLB_DEV static R load(const double* p) { return R(*p); }
  template <class L, int I> OLB_DEV static void store(double* p, R v) { *p = double(v); }
};
template <class R> struct Store<__half, R> {
  template <class L, int I> OLB_DEV static R load(const __half* p)
  {
    constexpr float inv = 1.f / storage_scale<L>(I);
    return R(__half2float(*p) * inv);
  }
  template <class L, int I> OLB_DEV static void store(__half* p, R v)
  {
    constexpr float s = storage_scale<L>(I);
    *p = __float2half_rn(float(v) * s);
  }
};
template <class R> struct Store<__nv_bfloat16, R> {
  template <class L, int I> OLB_DEV static R load(const __nv_bfloat16* p)
  {
    constexpr float inv = 1.f / storage_scale<L>(I);
    return R(__bfloat162float(*p) * inv);
  }
  template <class L, int I> OLB_DEV static void store(__nv_bfloat16* p, R v)
  {
    constexpr float s = storage_scale<L>(I);
    *p = __float2bfloat16_rn(float(v) * s);
  }
};

// ---------------------------------------------------------------------------
// neighbour offsets with per-axis wrap-around

struct Neighbours {
  uint32_t xo[3], yo[3], zo[3];
  OLB_DEV Neighbours(const Geometry& g, int x, int y, int z)
  {
    const uint32_t sxy = uint32_t(g.ny) * uint32_t(g.nz);
    xo[0] = uint32_t(x == 0 ? g.nx - 1 : x - 1) * sxy;
    xo[1] = uint32_t(x) * sxy;
    xo[2] = uint32_t(x == g.nx - 1 ? 0 : x + 1) * sxy;
    yo[0] = uint32_t(y == 0 ? g.ny - 1 : y - 1) * uint32_t(g.nz);
    yo[1] = uint32_t(y) * uint32_t(g.nz);
    yo[2] = uint32_t(y == g.ny - 1 ? 0 : y + 1) * uint32_t(g.nz);
    zo[0] = uint32_t(z == 0 ? g.nz - 1 : z - 1);
    zo[1] = uint32_t(z);
    zo[2] = uint32_t(z == g.nz - 1 ? 0 : z + 1);
  }
  template <int DX, int DY, int DZ>
  OLB_DEV uint32_t at() const { return xo[DX + 1] + yo[DY + 1] + zo[DZ + 1]; }
};

// ---------------------------------------------------------------------------
// block-level FP64 statistics reduction

OLB_DEV void warp_reduce(double& a, double& b, double& m, unsigned long long& n, unsigned long long& nf)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
    m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    n += __shfl_down_sync(0xffffffffu, n, o);
    nf += __shfl_down_sync(0xffffffffu, nf, o);
  }
}

OLB_DEV void block_stats(double a, double b, double m, unsigned long long n, unsigned long long nf,
                         StatPartial* out)
{
  __shared__ StatPartial warp_part[32];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthreads = blockDim.x * blockDim.y;
  warp_reduce(a, b, m, n, nf);
  const int lane = tid & 31, warp = tid >> 5;
  if (lane == 0) {
    warp_part[warp] = StatPartial{a, b, m, n, nf};
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = (nthreads + 31) >> 5;
    StatPartial p = lane < nw ? warp_part[lane] : StatPartial{0, 0, 0, 0, 0};
    warp_reduce(p.sum_rho, p.sum_usqr, p.max_usqr, p.n_cells, p.n_nonfinite);
    if (lane == 0) {
      const size_t bid = blockIdx.x + size_t(gridDim.x) * (blockIdx.y + size_t(gridDim.y) * blockIdx.z);
      out[bid] = p;
    }
  }
}

// ---------------------------------------------------------------------------
// the step kernel

// Step-kernel variants: cells per thread (along y, blockDim.y rows apart) and
// the register cap (__launch_bounds__(kStepThreads, min_blocks)).  All loads of
// a thread's cells are issued before any of them is collided, so more cells
// per thread — or more resident warps — means more bytes in flight per SM, the
// quantity that bounds this HBM-streaming kernel.  Which variant is fastest
// depends on the lattice, the storage type and the mask; the library picks a
// default per lattice and can time all of them (olb_b200_autotune).  Every
// variant performs the same arithmetic on every cell, so results are
// independent of the choice.
constexpr int kStepThreads = 256;
struct StepVariant {
  int cells_per_thread;
  int min_blocks;
};
#ifdef OLB_B200_SINGLE_VARIANT
// builds that only check arithmetic compile one variant; every id maps to it
constexpr StepVariant kStepVariants[] = {{1, 3}, {1, 3}, {1, 3}, {1, 3}};
#elif defined(OLB_B200_EXACT)
// the reference-order build serves parity, not speed: both work distributions
// (one and two cells per thread), one register cap each
constexpr StepVariant kStepVariants[] = {{1, 3}, {1, 3}, {2, 3}, {2, 3}};
#else
constexpr StepVariant kStepVariants[] = {{1, 3}, {1, 4}, {2, 2}, {2, 3}};
#endif
constexpr int kNumStepVariants = 4;

// running sums of the fused statistics of one thread
struct StatAcc {
  double rho = 0., usqr = 0., max = 0.;
  unsigned long long n = 0, nf = 0;
  OLB_DEV void add(double r, double u2)
  {
    if (isfinite(r) && isfinite(u2)) {
      rho += r; usqr += u2; max = fmax(max, u2); n += 1;
    } else {
      nf += 1;
    }
  }
};

// One tile of the step: the CPT cells (x, y0 + k*dy, z) of this thread.
// Masked lattices pass each cell's table entry in id[k] (loaded a tile ahead by
// aa_step_masked_kernel); unmasked lattices use `bulk` for every cell.
template <int Q, class S, class R, int KIND, bool ODD, bool MASKED, bool STATS, int CPT>
OLB_DEV void step_tile(S* __restrict__ pops, const Geometry& g, const DynDevice<R>* __restrict__ table,
                       const DynDevice<R>& bulk, int x, int y0, int z, int dy, const int (&id)[CPT], StatAcc& acc)
{
  using L = Lattice<Q>;
  using ST = Store<S, R>;
  constexpr bool kForced = KIND == K_FORCED_BGK || KIND == K_FORCED_TRT;
  R f[CPT][Q];
  R fc[CPT][3];  // the cell's FORCE when the lattice has a force field
  int kind[CPT];
  bool go[CPT];
  uint32_t n[CPT];

  // phase 1: issue all loads.  Masked lattices load every cell's populations
  // before its dynamics id has arrived (the id and the populations travel
  // together instead of one after the other); a full-way bounce-back cell
  // then stores nothing, its AA update being a no-op (see file comment).
  static_for<0, CPT>([&](auto k) {
    const int y = y0 + k.value * dy;
    go[k] = z < g.nz && y < g.ny;
    kind[k] = KIND;
    n[k] = 0;
    if (go[k]) {
      n[k] = (uint32_t(x) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z);
      Neighbours nb(g, x, y, z);
      static_for<0, Q>([&](auto i) {
        if constexpr (!ODD) {
          f[k][i] = ST::template load<L, i.value>(pops + size_t(i.value) * g.stride + n[k]);
        } else {
          constexpr int o = L::opp(i);
          const uint32_t src = nb.template at<-L::c(i, 0), -L::c(i, 1), -L::c(i, 2)>();
          f[k][i] = ST::template load<L, o>(pops + size_t(o) * g.stride + src);
        }
      });
      if constexpr (kForced) {
        fc[k][0] = fc[k][1] = fc[k][2] = R(0);
        if (g.force) {
          const R* __restrict__ F = static_cast<const R*>(g.force);
          fc[k][0] = __ldg(F + n[k]);
          fc[k][1] = __ldg(F + size_t(g.stride) + n[k]);
          fc[k][2] = __ldg(F + 2 * size_t(g.stride) + n[k]);
        }
      }
    }
  });
  if constexpr (MASKED) {
    static_for<0, CPT>([&](auto k) {
      if (go[k] && id[k] != kBoxCell) kind[k] = __ldg(&table[id[k]].kind);
      go[k] = go[k] && kind[k] != K_BOUNCE_BACK;
    });
  }

  // phase 2: collide and store
  static_for<0, CPT>([&](auto k) {
    if (!go[k]) return;
    const int y = y0 + k.value * dy;
    R st_rho = R(0), st_usqr = R(0);
    bool counted = false;
    if (kind[k] == KIND) {
      if constexpr (MASKED) {
        // the entry's collision constants (the bulk entry's for box cells)
        DynDevice<R> q;
        if (id[k] == kBoxCell || g.uniform) {
          q.omega = bulk.omega;
          q.omega_minus = bulk.omega_minus;
          q.smago_pre = bulk.smago_pre;
          q.tau_mol = bulk.tau_mol;
          q.force[0] = bulk.force[0];
          q.force[1] = bulk.force[1];
          q.force[2] = bulk.force[2];
          q.force_relax = bulk.force_relax;
        } else {
          const DynDevice<R>* e = table + id[k];
          q.omega = __ldg(&e->omega);
          q.omega_minus = __ldg(&e->omega_minus);
          q.smago_pre = __ldg(&e->smago_pre);
          q.tau_mol = __ldg(&e->tau_mol);
          q.force[0] = __ldg(&e->force[0]);
          q.force[1] = __ldg(&e->force[1]);
          q.force[2] = __ldg(&e->force[2]);
          q.force_relax = __ldg(&e->force_relax);
        }
        if constexpr (kForced) {
          if (g.force) {
            q.force[0] = fc[k][0]; q.force[1] = fc[k][1]; q.force[2] = fc[k][2];
          }
        }
        collide_bulk<L, KIND>(f[k], q, st_rho, st_usqr);
      } else if constexpr (kForced) {
        DynDevice<R> q;
        q.omega = bulk.omega;
        q.omega_minus = bulk.omega_minus;
        q.force_relax = bulk.force_relax;
        q.force[0] = g.force ? fc[k][0] : bulk.force[0];
        q.force[1] = g.force ? fc[k][1] : bulk.force[1];
        q.force[2] = g.force ? fc[k][2] : bulk.force[2];
        collide_bulk<L, KIND>(f[k], q, st_rho, st_usqr);
      } else {
        collide_bulk<L, KIND>(f[k], bulk, st_rho, st_usqr);
      }
      counted = true;
    } else if (MASKED && kind[k] == K_BOUNCE_BACK_VELOCITY) {
      const DynDevice<R>* e = table + id[k];
      revert<L>(f[k]);
      static_for<1, Q>([&](auto i) {
        f[k][i] += __ldg(&e->wall_term[i][0]);
        f[k][i] += __ldg(&e->wall_term[i][1]);
        f[k][i] += __ldg(&e->wall_term[i][2]);
      });
      st_rho = __ldg(&e->wall_rho);
      const R wu[3] = {__ldg(&e->wall_u[0]), __ldg(&e->wall_u[1]), __ldg(&e->wall_u[2])};
      st_usqr = norm_sqr(wu);
      counted = true;
    }
    // NoDynamics and the boundary cells that carry values (their collision
    // ran in place before this kernel, boundary_collide_kernel): populations
    // pass through unchanged.
    // The store offsets are recomputed here rather than kept live through
    // the collision.
    Neighbours nb(g, int(opaque(uint32_t(x))), int(opaque(uint32_t(y))), int(opaque(uint32_t(z))));
    const uint32_t stride = opaque(g.stride);
    const uint32_t nk = opaque(n[k]);
    static_for<0, Q>([&](auto i) {
      if constexpr (!ODD) {
        constexpr int o = L::opp(i);
        ST::template store<L, o>(pops + size_t(o) * stride + nk, f[k][i]);
      } else {
        const uint32_t dst = nb.template at<L::c(i, 0), L::c(i, 1), L::c(i, 2)>();
        ST::template store<L, i.value>(pops + size_t(i.value) * stride + dst, f[k][i]);
      }
    });
    if constexpr (STATS) {
      if (counted) acc.add(double(st_rho), double(st_usqr));
    }
  });
}

// Unmasked lattices (every cell uses `bulk`): one tile per block, grid
// step_grid().
template <int Q, class S, class R, int KIND, bool ODD, bool STATS, int CPT, int MINB>
__global__ void __launch_bounds__(kStepThreads, MINB)
aa_step_kernel(S* __restrict__ pops, const Geometry g, const DynDevice<R> bulk, StatPartial* __restrict__ partials)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y0 = blockIdx.y * (blockDim.y * CPT) + threadIdx.y;
  const int x = blockIdx.z;
  const int none[CPT] = {};
  StatAcc acc;
  step_tile<Q, S, R, KIND, ODD, false, STATS, CPT>(pops, g, nullptr, bulk, x, y0, z, int(blockDim.y), none, acc);
  if constexpr (STATS) {
    block_stats(acc.rho, acc.usqr, acc.max, acc.n, acc.nf, partials);
  }
}

// table entries of a tile's cells: kBoxCell for cells of the bulk box (they
// use the bulk entry, no load), -1 for cells outside the lattice (skipped)
template <int CPT>
OLB_DEV void load_tile_ids(int (&id)[CPT], const Geometry& g, const uint8_t* __restrict__ ids, int x, int y0,
                           int z, int dy)
{
  static_for<0, CPT>([&](auto k) {
    const int y = y0 + k.value * dy;
    id[k] = -1;
    if (z < g.nz && y < g.ny) {
      id[k] = in_bulk_box(g, x, y, z)
                ? kBoxCell
                : int(ids[(uint32_t(x) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z)]);
    }
  });
}

// Masked lattices: one tile per block, grid step_grid().  The ids of the
// thread's cells are loaded first (none for cells of the bulk box); the
// populations follow without waiting for them (step_tile).
template <int Q, class S, class R, int KIND, bool ODD, bool STATS, int CPT, int MINB>
__global__ void __launch_bounds__(kStepThreads, MINB)
aa_step_masked_kernel(S* __restrict__ pops, const Geometry g, const uint8_t* __restrict__ ids,
                      const DynDevice<R>* __restrict__ table, const DynDevice<R> bulk,
                      StatPartial* __restrict__ partials)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y0 = blockIdx.y * (blockDim.y * CPT) + threadIdx.y;
  const int x = blockIdx.z;
  const int dy = int(blockDim.y);
  int id[CPT];
  load_tile_ids(id, g, ids, x, y0, z, dy);
  StatAcc acc;
  step_tile<Q, S, R, KIND, ODD, true, STATS, CPT>(pops, g, table, bulk, x, y0, z, dy, id, acc);
  if constexpr (STATS) {
    block_stats(acc.rho, acc.usqr, acc.max, acc.n, acc.nf, partials);
  }
}

// ---------------------------------------------------------------------------
// the step kernel on the paired 16-bit layout
//
// Each thread updates the two cells of one 4-byte element, (x', y, z) and
// (x' + nx/2, y, z), with one aligned 32-bit load and one aligned 32-bit store
// per population — a warp moves 128 B per instruction instead of 64 B.  The
// grid's z dimension walks x' in [0, nx/2); a neighbour across the x seam is
// the element on the other side with its halves swapped, a condition that is
// uniform per block.  Cells of a pair may have different dynamics; full-way
// bounce-back cells then apply their swap in registers (it writes back what
// it read, so the result is the same as skipping them).

template <class S> struct Pair;
template <> struct Pair<__half> {
  using T = __half2;
  OLB_DEV static float2 to_float2(T v) { return __half22float2(v); }
  OLB_DEV static T from_floats(float lo, float hi) { return __floats2half2_rn(lo, hi); }
  OLB_DEV static T from_float2(float2 v) { return __float22half2_rn(v); }
};
template <> struct Pair<__nv_bfloat16> {
  using T = __nv_bfloat162;
  OLB_DEV static float2 to_float2(T v) { return __bfloat1622float2(v); }
  OLB_DEV static T from_floats(float lo, float hi) { return __floats2bfloat162_rn(lo, hi); }
  OLB_DEV static T from_float2(float2 v) { return __float22bfloat162_rn(v); }
};

// what a lane of the two-lane collision does: collide with the lattice's fluid
// kind, bounce back (full-way, collision::Revert), or pass its populations
// through unchanged (NoDynamics, and boundary cells, whose collision ran ahead
// of the step kernel)
enum LaneMode { kLaneFluid = 0, kLaneWall = 1, kLanePass = 2 };

// the fluid collision constants of a cell for the scaled collisions (KIND the
// lattice's fluid kind): its table entry's when `own` and it has one, else the
// bulk entry's (kernel argument); a wall or pass lane gets the constants that
// make the same arithmetic a swap or the identity (see ScaledParams)
template <int KIND>
OLB_DEV ScaledParams<float> scaled_params(const DynDevice<float>* pe, bool own, const DynDevice<float>& bulk,
                                          int lane = kLaneFluid)
{
  ScaledParams<float> q;
  if (own && pe) {
    q.omega = __ldg(&pe->omega);
    q.omega_b = __ldg(&pe->omega_minus);
    q.smago_pre = __ldg(&pe->smago_pre);
    q.tau_mol = __ldg(&pe->tau_mol);
    q.force_relax = __ldg(&pe->force_relax);
    q.force[0] = __ldg(&pe->force[0]);
    q.force[1] = __ldg(&pe->force[1]);
    q.force[2] = __ldg(&pe->force[2]);
  } else {
    q.omega = bulk.omega;
    q.omega_b = bulk.omega_minus;
    q.smago_pre = bulk.smago_pre;
    q.tau_mol = bulk.tau_mol;
    q.force_relax = bulk.force_relax;
    q.force[0] = bulk.force[0];
    q.force[1] = bulk.force[1];
    q.force[2] = bulk.force[2];
  }
  if (!(KIND == K_TRT || KIND == K_FORCED_TRT)) q.omega_b = q.omega;
  q.keep = 0.5f * (1.f - q.omega);
  q.keep_minus = 0.5f * (1.f - q.omega_b);
  q.live = 1.f;
  if (lane != kLaneFluid) {
    q.omega = q.omega_b = q.force_relax = 0.f;
    q.force[0] = q.force[1] = q.force[2] = 0.f;
    q.keep = 0.5f;
    q.keep_minus = lane == kLaneWall ? -0.5f : 0.5f;
    q.live = 0.f;
  }
  return q;
}

// the constants of two cells as the lanes of one pair
OLB_DEV ScaledParams<float2> zip_params(const ScaledParams<float>& a, const ScaledParams<float>& b)
{
  ScaledParams<float2> q;
  q.omega = make_float2(a.omega, b.omega);
  q.omega_b = make_float2(a.omega_b, b.omega_b);
  q.keep = make_float2(a.keep, b.keep);
  q.keep_minus = make_float2(a.keep_minus, b.keep_minus);
  q.smago_pre = make_float2(a.smago_pre, b.smago_pre);
  q.tau_mol = make_float2(a.tau_mol, b.tau_mol);
  q.live = make_float2(a.live, b.live);
  q.force_relax = make_float2(a.force_relax, b.force_relax);
  q.force[0] = make_float2(a.force[0], b.force[0]);
  q.force[1] = make_float2(a.force[1], b.force[1]);
  q.force[2] = make_float2(a.force[2], b.force[2]);
  return q;
}

// byte permutation of a packed pair (one PRMT): 0x3210 keeps it, 0x1032 swaps
// the halves; pair_merge_lo/hi take the low/high halves of a and b
template <class T>
OLB_DEV T pair_perm(T a, T b, uint32_t sel)
{
  static_assert(sizeof(T) == 4, "packed 16-bit pair");
  uint32_t ua, ub;
  memcpy(&ua, &a, 4);
  memcpy(&ub, &b, 4);
  const uint32_t r = __byte_perm(ua, ub, sel);
  T out;
  memcpy(&out, &r, 4);
  return out;
}

struct PairNeighbours {
  uint32_t xo[3], yo[3], zo[3];
  bool swap[3];
  OLB_DEV PairNeighbours(const Geometry& g, int xp, int y, int z)
  {
    const int nxh = g.nx >> 1;
    const uint32_t sxy = uint32_t(g.ny) * uint32_t(g.nz);
    xo[0] = uint32_t(xp == 0 ? nxh - 1 : xp - 1) * sxy;
    xo[1] = uint32_t(xp) * sxy;
    xo[2] = uint32_t(xp == nxh - 1 ? 0 : xp + 1) * sxy;
    swap[0] = xp == 0;
    swap[1] = false;
    swap[2] = xp == nxh - 1;
    yo[0] = uint32_t(y == 0 ? g.ny - 1 : y - 1) * uint32_t(g.nz);
    yo[1] = uint32_t(y) * uint32_t(g.nz);
    yo[2] = uint32_t(y == g.ny - 1 ? 0 : y + 1) * uint32_t(g.nz);
    zo[0] = uint32_t(z == 0 ? g.nz - 1 : z - 1);
    zo[1] = uint32_t(z);
    zo[2] = uint32_t(z == g.nz - 1 ? 0 : z + 1);
  }
  template <int DX, int DY, int DZ>
  OLB_DEV uint32_t at() const { return xo[DX + 1] + yo[DY + 1] + zo[DZ + 1]; }
};

// collision of one cell of a pair by its runtime kind (masked lattices);
// field: the Guo-forced dynamics take the cell's FORCE from fcell
template <class L, int KIND, bool MASKED>
OLB_DEV bool collide_any(float (&f)[L::q], int kind, const DynDevice<float>* e, const DynDevice<float>& bulk,
                         const float (&fcell)[3], bool field, bool uniform, float& st_rho, float& st_usqr)
{
  constexpr bool kForced = KIND == K_FORCED_BGK || KIND == K_FORCED_TRT;
  if (kind == KIND) {
    const bool own = MASKED && e && !uniform;  // the entry's constants, not the bulk entry's
    if (own || (kForced && field)) {
      DynDevice<float> q;
      if (own) {
        q.omega = __ldg(&e->omega);
        q.omega_minus = __ldg(&e->omega_minus);
        q.smago_pre = __ldg(&e->smago_pre);
        q.tau_mol = __ldg(&e->tau_mol);
        q.force[0] = __ldg(&e->force[0]);
        q.force[1] = __ldg(&e->force[1]);
        q.force[2] = __ldg(&e->force[2]);
        q.force_relax = __ldg(&e->force_relax);
      } else {
        q.omega = bulk.omega;
        q.omega_minus = bulk.omega_minus;
        q.smago_pre = bulk.smago_pre;
        q.tau_mol = bulk.tau_mol;
        q.force[0] = bulk.force[0];
        q.force[1] = bulk.force[1];
        q.force[2] = bulk.force[2];
        q.force_relax = bulk.force_relax;
      }
      if constexpr (kForced) {
        if (field) {
          q.force[0] = fcell[0]; q.force[1] = fcell[1]; q.force[2] = fcell[2];
        }
      }
      collide_bulk<L, KIND>(f, q, st_rho, st_usqr);
    } else {
      collide_bulk<L, KIND>(f, bulk, st_rho, st_usqr);
    }
    return true;
  }
  if constexpr (MASKED) {
    if (kind == K_BOUNCE_BACK) {
      revert<L>(f);
    } else if (kind == K_BOUNCE_BACK_VELOCITY) {
      revert<L>(f);
      static_for<1, L::q>([&](auto i) {
        f[i] += __ldg(&e->wall_term[i][0]);
        f[i] += __ldg(&e->wall_term[i][1]);
        f[i] += __ldg(&e->wall_term[i][2]);
      });
      st_rho = __ldg(&e->wall_rho);
      const float wu[3] = {__ldg(&e->wall_u[0]), __ldg(&e->wall_u[1]), __ldg(&e->wall_u[2])};
      st_usqr = norm_sqr(wu);
      return true;
    }
  }
  return false;  // NoDynamics / bounce-back / boundary cells (collided ahead): no statistic here
}

// One tile of the paired step: the CPT element rows (x', y0 + k*dy, z) of
// this thread, each the two cells x' and x' + nx/2.  Masked lattices pass the
// table entries of both cells (loaded a tile ahead); unmasked ones use `bulk`.
template <int Q, class S, int KIND, bool ODD, bool MASKED, bool STATS, int CPT>
OLB_DEV void paired_tile(S* __restrict__ pops_scalar, const Geometry& g, const DynDevice<float>* __restrict__ table,
                         const DynDevice<float>& bulk, int xp, int y0, int z, int dy, const int (&id_lo)[CPT],
                         const int (&id_hi)[CPT], StatAcc& acc)
{
  using L = Lattice<Q>;
  using P = Pair<S>;
  using T = typename P::T;
  constexpr bool kForced = KIND == K_FORCED_BGK || KIND == K_FORCED_TRT;
  T* __restrict__ pops = reinterpret_cast<T*>(pops_scalar);
  const uint32_t pstride = g.stride >> 1;  // elements per column

  // the loaded pairs stay packed (low half = cell x', high half = x' + nx/2):
  // one 32-bit register per population for both cells
  T raw[CPT][Q];
  int kind_lo[CPT], kind_hi[CPT];
  bool go[CPT];
  uint32_t e[CPT];

  static_for<0, CPT>([&](auto k) {
    const int y = y0 + k.value * dy;
    go[k] = z < g.nz && y < g.ny;
    kind_lo[k] = kind_hi[k] = KIND;
    e[k] = 0;
    if (go[k]) {
      // the pair's populations are loaded before its ids have arrived (as in
      // step_tile); a pair of two bounce-back cells then stores nothing
      e[k] = (uint32_t(xp) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z);
      PairNeighbours nb(g, xp, y, z);
      static_for<0, Q>([&](auto i) {
        // 32-bit element indices: the paired layout is only used while
        // q * pstride < 2^32 (olb_b200_create)
        if constexpr (!ODD) {
          raw[k][i] = pops[uint32_t(i.value) * pstride + e[k]];
        } else {
          constexpr int o = L::opp(i);
          const uint32_t src = nb.template at<-L::c(i, 0), -L::c(i, 1), -L::c(i, 2)>();
          const T v = pops[uint32_t(o) * pstride + src];
          if constexpr (L::c(i, 0) != 0) {
            raw[k][i] = pair_perm(v, v, nb.swap[1 - L::c(i, 0)] ? 0x1032u : 0x3210u);
          } else {
            raw[k][i] = v;
          }
        }
      });
    }
  });
  if constexpr (MASKED) {
    static_for<0, CPT>([&](auto k) {
      if (go[k]) {
        if (id_lo[k] != kBoxCell) kind_lo[k] = __ldg(&table[id_lo[k]].kind);
        if (id_hi[k] != kBoxCell) kind_hi[k] = __ldg(&table[id_hi[k]].kind);
        go[k] = !(kind_lo[k] == K_BOUNCE_BACK && kind_hi[k] == K_BOUNCE_BACK);
      }
    });
  }

  static_for<0, CPT>([&](auto k) {
    if (!go[k]) return;
    const int y = y0 + k.value * dy;
    // the table entries (nullptr: the bulk entry, the kernel argument)
    const DynDevice<float>* pe_lo = MASKED && id_lo[k] != kBoxCell ? table + id_lo[k] : nullptr;
    const DynDevice<float>* pe_hi = MASKED && id_hi[k] != kBoxCell ? table + id_hi[k] : nullptr;
    const bool field = kForced && g.force != nullptr;
    // the cell's FORCE when the lattice has a force field (Guo-forced
    // dynamics; loaded here, after the populations)
    auto load_force = [&](int x, float (&fc)[3]) {
      const float* __restrict__ F = static_cast<const float*>(g.force);
      const uint32_t nn = (uint32_t(x) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z);
      fc[0] = __ldg(F + nn);
      fc[1] = __ldg(F + size_t(g.stride) + nn);
      fc[2] = __ldg(F + 2 * size_t(g.stride) + nn);
    };
#ifndef OLB_B200_EXACT
    // both cells go through the two-lane collision unless one is a moving wall
    // (a pair of two bounce-back walls stores nothing)
    bool both = true;
    int lane_lo = kLaneFluid, lane_hi = kLaneFluid;
    if constexpr (MASKED) {
      auto mode = [](int kind) {
        return kind == KIND ? kLaneFluid : (kind == K_BOUNCE_BACK ? kLaneWall : kLanePass);
      };
      lane_lo = mode(kind_lo[k]);
      lane_hi = mode(kind_hi[k]);
      // a moving wall adds its momentum terms: one cell after the other
      both = kind_lo[k] != K_BOUNCE_BACK_VELOCITY && kind_hi[k] != K_BOUNCE_BACK_VELOCITY;
    }
    if (both) {
      // Both cells at once, in the scaled representation g_i = s_i (f_i - w_i)
      // of the storage: lane x the low cell, lane y the high one, straight
      // from and back to the packed pairs (packed FP32 arithmetic); a wall or
      // pass lane takes the constants that make the collision a bounce-back or
      // the identity.
      float2 g2[Q];
      static_for<0, Q>([&](auto i) { g2[i] = P::to_float2(raw[k][i]); });
      ScaledParams<float> lo = scaled_params<KIND>(pe_lo, MASKED && !g.uniform, bulk, lane_lo);
      ScaledParams<float> hi = scaled_params<KIND>(pe_hi, MASKED && !g.uniform, bulk, lane_hi);
      if constexpr (kForced) {
        if (field) {
          if (lane_lo == kLaneFluid) load_force(xp, lo.force);
          if (lane_hi == kLaneFluid) load_force(xp + (g.nx >> 1), hi.force);
        }
      }
      const ScaledParams<float2> q2 = zip_params(lo, hi);
      float2 r2, u22;
      collide_scaled<L, KIND>(g2, q2, r2, u22);
      static_for<0, Q>([&](auto i) { raw[k][i] = P::from_float2(g2[i]); });
      if constexpr (STATS) {
        if (lane_lo == kLaneFluid) acc.add(double(r2.x), double(u22.x));
        if (lane_hi == kLaneFluid) acc.add(double(r2.y), double(u22.y));
      }
    } else
#endif
    {
    // One cell after the other (a pair with a wall or boundary cell, and the
    // exact build).  BGK and TRT cells collide on g directly (collide_scaled);
    // any other dynamics decodes f_i = g_i / s_i, collides and re-encodes.
    // s_i of a population equals that of its opposite, so the column read or
    // written (i or opp(i)) does not change the scale.
    // the low cell's results wait in packed pairs of populations (half the
    // registers); the high cell's are packed the same way and the two are
    // merged with one byte permutation per population
    constexpr int QP = (Q + 1) / 2;
    T lo_pack[QP];
    auto cell = [&](auto half_tag, int kind, const DynDevice<float>* pe) {
      constexpr bool HI = decltype(half_tag)::value;
      const int x = HI ? xp + (g.nx >> 1) : xp;
      float gout[Q];
      static_for<0, Q>([&](auto i) {
        const float2 fv = P::to_float2(raw[k][i]);
        gout[i] = HI ? fv.y : fv.x;
      });
      float r = 0.f, u2 = 0.f;
      bool counted = false, done = false;
      float fcell[3] = {0.f, 0.f, 0.f};
      if constexpr (kForced) {
        if (field && (!MASKED || kind == KIND)) load_force(x, fcell);
      }
#ifndef OLB_B200_EXACT
      if (!MASKED || kind == KIND) {
        ScaledParams<float> q = scaled_params<KIND>(pe, MASKED && !g.uniform, bulk);
        if (field) {
          q.force[0] = fcell[0]; q.force[1] = fcell[1]; q.force[2] = fcell[2];
        }
        collide_scaled<L, KIND>(gout, q, r, u2);
        counted = true;
        done = true;
      }
#endif
      if (!done) {
        static_for<0, Q>([&](auto i) {
          constexpr float inv = 1.f / storage_scale<L>(i);
          gout[i] *= inv;
        });
        counted = collide_any<L, KIND, MASKED>(gout, kind, pe, bulk, fcell, field, g.uniform != 0, r, u2);
        static_for<0, Q>([&](auto i) {
          constexpr float sc = storage_scale<L>(i);
          gout[i] *= sc;
        });
      }
      static_for<0, QP>([&](auto jj) {
        constexpr int a = 2 * jj.value;
        constexpr int b = a + 1 < Q ? a + 1 : a;
        const T packed = P::from_floats(gout[a], gout[b]);
        if constexpr (!HI) {
          lo_pack[jj] = packed;
        } else {
          raw[k][a] = pair_perm(lo_pack[jj], packed, 0x5410u);
          if constexpr (a + 1 < Q) {
            raw[k][a + 1] = pair_perm(lo_pack[jj], packed, 0x7632u);
          }
        }
      });
      if constexpr (STATS) {
        if (counted) acc.add(double(r), double(u2));
      }
    };
    cell(std::integral_constant<bool, false>{}, kind_lo[k], pe_lo);
    cell(std::integral_constant<bool, true>{}, kind_hi[k], pe_hi);
    }
    // recomputed after the collision rather than kept live through it
    PairNeighbours nb(g, int(opaque(uint32_t(xp))), int(opaque(uint32_t(y))), int(opaque(uint32_t(z))));
    const uint32_t ps = opaque(pstride);
    const uint32_t ek = opaque(e[k]);
    static_for<0, Q>([&](auto i) {
      if constexpr (!ODD) {
        constexpr int o = L::opp(i);
        pops[uint32_t(o) * ps + ek] = raw[k][i];
      } else {
        const uint32_t dst = nb.template at<L::c(i, 0), L::c(i, 1), L::c(i, 2)>();
        T v = raw[k][i];
        if constexpr (L::c(i, 0) != 0) {
          v = pair_perm(v, v, nb.swap[1 + L::c(i, 0)] ? 0x1032u : 0x3210u);
        }
        pops[uint32_t(i.value) * ps + dst] = v;
      }
    });
  });
}

template <int Q, class S, int KIND, bool ODD, bool STATS, int CPT, int MINB>
__global__ void __launch_bounds__(kStepThreads, MINB)
aa_step_paired_kernel(S* __restrict__ pops, const Geometry g, const DynDevice<float> bulk,
                      StatPartial* __restrict__ partials)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y0 = blockIdx.y * (blockDim.y * CPT) + threadIdx.y;
  const int xp = blockIdx.z;
  const int none[CPT] = {};
  StatAcc acc;
  paired_tile<Q, S, KIND, ODD, false, STATS, CPT>(pops, g, nullptr, bulk, xp, y0, z, int(blockDim.y), none, none,
                                                 acc);
  if constexpr (STATS) {
    block_stats(acc.rho, acc.usqr, acc.max, acc.n, acc.nf, partials);
  }
}

// the masked paired kernel: one tile per block (aa_step_masked_kernel)
template <int Q, class S, int KIND, bool ODD, bool STATS, int CPT, int MINB>
__global__ void __launch_bounds__(kStepThreads, MINB)
aa_step_masked_paired_kernel(S* __restrict__ pops, const Geometry g, const uint8_t* __restrict__ ids,
                             const DynDevice<float>* __restrict__ table, const DynDevice<float> bulk,
                             StatPartial* __restrict__ partials)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y0 = blockIdx.y * (blockDim.y * CPT) + threadIdx.y;
  const int xp = blockIdx.z;
  const int dy = int(blockDim.y);
  int lo[CPT], hi[CPT];
  load_tile_ids(lo, g, ids, xp, y0, z, dy);
  load_tile_ids(hi, g, ids, xp + (g.nx >> 1), y0, z, dy);
  StatAcc acc;
  paired_tile<Q, S, KIND, ODD, true, STATS, CPT>(pops, g, table, bulk, xp, y0, z, dy, lo, hi, acc);
  if constexpr (STATS) {
    block_stats(acc.rho, acc.usqr, acc.max, acc.n, acc.nf, partials);
  }
}

// Deterministic second pass over the per-block partials (one block).
__global__ void reduce_partials_kernel(const StatPartial* __restrict__ parts, size_t count,
                                       StatPartial* __restrict__ out);

// ---------------------------------------------------------------------------
// logical-layout gather / scatter and moments

// Logical population i at cell (x,y,z): column i at the cell after an even
// number of steps, else column opp(i) at (x,y,z) - c_i (per-axis wrap).
template <int Q, class S, class R, int I>
OLB_DEV R logical_pop(const S* __restrict__ pops, const Geometry& g, int x, int y, int z, bool shifted)
{
  using L = Lattice<Q>;
  if (!shifted) {
    return Store<S, R>::template load<L, I>(pops + size_t(I) * g.stride + cell_slot(g, x, y, z));
  }
  constexpr int o = L::opp(I);
  const uint32_t src = cell_slot(g, wrap(x - L::c(I, 0), g.nx), wrap(y - L::c(I, 1), g.ny),
                                 wrap(z - L::c(I, 2), g.nz));
  return Store<S, R>::template load<L, o>(pops + size_t(o) * g.stride + src);
}

template <int Q, class S, class R>
__global__ void gather_logical_kernel(const S* __restrict__ pops, const Geometry g, bool shifted,
                                      R* __restrict__ out, int i_begin, int i_end)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= g.nz || y >= g.ny) return;
  const uint32_t n = (uint32_t(x) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z);
  const size_t cells = size_t(g.nx) * g.ny * g.nz;
  static_for<0, Q>([&](auto i) {
    if (i.value >= i_begin && i.value < i_end) {
      out[size_t(i.value - i_begin) * cells + n] = logical_pop<Q, S, R, i.value>(pops, g, x, y, z, shifted);
    }
  });
}

// write of logical populations in the unshifted order (resets the AA parity)
template <int Q, class S, class R>
__global__ void scatter_natural_kernel(S* __restrict__ pops, const Geometry g,
                                       const R* __restrict__ in, int i_begin, int i_end)
{
  using L = Lattice<Q>;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= g.nz || y >= g.ny) return;
  const uint32_t n = (uint32_t(x) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z);
  const size_t cells = size_t(g.nx) * g.ny * g.nz;
  const uint32_t slot = cell_slot(g, x, y, z);
  static_for<0, Q>([&](auto i) {
    if (i.value >= i_begin && i.value < i_end) {
      Store<S, R>::template store<L, i.value>(pops + size_t(i.value) * g.stride + slot,
                                              in[size_t(i.value - i_begin) * cells + n]);
    }
  });
}

// Cell::iniEquilibrium on every cell: the second-order equilibrium of the
// cell's density and velocity (equilibrium::secondOrder, src/dynamics/lbm.h:50-64,
// as the shifted value f_eq - w), written in the natural layout; rho_u holds
// rho of every cell, then u_x, u_y, u_z.
template <int Q, class S, class R>
__global__ void equilibrium_kernel(S* __restrict__ pops, const Geometry g, const R* __restrict__ rho_u)
{
  using L = Lattice<Q>;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= g.nz || y >= g.ny) return;
  const uint32_t n = (uint32_t(x) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z);
  const size_t cells = size_t(g.nx) * g.ny * g.nz;
  const uint32_t slot = cell_slot(g, x, y, z);
  const R rho = rho_u[n];
  const R u[3] = {rho_u[cells + n], rho_u[2 * cells + n], rho_u[3 * cells + n]};
  const R usqr = norm_sqr(u);
  static_for<0, Q>([&](auto i) {
    Store<S, R>::template store<L, i.value>(pops + size_t(i.value) * g.stride + slot,
                                            feq2<L, i.value>(rho, u, usqr));
  });
}

// FORCE of cell n of a Guo-forced dynamics: the lattice's force field when it
// has one, else the entry's constant
template <class R>
OLB_DEV void cell_force(const Geometry& g, const DynDevice<R>* e, uint32_t n, R (&gg)[3])
{
  if (g.force) {
    const R* F = static_cast<const R*>(g.force);
    gg[0] = F[n];
    gg[1] = F[size_t(g.stride) + n];
    gg[2] = F[2 * size_t(g.stride) + n];
  } else {
    gg[0] = e->force[0];
    gg[1] = e->force[1];
    gg[2] = e->force[2];
  }
}

// Density / velocity as the reference's Density3D / Velocity3D report them
// (per-dynamics momenta: src/dynamics/momenta/elements.h).
template <int Q, class S, class R>
__global__ void moments_kernel(const S* __restrict__ pops, const Geometry g, bool shifted,
                               const uint8_t* __restrict__ ids, const DynDevice<R>* __restrict__ table,
                               R* __restrict__ rho_out, R* __restrict__ u_out)
{
  using L = Lattice<Q>;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= g.nz || y >= g.ny) return;
  const uint32_t n = (uint32_t(x) * uint32_t(g.ny) + uint32_t(y)) * uint32_t(g.nz) + uint32_t(z);
  const size_t cells = size_t(g.nx) * g.ny * g.nz;
  const DynDevice<R>* p = table + (ids ? ids[n] : 0);
  const int kind = p->kind;
  R rho, u[3];
  if (kind == K_BGK || kind == K_TRT || kind == K_SMAGORINSKY || kind == K_FORCED_BGK ||
      kind == K_FORCED_TRT) {
    R f[Q];
    static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, x, y, z, shifted); });
    if (kind == K_FORCED_BGK || kind == K_FORCED_TRT) {
      R gg[3];
      cell_force(g, p, n, gg);
      compute_rho_u_forced<L>(f, gg, rho, u);
    } else {
      compute_rho_u<L>(f, rho, u);
    }
  } else if (kind == K_BOUNCE_BACK) {
    rho = p->wall_rho; u[0] = u[1] = u[2] = R(0);
  } else if (kind == K_BOUNCE_BACK_VELOCITY) {
    rho = p->wall_rho; u[0] = p->wall_u[0]; u[1] = p->wall_u[1]; u[2] = p->wall_u[2];
  } else if (is_interpolated(kind) || is_local(kind)) {
    R f[Q];
    static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, x, y, z, shifted); });
    bc_rho_u<L>(f, kind, p->bc_dir, p->bc_orient, p->bc_values + 4 * size_t(bc_index(p, x, y, z)), rho, u);
  } else if (is_inner(kind)) {
    // InnerEdge/CornerDensity3D + FixedVelocityMomentumGeneric
    R f[Q];
    static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, x, y, z, shifted); });
    const R* v = p->bc_values + 4 * size_t(bc_index(p, x, y, z));
    u[0] = v[1]; u[1] = v[2]; u[2] = v[3];
    const int32_t nn[3] = {p->nrm[0], p->nrm[1], p->nrm[2]};
    rho = inner_rho<L>(f, kind, nn, u);
  } else if (is_outer(kind)) {
    // BulkDensity + FixedVelocityMomentumGeneric
    R f[Q];
    static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, x, y, z, shifted); });
    rho = compute_rho<L>(f);
    const R* v = p->bc_values + 4 * size_t(bc_index(p, x, y, z));
    u[0] = v[1]; u[1] = v[2]; u[2] = v[3];
  } else {
    rho = R(1); u[0] = u[1] = u[2] = R(0);
  }
  rho_out[n] = rho;
  u_out[n] = u[0];
  u_out[cells + n] = u[1];
  u_out[2 * cells + n] = u[2];
}

// ---------------------------------------------------------------------------
// PostStream: PlaneFdBoundaryProcessor3D on the interpolated boundary cells
//
// src/boundary/boundaryPostProcessors3D.hh:39-92.  Each boundary cell is
// rebuilt from the post-stream state as feq(rho, u) + fneq(Pi), Pi from the
// finite-difference strain rate: one-sided second order along the normal
// (cells x - orient e and x - 2 orient e), central across it
// (fd::DirectedGradients3D, src/utilities/finiteDifference3D.h:58-200).
// Two passes: the first stores the velocity of every boundary cell (its
// momenta on the post-stream state), the second rebuilds every boundary cell;
// a boundary cell never reads another boundary cell's populations in the
// second pass, so the passes need no ordering among cells.

// Logical population I of cell (x,y,z) written back (inverse of logical_pop).
template <int Q, class S, class R, int I>
OLB_DEV void logical_store(S* __restrict__ pops, const Geometry& g, int x, int y, int z, bool shifted, R v)
{
  using L = Lattice<Q>;
  if (!shifted) {
    Store<S, R>::template store<L, I>(pops + size_t(I) * g.stride + cell_slot(g, x, y, z), v);
    return;
  }
  constexpr int o = L::opp(I);
  const uint32_t dst = cell_slot(g, wrap(x - L::c(I, 0), g.nx), wrap(y - L::c(I, 1), g.ny),
                                 wrap(z - L::c(I, 2), g.nz));
  Store<S, R>::template store<L, o>(pops + size_t(o) * g.stride + dst, v);
}

OLB_DEV void decode_cell(const Geometry& g, uint32_t n, int& x, int& y, int& z)
{
  const uint32_t nynz = uint32_t(g.ny) * uint32_t(g.nz);
  const uint32_t xx = n / nynz;
  const uint32_t r = n - xx * nynz;
  const uint32_t yy = r / uint32_t(g.nz);
  x = int(xx);
  y = int(yy);
  z = int(r - yy * uint32_t(g.nz));
}

// Cell::computeU through the cell's dynamics on the post-stream state: bulk
// (momenta/elements.h:466-475), forced bulk (:1480-1488), VELOCITY of moving
// walls, the stored velocity of interpolated cells, zero otherwise.  A cell
// beyond a non-periodic face is the reference's NoDynamics padding: zero.
template <int Q, class S, class R>
OLB_DEV void cell_velocity(const S* __restrict__ pops, const Geometry& g, bool shifted,
                           const uint8_t* __restrict__ ids, const DynDevice<R>* __restrict__ table,
                           int periodic, int x, int y, int z, R (&u)[3])
{
  using L = Lattice<Q>;
  u[0] = u[1] = u[2] = R(0);
  int p[3] = {x, y, z};
  const int ext[3] = {g.nx, g.ny, g.nz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (p[d] < 0 || p[d] >= ext[d]) {
      if (!((periodic >> d) & 1)) return;
      p[d] = p[d] < 0 ? p[d] + ext[d] : p[d] - ext[d];
    }
  }
  const uint32_t n = (uint32_t(p[0]) * uint32_t(g.ny) + uint32_t(p[1])) * uint32_t(g.nz) + uint32_t(p[2]);
  const DynDevice<R>* e = table + ids[n];
  const int kind = e->kind;
  if (kind == K_BGK || kind == K_TRT || kind == K_SMAGORINSKY || kind == K_FORCED_BGK || kind == K_FORCED_TRT) {
    R f[Q];
    static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, p[0], p[1], p[2], shifted); });
    R rho;
    if (kind == K_FORCED_BGK || kind == K_FORCED_TRT) {
      R gg[3];
      cell_force(g, e, n, gg);
      compute_rho_u_forced<L>(f, gg, rho, u);
    } else {
      compute_rho_u<L>(f, rho, u);
    }
  } else if (kind == K_BOUNCE_BACK_VELOCITY) {
    u[0] = e->wall_u[0]; u[1] = e->wall_u[1]; u[2] = e->wall_u[2];
  } else if (is_interpolated(kind)) {
    const R* bu = e->bc_u + 3 * size_t(bc_index(e, p[0], p[1], p[2]));
    u[0] = bu[0]; u[1] = bu[1]; u[2] = bu[2];
  } else if (kind == K_LOCAL_PRESSURE) {
    // FixedPressureMomentum::computeU: VELOCITY, the normal part from the populations
    R f[Q];
    static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, p[0], p[1], p[2], shifted); });
    R rho;
    bc_rho_u<L>(f, kind, e->bc_dir, e->bc_orient, e->bc_values + 4 * size_t(bc_index(e, p[0], p[1], p[2])), rho,
                u);
  } else if (kind == K_LOCAL_VELOCITY || is_outer(kind) || is_inner(kind)) {
    // FixedVelocityMomentumGeneric: the VELOCITY field
    const R* v = e->bc_values + 4 * size_t(bc_index(e, p[0], p[1], p[2]));
    u[0] = v[1]; u[1] = v[2]; u[2] = v[3];
  }
}

// Cell::computeRho through the cell's dynamics on the current state:
// BulkDensity (fluid, external edges and corners), velocityBMRho (flat velocity
// boundaries), FixedDensity RHO (walls, pressure boundaries), 1 for NoDynamics
// and for the reference's padding beyond a non-periodic face.
template <int Q, class S, class R>
OLB_DEV R cell_density(const S* __restrict__ pops, const Geometry& g, bool shifted,
                       const uint8_t* __restrict__ ids, const DynDevice<R>* __restrict__ table, int periodic,
                       int x, int y, int z)
{
  using L = Lattice<Q>;
  int p[3] = {x, y, z};
  const int ext[3] = {g.nx, g.ny, g.nz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (p[d] < 0 || p[d] >= ext[d]) {
      if (!((periodic >> d) & 1)) return R(1);
      p[d] = p[d] < 0 ? p[d] + ext[d] : p[d] - ext[d];
    }
  }
  const uint32_t n = (uint32_t(p[0]) * uint32_t(g.ny) + uint32_t(p[1])) * uint32_t(g.nz) + uint32_t(p[2]);
  const DynDevice<R>* e = table + ids[n];
  const int kind = e->kind;
  if (kind == K_BOUNCE_BACK || kind == K_BOUNCE_BACK_VELOCITY) return e->wall_rho;
  if (kind == K_NONE) return R(1);
  R f[Q];
  static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, p[0], p[1], p[2], shifted); });
  if (is_interpolated(kind) || is_local(kind)) {
    R rho, u[3];
    bc_rho_u<L>(f, kind, e->bc_dir, e->bc_orient, e->bc_values + 4 * size_t(bc_index(e, p[0], p[1], p[2])), rho,
                u);
    return rho;
  }
  if (is_inner(kind)) {
    const R* v = e->bc_values + 4 * size_t(bc_index(e, p[0], p[1], p[2]));
    const R u[3] = {v[1], v[2], v[3]};
    const int32_t nn[3] = {e->nrm[0], e->nrm[1], e->nrm[2]};
    return inner_rho<L>(f, kind, nn, u);
  }
  return compute_rho<L>(f);
}

// pass 1: velocity of every interpolated cell (its momenta, post-stream state)
template <int Q, class S, class R>
__global__ void bc_velocity_kernel(const S* __restrict__ pops, const Geometry g, bool shifted,
                                   const uint8_t* __restrict__ ids, const DynDevice<R>* __restrict__ table,
                                   const uint32_t* __restrict__ cells, uint32_t count)
{
  using L = Lattice<Q>;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint32_t n = cells[k];
  int x, y, z;
  decode_cell(g, n, x, y, z);
  const DynDevice<R>* e = table + ids[n];
  const uint32_t bi = bc_index(e, x, y, z);
  R f[Q];
  static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, x, y, z, shifted); });
  R rho, u[3];
  bc_rho_u<L>(f, e->kind, e->bc_dir, e->bc_orient, e->bc_values + 4 * size_t(bi), rho, u);
  R* bu = e->bc_u + 3 * size_t(bi);
  bu[0] = u[0];
  bu[1] = u[1];
  bu[2] = u[2];
}

// pass 2: PlaneFdBoundaryProcessor3D<direction,orientation>::apply
template <int Q, class S, class R>
__global__ void plane_fd_kernel(S* __restrict__ pops, const Geometry g, bool shifted,
                                const uint8_t* __restrict__ ids, const DynDevice<R>* __restrict__ table,
                                int periodic, const uint32_t* __restrict__ cells, uint32_t count)
{
  using L = Lattice<Q>;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint32_t n = cells[k];
  int x, y, z;
  decode_cell(g, n, x, y, z);
  const DynDevice<R>* e = table + ids[n];
  const int dir = e->bc_dir, orient = e->bc_orient;
  R f[Q];
  static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, x, y, z, shifted); });
  R rho, u[3];
  bc_rho_u<L>(f, e->kind, dir, orient, e->bc_values + 4 * size_t(bc_index(e, x, y, z)), rho, u);
  // grad[d][c]: derivative along axis d of velocity component c
  R grad[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int ex = d == 0, ey = d == 1, ez = d == 2;
    if (d == dir) {
      const int s = -orient;
      R u1[3], u2[3];
      cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x + s * ex, y + s * ey, z + s * ez, u1);
      cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x + 2 * s * ex, y + 2 * s * ey,
                             z + 2 * s * ez, u2);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        grad[d][c] = R(-orient) * ((-R(3) * u[c] + R(4) * u1[c] - R(1) * u2[c]) / R(2));
      }
    } else {
      R up[3], um[3];
      cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x + ex, y + ey, z + ez, up);
      cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x - ex, y - ey, z - ez, um);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        grad[d][c] = (up[c] - um[c]) / R(2);
      }
    }
  }
  const R s_to_pi = -rho / R(3) / e->omega;
  R pi[6];
  pi[0] = R(2) * grad[0][0] * s_to_pi;
  pi[3] = R(2) * grad[1][1] * s_to_pi;
  pi[5] = R(2) * grad[2][2] * s_to_pi;
  pi[1] = (grad[0][1] + grad[1][0]) * s_to_pi;
  pi[2] = (grad[0][2] + grad[2][0]) * s_to_pi;
  pi[4] = (grad[1][2] + grad[2][1]) * s_to_pi;
  const R usqr = norm_sqr(u);
  static_for<0, Q>([&](auto i) {
    const R v = feq2<L, i.value>(rho, u, usqr) + from_pi_to_fneq<L, i.value>(pi);
    logical_store<Q, S, R, i.value>(pops, g, x, y, z, shifted, v);
  });
}

// Collision of the boundary cells that carry values (interpolated, local
// velocity, external edges and corners), in place, ahead of the step kernel.
// Each cell's populations are read where the step kernel will read them
// (the current AA parity) and written back there, so the step kernel, which
// passes these cells through, streams the collided values.  Keeping the
// boundary collisions out of the step kernel leaves its register allocation
// to the bulk collision: inlined, they raised the register demand of every
// cell and the masked kernels spilled.  Statistics of the boundary cells go
// to the partials after the step kernel's blocks.
template <int Q, class S, class R, int KIND, bool STATS>
__global__ void boundary_collide_kernel(S* __restrict__ pops, const Geometry g, bool shifted,
                                        const uint8_t* __restrict__ ids, const DynDevice<R>* __restrict__ table,
                                        const uint32_t* __restrict__ cells, uint32_t count,
                                        StatPartial* __restrict__ partials)
{
  using L = Lattice<Q>;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  double s_rho = 0., s_usqr = 0., s_max = 0.;
  unsigned long long s_n = 0, s_nf = 0;
  if (k < count) {
    const uint32_t n = cells[k];
    int x, y, z;
    decode_cell(g, n, x, y, z);
    const DynDevice<R>* e = table + ids[n];
    R f[Q];
    static_for<0, Q>([&](auto i) { f[i] = logical_pop<Q, S, R, i.value>(pops, g, x, y, z, shifted); });
    R st_rho = R(0), st_usqr = R(0);
    collide_boundary<L, KIND>(f, e->kind, e, x, y, z, st_rho, st_usqr);
    static_for<0, Q>([&](auto i) { logical_store<Q, S, R, i.value>(pops, g, x, y, z, shifted, f[i]); });
    if constexpr (STATS) {
      const double r = double(st_rho), u2 = double(st_usqr);
      if (isfinite(r) && isfinite(u2)) {
        s_rho = r; s_usqr = u2; s_max = u2; s_n = 1;
      } else {
        s_nf = 1;
      }
    }
  }
  if constexpr (STATS) {
    block_stats(s_rho, s_usqr, s_max, s_n, s_nf, partials);
  }
}

// OuterVelocityEdgeProcessor3D<plane,normal1,normal2>::apply (pass 3) and
// OuterVelocityCornerProcessor3D<xN,yN,zN>::apply (pass 4),
// src/boundary/boundaryPostProcessors3D.hh:164-292: the density extrapolated
// from the cells inward along the normal(s), velocity gradients one-sided
// across the boundary and central along an edge, the cell rebuilt as
// feq(rho, VELOCITY) + fneq(Pi).  The corner pass runs after the edge pass
// (priority 1 after 0): a corner's density reads the edge cells it ends.
template <int Q, class S, class R, bool CORNER>
__global__ void outer_velocity_kernel(S* __restrict__ pops, const Geometry g, bool shifted,
                                      const uint8_t* __restrict__ ids, const DynDevice<R>* __restrict__ table,
                                      int periodic, const uint32_t* __restrict__ cells, uint32_t count)
{
  using L = Lattice<Q>;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint32_t n = cells[k];
  int x, y, z;
  decode_cell(g, n, x, y, z);
  const DynDevice<R>* e = table + ids[n];
  const int nrm[3] = {e->nrm[0], e->nrm[1], e->nrm[2]};
  const R* v = e->bc_values + 4 * size_t(bc_index(e, x, y, z));
  const R u[3] = {v[1], v[2], v[3]};
  R rho;
  R grad[3][3];  // grad[d][c]: derivative along axis d of velocity component c
  if constexpr (!CORNER) {
    const int plane = nrm[0] == 0 ? 0 : (nrm[1] == 0 ? 1 : 2);
    const int d1 = plane == 2 ? 0 : plane + 1, d2 = plane == 0 ? 2 : (plane == 1 ? 0 : 1);
    // getNeighborRho(step1, step2): offset -normal1 step1 along d1, -normal2 step2 along d2
    R r[4];  // rho10, rho01, rho20, rho02
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int s1 = m == 0 ? 1 : (m == 2 ? 2 : 0), s2 = m == 1 ? 1 : (m == 3 ? 2 : 0);
      int o[3] = {0, 0, 0};
      o[d1] = -nrm[d1] * s1;
      o[d2] = -nrm[d2] * s2;
      r[m] = cell_density<Q, S, R>(pops, g, shifted, ids, table, periodic, x + o[0], y + o[1], z + o[2]);
    }
    rho = R(2) / R(3) * (r[1] + r[0]) - R(1) / R(6) * (r[3] + r[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int ex = d == 0, ey = d == 1, ez = d == 2;
      if (d == plane) {
        R up[3], um[3];
        cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x + ex, y + ey, z + ez, up);
        cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x - ex, y - ey, z - ez, um);
#pragma unroll
        for (int c = 0; c < 3; ++c) grad[d][c] = (up[c] - um[c]) / R(2);
      } else {
        const int s = -nrm[d];
        R u1[3], u2[3];
        cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x + s * ex, y + s * ey, z + s * ez, u1);
        cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x + 2 * s * ex, y + 2 * s * ey,
                               z + 2 * s * ez, u2);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          grad[d][c] = R(-nrm[d]) * ((-R(3) * u[c] + R(4) * u1[c] - R(1) * u2[c]) / R(2));
        }
      }
    }
  } else {
    R r[6];  // rho100, rho010, rho001, rho200, rho020, rho002
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      int o[3] = {0, 0, 0};
      o[m % 3] = -(m / 3 + 1) * nrm[m % 3];
      r[m] = cell_density<Q, S, R>(pops, g, shifted, ids, table, periodic, x + o[0], y + o[1], z + o[2]);
    }
    rho = R(4) / R(9) * (r[2] + r[1] + r[0]) - R(1) / R(9) * (r[5] + r[4] + r[3]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int ex = d == 0, ey = d == 1, ez = d == 2;
      const int s = -nrm[d];
      R u1[3], u2[3];
      cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x + s * ex, y + s * ey, z + s * ez, u1);
      cell_velocity<Q, S, R>(pops, g, shifted, ids, table, periodic, x + 2 * s * ex, y + 2 * s * ey,
                             z + 2 * s * ez, u2);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        grad[d][c] = R(-nrm[d]) * ((-R(3) * u[c] + R(4) * u1[c] - R(1) * u2[c]) / R(2));
      }
    }
  }
  const R s_to_pi = -rho / R(3) / e->omega;
  R pi[6];
  pi[0] = R(2) * grad[0][0] * s_to_pi;
  pi[3] = R(2) * grad[1][1] * s_to_pi;
  pi[5] = R(2) * grad[2][2] * s_to_pi;
  pi[1] = (grad[0][1] + grad[1][0]) * s_to_pi;
  pi[2] = (grad[0][2] + grad[2][0]) * s_to_pi;
  pi[4] = (grad[1][2] + grad[2][1]) * s_to_pi;
  const R usqr = norm_sqr(u);
  static_for<0, Q>([&](auto i) {
    const R val = feq2<L, i.value>(rho, u, usqr) + from_pi_to_fneq<L, i.value>(pi);
    logical_store<Q, S, R, i.value>(pops, g, x, y, z, shifted, val);
  });
}

// ---------------------------------------------------------------------------
// host-side launch entry points (explicitly instantiated per lattice/storage)

struct StepLaunch {
  void* pops;
  Geometry g;
  const uint8_t* ids;      // device, or nullptr
  const void* table;       // device DynDevice<R>[]
  const void* bulk;        // host DynDevice<R>
  StatPartial* partials;   // device, gridDim product entries
  int block_z, block_y;
  int variant;             // index into kStepVariants
  cudaStream_t stream;
};

template <int Q, class S, class R>
cudaError_t launch_step(const StepLaunch& a, int kind, bool odd, bool masked, bool stats);

template <int Q, class S, class R>
cudaError_t launch_gather(const void* pops, const Geometry& g, bool shifted, void* out, int i_begin,
                          int i_end, cudaStream_t stream);

template <int Q, class S, class R>
cudaError_t launch_scatter(void* pops, const Geometry& g, const void* in, int i_begin, int i_end,
                           cudaStream_t stream);

// every cell's populations from its density and velocity (rho_u: 4 columns of R)
template <int Q, class S, class R>
cudaError_t launch_equilibrium(void* pops, const Geometry& g, const void* rho_u, cudaStream_t stream);

template <int Q, class S, class R>
cudaError_t launch_moments(const void* pops, const Geometry& g, bool shifted, const uint8_t* ids,
                           const void* table, void* rho, void* u, cudaStream_t stream);

// the boundary pre-pass over `count` cells; partials == nullptr: no statistics
template <int Q, class S, class R>
cudaError_t launch_boundary_collide(void* pops, const Geometry& g, bool shifted, const uint8_t* ids,
                                    const void* table, int kind, const uint32_t* cells, uint32_t count,
                                    StatPartial* partials, cudaStream_t stream);
constexpr int kBoundaryThreads = 128;

// the PostStream passes: cells[0, n_flat) are the interpolated flat cells
// (velocity pass, then PlaneFd), the next n_edge the external edge cells,
// the last n_corner the external corner cells
template <int Q, class S, class R>
cudaError_t launch_boundary(void* pops, const Geometry& g, bool shifted, const uint8_t* ids, const void* table,
                            int periodic, const uint32_t* cells, uint32_t n_flat, uint32_t n_edge,
                            uint32_t n_corner, cudaStream_t stream);

inline dim3 step_grid(const Geometry& g, int bz, int by, int cells_per_thread)
{
  const int rows = by * cells_per_thread;
  return dim3((g.nz + bz - 1) / bz, (g.ny + rows - 1) / rows, g.paired ? g.nx / 2 : g.nx);
}

// grid of the gather / moments kernels (one cell per thread)
inline dim3 cell_grid(const Geometry& g, int bz, int by)
{
  return dim3((g.nz + bz - 1) / bz, (g.ny + by - 1) / by, g.nx);
}

} // namespace olb_b200
