// C ABI of the B200-native collide-and-stream (declared in include/olb_b200.h).
//
// The handle owns: the population columns (AA layout, one array), the per-cell
// dynamics ids, the device dynamics table, a staging buffer for logical-layout
// transfers, the per-block statistics partials and one non-blocking stream.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/olb_b200.h"
#include "aa_kernels.cuh"

namespace olb_b200 {

// explicit instantiations live in step_q{19,27}_{f32,f64,f16,bf16}.cu
#define OLB_B200_EXTERN(Q, S, R)                                                                   \
  extern template cudaError_t launch_step<Q, S, R>(const StepLaunch&, int, bool, bool, bool);      \
  extern template cudaError_t launch_gather<Q, S, R>(const void*, const Geometry&, bool, void*,    \
                                                     int, int, cudaStream_t);                      \
  extern template cudaError_t launch_scatter<Q, S, R>(void*, const Geometry&, const void*, int,    \
                                                      int, cudaStream_t);                          \
  extern template cudaError_t launch_equilibrium<Q, S, R>(void*, const Geometry&, const void*,    \
                                                          cudaStream_t);                           \
  extern template cudaError_t launch_moments<Q, S, R>(const void*, const Geometry&, bool,          \
                                                      const uint8_t*, const void*, void*, void*,   \
                                                      cudaStream_t);                               \
  extern template cudaError_t launch_boundary_collide<Q, S, R>(void*, const Geometry&, bool,       \
                                                               const uint8_t*, const void*, int,   \
                                                               const uint32_t*, uint32_t,          \
                                                               StatPartial*, cudaStream_t);        \
  extern template cudaError_t launch_boundary<Q, S, R>(void*, const Geometry&, bool, const uint8_t*, \
                                                       const void*, int, const uint32_t*, uint32_t, \
                                                       uint32_t, uint32_t, cudaStream_t);
OLB_B200_EXTERN(19, float, float)
OLB_B200_EXTERN(19, double, double)
OLB_B200_EXTERN(19, __half, float)
OLB_B200_EXTERN(19, __nv_bfloat16, float)
OLB_B200_EXTERN(27, float, float)
OLB_B200_EXTERN(27, double, double)
OLB_B200_EXTERN(27, __half, float)
OLB_B200_EXTERN(27, __nv_bfloat16, float)

__global__ void reduce_partials_kernel(const StatPartial* __restrict__ parts, size_t count,
                                       StatPartial* __restrict__ out)
{
  // fixed assignment of partials to threads and a fixed tree: deterministic
  double a = 0., b = 0., m = 0.;
  unsigned long long n = 0, nf = 0;
  for (size_t k = threadIdx.x; k < count; k += blockDim.x) {
    const StatPartial p = parts[k];
    a += p.sum_rho;
    b += p.sum_usqr;
    m = fmax(m, p.max_usqr);
    n += p.n_cells;
    nf += p.n_nonfinite;
  }
  __shared__ StatPartial sh[32];
  warp_reduce(a, b, m, n, nf);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = StatPartial{a, b, m, n, nf};
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    StatPartial p = lane < nw ? sh[lane] : StatPartial{0, 0, 0, 0, 0};
    warp_reduce(p.sum_rho, p.sum_usqr, p.max_usqr, p.n_cells, p.n_nonfinite);
    if (lane == 0) *out = p;
  }
}

// velocity-change residual sums over the fluid cells; stores u as u_prev
template <class R>
__global__ void velocity_residual_kernel(const R* __restrict__ u_now, R* __restrict__ u_prev,
                                         const uint8_t* __restrict__ ids,
                                         const DynDevice<R>* __restrict__ table, size_t cells,
                                         StatPartial* __restrict__ partials)
{
  const size_t n = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  double du2 = 0., u2 = 0.;
  if (n < cells) {
    const int kind = table[ids ? ids[n] : 0].kind;
    if (kind == K_BGK || kind == K_TRT || kind == K_SMAGORINSKY || kind == K_FORCED_BGK ||
        kind == K_FORCED_TRT) {
      for (int d = 0; d < 3; ++d) {
        const R u = u_now[d * cells + n];
        const double du = double(u) - double(u_prev[d * cells + n]);
        du2 += du * du;
        u2 += double(u) * double(u);
        u_prev[d * cells + n] = u;
      }
    }
  }
  block_stats(du2, u2, 0., 0ull, 0ull, partials);
}

// splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): a counter-based uniform variate per key
OLB_HD uint64_t splitmix64(uint64_t x)
{
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Inlet fluctuations of step `step`: VELOCITY_d = base_d + amp |base| (2 r - 1)
// on every interpolated velocity cell, r = splitmix64(seed + (step*cells +
// cell)*3 + d) / 2^64 (53 bits).  Runs before the step's collision, so the
// collision and the PostStream pass of that step see the same values.
template <class R>
__global__ void bc_noise_kernel(const uint32_t* __restrict__ cells, uint32_t count,
                                const uint8_t* __restrict__ ids, const DynDevice<R>* __restrict__ table,
                                const R* __restrict__ base_all, R* __restrict__ values_all, Geometry g,
                                uint64_t step, uint64_t n_cells, double amp, uint64_t seed)
{
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint32_t n = cells[k];
  const DynDevice<R>* e = table + ids[n];
  if (e->kind != K_INTERP_VELOCITY) return;
  int x, y, z;
  decode_cell(g, n, x, y, z);
  const size_t slot = size_t(e->bc_values - static_cast<const R*>(values_all)) / 4 + bc_index(e, x, y, z);
  const R* b = base_all + 4 * slot;
  R* v = values_all + 4 * slot;
  const double bu[3] = {double(b[1]), double(b[2]), double(b[3])};
  const double mag = sqrt(bu[0] * bu[0] + bu[1] * bu[1] + bu[2] * bu[2]);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const uint64_t key = seed + (step * n_cells + n) * 3u + uint64_t(d);
    const double r = double(splitmix64(key) >> 11) * 0x1.0p-53;
    v[1 + d] = R(bu[d] + amp * mag * (2.0 * r - 1.0));
  }
}

} // namespace olb_b200

using namespace olb_b200;

namespace {

thread_local std::string g_last_error;

olb_b200_status fail(olb_b200_status code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

olb_b200_status cuda_fail(cudaError_t e, const char* what)
{
  return fail(e == cudaErrorMemoryAllocation ? OLB_B200_ERR_OOM : OLB_B200_ERR_CUDA, "%s: %s (%s)",
              what, cudaGetErrorString(e), cudaGetErrorName(e));
}

#define OLB_CUDA(call)                                                                             \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);                                            \
  } while (0)

bool is_fluid(int kind)
{
  return kind == K_BGK || kind == K_TRT || kind == K_SMAGORINSKY || kind == K_FORCED_BGK ||
         kind == K_FORCED_TRT;
}

template <class R>
DynDevice<R> make_device_params(int q, const olb_b200_dyn_params& in)
{
  // Cell-independent parts of each collision, evaluated in R with the
  // reference's operation order (the host compiler does not contract).
  DynDevice<R> d;
  std::memset(&d, 0, sizeof d);
  d.kind = in.kind;
  const R omega = R(in.omega);
  const R magic = R(in.magic);
  d.omega = omega;
  // collision::TRT  src/dynamics/collision.h:239 (double expression, rounded once)
  d.omega_minus = R(double(R(1)) / (double(magic) / (double(R(1) / omega) - 0.5) + double(R(0.5))));
  // detail::SmagorinskyEffectiveOmega  src/dynamics/collisionLES.h:67-71
  const R s = R(in.smagorinsky);
  R pre = s * s;
  pre = pre * R(3);
  pre = pre * R(3);
  pre = pre * R(2);
  d.smago_pre = R(double(pre) * std::sqrt(2.0));
  d.tau_mol = R(1) / omega;
  for (int e = 0; e < 3; ++e) {
    d.force[e] = R(in.force[e]);
    d.wall_u[e] = R(in.wall_u[e]);
  }
  // lbm::addExternalForce  src/dynamics/lbm.h:562
  d.force_relax = R(1) - omega * R(0.5);
  d.wall_rho = R(in.wall_rho);
  // collision::NguyenLaddCorrection  src/dynamics/collision.h:341-343
  for (int i = 0; i < q; ++i) {
    int c[3];
    R w;
    if (q == 19) {
      for (int e = 0; e < 3; ++e) c[e] = Lattice<19>::c(i, e);
      w = R(Lattice<19>::wnum(i)) / R(Lattice<19>::wden(i));
    } else {
      for (int e = 0; e < 3; ++e) c[e] = Lattice<27>::c(i, e);
      w = R(Lattice<27>::wnum(i)) / R(Lattice<27>::wden(i));
    }
    for (int e = 0; e < 3; ++e) {
      R t = R(2) * d.wall_rho;
      t = t * d.wall_u[e];
      t = t * R(c[e]);
      t = t * w;
      t = t * R(3);
      d.wall_term[i][e] = t;
    }
  }
  return d;
}

} // namespace

namespace olb_b200 {
namespace detail {
// entry points for other translation units of the library
DynDevice<float> device_params_f32(int q, const olb_b200_dyn_params& in) { return make_device_params<float>(q, in); }
DynDevice<double> device_params_f64(int q, const olb_b200_dyn_params& in) { return make_device_params<double>(q, in); }
bool fluid_kind(int kind) { return is_fluid(kind); }
void set_last_error(const std::string& message) { g_last_error = message; }
} // namespace detail
} // namespace olb_b200

struct olb_b200_lattice {
  olb_b200_desc desc{};
  int q = 19;
  size_t cells = 0;
  size_t stride = 0;
  size_t elem = 4;          // storage element size
  size_t real = 4;          // compute element size (ABI element)
  int device = 0;
  Geometry g{};
  void* pops = nullptr;
  uint8_t* ids = nullptr;   // device, n bytes (masked lattices only)
  void* table = nullptr;    // device DynDevice<R>[256]
  alignas(16) unsigned char bulk[sizeof(DynDevice<double>)];  // host DynDevice<R>
  int bulk_kind = K_BGK;
  bool masked = true;
  int n_entries = 0;
  int parity = 0;           // 1 after an odd number of steps (shifted layout)
  int64_t steps_done = 0;
  void* scratch = nullptr;  // staging, 4 * cells * real bytes
  StatPartial* partials = nullptr;
  size_t n_partials = 0;
  void* uprev = nullptr;    // velocity at the last residual call (3 * cells * real)
  StatPartial* stat_dev = nullptr;
  StatPartial* stat_host = nullptr;  // pinned
  int block_z = 0, block_y = 0;
  int variant = 0;          // index into kStepVariants
  void* force = nullptr;    // FORCE per cell, 3 columns of `stride` R (olb_b200_set_force_field)
  bool tuned = false;       // variant and shape chosen by olb_b200_autotune
  float tuned_ms = 0.f;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  size_t device_bytes = 0;
  // interpolated velocity / pressure boundaries
  struct BcBox {
    int box[6];             // x0, y0, z0, extents (0 extents: not a boundary entry)
    size_t slot0;           // first value slot
  };
  std::vector<BcBox> bc_box;        // per table entry
  std::vector<uint8_t> ids_host;    // per cell (kept while boundary entries exist)
  std::vector<double> bc_host;      // 4 values per slot, host copy
  uint32_t* bc_cells = nullptr;     // device: flat interpolated, then edge, then corner cells
  uint32_t n_bc = 0;                // cells in bc_cells
  uint32_t n_bc_flat = 0, n_bc_edge = 0, n_bc_corner = 0;  // PostStream segments; local faces follow
  void* bc_values = nullptr;        // device: 4 R per slot
  void* bc_u = nullptr;             // device: 3 R per slot
  size_t bc_slots = 0;
  size_t bc_bytes = 0;
  void* bc_base = nullptr;          // device: 4 R per slot, the values before fluctuations
  double noise_amp = 0.0;           // inlet fluctuations (olb_b200_set_boundary_noise)
  uint64_t noise_seed = 0;
  bool initialized = false;         // PostStream post-processors applied to the initial state
  // bounded pipeline of collide_and_stream calls (olb_b200_set_max_steps_in_flight)
  std::vector<cudaEvent_t> flight;  // ring: event after the call k - flight.size()
  std::vector<bool> flight_used;
  size_t flight_pos = 0;
};

namespace {

olb_b200_status select_device(olb_b200_lattice* L)
{
  OLB_CUDA(cudaSetDevice(L->device));
  return OLB_B200_OK;
}

void default_shape(const olb_b200_lattice* L, int& bz, int& by)
{
  // 256 threads: a full z-row segment per warp; rows stacked along y
  bz = L->desc.nz >= 128 ? 128 : (L->desc.nz >= 64 ? 64 : 32);
  by = 256 / bz;
}

// Default step variant per lattice class, from a 256^3 sweep on B200 (the
// autotuner refines it on the actual lattice): masked lattices and 16-bit
// storage keep one cell per thread at high occupancy; FP64 and unmasked
// FP32 lattices issue the loads of two cells per thread.
int default_variant(const olb_b200_lattice* L)
{
  const int storage = L->desc.storage;
  // 16-bit: D3Q19's two-lane collision fits the 64-register cap of {1,4};
  // D3Q27's needs the 80 registers of {1,3}
  if (storage == OLB_B200_STORAGE_F16 || storage == OLB_B200_STORAGE_BF16) return L->q == 27 ? 0 : 1;
  if (L->masked) return storage == OLB_B200_STORAGE_F64 ? 0 : 1;                  // {1,3} / {1,4}
  if (storage == OLB_B200_STORAGE_F64) return 2;                                     // {2,2}
  return 3;                                                                          // {2,3}
}

int cells_per_thread(const olb_b200_lattice* L) { return kStepVariants[L->variant].cells_per_thread; }

template <class F>
cudaError_t dispatch(const olb_b200_lattice* L, F&& f)
{
  switch (L->desc.storage) {
  case OLB_B200_STORAGE_F32:
    return L->q == 19 ? f(std::integral_constant<int, 19>{}, float{}, float{})
                      : f(std::integral_constant<int, 27>{}, float{}, float{});
  case OLB_B200_STORAGE_F64:
    return L->q == 19 ? f(std::integral_constant<int, 19>{}, double{}, double{})
                      : f(std::integral_constant<int, 27>{}, double{}, double{});
  case OLB_B200_STORAGE_F16:
    return L->q == 19 ? f(std::integral_constant<int, 19>{}, __half{}, float{})
                      : f(std::integral_constant<int, 27>{}, __half{}, float{});
  case OLB_B200_STORAGE_BF16:
    return L->q == 19 ? f(std::integral_constant<int, 19>{}, __nv_bfloat16{}, float{})
                      : f(std::integral_constant<int, 27>{}, __nv_bfloat16{}, float{});
  }
  return cudaErrorInvalidValue;
}

olb_b200_status ensure_partial_count(olb_b200_lattice* L, size_t need);

// blocks of the boundary collision pre-pass (their statistics follow the step kernel's)
size_t boundary_blocks(const olb_b200_lattice* L)
{
  return (size_t(L->n_bc) + kBoundaryThreads - 1) / kBoundaryThreads;
}

size_t step_blocks(const olb_b200_lattice* L)
{
  const dim3 grid = step_grid(L->g, L->block_z, L->block_y, cells_per_thread(L));
  return size_t(grid.x) * grid.y * grid.z;
}

// The bulk box of a masked lattice: a box all of whose cells use the bulk
// entry, so the step kernel loads no dynamics id for them.  The box starts as
// the whole lattice and loses any face layer that holds another entry until
// no face does (for a lattice with walls on its faces, such as the lid-driven
// cavity, that is the interior).  If the box's interior still holds other
// entries (an obstacle inside, such as a cylinder in a channel), the box
// becomes the largest of the six slabs of it beside the obstacles' bounding
// box that holds the bulk entry only, if any.
void compute_bulk_box(olb_b200_lattice* L, const uint8_t* ids, int bulk_entry)
{
  Geometry& g = L->g;
  for (int d = 0; d < 3; ++d) g.bulk_lo[d] = g.bulk_hi[d] = 0;
  if (!ids || bulk_entry < 0) return;
  const int n[3] = {L->desc.nx, L->desc.ny, L->desc.nz};
  auto id_at = [&](int x, int y, int z) { return int(ids[(size_t(x) * n[1] + y) * n[2] + z]); };
  int lo[3] = {0, 0, 0}, hi[3] = {n[0], n[1], n[2]};
  auto face_clean = [&](int axis, int layer) {
    int a[3], b[3];
    for (int d = 0; d < 3; ++d) { a[d] = lo[d]; b[d] = hi[d]; }
    a[axis] = layer;
    b[axis] = layer + 1;
    for (int x = a[0]; x < b[0]; ++x)
      for (int y = a[1]; y < b[1]; ++y)
        for (int z = a[2]; z < b[2]; ++z)
          if (id_at(x, y, z) != bulk_entry) return false;
    return true;
  };
  for (bool changed = true; changed;) {
    changed = false;
    for (int d = 0; d < 3 && lo[0] < hi[0] && lo[1] < hi[1] && lo[2] < hi[2]; ++d) {
      if (!face_clean(d, lo[d])) { ++lo[d]; changed = true; }
      if (lo[d] < hi[d] && !face_clean(d, hi[d] - 1)) { --hi[d]; changed = true; }
    }
    if (!(lo[0] < hi[0] && lo[1] < hi[1] && lo[2] < hi[2])) return;
  }
  // the bounding box of the other entries inside the box
  int olo[3] = {hi[0], hi[1], hi[2]}, ohi[3] = {lo[0] - 1, lo[1] - 1, lo[2] - 1};
  for (int x = lo[0]; x < hi[0]; ++x)
    for (int y = lo[1]; y < hi[1]; ++y)
      for (int z = lo[2]; z < hi[2]; ++z)
        if (id_at(x, y, z) != bulk_entry) {
          const int p[3] = {x, y, z};
          for (int d = 0; d < 3; ++d) {
            olo[d] = std::min(olo[d], p[d]);
            ohi[d] = std::max(ohi[d], p[d]);
          }
        }
  if (ohi[0] >= lo[0]) {
    // six slabs beside the obstacles: below olo[d] or above ohi[d] along axis d
    size_t best = 0;
    int blo[3] = {0, 0, 0}, bhi[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d) {
      for (int side = 0; side < 2; ++side) {
        int a[3] = {lo[0], lo[1], lo[2]}, b[3] = {hi[0], hi[1], hi[2]};
        if (side == 0) b[d] = olo[d]; else a[d] = ohi[d] + 1;
        if (!(a[d] < b[d])) continue;
        const size_t vol = size_t(b[0] - a[0]) * size_t(b[1] - a[1]) * size_t(b[2] - a[2]);
        if (vol > best) {
          best = vol;
          for (int e = 0; e < 3; ++e) { blo[e] = a[e]; bhi[e] = b[e]; }
        }
      }
    }
    if (best == 0) return;
    for (int d = 0; d < 3; ++d) { lo[d] = blo[d]; hi[d] = bhi[d]; }
  }
  for (int d = 0; d < 3; ++d) { g.bulk_lo[d] = lo[d]; g.bulk_hi[d] = hi[d]; }
}

olb_b200_status ensure_partials(olb_b200_lattice* L)
{
  return ensure_partial_count(L, step_blocks(L) + boundary_blocks(L));
}

olb_b200_status ensure_partial_count(olb_b200_lattice* L, size_t need)
{
  if (need > L->n_partials) {
    if (L->partials) cudaFree(L->partials);
    L->partials = nullptr;
    L->n_partials = 0;
    OLB_CUDA(cudaMalloc(&L->partials, need * sizeof(StatPartial)));
    L->n_partials = need;
  }
  return OLB_B200_OK;
}

olb_b200_status upload_boundary_values(olb_b200_lattice* L);

int periodic_mask(const olb_b200_lattice* L)
{
  return (L->desc.periodic[0] ? 1 : 0) | (L->desc.periodic[1] ? 2 : 0) | (L->desc.periodic[2] ? 4 : 0);
}

// The PostStream stage (SuperLattice::collideAndStream, src/core/superLattice.hh:640-641):
// PlaneFdBoundaryProcessor3D on every interpolated boundary cell.
olb_b200_status post_stream(olb_b200_lattice* L)
{
  if (L->n_bc == 0) return OLB_B200_OK;
  cudaError_t e = dispatch(L, [&](auto qc, auto s_, auto r_) {
    return launch_boundary<decltype(qc)::value, decltype(s_), decltype(r_)>(
      L->pops, L->g, L->parity == 1, L->ids, L->table, periodic_mask(L), L->bc_cells, L->n_bc_flat,
      L->n_bc_edge, L->n_bc_corner, L->stream);
  });
  if (e != cudaSuccess) return cuda_fail(e, "boundary post-processing kernels");
  return OLB_B200_OK;
}

// BlockLattice::initialize (src/core/blockLattice.hh:56-67): the PostStream
// post-processors run once on the initial state, before the first collision.
olb_b200_status initialize_once(olb_b200_lattice* L)
{
  if (L->initialized) return OLB_B200_OK;
  olb_b200_status st = post_stream(L);
  if (st != OLB_B200_OK) return st;
  L->initialized = true;
  return OLB_B200_OK;
}

olb_b200_status boundary_noise(olb_b200_lattice* L);

olb_b200_status enqueue_steps(olb_b200_lattice* L, int steps, bool stats_last)
{
  for (int s = 0; s < steps; ++s) {
    olb_b200_status nst = boundary_noise(L);
    if (nst != OLB_B200_OK) return nst;
    const bool stats = stats_last && s == steps - 1;
    StepLaunch a;
    a.pops = L->pops;
    a.g = L->g;
    a.ids = L->masked ? L->ids : nullptr;
    a.table = L->table;
    a.bulk = L->bulk;
    a.partials = stats ? L->partials : nullptr;
    a.block_z = L->block_z;
    a.block_y = L->block_y;
    a.variant = L->variant;
    a.stream = L->stream;
    const bool odd = L->parity == 1;
    cudaError_t e = cudaSuccess;
    if (L->n_bc) {
      // collision of the boundary cells in place, ahead of the step kernel
      StatPartial* bp = stats ? L->partials + step_blocks(L) : nullptr;
      e = dispatch(L, [&](auto qc, auto s_, auto r_) {
        return launch_boundary_collide<decltype(qc)::value, decltype(s_), decltype(r_)>(
          L->pops, L->g, odd, L->ids, L->table, L->bulk_kind, L->bc_cells, L->n_bc, bp, L->stream);
      });
      if (e != cudaSuccess) return cuda_fail(e, "boundary collision launch");
    }
    e = dispatch(L, [&](auto qc, auto s_, auto r_) {
      using S = decltype(s_);
      using R = decltype(r_);
      return launch_step<decltype(qc)::value, S, R>(a, L->bulk_kind, odd, L->masked, stats);
    });
    if (e != cudaSuccess) return cuda_fail(e, "step kernel launch");
    L->parity ^= 1;
    L->steps_done += 1;
    olb_b200_status st = post_stream(L);
    if (st != OLB_B200_OK) return st;
  }
  return OLB_B200_OK;
}

// Per boundary entry: the bounding box of its cells, which indexes its values
// (RHO, VELOCITY per cell, as defineRho / defineU set them); the list of all
// boundary cells for the PostStream passes.  Values start at RHO = 1, VELOCITY
// = 0 (FixedDensity / FixedVelocityMomentumGeneric::initialize,
// src/dynamics/momenta/elements.h:251-255, 560-565).
olb_b200_status setup_boundaries(olb_b200_lattice* L, const uint8_t* ids, const olb_b200_dyn_params* table,
                                 int n_entries, bool any)
{
  if (L->bc_cells) cudaFree(L->bc_cells);
  if (L->bc_values) cudaFree(L->bc_values);
  if (L->bc_u) cudaFree(L->bc_u);
  if (L->bc_base) cudaFree(L->bc_base);
  if (L->force) cudaFree(L->force);
  L->bc_base = nullptr;
  L->bc_cells = nullptr;
  L->bc_values = nullptr;
  L->bc_u = nullptr;
  L->device_bytes -= L->bc_bytes;
  L->bc_bytes = 0;
  L->n_bc = 0;
  L->n_bc_flat = L->n_bc_edge = L->n_bc_corner = 0;
  L->bc_slots = 0;
  L->bc_box.assign(size_t(n_entries), olb_b200_lattice::BcBox{{0, 0, 0, 0, 0, 0}, 0});
  L->bc_host.clear();
  L->ids_host.clear();
  if (!any) return OLB_B200_OK;
  const int nx = L->desc.nx, ny = L->desc.ny, nz = L->desc.nz;
  std::vector<int> lo(size_t(n_entries) * 3, INT32_MAX), hi(size_t(n_entries) * 3, -1);
  // PostStream order: flat interpolated cells (velocity pass, PlaneFd), then
  // external edges, then external corners; local faces and internal edges and
  // corners need no PostStream pass and come last (the boundary collision
  // pre-pass takes all)
  std::vector<uint32_t> flat, edges, corners, local;
  for (int x = 0; x < nx; ++x) {
    for (int y = 0; y < ny; ++y) {
      for (int z = 0; z < nz; ++z) {
        const size_t c = (size_t(x) * ny + y) * nz + z;
        const int k = ids[c];
        const int kind = table[k].kind;
        if (!has_values(kind)) continue;
        if (is_interpolated(kind)) flat.push_back(uint32_t(c));
        else if (kind == K_VELOCITY_EDGE) edges.push_back(uint32_t(c));
        else if (kind == K_VELOCITY_CORNER) corners.push_back(uint32_t(c));
        else local.push_back(uint32_t(c));
        const int p[3] = {x, y, z};
        for (int d = 0; d < 3; ++d) {
          lo[3 * k + d] = std::min(lo[3 * k + d], p[d]);
          hi[3 * k + d] = std::max(hi[3 * k + d], p[d]);
        }
      }
    }
  }
  size_t slots = 0;
  for (int k = 0; k < n_entries; ++k) {
    if (hi[3 * k] < 0) continue;
    auto& b = L->bc_box[size_t(k)];
    for (int d = 0; d < 3; ++d) {
      b.box[d] = lo[3 * k + d];
      b.box[3 + d] = hi[3 * k + d] - lo[3 * k + d] + 1;
    }
    b.slot0 = slots;
    slots += size_t(b.box[3]) * b.box[4] * b.box[5];
  }
  if (slots == 0) return OLB_B200_OK;
  std::vector<uint32_t> cells(flat);
  cells.insert(cells.end(), edges.begin(), edges.end());
  cells.insert(cells.end(), corners.begin(), corners.end());
  cells.insert(cells.end(), local.begin(), local.end());
  L->n_bc_flat = uint32_t(flat.size());
  L->n_bc_edge = uint32_t(edges.size());
  L->n_bc_corner = uint32_t(corners.size());
  L->ids_host.assign(ids, ids + L->cells);
  L->bc_slots = slots;
  L->bc_host.assign(4 * slots, 0.0);
  for (size_t k = 0; k < slots; ++k) L->bc_host[4 * k] = 1.0;
  L->n_bc = uint32_t(cells.size());
  OLB_CUDA(cudaMalloc(&L->bc_cells, std::max<size_t>(cells.size(), 1) * sizeof(uint32_t)));
  OLB_CUDA(cudaMalloc(&L->bc_values, 4 * slots * L->real));
  OLB_CUDA(cudaMalloc(&L->bc_u, 3 * slots * L->real));
  OLB_CUDA(cudaMemset(L->bc_u, 0, 3 * slots * L->real));
  L->bc_bytes = cells.size() * sizeof(uint32_t) + 7 * slots * L->real;
  L->device_bytes += L->bc_bytes;
  if (!cells.empty())
    OLB_CUDA(cudaMemcpy(L->bc_cells, cells.data(), cells.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  return upload_boundary_values(L);
}

olb_b200_status upload_boundary_values(olb_b200_lattice* L)
{
  if (!L->bc_slots) return OLB_B200_OK;
  if (!L->bc_base) {
    OLB_CUDA(cudaMalloc(&L->bc_base, 4 * L->bc_slots * L->real));
    L->bc_bytes += 4 * L->bc_slots * L->real;
    L->device_bytes += 4 * L->bc_slots * L->real;
  }
  if (L->real == 8) {
    OLB_CUDA(cudaMemcpy(L->bc_values, L->bc_host.data(), L->bc_host.size() * sizeof(double),
                        cudaMemcpyHostToDevice));
    OLB_CUDA(cudaMemcpy(L->bc_base, L->bc_host.data(), L->bc_host.size() * sizeof(double),
                        cudaMemcpyHostToDevice));
  } else {
    std::vector<float> v(L->bc_host.begin(), L->bc_host.end());
    OLB_CUDA(cudaMemcpy(L->bc_values, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice));
    OLB_CUDA(cudaMemcpy(L->bc_base, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  return OLB_B200_OK;
}

// inlet fluctuations of the step about to run (no-op unless enabled)
olb_b200_status boundary_noise(olb_b200_lattice* L)
{
  if (L->noise_amp == 0.0 || L->n_bc == 0) return OLB_B200_OK;
  const unsigned threads = 128, blocks = (L->n_bc + threads - 1) / threads;
  if (L->real == 8) {
    bc_noise_kernel<double><<<blocks, threads, 0, L->stream>>>(
      L->bc_cells, L->n_bc, L->ids, static_cast<const DynDevice<double>*>(L->table),
      static_cast<const double*>(L->bc_base), static_cast<double*>(L->bc_values), L->g, uint64_t(L->steps_done),
      uint64_t(L->cells), L->noise_amp, L->noise_seed);
  } else {
    bc_noise_kernel<float><<<blocks, threads, 0, L->stream>>>(
      L->bc_cells, L->n_bc, L->ids, static_cast<const DynDevice<float>*>(L->table),
      static_cast<const float*>(L->bc_base), static_cast<float*>(L->bc_values), L->g, uint64_t(L->steps_done),
      uint64_t(L->cells), L->noise_amp, L->noise_seed);
  }
  OLB_CUDA(cudaGetLastError());
  return OLB_B200_OK;
}

template <class R>
void attach_boundary(const olb_b200_lattice* L, int k, const olb_b200_dyn_params& in, DynDevice<R>& d)
{
  if (!has_values(in.kind)) return;
  const auto& b = L->bc_box[size_t(k)];
  d.bc_dir = in.direction;
  d.bc_orient = in.orientation;
  for (int e = 0; e < 3; ++e) d.nrm[e] = in.normal[e];
  for (int e = 0; e < 6; ++e) d.box[e] = b.box[e];
  d.bc_values = L->bc_values ? static_cast<const R*>(L->bc_values) + 4 * b.slot0 : nullptr;
  d.bc_u = L->bc_u ? static_cast<R*>(L->bc_u) + 3 * b.slot0 : nullptr;
}

} // namespace

extern "C" {

const char* olb_b200_last_error(void) { return g_last_error.c_str(); }

int32_t olb_b200_abi_version(void) { return OLB_B200_ABI_VERSION; }

const char* olb_b200_build_info(void)
{
  static const std::string info = std::string("openlb_b200 abi ") + std::to_string(OLB_B200_ABI_VERSION) +
                                  "; nvcc " + std::to_string(__CUDACC_VER_MAJOR__) + "." +
                                  std::to_string(__CUDACC_VER_MINOR__) +
#ifdef OLB_B200_EXACT
                                  "; sm_100a; -fmad=false (exact arithmetic build)";
#else
                                  "; sm_100a; -fmad=true";
#endif
  return info.c_str();
}

olb_b200_status olb_b200_create(const olb_b200_desc* desc, olb_b200_lattice** out)
{
  g_last_error.clear();
  if (!desc || !out) return fail(OLB_B200_ERR_ARG, "create: null argument");
  *out = nullptr;
  if (desc->q != 19 && desc->q != 27) return fail(OLB_B200_ERR_ARG, "create: q must be 19 or 27, got %d", desc->q);
  if (desc->nx < 1 || desc->ny < 1 || desc->nz < 1)
    return fail(OLB_B200_ERR_ARG, "create: extent must be positive (%d,%d,%d)", desc->nx, desc->ny, desc->nz);
  if (desc->storage < 0 || desc->storage > 3) return fail(OLB_B200_ERR_ARG, "create: unknown storage %d", desc->storage);
  if (desc->reserved[0] || desc->reserved[1] || desc->reserved[2])
    return fail(OLB_B200_ERR_ARG, "create: reserved fields must be zero");
  const size_t cells = size_t(desc->nx) * desc->ny * desc->nz;
  if (cells > (size_t(1) << 31)) return fail(OLB_B200_ERR_ARG, "create: %zu cells exceed 2^31", cells);
  if (desc->nx > 65535) return fail(OLB_B200_ERR_ARG, "create: nx %d exceeds 65535", desc->nx);
  // 16-bit storage with an even nx uses the paired layout (two cells per
  // 4-byte element); its element columns start on 256-byte boundaries too
  // (its kernel indexes elements with 32 bits: q * stride/2 < 2^32)
  const bool paired = (desc->storage == OLB_B200_STORAGE_F16 || desc->storage == OLB_B200_STORAGE_BF16) &&
                      desc->nx % 2 == 0 &&
                      uint64_t(desc->q) * ((cells + 127) / 128 * 64) < (uint64_t(1) << 32);
  const size_t stride = paired ? (cells + 127) / 128 * 128 : (cells + 63) / 64 * 64;
  if (stride * size_t(desc->q) > (size_t(1) << 40)) return fail(OLB_B200_ERR_ARG, "create: lattice too large");

  auto* L = new olb_b200_lattice;
  L->desc = *desc;
  L->q = desc->q;
  L->cells = cells;
  L->stride = stride;
  L->device = desc->device;
  L->elem = desc->storage == OLB_B200_STORAGE_F64 ? 8 : (desc->storage == OLB_B200_STORAGE_F32 ? 4 : 2);
  L->real = desc->storage == OLB_B200_STORAGE_F64 ? 8 : 4;
  L->g = Geometry{desc->nx, desc->ny, desc->nz, uint32_t(stride), paired ? 1 : 0};
  default_shape(L, L->block_z, L->block_y);

  auto cleanup = [&](olb_b200_status st) {
    olb_b200_destroy(L);
    return st;
  };
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return cleanup(st);
#define OLB_CUDA_C(call)                                                                           \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return cleanup(cuda_fail(e_, #call));                                   \
  } while (0)
  OLB_CUDA_C(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking));
  OLB_CUDA_C(cudaEventCreate(&L->ev0));
  OLB_CUDA_C(cudaEventCreate(&L->ev1));
  const size_t pop_bytes = stride * size_t(L->q) * L->elem;
  OLB_CUDA_C(cudaMalloc(&L->pops, pop_bytes));
  OLB_CUDA_C(cudaMemsetAsync(L->pops, 0, pop_bytes, L->stream));
  OLB_CUDA_C(cudaMalloc(&L->ids, cells));
  OLB_CUDA_C(cudaMemsetAsync(L->ids, 0, cells, L->stream));
  OLB_CUDA_C(cudaMalloc(&L->table, 256 * sizeof(DynDevice<double>)));
  OLB_CUDA_C(cudaMalloc(&L->scratch, 4 * cells * L->real));
  OLB_CUDA_C(cudaMalloc(&L->stat_dev, sizeof(StatPartial)));
  OLB_CUDA_C(cudaMallocHost(&L->stat_host, sizeof(StatPartial)));
  L->device_bytes = pop_bytes + cells + 256 * sizeof(DynDevice<double>) + 4 * cells * L->real;
  // default: every cell NoDynamics
  olb_b200_dyn_params none{};
  none.kind = OLB_B200_DYN_NONE;
  none.wall_rho = 1.0;
  st = olb_b200_set_dynamics(L, nullptr, &none, 1);
  if (st != OLB_B200_OK) return cleanup(st);
  OLB_CUDA_C(cudaStreamSynchronize(L->stream));
#undef OLB_CUDA_C
  *out = L;
  return OLB_B200_OK;
}

void olb_b200_destroy(olb_b200_lattice* L)
{
  if (!L) return;
  cudaSetDevice(L->device);
  if (L->stream) cudaStreamSynchronize(L->stream);
  if (L->pops) cudaFree(L->pops);
  if (L->ids) cudaFree(L->ids);
  if (L->table) cudaFree(L->table);
  if (L->scratch) cudaFree(L->scratch);
  if (L->partials) cudaFree(L->partials);
  if (L->uprev) cudaFree(L->uprev);
  if (L->bc_cells) cudaFree(L->bc_cells);
  if (L->bc_values) cudaFree(L->bc_values);
  if (L->bc_u) cudaFree(L->bc_u);
  if (L->bc_base) cudaFree(L->bc_base);
  if (L->force) cudaFree(L->force);
  if (L->stat_dev) cudaFree(L->stat_dev);
  if (L->stat_host) cudaFreeHost(L->stat_host);
  if (L->ev0) cudaEventDestroy(L->ev0);
  if (L->ev1) cudaEventDestroy(L->ev1);
  for (cudaEvent_t e : L->flight) cudaEventDestroy(e);
  if (L->stream) cudaStreamDestroy(L->stream);
  delete L;
}

olb_b200_status olb_b200_set_dynamics(olb_b200_lattice* L, const uint8_t* ids,
                                      const olb_b200_dyn_params* table, int32_t n_entries)
{
  g_last_error.clear();
  if (!L || !table) return fail(OLB_B200_ERR_ARG, "set_dynamics: null argument");
  if (n_entries < 1 || n_entries > 256)
    return fail(OLB_B200_ERR_ARG, "set_dynamics: table needs 1..256 entries, got %d", n_entries);
  int bulk = -1, first_bc = -1;
  for (int k = 0; k < n_entries; ++k) {
    const int kind = table[k].kind;
    if (kind < OLB_B200_DYN_NONE || kind > OLB_B200_DYN_LOCAL_PRESSURE)
      return fail(OLB_B200_ERR_ARG, "set_dynamics: entry %d has unknown kind %d", k, kind);
    if (table[k].reserved != 0)
      return fail(OLB_B200_ERR_ARG, "set_dynamics: entry %d: reserved field must be 0", k);
    if (has_values(kind)) {
      const int m = table[k].mixin;
      if (m != OLB_B200_DYN_BGK && m != OLB_B200_DYN_TRT && m != OLB_B200_DYN_SMAGORINSKY)
        return fail(OLB_B200_ERR_UNSUPPORTED, "set_dynamics: entry %d: boundaries take a BGK, TRT "
                    "or Smagorinsky-BGK mixin, got kind %d", k, m);
      if ((is_local(kind) || is_inner(kind)) && m == OLB_B200_DYN_SMAGORINSKY)
        return fail(OLB_B200_ERR_UNSUPPORTED, "set_dynamics: entry %d: regularised (local velocity or pressure, "
                    "internal edge or corner) boundaries with a Smagorinsky-BGK mixin are not implemented", k);
      if (is_outer(kind) || is_inner(kind)) {
        int nonzero = 0;
        bool valid = true;
        for (int e = 0; e < 3; ++e) {
          const int v = table[k].normal[e];
          valid &= v >= -1 && v <= 1;
          nonzero += v != 0;
        }
        const bool edge = kind == OLB_B200_DYN_VELOCITY_EDGE || kind == OLB_B200_DYN_VELOCITY_INNER_EDGE;
        if (!valid || nonzero != (edge ? 2 : 3))
          return fail(OLB_B200_ERR_ARG, "set_dynamics: entry %d: normal (%d,%d,%d) is not an %s normal", k,
                      table[k].normal[0], table[k].normal[1], table[k].normal[2], edge ? "edge" : "corner");
      } else if (table[k].direction < 0 || table[k].direction > 2 ||
                 (table[k].orientation != 1 && table[k].orientation != -1)) {
        return fail(OLB_B200_ERR_ARG, "set_dynamics: entry %d: normal axis %d / sign %d invalid", k,
                    table[k].direction, table[k].orientation);
      }
      if (!(table[k].omega > 0.0 && table[k].omega < 2.0))
        return fail(OLB_B200_ERR_ARG, "set_dynamics: entry %d omega %g outside (0,2)", k, table[k].omega);
      if (first_bc < 0) {
        first_bc = k;
      } else if (table[first_bc].mixin != m) {
        return fail(OLB_B200_ERR_UNSUPPORTED, "set_dynamics: entries %d and %d use different boundary mixins",
                    first_bc, k);
      }
    }
    if (is_fluid(kind)) {
      if (!(table[k].omega > 0.0 && table[k].omega < 2.0))
        return fail(OLB_B200_ERR_ARG, "set_dynamics: entry %d omega %g outside (0,2)", k, table[k].omega);
      if (bulk < 0) {
        bulk = k;
      } else if (table[bulk].kind != kind) {
        return fail(OLB_B200_ERR_UNSUPPORTED,
                    "set_dynamics: entries %d and %d use different fluid collisions (%d, %d); one "
                    "fluid collision kind per lattice is supported", bulk, k, table[bulk].kind, kind);
      }
    }
  }
  if (first_bc >= 0) {
    if (bulk >= 0 && table[bulk].kind != table[first_bc].mixin)
      return fail(OLB_B200_ERR_UNSUPPORTED, "set_dynamics: the boundary mixin (kind %d) must be the lattice's "
                  "fluid collision (kind %d)", table[first_bc].mixin, table[bulk].kind);
    if (!ids) return fail(OLB_B200_ERR_ARG, "set_dynamics: boundary entries need per-cell ids");
  }
  bool uniform = ids == nullptr;
  uint8_t first = 0;
  if (ids) {
    first = ids[0];
    uniform = true;
    for (size_t c = 0; c < L->cells; ++c) {
      if (ids[c] >= n_entries)
        return fail(OLB_B200_ERR_ARG, "set_dynamics: cell %zu has id %u >= %d entries", c, unsigned(ids[c]), n_entries);
      uniform &= ids[c] == first;
    }
  }
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  st = setup_boundaries(L, ids, table, n_entries, first_bc >= 0);
  if (st != OLB_B200_OK) return st;
  // device table and the host copy of the bulk entry
  const bool f64 = L->desc.storage == OLB_B200_STORAGE_F64;
  std::vector<unsigned char> host(size_t(n_entries) * (f64 ? sizeof(DynDevice<double>) : sizeof(DynDevice<float>)));
  for (int k = 0; k < n_entries; ++k) {
    if (f64) {
      auto d = make_device_params<double>(L->q, table[k]);
      attach_boundary(L, k, table[k], d);
      std::memcpy(host.data() + k * sizeof d, &d, sizeof d);
    } else {
      auto d = make_device_params<float>(L->q, table[k]);
      attach_boundary(L, k, table[k], d);
      std::memcpy(host.data() + k * sizeof d, &d, sizeof d);
    }
  }
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  OLB_CUDA(cudaMemcpy(L->table, host.data(), host.size(), cudaMemcpyHostToDevice));
  if (ids) {
    OLB_CUDA(cudaMemcpy(L->ids, ids, L->cells, cudaMemcpyHostToDevice));
  } else {
    OLB_CUDA(cudaMemset(L->ids, 0, L->cells));
  }
  const int bulk_entry = bulk >= 0 ? bulk : (first_bc >= 0 ? first_bc : 0);
  L->bulk_kind = bulk >= 0 ? table[bulk].kind : (first_bc >= 0 ? table[first_bc].mixin : K_BGK);
  const size_t esz = f64 ? sizeof(DynDevice<double>) : sizeof(DynDevice<float>);
  std::memcpy(L->bulk, host.data() + bulk_entry * esz, esz);
  // the unmasked kernel serves lattices where every cell uses one fluid entry
  const int only = ids ? first : 0;
  const bool was_masked = L->masked;
  L->masked = !(uniform && is_fluid(table[only].kind));
  if (!L->masked) {
    std::memcpy(L->bulk, host.data() + only * esz, esz);
  }
  compute_bulk_box(L, L->masked ? ids : nullptr, bulk);
  // the masked kernels take the bulk entry's constants for every cell of its
  // kind when no other entry of that kind differs from it
  L->g.uniform = 0;
  if (L->masked && bulk >= 0) {
    bool same = true;
    const olb_b200_dyn_params& b = table[bulk];
    for (int k = 0; k < n_entries && same; ++k) {
      const olb_b200_dyn_params& e = table[k];
      if (e.kind != b.kind) continue;
      same = e.omega == b.omega && e.magic == b.magic && e.smagorinsky == b.smagorinsky &&
             e.force[0] == b.force[0] && e.force[1] == b.force[1] && e.force[2] == b.force[2];
    }
    L->g.uniform = same ? 1 : 0;
  }
  L->n_entries = n_entries;
  // a change of kernel class invalidates an earlier tuning
  if (!L->tuned || was_masked != L->masked) {
    L->variant = default_variant(L);
    L->tuned = false;
  }
  return OLB_B200_OK;
}

olb_b200_status olb_b200_set_populations(olb_b200_lattice* L, const void* host_pops)
{
  g_last_error.clear();
  if (!L || !host_pops) return fail(OLB_B200_ERR_ARG, "set_populations: null argument");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  const size_t col = L->cells * L->real;
  const char* src = static_cast<const char*>(host_pops);
  if (L->elem == L->real) {
    for (int i = 0; i < L->q; ++i) {
      OLB_CUDA(cudaMemcpyAsync(static_cast<char*>(L->pops) + size_t(i) * L->stride * L->elem,
                               src + size_t(i) * col, col, cudaMemcpyHostToDevice, L->stream));
    }
  } else {
    for (int i0 = 0; i0 < L->q; i0 += 4) {
      const int i1 = std::min(L->q, i0 + 4);
      OLB_CUDA(cudaMemcpyAsync(L->scratch, src + size_t(i0) * col, size_t(i1 - i0) * col,
                               cudaMemcpyHostToDevice, L->stream));
      cudaError_t e = dispatch(L, [&](auto qc, auto s_, auto r_) {
        return launch_scatter<decltype(qc)::value, decltype(s_), decltype(r_)>(L->pops, L->g, L->scratch, i0, i1,
                                                                              L->stream);
      });
      if (e != cudaSuccess) return cuda_fail(e, "scatter kernel");
    }
  }
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  L->parity = 0;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_ini_equilibrium(olb_b200_lattice* L, const void* rho, const void* u)
{
  g_last_error.clear();
  if (!L || !rho || !u) return fail(OLB_B200_ERR_ARG, "ini_equilibrium: null argument");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  // rho and u staged in the scratch buffer (4 columns of R), expanded on the device
  const size_t col = L->cells * L->real;
  char* stage = static_cast<char*>(L->scratch);
  OLB_CUDA(cudaMemcpyAsync(stage, rho, col, cudaMemcpyHostToDevice, L->stream));
  OLB_CUDA(cudaMemcpyAsync(stage + col, u, 3 * col, cudaMemcpyHostToDevice, L->stream));
  cudaError_t e = dispatch(L, [&](auto qc, auto s_, auto r_) {
    return launch_equilibrium<decltype(qc)::value, decltype(s_), decltype(r_)>(L->pops, L->g, L->scratch,
                                                                              L->stream);
  });
  if (e != cudaSuccess) return cuda_fail(e, "equilibrium kernel");
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  L->parity = 0;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_get_populations(olb_b200_lattice* L, void* host_pops)
{
  g_last_error.clear();
  if (!L || !host_pops) return fail(OLB_B200_ERR_ARG, "get_populations: null argument");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  const size_t col = L->cells * L->real;
  char* dst = static_cast<char*>(host_pops);
  if (L->elem == L->real && L->parity == 0) {
    for (int i = 0; i < L->q; ++i) {
      OLB_CUDA(cudaMemcpyAsync(dst + size_t(i) * col,
                               static_cast<const char*>(L->pops) + size_t(i) * L->stride * L->elem, col,
                               cudaMemcpyDeviceToHost, L->stream));
    }
  } else {
    for (int i0 = 0; i0 < L->q; i0 += 4) {
      const int i1 = std::min(L->q, i0 + 4);
      cudaError_t e = dispatch(L, [&](auto qc, auto s_, auto r_) {
        return launch_gather<decltype(qc)::value, decltype(s_), decltype(r_)>(L->pops, L->g, L->parity == 1,
                                                                             L->scratch, i0, i1, L->stream);
      });
      if (e != cudaSuccess) return cuda_fail(e, "gather kernel");
      OLB_CUDA(cudaMemcpyAsync(dst + size_t(i0) * col, L->scratch, size_t(i1 - i0) * col,
                               cudaMemcpyDeviceToHost, L->stream));
    }
  }
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  return OLB_B200_OK;
}

olb_b200_status olb_b200_collide_and_stream(olb_b200_lattice* L, int32_t steps, olb_b200_stats* stats)
{
  g_last_error.clear();
  if (!L) return fail(OLB_B200_ERR_ARG, "collide_and_stream: null lattice");
  if (steps < 0) return fail(OLB_B200_ERR_ARG, "collide_and_stream: negative step count %d", steps);
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  if (steps == 0) {
    if (stats) std::memset(stats, 0, sizeof *stats);
    return OLB_B200_OK;
  }
  if (stats) {
    st = ensure_partials(L);
    if (st != OLB_B200_OK) return st;
  }
  st = initialize_once(L);
  if (st != OLB_B200_OK) return st;
  const bool bounded = !stats && !L->flight.empty();
  if (bounded && L->flight_used[L->flight_pos]) {
    // wait for the call issued flight.size() calls ago
    OLB_CUDA(cudaEventSynchronize(L->flight[L->flight_pos]));
  }
  st = enqueue_steps(L, steps, stats != nullptr);
  if (st != OLB_B200_OK) return st;
  if (bounded) {
    OLB_CUDA(cudaEventRecord(L->flight[L->flight_pos], L->stream));
    L->flight_used[L->flight_pos] = true;
    L->flight_pos = (L->flight_pos + 1) % L->flight.size();
  }
  if (!stats) return OLB_B200_OK;
  const size_t count = step_blocks(L) + boundary_blocks(L);
  reduce_partials_kernel<<<1, 1024, 0, L->stream>>>(L->partials, count, L->stat_dev);
  OLB_CUDA(cudaGetLastError());
  OLB_CUDA(cudaMemcpyAsync(L->stat_host, L->stat_dev, sizeof(StatPartial), cudaMemcpyDeviceToHost, L->stream));
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  const StatPartial p = *L->stat_host;
  stats->sum_rho = p.sum_rho;
  stats->sum_usqr = p.sum_usqr;
  stats->max_usqr = p.max_usqr;
  stats->n_cells = int64_t(p.n_cells);
  // LatticeStatistics::reset: energy = 0.5 <|u|^2>, maxU = sqrt(max |u|^2)
  // (src/core/latticeStatistics.hh:88-89)
  stats->average_rho = p.n_cells ? p.sum_rho / double(p.n_cells) : 0.0;
  stats->average_energy = p.n_cells ? 0.5 * p.sum_usqr / double(p.n_cells) : 0.0;
  stats->max_u = std::sqrt(p.max_usqr);
  stats->n_nonfinite = int64_t(p.n_nonfinite);
  if (p.n_nonfinite) {
    return fail(OLB_B200_ERR_DIVERGED, "collide_and_stream: %llu cells with non-finite density or "
                "velocity after step %lld (simulation diverged)", p.n_nonfinite, (long long)L->steps_done);
  }
  return OLB_B200_OK;
}

olb_b200_status olb_b200_get_moments(olb_b200_lattice* L, void* host_rho, void* host_u)
{
  g_last_error.clear();
  if (!L || !host_rho || !host_u) return fail(OLB_B200_ERR_ARG, "get_moments: null argument");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  char* rho_d = static_cast<char*>(L->scratch);
  char* u_d = rho_d + L->cells * L->real;
  cudaError_t e = dispatch(L, [&](auto qc, auto s_, auto r_) {
    return launch_moments<decltype(qc)::value, decltype(s_), decltype(r_)>(
      L->pops, L->g, L->parity == 1, L->ids, L->table, rho_d, u_d, L->stream);
  });
  if (e != cudaSuccess) return cuda_fail(e, "moments kernel");
  OLB_CUDA(cudaMemcpyAsync(host_rho, rho_d, L->cells * L->real, cudaMemcpyDeviceToHost, L->stream));
  OLB_CUDA(cudaMemcpyAsync(host_u, u_d, 3 * L->cells * L->real, cudaMemcpyDeviceToHost, L->stream));
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  return OLB_B200_OK;
}

olb_b200_status olb_b200_synchronize(olb_b200_lattice* L)
{
  g_last_error.clear();
  if (!L) return fail(OLB_B200_ERR_ARG, "synchronize: null lattice");
  OLB_CUDA(cudaSetDevice(L->device));
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  return OLB_B200_OK;
}

olb_b200_status olb_b200_time_steps(olb_b200_lattice* L, int32_t steps, float* ms)
{
  g_last_error.clear();
  if (!L || !ms || steps < 1) return fail(OLB_B200_ERR_ARG, "time_steps: bad argument");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  st = initialize_once(L);
  if (st != OLB_B200_OK) return st;
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  OLB_CUDA(cudaEventRecord(L->ev0, L->stream));
  st = enqueue_steps(L, steps, false);
  if (st != OLB_B200_OK) return st;
  OLB_CUDA(cudaEventRecord(L->ev1, L->stream));
  OLB_CUDA(cudaEventSynchronize(L->ev1));
  OLB_CUDA(cudaEventElapsedTime(ms, L->ev0, L->ev1));
  return OLB_B200_OK;
}

olb_b200_status olb_b200_set_max_steps_in_flight(olb_b200_lattice* L, int32_t calls)
{
  g_last_error.clear();
  if (!L) return fail(OLB_B200_ERR_ARG, "set_max_steps_in_flight: null lattice");
  if (calls < 0 || calls > 64) return fail(OLB_B200_ERR_ARG, "set_max_steps_in_flight: %d not in [0, 64]", calls);
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  for (cudaEvent_t e : L->flight) cudaEventDestroy(e);
  L->flight.assign(size_t(calls), nullptr);
  L->flight_used.assign(size_t(calls), false);
  L->flight_pos = 0;
  for (cudaEvent_t& e : L->flight) OLB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return OLB_B200_OK;
}

olb_b200_status olb_b200_get_stream(olb_b200_lattice* L, void** stream)
{
  if (!L || !stream) return fail(OLB_B200_ERR_ARG, "get_stream: null argument");
  *stream = L->stream;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_get_info(olb_b200_lattice* L, int64_t* steps_done, int64_t* device_bytes,
                                  int32_t* block_z, int32_t* block_y)
{
  if (!L) return fail(OLB_B200_ERR_ARG, "get_info: null lattice");
  if (steps_done) *steps_done = L->steps_done;
  if (device_bytes) *device_bytes = int64_t(L->device_bytes + L->n_partials * sizeof(StatPartial));
  if (block_z) *block_z = L->block_z;
  if (block_y) *block_y = L->block_y;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_set_launch_shape(olb_b200_lattice* L, int32_t block_z, int32_t block_y)
{
  g_last_error.clear();
  if (!L) return fail(OLB_B200_ERR_ARG, "set_launch_shape: null lattice");
  if (block_z == 0 && block_y == 0) {
    default_shape(L, L->block_z, L->block_y);
    return OLB_B200_OK;
  }
  if (block_z < 32 || block_z % 32 != 0 || block_y < 1 || block_z * block_y > kStepThreads)
    return fail(OLB_B200_ERR_ARG, "set_launch_shape: block (%d,%d) invalid: block_z a positive multiple "
                "of 32, block_z*block_y <= %d", block_z, block_y, kStepThreads);
  L->block_z = block_z;
  L->block_y = block_y;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_velocity_residual(olb_b200_lattice* L, double* residual)
{
  g_last_error.clear();
  if (!L || !residual) return fail(OLB_B200_ERR_ARG, "velocity_residual: null argument");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  const size_t ubytes = 3 * L->cells * L->real;
  if (!L->uprev) {
    OLB_CUDA(cudaMalloc(&L->uprev, ubytes));
    OLB_CUDA(cudaMemsetAsync(L->uprev, 0, ubytes, L->stream));
    L->device_bytes += ubytes;
  }
  char* rho_d = static_cast<char*>(L->scratch);
  char* u_d = rho_d + L->cells * L->real;
  cudaError_t e = dispatch(L, [&](auto qc, auto s_, auto r_) {
    return launch_moments<decltype(qc)::value, decltype(s_), decltype(r_)>(
      L->pops, L->g, L->parity == 1, L->ids, L->table, rho_d, u_d, L->stream);
  });
  if (e != cudaSuccess) return cuda_fail(e, "moments kernel");
  const unsigned threads = 256;
  const size_t blocks = (L->cells + threads - 1) / threads;
  st = ensure_partial_count(L, blocks);
  if (st != OLB_B200_OK) return st;
  if (L->real == 8) {
    velocity_residual_kernel<double><<<unsigned(blocks), threads, 0, L->stream>>>(
      reinterpret_cast<const double*>(u_d), static_cast<double*>(L->uprev), L->ids,
      static_cast<const DynDevice<double>*>(L->table), L->cells, L->partials);
  } else {
    velocity_residual_kernel<float><<<unsigned(blocks), threads, 0, L->stream>>>(
      reinterpret_cast<const float*>(u_d), static_cast<float*>(L->uprev), L->ids,
      static_cast<const DynDevice<float>*>(L->table), L->cells, L->partials);
  }
  OLB_CUDA(cudaGetLastError());
  reduce_partials_kernel<<<1, 1024, 0, L->stream>>>(L->partials, blocks, L->stat_dev);
  OLB_CUDA(cudaGetLastError());
  OLB_CUDA(cudaMemcpyAsync(L->stat_host, L->stat_dev, sizeof(StatPartial), cudaMemcpyDeviceToHost, L->stream));
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  const StatPartial p = *L->stat_host;
  *residual = p.sum_usqr > 0. ? std::sqrt(p.sum_rho / p.sum_usqr) : (p.sum_rho > 0. ? INFINITY : 0.);
  return OLB_B200_OK;
}

olb_b200_status olb_b200_set_boundary_values(olb_b200_lattice* L, const int64_t* cells, int64_t count,
                                             const double* values)
{
  g_last_error.clear();
  if (!L || (count > 0 && (!cells || !values))) return fail(OLB_B200_ERR_ARG, "set_boundary_values: null argument");
  if (count < 0) return fail(OLB_B200_ERR_ARG, "set_boundary_values: negative count");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  const int ny = L->desc.ny, nz = L->desc.nz;
  for (int64_t j = 0; j < count; ++j) {
    const int64_t c = cells[j];
    if (c < 0 || size_t(c) >= L->cells)
      return fail(OLB_B200_ERR_ARG, "set_boundary_values: cell %lld out of range", (long long)c);
    if (L->ids_host.empty() || L->bc_box[L->ids_host[size_t(c)]].box[3] == 0)
      return fail(OLB_B200_ERR_ARG, "set_boundary_values: cell %lld is not an interpolated boundary cell",
                  (long long)c);
    const auto& b = L->bc_box[L->ids_host[size_t(c)]];
    const int x = int(c / (int64_t(ny) * nz));
    const int y = int((c / nz) % ny);
    const int z = int(c % nz);
    const size_t slot = b.slot0 + (size_t(x - b.box[0]) * b.box[4] + size_t(y - b.box[1])) * b.box[5] +
                        size_t(z - b.box[2]);
    for (int e = 0; e < 4; ++e) L->bc_host[4 * slot + e] = values[4 * j + e];
  }
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  return upload_boundary_values(L);
}

olb_b200_status olb_b200_set_force_field(olb_b200_lattice* L, const void* force)
{
  g_last_error.clear();
  if (!L) return fail(OLB_B200_ERR_ARG, "set_force_field: null lattice");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  const size_t column = L->stride * L->real;  // bytes per component column
  if (!force) {
    if (L->force) {
      cudaFree(L->force);
      L->device_bytes -= 3 * column;
    }
    L->force = nullptr;
    L->g.force = nullptr;
    return OLB_B200_OK;
  }
  if (!L->force) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, 3 * column);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return fail(OLB_B200_ERR_OOM, "set_force_field: cudaMalloc(%zu) failed", 3 * column);
    }
    L->force = p;
    L->device_bytes += 3 * column;
    OLB_CUDA(cudaMemset(L->force, 0, 3 * column));
  }
  for (int d = 0; d < 3; ++d) {
    OLB_CUDA(cudaMemcpy(static_cast<char*>(L->force) + d * column,
                        static_cast<const char*>(force) + d * L->cells * L->real, L->cells * L->real,
                        cudaMemcpyHostToDevice));
  }
  L->g.force = L->force;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_set_boundary_noise(olb_b200_lattice* L, double amplitude, uint64_t seed)
{
  g_last_error.clear();
  if (!L) return fail(OLB_B200_ERR_ARG, "set_boundary_noise: null lattice");
  if (!(amplitude >= 0.0 && amplitude < 1.0))
    return fail(OLB_B200_ERR_ARG, "set_boundary_noise: amplitude %g outside [0,1)", amplitude);
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  L->noise_amp = amplitude;
  L->noise_seed = seed;
  if (amplitude == 0.0) return upload_boundary_values(L);  // back to the defined values
  return OLB_B200_OK;
}

olb_b200_status olb_b200_initialize(olb_b200_lattice* L)
{
  g_last_error.clear();
  if (!L) return fail(OLB_B200_ERR_ARG, "initialize: null lattice");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  st = initialize_once(L);
  if (st != OLB_B200_OK) return st;
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  return OLB_B200_OK;
}

olb_b200_status olb_b200_set_step_variant(olb_b200_lattice* L, int32_t variant)
{
  g_last_error.clear();
  if (!L) return fail(OLB_B200_ERR_ARG, "set_step_variant: null lattice");
  if (variant < -1 || variant >= kNumStepVariants)
    return fail(OLB_B200_ERR_ARG, "set_step_variant: variant %d outside [-1, %d)", variant, kNumStepVariants);
  L->variant = variant < 0 ? default_variant(L) : variant;
  L->tuned = false;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_get_tuning(olb_b200_lattice* L, olb_b200_tuning* out)
{
  if (!L || !out) return fail(OLB_B200_ERR_ARG, "get_tuning: null argument");
  out->variant = L->variant;
  out->cells_per_thread = kStepVariants[L->variant].cells_per_thread;
  out->min_blocks_per_sm = kStepVariants[L->variant].min_blocks;
  out->block_z = L->block_z;
  out->block_y = L->block_y;
  out->tuned = L->tuned ? 1 : 0;
  out->candidates = 0;
  out->ms_per_step = L->tuned ? L->tuned_ms : 0.f;
  return OLB_B200_OK;
}

olb_b200_status olb_b200_autotune(olb_b200_lattice* L, int32_t trial_steps, olb_b200_tuning* out)
{
  g_last_error.clear();
  if (!L) return fail(OLB_B200_ERR_ARG, "autotune: null lattice");
  if (trial_steps < 0) return fail(OLB_B200_ERR_ARG, "autotune: negative trial steps");
  olb_b200_status st = select_device(L);
  if (st != OLB_B200_OK) return st;
  const int trials = trial_steps == 0 ? 4 : (trial_steps + 1) / 2 * 2;  // even: same layout parity
  // the trials advance the state; keep a device copy and restore it afterwards
  const size_t pop_bytes = L->stride * size_t(L->q) * L->elem;
  void* backup = nullptr;
  OLB_CUDA(cudaStreamSynchronize(L->stream));
  OLB_CUDA(cudaMalloc(&backup, pop_bytes));
  cudaError_t e = cudaMemcpyAsync(backup, L->pops, pop_bytes, cudaMemcpyDeviceToDevice, L->stream);
  if (e != cudaSuccess) {
    cudaFree(backup);
    return cuda_fail(e, "autotune backup copy");
  }
  const int parity = L->parity;
  const int64_t steps_done = L->steps_done;
  const int zmax = std::max(32, (L->desc.nz + 31) / 32 * 32);
  float best = 0.f;
  int best_v = L->variant, best_bz = L->block_z, best_by = L->block_y, tried = 0;
  for (int v = 0; v < kNumStepVariants && st == OLB_B200_OK; ++v) {
    bool duplicate = false;
    for (int w = 0; w < v; ++w) {
      duplicate |= kStepVariants[w].cells_per_thread == kStepVariants[v].cells_per_thread &&
                   kStepVariants[w].min_blocks == kStepVariants[v].min_blocks;
    }
    if (duplicate) continue;
    for (int bz = 256; bz >= 32 && st == OLB_B200_OK; bz /= 2) {
      if (bz > zmax) continue;
      L->variant = v;
      L->block_z = bz;
      L->block_y = kStepThreads / bz;
      st = enqueue_steps(L, 2, false);  // warm-up
      if (st != OLB_B200_OK) break;
      if ((e = cudaEventRecord(L->ev0, L->stream)) != cudaSuccess) { st = cuda_fail(e, "autotune event"); break; }
      st = enqueue_steps(L, trials, false);
      if (st != OLB_B200_OK) break;
      float ms = 0.f;
      if ((e = cudaEventRecord(L->ev1, L->stream)) != cudaSuccess ||
          (e = cudaEventSynchronize(L->ev1)) != cudaSuccess ||
          (e = cudaEventElapsedTime(&ms, L->ev0, L->ev1)) != cudaSuccess) {
        st = cuda_fail(e, "autotune timing");
        break;
      }
      ms /= float(trials);
      ++tried;
      if (tried == 1 || ms < best) {
        best = ms;
        best_v = v;
        best_bz = bz;
        best_by = kStepThreads / bz;
      }
    }
  }
  // restore the state whatever happened
  e = cudaMemcpyAsync(L->pops, backup, pop_bytes, cudaMemcpyDeviceToDevice, L->stream);
  const cudaError_t e2 = cudaStreamSynchronize(L->stream);
  cudaFree(backup);
  L->parity = parity;
  L->steps_done = steps_done;
  if (st != OLB_B200_OK) return st;
  if (e != cudaSuccess) return cuda_fail(e, "autotune restore copy");
  if (e2 != cudaSuccess) return cuda_fail(e2, "autotune synchronize");
  L->variant = best_v;
  L->block_z = best_bz;
  L->block_y = best_by;
  L->tuned = true;
  L->tuned_ms = best;
  if (out) {
    olb_b200_get_tuning(L, out);
    out->candidates = tried;
  }
  return OLB_B200_OK;
}

} // extern "C"
