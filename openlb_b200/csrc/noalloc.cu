// olb_b200_collide_and_stream_noalloc: the fused step on caller-owned device
// memory, allocating nothing.
//
// Who needs it: callers that must not allocate device memory themselves or
// through this library — a solver embedded in a host application that owns a
// fixed device-memory pool (its allocator hands out every byte and forbids
// cudaMalloc/cudaFree from plug-ins), or a service that sizes its memory once
// at start-up and must not allocate on the request path.  Such a caller keeps
// the populations in its own buffer and still wants OpenLB's per-step
// statistics, whose reduction needs per-block scratch.
//
// The scratch is a file-scope __device__ array of fixed size (below).  Every
// GPU that loads this library holds it until the process exits.  Host code
// cannot pass the array's name to a kernel (on the host it names a host-side
// stand-in, not device memory), so the first call on each device looks up the
// device address with cudaGetSymbolAddress, with that device current, and
// keeps it.  That first call should come before any stream capture.
//
// All calls share the one array: calls whose device work overlaps (two host
// threads, or two streams) race on it and must be serialised by the caller.
// Each call overwrites every scratch slot it later reads, so nothing needs to
// start at zero; the array keeps the last call's contents.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/olb_b200.h"
#include "aa_kernels.cuh"

namespace olb_b200 {

#define OLB_B200_EXTERN_STEP(Q, S, R)                                                              \
  extern template cudaError_t launch_step<Q, S, R>(const StepLaunch&, int, bool, bool, bool);
OLB_B200_EXTERN_STEP(19, float, float)
OLB_B200_EXTERN_STEP(19, double, double)
OLB_B200_EXTERN_STEP(19, __half, float)
OLB_B200_EXTERN_STEP(19, __nv_bfloat16, float)
OLB_B200_EXTERN_STEP(27, float, float)
OLB_B200_EXTERN_STEP(27, double, double)
OLB_B200_EXTERN_STEP(27, __half, float)
OLB_B200_EXTERN_STEP(27, __nv_bfloat16, float)

namespace detail {
DynDevice<float> device_params_f32(int q, const olb_b200_dyn_params& in);
DynDevice<double> device_params_f64(int q, const olb_b200_dyn_params& in);
bool fluid_kind(int kind);
void set_last_error(const std::string& message);  // read by olb_b200_last_error()
} // namespace detail

} // namespace olb_b200

using namespace olb_b200;

namespace {

// Scratch for the per-block statistics partials plus one slot for the reduced
// result: (65536 + 1) * 40 B = 2.5 MiB per device.  A call with statistics
// launches ceil(nz/bz) * ceil(ny/by) * nx blocks, (bz, by) = (128, 2) for
// nz >= 128, (64, 4) for nz >= 64, else (32, 8): 65536 blocks cover a
// 256 x 256 x 256 lattice, but only 2048 x 256 x 16 for a thin one.
constexpr size_t kMaxBlocks = 65536;
static __device__ __align__(256) StatPartial g_noalloc_scratch[kMaxBlocks + 1];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
StatPartial* g_scratch_addr[kMaxDevices] = {};

olb_b200_status noalloc_fail(olb_b200_status code, const std::string& msg)
{
  detail::set_last_error(msg);
  return code;
}

olb_b200_status noalloc_cuda(cudaError_t e, const char* what)
{
  return noalloc_fail(OLB_B200_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Device address of the scratch array on `device` (the current device),
// looked up on the first call on that device and kept for the process: after
// cudaDeviceReset on that device the kept address is stale, so callers that
// reset a device must not use this entry point on it afterwards.
olb_b200_status scratch_address(int device, StatPartial** out)
{
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return noalloc_cuda(e, "cudaGetSymbolAddress(scratch)");
    g_scratch_addr[device] = static_cast<StatPartial*>(ptr);
  }
  *out = g_scratch_addr[device];
  return OLB_B200_OK;
}

} // namespace

extern "C" olb_b200_status olb_b200_collide_and_stream_noalloc(
  const olb_b200_desc* desc, void* device_pops, int64_t steps_done, const olb_b200_dyn_params* bulk,
  int32_t steps, olb_b200_stats* stats, void* stream)
{
  detail::set_last_error("");
  if (!desc || !device_pops || !bulk) return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: null argument");
  if (desc->q != 19 && desc->q != 27) return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: q must be 19 or 27");
  if (desc->nx < 1 || desc->ny < 1 || desc->nz < 1 || desc->storage < 0 || desc->storage > 3)
    return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: invalid lattice description");
  if (desc->reserved[0] || desc->reserved[1] || desc->reserved[2])
    return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: reserved fields must be zero");
  // the step grid puts x in gridDim.z
  if (desc->nx > 65535) return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: nx exceeds 65535");
  // One bulk dynamics and no walls: the step wraps every axis.  A box with
  // closed faces needs wall cells (per-cell dynamics), which only a lattice
  // handle carries.
  if (desc->periodic[0] != 1 || desc->periodic[1] != 1 || desc->periodic[2] != 1)
    return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: every axis must be periodic "
                        "(periodic = {1,1,1}); lattices with walls need a lattice handle");
  if (desc->device < 0 || desc->device >= kMaxDevices)
    return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: device ordinal out of range");
  if (steps < 1 || steps_done < 0) return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: steps must be >= 1");
  if (!detail::fluid_kind(bulk->kind) || !(bulk->omega > 0.0 && bulk->omega < 2.0))
    return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: bulk dynamics must be a fluid "
                        "collision with omega in (0,2)");
  const size_t cells = size_t(desc->nx) * desc->ny * desc->nz;
  if (cells > (size_t(1) << 31)) return noalloc_fail(OLB_B200_ERR_ARG, "collide_and_stream_noalloc: too many cells");

  Geometry g{desc->nx, desc->ny, desc->nz, uint32_t((cells + 63) / 64 * 64)};
  // the library's default launch shape
  const int bz = desc->nz >= 128 ? 128 : (desc->nz >= 64 ? 64 : 32);
  const int by = 256 / bz;
  // one cell per thread (step variant 0): 65536 blocks cover 256^3 cells
  const int variant = 0;
  const dim3 grid = step_grid(g, bz, by, kStepVariants[variant].cells_per_thread);
  const size_t blocks = size_t(grid.x) * grid.y * grid.z;
  if (stats && blocks > kMaxBlocks) {
    char buf[256];
    snprintf(buf, sizeof buf, "collide_and_stream_noalloc: with statistics the lattice needs "
             "ceil(nz/%d)*ceil(ny/%d)*nx = %zu reduction blocks; the fixed scratch holds %zu",
             bz, by, blocks, kMaxBlocks);
    return noalloc_fail(OLB_B200_ERR_ARG, buf);
  }

  cudaError_t e = cudaSetDevice(desc->device);
  if (e != cudaSuccess) return noalloc_cuda(e, "cudaSetDevice");
  StatPartial* scratch = nullptr;
  olb_b200_status st = scratch_address(desc->device, &scratch);
  if (st != OLB_B200_OK) return st;

  const bool f64 = desc->storage == OLB_B200_STORAGE_F64;
  alignas(16) unsigned char params[sizeof(DynDevice<double>)];
  if (f64) {
    const DynDevice<double> d = detail::device_params_f64(desc->q, *bulk);
    std::memcpy(params, &d, sizeof d);
  } else {
    const DynDevice<float> d = detail::device_params_f32(desc->q, *bulk);
    std::memcpy(params, &d, sizeof d);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int k = 0; k < steps; ++k) {
    const bool last_stats = stats && k == steps - 1;
    StepLaunch a;
    a.pops = device_pops;
    a.g = g;
    a.ids = nullptr;
    a.table = nullptr;
    a.bulk = params;
    a.partials = last_stats ? scratch : nullptr;
    a.block_z = bz;
    a.block_y = by;
    a.variant = variant;
    a.stream = s;
    const bool odd = ((steps_done + k) & 1) != 0;
    switch (desc->storage) {
    case OLB_B200_STORAGE_F32:
      e = desc->q == 19 ? launch_step<19, float, float>(a, bulk->kind, odd, false, last_stats)
                        : launch_step<27, float, float>(a, bulk->kind, odd, false, last_stats);
      break;
    case OLB_B200_STORAGE_F64:
      e = desc->q == 19 ? launch_step<19, double, double>(a, bulk->kind, odd, false, last_stats)
                        : launch_step<27, double, double>(a, bulk->kind, odd, false, last_stats);
      break;
    case OLB_B200_STORAGE_F16:
      e = desc->q == 19 ? launch_step<19, __half, float>(a, bulk->kind, odd, false, last_stats)
                        : launch_step<27, __half, float>(a, bulk->kind, odd, false, last_stats);
      break;
    default:
      e = desc->q == 19 ? launch_step<19, __nv_bfloat16, float>(a, bulk->kind, odd, false, last_stats)
                        : launch_step<27, __nv_bfloat16, float>(a, bulk->kind, odd, false, last_stats);
      break;
    }
    if (e != cudaSuccess) return noalloc_cuda(e, "step kernel launch");
  }
  if (!stats) return OLB_B200_OK;

  StatPartial* result = scratch + kMaxBlocks;
  reduce_partials_kernel<<<1, 1024, 0, s>>>(scratch, blocks, result);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_cuda(e, "statistics reduction launch");
  StatPartial p;
  e = cudaMemcpyAsync(&p, result, sizeof p, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return noalloc_cuda(e, "statistics read-back");
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return noalloc_cuda(e, "cudaStreamSynchronize");
  stats->sum_rho = p.sum_rho;
  stats->sum_usqr = p.sum_usqr;
  stats->max_usqr = p.max_usqr;
  stats->n_cells = int64_t(p.n_cells);
  stats->average_rho = p.n_cells ? p.sum_rho / double(p.n_cells) : 0.0;
  stats->average_energy = p.n_cells ? 0.5 * p.sum_usqr / double(p.n_cells) : 0.0;
  stats->max_u = std::sqrt(p.max_usqr);
  stats->n_nonfinite = int64_t(p.n_nonfinite);
  if (p.n_nonfinite) return noalloc_fail(OLB_B200_ERR_DIVERGED, "collide_and_stream_noalloc: non-finite cells");
  return OLB_B200_OK;
}
