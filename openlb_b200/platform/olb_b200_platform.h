/* Platform::GPU_B200 — OpenLB's platform seam bound to libolb_b200.
 *
 * This header is compiled by the host C++ compiler as part of OpenLB (it is
 * included at the end of src/core/blockLattice.h when PLATFORM_GPU_B200 is
 * defined; patch_openlb.py adds the tag, the dispatch cases, the default
 * platform and that include to a copy of OpenLB's sources).  An unmodified
 * example built with PLATFORMS := CPU_SISD GPU_B200 then gets
 * ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200> blocks from the load
 * balancer (src/communication/loadBalancer.h:102-118) and every collision
 * step runs as one fused collide-and-stream kernel on the GPU behind the C ABI
 * of include/olb_b200.h.  Nothing here is CUDA: host code stays C++ and the
 * only device entry points are the ABI's.
 *
 * Design.
 *  - Host side = CPU_SISD data structures.  The block's fields, masks,
 *    parameters and dynamics map live in host memory exactly as on CPU_SISD
 *    (columns: src/core/platform/cpu/sisd/column.h:229-238), so set-up
 *    (defineDynamics, boundary::set, setParameter, defineU/defineRho,
 *    iniEquilibrium) and evaluation (functors, VTK output) run unchanged on
 *    the host copy.
 *  - Device side = one olb_b200_lattice per block (DeviceLattice below),
 *    registered in the block's Data like any field type, so the block's
 *    setProcessingContext reaches it: Simulation uploads the host state
 *    (populations, dynamics of every cell, boundary values), Evaluation
 *    downloads the populations.  The host copy is stale while the device
 *    owns the simulation, as on GPU_CUDA (src/core/platform/gpu/cuda/
 *    column.hh:157-187).
 *  - Collision: the block's custom collision operator (setCollisionO,
 *    src/core/blockLattice.h:523-531) calls olb_b200_collide_and_stream, which
 *    collides, streams (AA pattern, periodic wrap included) and applies the
 *    PostStream boundary post-processors in one call.  The host's stream()
 *    still rotates the host columns (pointer arithmetic only,
 *    src/core/platform/cpu/sisd/column.h:189-200), which the logical
 *    population access of the upload/download absorbs.
 *  - Communication: a block communicator that copies nothing.  The step
 *    kernel wraps periodic axes itself; the communicator's neighbourhood is
 *    read once to learn which axes are periodic (a single cuboid requests its
 *    own opposite face for each periodic axis).  More than one cuboid per
 *    process is rejected: halo exchange between device blocks is not built.
 *  - Dynamics: ConcreteBlockCollisionO<...,GPU_B200,DYNAMICS> records which
 *    cells a dynamics covers and describes it for the device table (kind and
 *    parameters, per cell where the reference reads per-cell fields: wall
 *    velocity and density, FORCE).  Dynamics the device does not implement
 *    raise std::runtime_error naming them when the table is built; there is
 *    no CPU fallback.
 *  - Post-processors: the statistics post-processor, the interpolated
 *    boundaries' PlaneFdBoundaryProcessor3D and the outer edge and corner
 *    processors of velocity boundaries run inside the device step (an edge
 *    or corner processor also tells the device lattice its cell's normal);
 *    any other post-processor raises std::runtime_error at set-up.
 *
 * Environment (read when a block's device lattice is created):
 *   OLB_B200_DEVICE   CUDA device ordinal (default 0)
 *   OLB_B200_STORAGE  f32 (default for float), f64 (default for double),
 *                     f16 or bf16: 16-bit shifted population storage, FP32 math
 *   OLB_B200_AUTOTUNE 0 disables the step-kernel autotuning at the first upload
 *   OLB_B200_INFLIGHT collide_and_stream calls allowed in flight (default 2):
 *                     keeps wall-clock timers of examples honest without
 *                     synchronising the device every step
 */
#ifndef OLB_B200_PLATFORM_H
#define OLB_B200_PLATFORM_H

#include <olb_b200.h>

#include <array>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

namespace olb {

/// Host storage of GPU_B200 blocks: CPU_SISD's columns
template <typename T>
struct ImplementationOf<AbstractColumn<T>,Platform::GPU_B200> {
  using type = cpu::sisd::Column<T>;
};

template <typename T>
struct ImplementationOf<AbstractCyclicColumn<T>,Platform::GPU_B200> {
  using type = cpu::sisd::CyclicColumn<T>;
};

namespace gpu {

namespace b200 {

/// Counts changes of any GPU_B200 cell's dynamics; a device lattice rebuilds
/// its dynamics table when the count moved since its last upload.
inline std::atomic<std::uint64_t>& dynamicsEpoch()
{
  static std::atomic<std::uint64_t> epoch{0};
  return epoch;
}

inline void check(olb_b200_status status, const char* what)
{
  if (status != OLB_B200_OK) {
    throw std::runtime_error(std::string("GPU_B200 ") + what + ": " + olb_b200_last_error());
  }
}

inline int envInt(const char* name, int fallback)
{
  const char* v = std::getenv(name);
  return (v && *v) ? std::atoi(v) : fallback;
}

}

}

/// Cells covered by one dynamics (or the core of the block), on the host
template <typename T>
class ConcreteBlockMask<T,Platform::GPU_B200> final : public Serializable {
private:
  cpu::sisd::Column<bool> _cells;
  std::size_t _count;

public:
  ConcreteBlockMask(std::size_t size):
    _cells(size),
    _count(0)
  { }

  AbstractColumn<bool>& asAbstract()
  {
    return _cells;
  }

  bool operator[](std::size_t iCell) const
  {
    return _cells[iCell];
  }

  void set(std::size_t iCell, bool active)
  {
    const bool was = _cells[iCell];
    if (was == active) {
      return;
    }
    _cells[iCell] = active;
    if (active) {
      ++_count;
    } else {
      --_count;
    }
    gpu::b200::dynamicsEpoch().fetch_add(1, std::memory_order_relaxed);
  }

  std::size_t weight() const
  {
    return _count;
  }

  void setProcessingContext(ProcessingContext) { }

  std::size_t getNblock() const override
  {
    return 1 + _cells.getNblock();
  }

  std::size_t getSerializableSize() const override
  {
    return sizeof(_count) + _cells.getSerializableSize();
  }

  bool* getBlock(std::size_t iBlock, std::size_t& sizeBlock, bool loadingMode) override
  {
    std::size_t currentBlock = 0;
    bool* dataPtr = nullptr;
    registerVar(iBlock, sizeBlock, currentBlock, dataPtr, _count);
    registerSerializableOfConstSize(iBlock, sizeBlock, currentBlock, dataPtr, _cells, loadingMode);
    return dataPtr;
  }
};

namespace gpu {

namespace b200 {

/// The device-table entry a dynamics maps to (olb_b200_dyn_params).  kind < 0:
/// the device has no implementation of this dynamics.
template <typename T, typename DESCRIPTOR, typename DYNAMICS>
struct Describe {
  static constexpr int kind = -1;
  static constexpr bool perCell = false;
  template <typename PARAMETERS>
  static void shared(PARAMETERS&, olb_b200_dyn_params&) { }
  template <typename BLOCK>
  static void cell(BLOCK&, CellID, olb_b200_dyn_params&) { }
};

/// RHO and VELOCITY of a boundary cell (specialised for the boundary
/// dynamics in olb_b200_dynamics.h); valued == false for all others
template <typename T, typename DESCRIPTOR, typename DYNAMICS>
struct BoundaryValues {
  static constexpr bool valued = false;
  template <typename BLOCK>
  static void get(BLOCK&, CellID, double (&v)[4])
  {
    v[0] = 1.0;
    v[1] = v[2] = v[3] = 0.0;
  }
};

/// CSE-optimized dynamics (src/cse/wrapper.h) compute what DYNAMICS computes
template <typename D>
struct Unwrap {
  using type = D;
};

template <typename D>
struct Unwrap<CSE<D>> {
  using type = D;
};

/// Value of a per-cell field of `block` at iCell, or `fallback` when the
/// field was never allocated (nothing defined it)
template <typename FIELD, typename BLOCK>
std::array<double,3> cellField(BLOCK& block, CellID iCell, double fallback)
{
  using T = typename BLOCK::value_t;
  using DESCRIPTOR = typename BLOCK::descriptor_t;
  std::array<double,3> out{fallback, fallback, fallback};
  if (block.template hasData<Array<FIELD>>()) {
    auto& field = block.template getField<FIELD>();
    for (unsigned iD = 0; iD < DESCRIPTOR::template size<FIELD>() && iD < 3; ++iD) {
      out[iD] = static_cast<double>(static_cast<T>(field[iD][iCell]));
    }
  }
  return out;
}

template <typename FIELD, typename PARAMETERS>
double parameter(PARAMETERS& parameters)
{
  return static_cast<double>(parameters.template get<FIELD>());
}

/// What a GPU_B200 collision operator tells its block's device lattice
template <typename T, typename DESCRIPTOR>
struct DeviceDynamics {
  virtual ~DeviceDynamics() = default;
  /// The host dynamics object cells of this operator point to
  virtual const Dynamics<T,DESCRIPTOR>* hostDynamics() const = 0;
  /// olb_b200_dyn_kind, or -1 if the device does not implement the dynamics
  virtual int kind() const = 0;
  virtual bool perCell() const = 0;
  virtual std::string name() const = 0;
  /// Fills the operator-wide parameters (OMEGA, MAGIC, SMAGORINSKY)
  virtual void shared(olb_b200_dyn_params& p) = 0;
  /// Fills the per-cell values (FORCE, wall VELOCITY / RHO)
  virtual void cell(ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>& block, CellID iCell,
                    olb_b200_dyn_params& p) = 0;
  /// Boundary cells (interpolated, local velocity, edges, corners): RHO and
  /// VELOCITY of the cell as defineRho / defineU set them
  virtual bool valued() const = 0;
  virtual void values(ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>& block, CellID iCell,
                      double (&v)[4]) = 0;
};

/// Kind of a post-processor that marks an external edge or corner of a
/// velocity boundary, with its discrete normal (specialised in
/// olb_b200_dynamics.h for OuterVelocityEdgeProcessor3D / CornerProcessor3D)
template <typename OPERATOR>
struct OuterNormal {
  static constexpr int kind = -1;
  static constexpr int normal[3] = {0, 0, 0};
};

/// Table kind placeholder of FixedVelocityBoundaryTuple cells: the cell's
/// edge or corner post-processor decides which one it is and its normal
constexpr int kOuterPlaceholder = 1000;

/// Device twin of one GPU_B200 block: owns the olb_b200_lattice
template <typename T, typename DESCRIPTOR>
class DeviceLattice final : public Serializable {
private:
  using BLOCK = ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>;

  BLOCK* _block = nullptr;
  olb_b200_lattice* _handle = nullptr;
  int _periodic[3] = {0, 0, 0};
  std::vector<DeviceDynamics<T,DESCRIPTOR>*> _operators;
  /// operator-wide parameters of each operator at the last table upload
  std::vector<olb_b200_dyn_params> _sharedAtUpload;
  std::uint64_t _epochAtUpload = ~std::uint64_t(0);
  bool _onDevice = false;
  /// external edge / corner cells announced by their post-processors: kind, normal
  std::unordered_map<CellID, std::array<int,4>> _outer;

  static olb_b200_dyn_params blank()
  {
    olb_b200_dyn_params p;
    std::memset(&p, 0, sizeof p);
    p.omega = 1.0;
    p.wall_rho = 1.0;
    return p;
  }

  int storage() const
  {
    const char* s = std::getenv("OLB_B200_STORAGE");
    const std::string v = s ? s : "";
    if (v == "f16") {
      return OLB_B200_STORAGE_F16;
    }
    if (v == "bf16") {
      return OLB_B200_STORAGE_BF16;
    }
    if (v == "f64" || (v.empty() && std::is_same_v<T,double>)) {
      if (!std::is_same_v<T,double>) {
        throw std::runtime_error("GPU_B200: OLB_B200_STORAGE=f64 needs a double-precision lattice");
      }
      return OLB_B200_STORAGE_F64;
    }
    if (std::is_same_v<T,double>) {
      throw std::runtime_error("GPU_B200: a double-precision lattice stores f64 populations");
    }
    return OLB_B200_STORAGE_F32;
  }

  void create()
  {
    static_assert(DESCRIPTOR::d == 3 && (DESCRIPTOR::q == 19 || DESCRIPTOR::q == 27),
                  "Platform::GPU_B200 implements the D3Q19 and D3Q27 lattices");
    static_assert(std::is_same_v<T,float> || std::is_same_v<T,double>,
                  "Platform::GPU_B200 computes in float or double");
    olb_b200_desc d;
    std::memset(&d, 0, sizeof d);
    d.q = DESCRIPTOR::q;
    d.nx = _block->getNx();
    d.ny = _block->getNy();
    d.nz = _block->getNz();
    for (int iD = 0; iD < 3; ++iD) {
      d.periodic[iD] = _periodic[iD];
    }
    d.storage = storage();
    d.device = envInt("OLB_B200_DEVICE", 0);
    check(olb_b200_create(&d, &_handle), "create");
    check(olb_b200_set_max_steps_in_flight(_handle, envInt("OLB_B200_INFLIGHT", 2)), "set_max_steps_in_flight");
  }

  /// Per-cell dynamics ids and the entries they index, from the host's dynamics map
  std::vector<std::uint8_t> _ids;
  std::vector<olb_b200_dyn_params> _table;
  std::vector<std::int64_t> _valueCells;  // boundary cells with values, logical index
  std::vector<double> _values;            // 4 per cell: RHO, VELOCITY x, y, z
  /// FORCE per cell (x of every cell, then y, then z) when the Guo-forced
  /// cells do not all share one value; empty: the entries carry the force
  std::vector<T> _forceField;

  void buildTable()
  {
    const int nx = _block->getNx(), ny = _block->getNy(), nz = _block->getNz();
    std::unordered_map<const Dynamics<T,DESCRIPTOR>*, DeviceDynamics<T,DESCRIPTOR>*> byDynamics;
    for (auto* op : _operators) {
      byDynamics[op->hostDynamics()] = op;
    }
    _sharedAtUpload.clear();
    std::unordered_map<DeviceDynamics<T,DESCRIPTOR>*, olb_b200_dyn_params> shared;
    for (auto* op : _operators) {
      olb_b200_dyn_params p = blank();
      p.kind = op->kind();
      op->shared(p);
      shared[op] = p;
      _sharedAtUpload.push_back(p);
    }
    std::map<std::string, std::uint8_t> entryOf;  // parameter bytes -> id
    std::vector<olb_b200_dyn_params> table;
    std::vector<std::uint8_t> ids(std::size_t(nx) * ny * nz);
    const Dynamics<T,DESCRIPTOR>* lastDynamics = nullptr;
    DeviceDynamics<T,DESCRIPTOR>* lastOp = nullptr;
    std::uint8_t lastSharedId = 0;
    bool lastSharedValid = false;
    std::size_t n = 0;
    _valueCells.clear();
    _values.clear();
    // FORCE of the forced cells, gathered while their entries are keyed
    // without it (one entry per forced dynamics and parameter set)
    std::vector<double> force;
    bool anyForced = false, uniformForce = true;
    double firstForce[3] = {0., 0., 0.};
    const std::size_t cells = std::size_t(nx) * ny * nz;
    for (int iX = 0; iX < nx; ++iX) {
      for (int iY = 0; iY < ny; ++iY) {
        for (int iZ = 0; iZ < nz; ++iZ, ++n) {
          const CellID iCell = _block->getCellId(iX, iY, iZ);
          const Dynamics<T,DESCRIPTOR>* dynamics = _block->getDynamics(iCell);
          if (dynamics != lastDynamics) {
            auto it = byDynamics.find(dynamics);
            if (it == byDynamics.end()) {
              throw std::runtime_error("GPU_B200: a cell's dynamics was not created by this block's dynamics map");
            }
            lastDynamics = dynamics;
            lastOp = it->second;
            lastSharedValid = false;
            if (lastOp->kind() < 0) {
              throw std::runtime_error("GPU_B200: dynamics " + lastOp->name()
                                       + " has no device implementation on this platform");
            }
          }
          if (!lastOp->perCell() && !lastOp->valued() && lastSharedValid) {
            ids[n] = lastSharedId;
            continue;
          }
          olb_b200_dyn_params p = shared[lastOp];
          if (lastOp->perCell()) {
            lastOp->cell(*_block, iCell, p);
          }
          if (p.kind == kOuterPlaceholder) {
            auto it = _outer.find(iCell);
            if (it == _outer.end()) {
              throw std::runtime_error("GPU_B200: a fixed-velocity boundary cell without an outer edge or corner "
                                       "post-processor (" + lastOp->name() + ")");
            }
            p.kind = it->second[0];
            for (int iD = 0; iD < 3; ++iD) {
              p.normal[iD] = it->second[1 + iD];
            }
          }
          if (p.kind == OLB_B200_DYN_FORCED_BGK || p.kind == OLB_B200_DYN_FORCED_TRT) {
            if (force.empty()) {
              force.assign(3 * cells, 0.);
            }
            for (int iD = 0; iD < 3; ++iD) {
              force[iD * cells + n] = p.force[iD];
              if (!anyForced) {
                firstForce[iD] = p.force[iD];
              }
              uniformForce = uniformForce && p.force[iD] == firstForce[iD];
              p.force[iD] = 0.;
            }
            anyForced = true;
          }
          if (lastOp->valued()) {
            double v[4];
            lastOp->values(*_block, iCell, v);
            _valueCells.push_back(std::int64_t(n));
            _values.insert(_values.end(), v, v + 4);
          }
          const std::string key(reinterpret_cast<const char*>(&p), sizeof p);
          auto found = entryOf.find(key);
          std::uint8_t id;
          if (found == entryOf.end()) {
            if (table.size() == 256) {
              throw std::runtime_error("GPU_B200: more than 256 distinct (dynamics, parameter) combinations; "
                                       "per-cell values that vary cell by cell are not supported");
            }
            id = std::uint8_t(table.size());
            entryOf.emplace(key, id);
            table.push_back(p);
          } else {
            id = found->second;
          }
          ids[n] = id;
          if (!lastOp->perCell()) {
            lastSharedId = id;
            lastSharedValid = true;
          }
        }
      }
    }
    _forceField.clear();
    if (anyForced && uniformForce) {
      // one value everywhere: it goes back into the entries
      for (auto& e : table) {
        if (e.kind == OLB_B200_DYN_FORCED_BGK || e.kind == OLB_B200_DYN_FORCED_TRT) {
          for (int iD = 0; iD < 3; ++iD) {
            e.force[iD] = firstForce[iD];
          }
        }
      }
    } else if (anyForced) {
      _forceField.assign(force.begin(), force.end());
    }
    _ids = std::move(ids);
    _table = std::move(table);
    _epochAtUpload = dynamicsEpoch().load(std::memory_order_relaxed);
  }

  void uploadDynamics()
  {
    bool needIds = _table.size() > 1;
    for (const auto& e : _table) {
      needIds |= e.kind >= OLB_B200_DYN_INTERPOLATED_VELOCITY;
    }
    check(olb_b200_set_dynamics(_handle, needIds ? _ids.data() : nullptr, _table.data(),
                                int32_t(_table.size())), "set_dynamics");
    check(olb_b200_set_force_field(_handle, _forceField.empty() ? nullptr : _forceField.data()),
          "set_force_field");
    if (!_valueCells.empty()) {
      check(olb_b200_set_boundary_values(_handle, _valueCells.data(), std::int64_t(_valueCells.size()),
                                         _values.data()), "set_boundary_values");
    }
  }

  /// Re-uploads the table when setParameter changed an operator-wide parameter
  bool parametersChanged()
  {
    if (_sharedAtUpload.size() != _operators.size()) {
      return true;
    }
    for (std::size_t i = 0; i < _operators.size(); ++i) {
      olb_b200_dyn_params p = blank();
      p.kind = _operators[i]->kind();
      _operators[i]->shared(p);
      if (std::memcmp(&p, &_sharedAtUpload[i], sizeof p) != 0) {
        return true;
      }
    }
    return false;
  }

  /// Core cells' populations, logical (post-stream) layout, shifted f - w
  void uploadPopulations()
  {
    const int nx = _block->getNx(), ny = _block->getNy(), nz = _block->getNz();
    const std::size_t n = std::size_t(nx) * ny * nz;
    std::vector<T> buffer(DESCRIPTOR::q * n);
    auto& pops = _block->template getField<descriptors::POPULATION>();
    for (unsigned iPop = 0; iPop < DESCRIPTOR::q; ++iPop) {
      auto& column = pops[iPop];
      T* out = buffer.data() + iPop * n;
      for (int iX = 0; iX < nx; ++iX) {
        for (int iY = 0; iY < ny; ++iY) {
          const CellID row = _block->getCellId(iX, iY, 0);
          for (int iZ = 0; iZ < nz; ++iZ) {
            *out++ = column[row + iZ];
          }
        }
      }
    }
    check(olb_b200_set_populations(_handle, buffer.data()), "set_populations");
  }

  void downloadPopulations()
  {
    const int nx = _block->getNx(), ny = _block->getNy(), nz = _block->getNz();
    const std::size_t n = std::size_t(nx) * ny * nz;
    std::vector<T> buffer(DESCRIPTOR::q * n);
    check(olb_b200_get_populations(_handle, buffer.data()), "get_populations");
    auto& pops = _block->template getField<descriptors::POPULATION>();
    for (unsigned iPop = 0; iPop < DESCRIPTOR::q; ++iPop) {
      auto& column = pops[iPop];
      const T* in = buffer.data() + iPop * n;
      for (int iX = 0; iX < nx; ++iX) {
        for (int iY = 0; iY < ny; ++iY) {
          const CellID row = _block->getCellId(iX, iY, 0);
          for (int iZ = 0; iZ < nz; ++iZ) {
            column[row + iZ] = *in++;
          }
        }
      }
    }
  }

public:
  DeviceLattice(std::size_t) { }

  ~DeviceLattice()
  {
    if (_handle) {
      olb_b200_destroy(_handle);
    }
  }

  DeviceLattice(const DeviceLattice&) = delete;
  DeviceLattice& operator=(const DeviceLattice&) = delete;

  /// Platform-independent view, as BlockLattice::getData returns it
  DeviceLattice& asAbstract()
  {
    return *this;
  }

  /// The device twin of `block`, created with the block's first dynamics
  static DeviceLattice& of(BLOCK& block);

  void attach(BLOCK& block)
  {
    if (_block) {
      return;
    }
    _block = &block;
    block.setCollisionO([this](BLOCK&) {
      collide();
    });
  }

  void enroll(DeviceDynamics<T,DESCRIPTOR>* op)
  {
    _operators.push_back(op);
  }

  /// An external edge or corner cell, announced by its post-processor
  void setOuter(CellID iCell, int kind, const int (&normal)[3])
  {
    _outer[iCell] = {kind, normal[0], normal[1], normal[2]};
    dynamicsEpoch().fetch_add(1, std::memory_order_relaxed);
  }

  void setPeriodic(int axis)
  {
    if (_periodic[axis]) {
      return;
    }
    if (_handle) {
      throw std::runtime_error("GPU_B200: periodicity changed after the device lattice was created");
    }
    _periodic[axis] = 1;
  }

  /// Host -> device on Simulation, device -> host on Evaluation
  void setProcessingContext(ProcessingContext context)
  {
    if (!_block) {
      return;
    }
    if (context == ProcessingContext::Simulation) {
      buildTable();
      const bool first = !_handle;
      if (first) {
        create();
      }
      uploadDynamics();
      uploadPopulations();
      if (first && envInt("OLB_B200_AUTOTUNE", 1) != 0) {
        olb_b200_tuning tuning;
        check(olb_b200_autotune(_handle, 0, &tuning), "autotune");
      }
      _onDevice = true;
    } else if (_onDevice) {
      downloadPopulations();
      _onDevice = false;
    }
  }

  /// One collide-and-stream step of the block on the device
  void collide()
  {
    if (!_onDevice) {
      setProcessingContext(ProcessingContext::Simulation);
    }
    if (_epochAtUpload != dynamicsEpoch().load(std::memory_order_relaxed) || parametersChanged()) {
      buildTable();
      uploadDynamics();
    }
    if (_block->statisticsEnabled()) {
      olb_b200_stats stats;
      check(olb_b200_collide_and_stream(_handle, 1, &stats), "collide_and_stream");
      typename LatticeStatistics<T>::Aggregatable sums{};
      sums.nCells = std::size_t(stats.n_cells);
      sums.avRho = T(stats.sum_rho);
      sums.avEnergy = T(stats.sum_usqr);
      sums.maxU = T(stats.max_usqr);
      _block->getStatistics().incrementStats(sums);
    } else {
      check(olb_b200_collide_and_stream(_handle, 1, nullptr), "collide_and_stream");
    }
  }

  olb_b200_lattice* handle()
  {
    return _handle;
  }

  // not serialized: the populations are the block's POPULATION field
  std::size_t getNblock() const override
  {
    return 0;
  }
  std::size_t getSerializableSize() const override
  {
    return 0;
  }
  bool* getBlock(std::size_t, std::size_t& sizeBlock, bool) override
  {
    sizeBlock = 0;
    return nullptr;
  }
};

}

}

/// Data type of a block's device twin (allocated through ConcreteData like a field)
struct GPU_B200_DEVICE_LATTICE {
  template <typename T, typename DESCRIPTOR, Platform PLATFORM>
  using type = gpu::b200::DeviceLattice<T,DESCRIPTOR>;
};

template <typename T, typename DESCRIPTOR>
gpu::b200::DeviceLattice<T,DESCRIPTOR>& gpu::b200::DeviceLattice<T,DESCRIPTOR>::of(BLOCK& block)
{
  auto& device = block.template getData<GPU_B200_DEVICE_LATTICE>();
  device.attach(block);
  return device;
}

/// Collision operator of DYNAMICS on a GPU_B200 block: bookkeeping on the
/// host, the collision itself runs in the block's fused device step
template <typename T, typename DESCRIPTOR, typename DYNAMICS>
class ConcreteBlockCollisionO<T,DESCRIPTOR,Platform::GPU_B200,DYNAMICS> final
  : public BlockCollisionO<T,DESCRIPTOR,Platform::GPU_B200>
  , public gpu::b200::DeviceDynamics<T,DESCRIPTOR> {
private:
  using describe_t = gpu::b200::Describe<T,DESCRIPTOR,typename gpu::b200::Unwrap<DYNAMICS>::type>;

  std::unique_ptr<DYNAMICS> _dynamics;
  ParametersOfOperatorD<T,DESCRIPTOR,DYNAMICS>* _parameters;
  ConcreteBlockMask<T,Platform::GPU_B200>* _mask;

public:
  ConcreteBlockCollisionO():
    _dynamics(new DYNAMICS()),
    _parameters(nullptr),
    _mask(nullptr)
  { }

  std::type_index id() const override
  {
    return typeid(DYNAMICS);
  }

  std::size_t weight() const override
  {
    return _mask->weight();
  }

  void set(CellID iCell, bool state, bool overlap) override
  {
    if (!overlap) {
      _mask->set(iCell, state);
    }
  }

  Dynamics<T,DESCRIPTOR>* getDynamics() override
  {
    return _dynamics.get();
  }

  void setup(ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>& block) override
  {
    _parameters = &block.template getData<OperatorParameters<DYNAMICS>>().parameters;
    _mask = &block.template getData<DynamicsMask<DYNAMICS>>();
    if constexpr (dynamics::has_parametrized_momenta_v<DYNAMICS>) {
      _dynamics->setMomentaParameters(_parameters);
    }
    gpu::b200::DeviceLattice<T,DESCRIPTOR>::of(block).enroll(this);
  }

  void apply(ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>&,
             ConcreteBlockMask<T,Platform::GPU_B200>&,
             CollisionDispatchStrategy) override
  {
    throw std::logic_error("GPU_B200: collisions run in the block's fused device step");
  }

  // DeviceDynamics
  const Dynamics<T,DESCRIPTOR>* hostDynamics() const override
  {
    return _dynamics.get();
  }
  int kind() const override
  {
    return describe_t::kind;
  }
  bool perCell() const override
  {
    return describe_t::perCell;
  }
  std::string name() const override
  {
    return fields::name<DYNAMICS>();
  }
  void shared(olb_b200_dyn_params& p) override
  {
    describe_t::shared(*_parameters, p);
  }
  void cell(ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>& block, CellID iCell,
            olb_b200_dyn_params& p) override
  {
    describe_t::cell(block, iCell, p);
  }
  bool valued() const override
  {
    return gpu::b200::BoundaryValues<T,DESCRIPTOR,typename gpu::b200::Unwrap<DYNAMICS>::type>::valued;
  }
  void values(ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>& block, CellID iCell,
              double (&v)[4]) override
  {
    gpu::b200::BoundaryValues<T,DESCRIPTOR,typename gpu::b200::Unwrap<DYNAMICS>::type>::get(block, iCell, v);
  }
};

namespace gpu {

namespace b200 {

/// Post-processors the fused device step performs itself (the boundary
/// post-processors are added in olb_b200_dynamics.h)
template <typename OPERATOR>
struct RunsInDeviceStep : std::false_type { };

template <>
struct RunsInDeviceStep<StatisticsPostProcessor> : std::true_type { };

/// CSE-optimized post-processors (src/cse/wrapper.h) compute what OPERATOR computes
template <typename OPERATOR>
struct UnwrapOperator {
  using type = OPERATOR;
};

template <typename OPERATOR, typename D>
struct UnwrapOperator<CSE_O<OPERATOR,D>> {
  using type = OPERATOR;
};

}

}

/// Post-processor on a GPU_B200 block: accepted only when the device step
/// already performs it
template <typename T, typename DESCRIPTOR, typename OPERATOR, OperatorScope SCOPE>
class ConcreteBlockO<T,DESCRIPTOR,Platform::GPU_B200,OPERATOR,SCOPE> final
  : public BlockO<T,DESCRIPTOR,Platform::GPU_B200> {
private:
  using op_t = typename gpu::b200::UnwrapOperator<OPERATOR>::type;
  using outer_t = gpu::b200::OuterNormal<op_t>;

  std::size_t _cells = 0;
  gpu::b200::DeviceLattice<T,DESCRIPTOR>* _device = nullptr;

public:
  std::type_index id() const override
  {
    return typeid(OPERATOR);
  }

  void set(CellID iCell, bool state) override
  {
    if (state) {
      ++_cells;
      if constexpr (outer_t::kind >= 0) {
        _device->setOuter(iCell, outer_t::kind, outer_t::normal);
      }
    }
  }

  void setup(ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>& block) override
  {
    if constexpr (!gpu::b200::RunsInDeviceStep<op_t>::value) {
      throw std::runtime_error("GPU_B200: post-processor " + fields::name<OPERATOR>()
                               + " has no device implementation on this platform");
    }
    _device = &gpu::b200::DeviceLattice<T,DESCRIPTOR>::of(block);
  }

  void apply(ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>&) override { }

  std::size_t weight() const override
  {
    return _cells;
  }
};

/// Overlap communication of a GPU_B200 block: nothing to copy (the device
/// step wraps periodic axes itself); the neighbourhood tells which axes wrap
template <typename T, typename DESCRIPTOR>
class ConcreteBlockCommunicator<ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>>
  final : public BlockCommunicator {
public:
  ConcreteBlockCommunicator(SuperLattice<T,DESCRIPTOR>& super,
                            LoadBalancer<T>& loadBalancer,
#ifdef PARALLEL_MODE_MPI
                            SuperCommunicationTagCoordinator<T>&,
                            MPI_Comm,
#endif
                            int iC,
                            const BlockCommunicationNeighborhood<T,DESCRIPTOR::d>& neighborhood)
  {
    using BLOCK = ConcreteBlockLattice<T,DESCRIPTOR,Platform::GPU_B200>;
    auto& block = super.template getBlock<BLOCK>(iC);
    auto& device = gpu::b200::DeviceLattice<T,DESCRIPTOR>::of(block);
    const int self = loadBalancer.glob(iC);
    neighborhood.forNeighbors([&](int remoteC) {
      if (remoteC != self) {
        throw std::runtime_error("GPU_B200 runs one cuboid per process: cuboid " + std::to_string(self)
                                 + " exchanges overlap with cuboid " + std::to_string(remoteC));
      }
      const auto core = block.getExtent();
      for (CellID iCell : neighborhood.getCellsInboundFrom(remoteC)) {
        const auto r = block.getLatticeR(iCell);
        for (int iD = 0; iD < 3; ++iD) {
          if (r[iD] < 0 || r[iD] >= core[iD]) {
            device.setPeriodic(iD);
          }
        }
      }
    });
  }

#ifdef PARALLEL_MODE_MPI
  void receive() override { }
  void send() override { }
  void unpack() override { }
  void wait() override { }
#else
  void copy() override { }
#endif
};

}

#endif
