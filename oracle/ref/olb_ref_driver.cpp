/* Reference driver: runs OpenLB's own SuperLattice on a case described by
 * plain files and dumps the post-stream state.  It is test infrastructure —
 * it produces the golden fixtures and the timed CPU baseline; it is never part
 * of the product.  It is compiled from the reference's sources where they lie
 * by oracle/ref/Makefile into oracle/_ref/ (git-ignored).
 *
 * Everything it does goes through OpenLB's public user API, exactly like an
 * example program (examples/laminar/cavity3dBenchmark/cavity3d.cpp:154-243):
 *   CuboidDecomposition3D + setPeriodicity      geometry/cuboidDecomposition.h:66
 *   SuperGeometry material numbers              geometry/blockGeometry.h:108-121
 *   SuperLattice::defineDynamics<...>           core/superLattice.hh:286-291
 *   setParameter<OMEGA/MAGIC/SMAGORINSKY>       core/blockLattice.h:562-572
 *   defineField<FORCE>, defineU (lid velocity)  core/superLattice.h:287-303
 *   Cell::operator[] for populations            core/platform/cpu/cell.h:174-176
 *   collideAndStream                            core/superLattice.hh:601-663
 *   SuperLatticeDensity3D / Velocity3D          functors/lattice/latticeVelocity3D.hh:44-71
 *
 * Case directory layout (all arrays z fastest, x slowest, core cells only):
 *   case.txt        key/value lines (see parse_case)
 *   materials.i32   int32[nx*ny*nz]
 *   init.bin        T[q][nx*ny*nz] shifted populations (f_i - w_i)   (init pops)
 *   rhou.bin        T[4][nx*ny*nz] rho, ux, uy, uz for iniEquilibrium (init eq)
 *   bcvalues.bin    T[4][nx*ny*nz] rho, ux, uy, uz defined on the cells of
 *                   interpolated velocity / pressure materials   (bcvalues 1)
 * Outputs written into the same directory:
 *   out_pops.bin    T[q][nx*ny*nz]   populations after `steps` collideAndStream
 *   out_rho.bin     T[nx*ny*nz]      SuperLatticeDensity3D
 *   out_u.bin       T[3][nx*ny*nz]   SuperLatticeVelocity3D
 *   out_stats.txt   one line per step: avgRho avgEnergy maxU  (when `stats 1`)
 *   out_normals.i32 int32[4][nx*ny*nz] discrete normal type, n_x, n_y, n_z of
 *                   every boundary-condition cell, type -1 elsewhere (`normals 1`;
 *                   `normals 2` stops after writing it)
 *
 * Interpolated boundaries (`dyn <m> interpolated_velocity|interpolated_pressure`)
 * and local boundaries (`dyn <m> local_velocity|local_pressure`) are set like the
 * examples do, boundary::set<InterpolatedVelocity<T,D,MIXIN>>,
 * boundary::set<LocalVelocity<T,D,MIXIN>> or boundary::set<LocalPressure<T,D,MIXIN>>
 * (boundary/setBoundary.h:150-157, boundary/interpolatedVelocity3D.h:36-98,
 * boundary/localVelocity3D.h:36-120, boundary/localPressure3D.h:36-66),
 * with the fluid material 1 and the outside material 0; MIXIN is the bulk
 * dynamics named by `bcmixin`.  Their boundary values go through Cell::defineRho
 * and Cell::defineU (core/cell.h:194-198).
 * Checkpoints: `save <name>` writes the lattice after the steps with
 * SuperLattice::save (core/superLattice.hh:807-842) into <name>_rank0_size1.dat;
 * `load <name>` resumes from such a file after initialize() instead of the
 * initial state.
 * Bench mode (`bench <warmup> <steps>` in case.txt) prints one JSON line with
 * MLUPS measured by OpenLB's own util::Timer (utilities/timer.hh:36-76).
 */
#include <olb.h>

#include <chrono>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

using namespace olb;

#ifndef DRV_T
#define DRV_T float
#endif
#ifndef DRV_Q
#define DRV_Q 19
#endif

using T = DRV_T;
#if DRV_Q == 19
using DESCRIPTOR = descriptors::D3Q19<descriptors::FORCE>;
#else
using DESCRIPTOR = descriptors::D3Q27<descriptors::FORCE>;
#endif

namespace {

struct Case {
  int nx = 0, ny = 0, nz = 0;
  bool periodic[3] = {false, false, false};
  std::map<int, std::string> dyn;             // material -> dynamics kind
  std::map<int, std::array<double, 3>> vel;   // material -> wall velocity
  std::map<int, std::array<double, 3>> force; // material -> body force
  double omega = 1.0, magic = 0.25, smagorinsky = 0.1;
  std::string init = "pops";
  int steps = 0;
  bool stats = false;
  bool statisticsOn = false;
  int benchWarmup = -1, benchSteps = 0;
  std::string bcMixin = "bgk";
  bool bcValues = false;
  bool forceField = false;                    // FORCE per cell from forcefield.bin
  int dumpNormals = 0;
  std::string loadPath, savePath;             // checkpoints (Serializable), relative to the case dir
};

Case parse_case(const std::string& dir)
{
  Case c;
  std::ifstream in(dir + "/case.txt");
  if (!in) {
    throw std::runtime_error("cannot open " + dir + "/case.txt");
  }
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string key;
    if (!(ls >> key) || key[0] == '#') {
      continue;
    }
    if (key == "size") { ls >> c.nx >> c.ny >> c.nz; }
    else if (key == "periodic") { int a, b, d; ls >> a >> b >> d; c.periodic[0] = a; c.periodic[1] = b; c.periodic[2] = d; }
    else if (key == "dyn") { int m; std::string k; ls >> m >> k; c.dyn[m] = k; }
    else if (key == "velocity") { int m; std::array<double,3> u; ls >> m >> u[0] >> u[1] >> u[2]; c.vel[m] = u; }
    else if (key == "force") { int m; std::array<double,3> g; ls >> m >> g[0] >> g[1] >> g[2]; c.force[m] = g; }
    else if (key == "omega") { ls >> c.omega; }
    else if (key == "magic") { ls >> c.magic; }
    else if (key == "smagorinsky") { ls >> c.smagorinsky; }
    else if (key == "init") { ls >> c.init; }
    else if (key == "steps") { ls >> c.steps; }
    else if (key == "stats") { int s; ls >> s; c.stats = s; c.statisticsOn = s; }
    else if (key == "bench") { ls >> c.benchWarmup >> c.benchSteps; }
    else if (key == "bcmixin") { ls >> c.bcMixin; }
    else if (key == "bcvalues") { int b; ls >> b; c.bcValues = b; }
    else if (key == "forcefield") { int b; ls >> b; c.forceField = b; }
    else if (key == "normals") { ls >> c.dumpNormals; }
    else if (key == "load") { ls >> c.loadPath; }
    else if (key == "save") { ls >> c.savePath; }
    else if (key == "lattice" || key == "dtype") { /* informational, checked below */ }
    else { throw std::runtime_error("unknown key " + key); }
  }
  return c;
}

template <typename V>
std::vector<V> read_array(const std::string& path, std::size_t n)
{
  std::vector<V> v(n);
  std::ifstream in(path, std::ios::binary);
  if (!in) {
    throw std::runtime_error("cannot open " + path);
  }
  in.read(reinterpret_cast<char*>(v.data()), n * sizeof(V));
  if (!in) {
    throw std::runtime_error("short read " + path);
  }
  return v;
}

template <typename V>
void write_array(const std::string& path, const std::vector<V>& v)
{
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(V));
}

template <typename DYN>
void define(SuperLattice<T,DESCRIPTOR>& lattice, SuperGeometry<T,3>& geometry, int m)
{
  lattice.template defineDynamics<DYN>(geometry, m);
}

// boundary conditions set with boundary::set<...> (per-cell discrete normals,
// per-cell boundary values through defineRho / defineU)
bool is_interpolated(const std::string& kind)
{
  return kind == "interpolated_velocity" || kind == "interpolated_pressure" || kind == "local_velocity" ||
         kind == "local_pressure";
}

template <typename MIXIN>
void set_interpolated(SuperLattice<T,DESCRIPTOR>& lattice, SuperGeometry<T,3>& geometry, int m,
                      const std::string& kind)
{
  if (kind == "interpolated_velocity") {
    boundary::set<boundary::InterpolatedVelocity<T,DESCRIPTOR,MIXIN>>(lattice, geometry, m);
  } else if (kind == "local_velocity") {
    boundary::set<boundary::LocalVelocity<T,DESCRIPTOR,MIXIN>>(lattice, geometry, m);
  } else if (kind == "local_pressure") {
    boundary::set<boundary::LocalPressure<T,DESCRIPTOR,MIXIN>>(lattice, geometry, m);
  } else {
    boundary::set<boundary::InterpolatedPressure<T,DESCRIPTOR,MIXIN>>(lattice, geometry, m);
  }
}

} // namespace

int main(int argc, char* argv[])
{
  initialize(&argc, &argv, false, false);
  if (argc < 2) {
    std::cerr << "usage: " << argv[0] << " <case-dir>" << std::endl;
    return 2;
  }
  const std::string dir = argv[1];
  Case cs = parse_case(dir);
  const int nx = cs.nx, ny = cs.ny, nz = cs.nz;
  const std::size_t n = std::size_t(nx) * ny * nz;
  constexpr int q = DESCRIPTOR::q;

  CuboidDecomposition3D<T> cuboids(Vector<T,3>(T(0)), T(1), Vector<int,3>(nx, ny, nz), 1);
  cuboids.setPeriodicity({cs.periodic[0], cs.periodic[1], cs.periodic[2]});
  BlockLoadBalancer<T> loadBalancer(0, 1, cuboids.size(), 0);
  SuperGeometry<T,3> geometry(cuboids, loadBalancer, 3);

  {
    auto materials = read_array<std::int32_t>(dir + "/materials.i32", n);
    auto& block = geometry.getBlockGeometry(0);
    for (int x = 0; x < nx; ++x) {
      for (int y = 0; y < ny; ++y) {
        for (int z = 0; z < nz; ++z) {
          block.set({x, y, z}, materials[(std::size_t(x) * ny + y) * nz + z]);
        }
      }
    }
    geometry.communicate();
    geometry.getStatisticsStatus() = true;
  }

  SuperLattice<T,DESCRIPTOR> lattice(geometry);
  if (!cs.statisticsOn) {
    lattice.statisticsOff();
  }

  for (auto& [m, kind] : cs.dyn) {
    if (kind == "bgk") { define<BGKdynamics<T,DESCRIPTOR>>(lattice, geometry, m); }
    else if (kind == "trt") { define<TRTdynamics<T,DESCRIPTOR>>(lattice, geometry, m); }
    else if (kind == "forced_trt") { define<ForcedTRTdynamics<T,DESCRIPTOR>>(lattice, geometry, m); }
    else if (kind == "forced_bgk") { define<ForcedBGKdynamics<T,DESCRIPTOR>>(lattice, geometry, m); }
    else if (kind == "smagorinsky") { define<SmagorinskyBGKdynamics<T,DESCRIPTOR>>(lattice, geometry, m); }
    else if (kind == "bounce_back") { define<BounceBack<T,DESCRIPTOR>>(lattice, geometry, m); }
    else if (kind == "bounce_back_velocity") { define<BounceBackVelocity<T,DESCRIPTOR>>(lattice, geometry, m); }
    else if (kind == "none" || is_interpolated(kind)) { }
    else { throw std::runtime_error("unknown dynamics " + kind); }
  }
  if (cs.dumpNormals) {
    auto& bg = geometry.getBlockGeometry(0);
    BlockIndicatorMaterial3D<T> fluidI(bg, 1);
    BlockIndicatorMaterial3D<T> outsideI(bg, 0);
    auto materials = read_array<std::int32_t>(dir + "/materials.i32", n);
    std::vector<std::int32_t> normals(4 * n, 0);
    for (int x = 0; x < nx; ++x) {
      for (int y = 0; y < ny; ++y) {
        for (int z = 0; z < nz; ++z) {
          const std::size_t i = (std::size_t(x) * ny + y) * nz + z;
          normals[i] = -1;
          auto it = cs.dyn.find(materials[i]);
          if (it == cs.dyn.end() || !is_interpolated(it->second)) {
            continue;
          }
          const auto [type, normal] = computeBoundaryTypeAndNormal(fluidI, outsideI, {x, y, z});
          normals[i] = static_cast<std::int32_t>(type);
          for (int d = 0; d < 3; ++d) {
            normals[(d + 1) * n + i] = normal[d];
          }
        }
      }
    }
    write_array(dir + "/out_normals.i32", normals);
    if (cs.dumpNormals == 2) {
      return 0;  // classification only
    }
  }
  for (auto& [m, kind] : cs.dyn) {
    if (!is_interpolated(kind)) {
      continue;
    }
    if (cs.bcMixin == "bgk") { set_interpolated<BGKdynamics<T,DESCRIPTOR>>(lattice, geometry, m, kind); }
    else if (cs.bcMixin == "trt") { set_interpolated<TRTdynamics<T,DESCRIPTOR>>(lattice, geometry, m, kind); }
    else if (cs.bcMixin == "smagorinsky") { set_interpolated<SmagorinskyBGKdynamics<T,DESCRIPTOR>>(lattice, geometry, m, kind); }
    else { throw std::runtime_error("unknown bcmixin " + cs.bcMixin); }
  }

  lattice.template setParameter<descriptors::OMEGA>(T(cs.omega));
  lattice.template setParameter<collision::TRT::MAGIC>(T(cs.magic));
  lattice.template setParameter<collision::LES::SMAGORINSKY>(T(cs.smagorinsky));

  for (auto& [m, g] : cs.force) {
    AnalyticalConst3D<T,T> forceF(std::vector<T>{T(g[0]), T(g[1]), T(g[2])});
    lattice.template defineField<descriptors::FORCE>(geometry, m, forceF);
  }
  // a FORCE value per cell (every cell; only the forced dynamics read it)
  if (cs.forceField) {
    auto force = read_array<T>(dir + "/forcefield.bin", 3 * n);
    auto& block = lattice.getBlock(0);
    for (int x = 0; x < nx; ++x) {
      for (int y = 0; y < ny; ++y) {
        for (int z = 0; z < nz; ++z) {
          const std::size_t i = (std::size_t(x) * ny + y) * nz + z;
          auto cell = block.get({x, y, z});
          cell.template setField<descriptors::FORCE>(Vector<T,3>{force[i], force[n + i], force[2 * n + i]});
        }
      }
    }
  }

  // Initial populations: either given directly, or the equilibrium of given
  // (rho, u) through Cell::iniEquilibrium (dynamics/interface.h:111-121).
  {
    auto& block = lattice.getBlock(0);
    if (cs.init == "pops") {
      auto pops = read_array<T>(dir + "/init.bin", q * n);
      for (int x = 0; x < nx; ++x) {
        for (int y = 0; y < ny; ++y) {
          for (int z = 0; z < nz; ++z) {
            auto cell = block.get({x, y, z});
            const std::size_t i = (std::size_t(x) * ny + y) * nz + z;
            for (int iPop = 0; iPop < q; ++iPop) {
              cell[iPop] = pops[iPop * n + i];
            }
          }
        }
      }
    } else if (cs.init == "eq") {
      auto rhou = read_array<T>(dir + "/rhou.bin", 4 * n);
      for (int x = 0; x < nx; ++x) {
        for (int y = 0; y < ny; ++y) {
          for (int z = 0; z < nz; ++z) {
            auto cell = block.get({x, y, z});
            const std::size_t i = (std::size_t(x) * ny + y) * nz + z;
            T u[3] = {rhou[n + i], rhou[2 * n + i], rhou[3 * n + i]};
            cell.iniEquilibrium(rhou[i], u);
          }
        }
      }
    } else {
      throw std::runtime_error("unknown init " + cs.init);
    }
  }

  // Wall velocity of moving-wall bounce-back (VELOCITY field), as the cavity
  // example does with defineU (cavity3d.cpp:131-135).
  for (auto& [m, u] : cs.vel) {
    AnalyticalConst3D<T,T> uF(std::vector<T>{T(u[0]), T(u[1]), T(u[2])});
    lattice.defineU(geometry, m, uF);
  }

  // Boundary values of interpolated velocity / pressure cells: RHO (fixed
  // density of pressure cells) and VELOCITY, per cell.
  if (cs.bcValues) {
    auto materials = read_array<std::int32_t>(dir + "/materials.i32", n);
    auto values = read_array<T>(dir + "/bcvalues.bin", 4 * n);
    auto& block = lattice.getBlock(0);
    for (int x = 0; x < nx; ++x) {
      for (int y = 0; y < ny; ++y) {
        for (int z = 0; z < nz; ++z) {
          const std::size_t i = (std::size_t(x) * ny + y) * nz + z;
          auto it = cs.dyn.find(materials[i]);
          if (it == cs.dyn.end() || !is_interpolated(it->second)) {
            continue;
          }
          auto cell = block.get({x, y, z});
          T u[3] = {values[n + i], values[2 * n + i], values[3 * n + i]};
          cell.defineRho(values[i]);
          cell.defineU(u);
        }
      }
    }
  }

  lattice.initialize();

  // Resume from a checkpoint as the examples do (bifurcation3d.cpp:560):
  // Serializable::load reads <name>_rank0_size1.dat (core/serializer.hh:64-79,
  // io/fileName.hh:51-63) and postLoad() refreshes the cyclic columns.
  if (!cs.loadPath.empty()) {
    if (!lattice.template load<false>(dir + "/" + cs.loadPath)) {
      throw std::runtime_error("cannot load checkpoint " + cs.loadPath);
    }
  }

  if (cs.benchWarmup >= 0) {
    for (int iT = 0; iT < cs.benchWarmup; ++iT) {
      lattice.collideAndStream();
    }
    util::Timer<T> timer(cs.benchSteps, geometry.getStatistics().getNvoxel());
    timer.start();
    auto t0 = std::chrono::steady_clock::now();
    for (int iT = 0; iT < cs.benchSteps; ++iT) {
      lattice.collideAndStream();
    }
    auto t1 = std::chrono::steady_clock::now();
    timer.stop();
    timer.update(cs.benchSteps);
    const double sec = std::chrono::duration<double>(t1 - t0).count();
    std::cout << "{\"mlups\": " << timer.getTotalMLUPs()
              << ", \"seconds\": " << sec
              << ", \"steps\": " << cs.benchSteps
              << ", \"nvoxel\": " << geometry.getStatistics().getNvoxel()
#ifdef PARALLEL_MODE_OMP
              << ", \"threads\": " << singleton::omp().getSize()
#else
              << ", \"threads\": 1"
#endif
              << "}" << std::endl;
    return 0;
  }

  std::ofstream statsOut;
  if (cs.stats) {
    statsOut.open(dir + "/out_stats.txt");
    statsOut.precision(17);
  }
  for (int iT = 0; iT < cs.steps; ++iT) {
    lattice.collideAndStream();
    if (cs.stats) {
      auto& st = lattice.getStatistics();
      statsOut << double(st.getAverageRho()) << " " << double(st.getAverageEnergy())
               << " " << double(st.getMaxU()) << "\n";
    }
  }
  if (!cs.savePath.empty()) {
    if (!lattice.template save<false>(dir + "/" + cs.savePath)) {
      throw std::runtime_error("cannot save checkpoint " + cs.savePath);
    }
  }
  lattice.setProcessingContext(ProcessingContext::Evaluation);

  std::vector<T> pops(q * n), rho(n), vel(3 * n);
  SuperLatticeDensity3D<T,DESCRIPTOR> densityF(lattice);
  SuperLatticeVelocity3D<T,DESCRIPTOR> velocityF(lattice);
  auto& block = lattice.getBlock(0);
  for (int x = 0; x < nx; ++x) {
    for (int y = 0; y < ny; ++y) {
      for (int z = 0; z < nz; ++z) {
        const std::size_t i = (std::size_t(x) * ny + y) * nz + z;
        auto cell = block.get({x, y, z});
        for (int iPop = 0; iPop < q; ++iPop) {
          pops[iPop * n + i] = cell[iPop];
        }
        int input[4] = {0, x, y, z};
        T r[1] = {};
        T u[3] = {};
        densityF(r, input);
        velocityF(u, input);
        rho[i] = r[0];
        vel[i] = u[0];
        vel[n + i] = u[1];
        vel[2 * n + i] = u[2];
      }
    }
  }
  write_array(dir + "/out_pops.bin", pops);
  write_array(dir + "/out_rho.bin", rho);
  write_array(dir + "/out_u.bin", vel);
  return 0;
}
