// Per-cell lattice-Boltzmann arithmetic for the sm_100a step kernels.
//
// Lattice tables follow OpenLB's descriptors bit for bit (direction order and
// weights: src/descriptor/definition/common.h:120-168 for D3Q19, :313-366 for
// D3Q27).  The collision functions restate OpenLB's generic templates; the
// order of the floating-point operations is kept identical to theirs (cited
// per function) so that a build with -fmad=false reproduces the reference's
// CPU_SISD results exactly, while the default build lets nvcc contract
// multiply-adds into FMAs.  Multiplications by a lattice vector component of
// 0 or +-1 are resolved at compile time (they are exact).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>
#include <utility>

#define OLB_DEV __device__ __forceinline__
#define OLB_HD __host__ __device__ __forceinline__

namespace olb_b200 {

// ---------------------------------------------------------------------------
// compile-time iteration

template <int B, int E, class F>
OLB_HD void static_for(F&& f)
{
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(static_cast<F&&>(f));
  }
}

// ---------------------------------------------------------------------------
// lattice descriptors

template <int Q> struct Lattice;

template <> struct Lattice<19> {
  static constexpr int q = 19;
  static constexpr int half = 9;
  OLB_HD static constexpr int c(int i, int d)
  {
    constexpr int tab[19][3] = {
      { 0, 0, 0},
      {-1, 0, 0}, { 0,-1, 0}, { 0, 0,-1}, {-1,-1, 0}, {-1, 1, 0}, {-1, 0,-1},
      {-1, 0, 1}, { 0,-1,-1}, { 0,-1, 1},
      { 1, 0, 0}, { 0, 1, 0}, { 0, 0, 1}, { 1, 1, 0}, { 1,-1, 0}, { 1, 0, 1},
      { 1, 0,-1}, { 0, 1, 1}, { 0, 1,-1}};
    return tab[i][d];
  }
  OLB_HD static constexpr int opp(int i) { return i == 0 ? 0 : (i <= 9 ? i + 9 : i - 9); }
  OLB_HD static constexpr int wnum(int) { return 1; }
  OLB_HD static constexpr int wden(int i)
  {
    return i == 0 ? 3 : ((i % 9 >= 1 && i % 9 <= 3) ? 18 : 36);
  }
};

template <> struct Lattice<27> {
  static constexpr int q = 27;
  static constexpr int half = 13;
  OLB_HD static constexpr int c(int i, int d)
  {
    constexpr int tab[27][3] = {
      { 0, 0, 0},
      {-1, 0, 0}, { 0,-1, 0}, { 0, 0,-1}, {-1,-1, 0}, {-1, 1, 0}, {-1, 0,-1},
      {-1, 0, 1}, { 0,-1,-1}, { 0,-1, 1}, {-1,-1,-1}, {-1,-1, 1}, {-1, 1,-1}, {-1, 1, 1},
      { 1, 0, 0}, { 0, 1, 0}, { 0, 0, 1}, { 1, 1, 0}, { 1,-1, 0}, { 1, 0, 1},
      { 1, 0,-1}, { 0, 1, 1}, { 0, 1,-1}, { 1, 1, 1}, { 1, 1,-1}, { 1,-1, 1}, { 1,-1,-1}};
    return tab[i][d];
  }
  OLB_HD static constexpr int opp(int i) { return i == 0 ? 0 : (i <= 13 ? i + 13 : i - 13); }
  OLB_HD static constexpr int wnum(int i)
  {
    const int k = i == 0 ? 0 : (i <= 13 ? i : i - 13);
    return k == 0 ? 8 : (k <= 3 ? 2 : 1);
  }
  OLB_HD static constexpr int wden(int i)
  {
    const int k = i == 0 ? 0 : (i <= 13 ? i : i - 13);
    return k == 0 ? 27 : (k <= 3 ? 27 : (k <= 9 ? 54 : 216));
  }
};

// Fraction::as<T>() = T(num)/T(den), rounded in T (src/utilities/fraction.h:58-62)
template <class L, class R>
OLB_HD constexpr R weight(int i) { return R(L::wnum(i)) / R(L::wden(i)); }

// Power-of-two scale applied to shifted populations in 16-bit storage: the
// power of two nearest to 1/w_i, so that (f_i - w_i)/w_i-sized deviations use
// the format's full mantissa.  Exact in binary floating point.
template <class L>
OLB_HD constexpr float storage_scale(int i)
{
  const int den = L::wden(i), num = L::wnum(i);
  // nearest power of two to den/num
  float r = float(den) / float(num);
  float p = 1.f;
  while (p * 1.41421356f < r) p *= 2.f;
  return p;
}

// ---------------------------------------------------------------------------
// per-dynamics device parameters (precomputed on the host in R, in the same
// order the reference evaluates the cell-independent parts)

enum DynKind : int32_t {
  K_NONE = 0, K_BGK = 1, K_TRT = 2, K_SMAGORINSKY = 3, K_BOUNCE_BACK = 4,
  K_BOUNCE_BACK_VELOCITY = 5, K_FORCED_BGK = 6, K_FORCED_TRT = 7,
  K_INTERP_VELOCITY = 8, K_INTERP_PRESSURE = 9,
  K_LOCAL_VELOCITY = 10, K_VELOCITY_EDGE = 11, K_VELOCITY_CORNER = 12,
  K_VELOCITY_INNER_EDGE = 13, K_VELOCITY_INNER_CORNER = 14, K_LOCAL_PRESSURE = 15
};

OLB_HD bool is_interpolated(int kind) { return kind == K_INTERP_VELOCITY || kind == K_INTERP_PRESSURE; }
// regularised flat faces (CombinedRLBdynamics with a Regularized*BoundaryTuple)
OLB_HD bool is_local(int kind) { return kind == K_LOCAL_VELOCITY || kind == K_LOCAL_PRESSURE; }
// faces whose density is fixed and whose normal velocity follows the populations
OLB_HD bool is_pressure(int kind) { return kind == K_INTERP_PRESSURE || kind == K_LOCAL_PRESSURE; }
// external edges and corners of velocity boundaries (OuterVelocity*Processor3D)
OLB_HD bool is_outer(int kind) { return kind == K_VELOCITY_EDGE || kind == K_VELOCITY_CORNER; }
// internal edges and corners of velocity boundaries (InnerEdge/InnerCornerVelocityTuple3D)
OLB_HD bool is_inner(int kind) { return kind == K_VELOCITY_INNER_EDGE || kind == K_VELOCITY_INNER_CORNER; }
// boundary cells whose values (RHO, VELOCITY) live in their entry's value box
OLB_HD bool has_values(int kind)
{
  return is_interpolated(kind) || is_local(kind) || is_outer(kind) || is_inner(kind);
}

template <class R>
struct DynDevice {
  int32_t kind;
  int32_t pad;
  R omega;          // OMEGA
  R omega_minus;    // TRT: 1/(magic/(1/omega - 1/2) + 1/2), rounded once (collision.h:239)
  R smago_pre;      // Smagorinsky prefactor Cs^2 cs^-4 2 sqrt(2)  (collisionLES.h:67-69)
  R tau_mol;        // 1/omega  (collisionLES.h:71)
  R force[3];       // FORCE
  R force_relax;    // 1 - omega/2  (lbm.h:562)
  R wall_u[3];      // VELOCITY (moving wall)
  R wall_rho;       // RHO (FixedDensity)
  R wall_term[27][3]; // 2 rho u_d c_id w_i cs^-2, evaluated as the reference does (collision.h:341-343)
  // interpolated velocity / pressure boundaries (flat faces)
  int32_t bc_dir;     // axis of the outward normal
  int32_t bc_orient;  // its sign, -1 or +1
  int32_t box[6];     // x0, y0, z0 and extents of the bounding box of the entry's cells
  int32_t nrm[3];     // edges and corners: the discrete normal
  int32_t nrm_pad;
  const R* bc_values; // per box cell: RHO, VELOCITY x, y, z (4 values)
  R* bc_u;            // per box cell: velocity of the post-stream state (3 values)
};

// index of cell (x,y,z) in the value box of its boundary entry
template <class R>
OLB_DEV uint32_t bc_index(const DynDevice<R>* e, int x, int y, int z)
{
  return (uint32_t(x - e->box[0]) * uint32_t(e->box[4]) + uint32_t(y - e->box[1])) * uint32_t(e->box[5]) +
         uint32_t(z - e->box[2]);
}

// ---------------------------------------------------------------------------
// moments

// lbm::computeRho  src/dynamics/lbm.h:266-275
template <class L, class R>
OLB_DEV R compute_rho(const R (&f)[L::q])
{
  R rho = f[0];
  static_for<1, L::q>([&](auto i) { rho += f[i]; });
  rho += R(1);
  return rho;
}

// lbm::computeJ  src/dynamics/lbm.h:279-290 (terms with c = 0 add nothing)
template <class L, class R>
OLB_DEV void compute_j(const R (&f)[L::q], R (&j)[3])
{
  j[0] = R(0); j[1] = R(0); j[2] = R(0);
  static_for<0, L::q>([&](auto i) {
    static_for<0, 3>([&](auto d) {
      constexpr int cc = L::c(i, d);
      if constexpr (cc == 1) { j[d] += f[i]; }
      else if constexpr (cc == -1) { j[d] += -f[i]; }
    });
  });
}

// lbm::computeRhoU  src/dynamics/lbm.h:300-307.  The exact build divides each
// component as the reference does; the fast build multiplies by one
// reciprocal (within one ulp of the quotient).
template <class L, class R>
OLB_DEV void compute_rho_u(const R (&f)[L::q], R& rho, R (&u)[3])
{
  rho = compute_rho<L>(f);
  compute_j<L>(f, u);
#ifdef OLB_B200_EXACT
  u[0] /= rho; u[1] /= rho; u[2] /= rho;
#else
  const R inv = R(1) / rho;
  u[0] *= inv; u[1] *= inv; u[2] *= inv;
#endif
}

// ForcedMomentum<BulkMomentum>::computeU after BulkDensity
// (src/dynamics/momenta/elements.h:1480-1488, :466-475): rho is summed twice
// in the reference; the second sum is the same value.
template <class L, class R>
OLB_DEV void compute_rho_u_forced(const R (&f)[L::q], const R (&g)[3], R& rho, R (&u)[3])
{
  compute_rho_u<L>(f, rho, u);
  u[0] += g[0] * R(0.5); u[1] += g[1] * R(0.5); u[2] += g[2] * R(0.5);
}

// The same moments plus the density deviation delta = rho - 1.  The shifted
// populations sum to delta directly; rho = delta + 1 is then the value
// lbm::computeRho gives.  The fast build's collisions use delta to form the
// equilibrium without the rho*t - t cancellation, which at low Mach numbers
// would cost FP32 most of the bits of the velocity term.
template <class L, class R>
OLB_DEV void compute_rho_delta_u(const R (&f)[L::q], R& rho, R& delta, R (&u)[3])
{
  R s = f[0];
  static_for<1, L::q>([&](auto i) { s += f[i]; });
  delta = s;
  rho = s + R(1);
  compute_j<L>(f, u);
#ifdef OLB_B200_EXACT
  u[0] /= rho; u[1] /= rho; u[2] /= rho;
#else
  const R inv = R(1) / rho;
  u[0] *= inv; u[1] *= inv; u[2] *= inv;
#endif
}

template <class L, class R>
OLB_DEV void compute_rho_delta_u_forced(const R (&f)[L::q], const R (&g)[3], R& rho, R& delta, R (&u)[3])
{
  compute_rho_delta_u<L>(f, rho, delta, u);
  u[0] += g[0] * R(0.5); u[1] += g[1] * R(0.5); u[2] += g[2] * R(0.5);
}

// util::normSqr  src/core/util.h:161-168
template <class R>
OLB_DEV R norm_sqr(const R (&u)[3])
{
  R s = u[0] * u[0];
  s += u[1] * u[1];
  s += u[2] * u[2];
  return s;
}

// c_i . u accumulated over d as equilibrium::secondOrder does (lbm.h:53-56)
template <class L, int I, class R>
OLB_DEV R c_dot(const R (&u)[3])
{
  R cu = R(0);
  bool first = true;
  static_for<0, 3>([&](auto d) {
    constexpr int cc = L::c(I, d);
    if constexpr (cc != 0) {
      const R term = cc == 1 ? u[d] : -u[d];
      if (first) { cu = term; first = false; } else { cu += term; }
    }
  });
  return cu;
}

// equilibrium::secondOrder  src/dynamics/lbm.h:50-64
template <class L, int I, class R>
OLB_DEV R feq2(R rho, const R (&u)[3], R usqr)
{
  constexpr R t = weight<L, R>(I);
  constexpr R inv_cs2 = R(3);
  const R cu = c_dot<L, I>(u);
  return rho * t * (R(1) + inv_cs2 * cu + inv_cs2 * inv_cs2 * R(0.5) * cu * cu
                    - inv_cs2 * R(0.5) * usqr) - t;
}

// ---------------------------------------------------------------------------
// collisions (in place on f; return the CellStatistic {rho, uSqr})

// collision::BGK  src/dynamics/collision.h:67-78 with equilibria::SecondOrder
// (src/dynamics/equilibrium.h:160-167), in the reference's operation order
template <class L, class R>
OLB_DEV void relax_bgk_reference(R (&f)[L::q], R rho, const R (&u)[3], R omega)
{
  const R usqr = norm_sqr(u);
  static_for<0, L::q>([&](auto i) {
    const R fe = feq2<L, i.value>(rho, u, usqr);
    f[i] *= R(1) - omega;
    f[i] += omega * fe;
  });
}

// collision::TRT  src/dynamics/collision.h:220-245, reference operation order
template <class L, class R>
OLB_DEV void relax_trt_reference(R (&f)[L::q], R rho, const R (&u)[3], R omega, R omega_minus)
{
  const R usqr = norm_sqr(u);
  R fe[L::q];
  static_for<0, L::q>([&](auto i) { fe[i] = feq2<L, i.value>(rho, u, usqr); });
  R out[L::q];
  static_for<0, L::q>([&](auto i) {
    constexpr int o = L::opp(i);
    const R fp = R(0.5) * (f[i] + f[o]);
    const R fm = R(0.5) * (f[i] - f[o]);
    const R fep = R(0.5) * (fe[i] + fe[o]);
    const R fem = R(0.5) * (fe[i] - fe[o]);
    out[i] = f[i] - (omega * (fp - fep) + omega_minus * (fm - fem));
  });
  static_for<0, L::q>([&](auto i) { f[i] = out[i]; });
}

// The equilibrium's momentum coefficient 3 w_i (with inv_cs2 = 3) applied to
// x = rho (c_i . u), with 3 w_i held as an unevaluated sum hi + lo of two R
// values (FP32 / FP64 storage; the 16-bit collisions keep one coefficient,
// their storage rounding being far larger than its bias).  hi alone is biased: in FP32
// fl(1/6) = fl(3/18) and fl(1/12) = fl(3/36) both exceed the exact value by
// the same 3.0e-8 relative, so the equilibrium's momentum sum_i hi_i c_i c_i
// rho u = (1 + 3.0e-8) rho u, and each relaxation adds omega times that bias
// to the fluid's momentum: a velocity drift that grows linearly with the step
// count (3e-4 of the velocity after 5000 steps of the 256^3 Taylor-Green
// vortex).  x hi + x lo, fused, keeps the coefficient to within rounding of
// x; the reference's form rho t (1 + 3 c.u + ...) carries the smaller bias
// of fl(1/18) (7.5e-9).  In FP64 lo is zero.
template <class L, class R, int I>
OLB_DEV R momentum_term(R x)
{
  constexpr double exact = 3.0 * double(L::wnum(I)) / double(L::wden(I));
  constexpr R hi = R(exact);
  constexpr R lo = R(exact - double(hi));
  return fma(x, hi, x * lo);
}

// The same two collisions evaluated over opposite pairs.  For c_o = -c_i the
// second-order equilibria share their even part:
//   feq_i = A + B,  feq_o = A - B,
//   A = t (delta + rho (9/2 (c.u)^2 - 3/2 |u|^2)),   B = 3 rho t (c.u),
// with delta = rho - 1 from the populations' sum (A = rho t X - t regrouped so
// nothing cancels), so each pair costs one c.u, one even and one odd term.
// Algebraically identical to the reference; rounding differs by a few ulp of
// the populations, and at low Mach numbers FP32 keeps the velocity terms the
// reference's form loses to the cancellation.
template <class L, class R>
OLB_DEV void relax_bgk_paired(R (&f)[L::q], R rho, R delta, const R (&u)[3], R omega)
{
  const R usqr = norm_sqr(u);
  const R e0 = R(-1.5) * usqr;
  const R keep = R(1) - omega;
  {
    constexpr R t = weight<L, R>(0);
    f[0] = keep * f[0] + omega * (t * (delta + rho * e0));
  }
  static_for<1, L::half + 1>([&](auto i) {
    constexpr int o = L::opp(i);
    constexpr R t = weight<L, R>(i);
    const R cu = c_dot<L, i.value>(u);
    const R ev = R(4.5) * cu * cu + e0;
    const R a = t * (delta + rho * ev);
    const R b = momentum_term<L, R, i.value>(rho * cu);
    const R fi = keep * f[i] + omega * (a + b);
    const R fo = keep * f[o] + omega * (a - b);
    f[i] = fi;
    f[o] = fo;
  });
}

template <class L, class R>
OLB_DEV void relax_trt_paired(R (&f)[L::q], R rho, R delta, const R (&u)[3], R omega, R omega_minus)
{
  const R usqr = norm_sqr(u);
  const R e0 = R(-1.5) * usqr;
  {
    constexpr R t = weight<L, R>(0);
    f[0] -= omega * (f[0] - t * (delta + rho * e0));
  }
  static_for<1, L::half + 1>([&](auto i) {
    constexpr int o = L::opp(i);
    constexpr R t = weight<L, R>(i);
    const R cu = c_dot<L, i.value>(u);
    const R ev = R(4.5) * cu * cu + e0;
    const R a = t * (delta + rho * ev);                 // symmetric part of feq
    const R b = momentum_term<L, R, i.value>(rho * cu);   // antisymmetric part
    const R dp = omega * (R(0.5) * (f[i] + f[o]) - a);
    const R dm = omega_minus * (R(0.5) * (f[i] - f[o]) - b);
    const R fi = f[i] - dp - dm;
    const R fo = f[o] - dp + dm;
    f[i] = fi;
    f[o] = fo;
  });
}

// The exact (-fmad=false) build keeps the reference's operation order so it
// reproduces the reference bit for bit; the fast build uses the pair form.
template <class L, class R>
OLB_DEV void relax_bgk(R (&f)[L::q], R rho, R delta, const R (&u)[3], R omega)
{
#ifdef OLB_B200_EXACT
  (void)delta;
  relax_bgk_reference<L>(f, rho, u, omega);
#else
  relax_bgk_paired<L>(f, rho, delta, u, omega);
#endif
}

template <class L, class R>
OLB_DEV void relax_trt(R (&f)[L::q], R rho, R delta, const R (&u)[3], R omega, R omega_minus)
{
#ifdef OLB_B200_EXACT
  (void)delta;
  relax_trt_reference<L>(f, rho, u, omega, omega_minus);
#else
  relax_trt_paired<L>(f, rho, delta, u, omega, omega_minus);
#endif
}

// lbm::addExternalForce (Guo)  src/dynamics/lbm.h:544-566, reference operation order
template <class L, class R>
OLB_DEV void add_force_reference(R (&f)[L::q], R rho, const R (&u)[3], R force_relax, const R (&g)[3])
{
  constexpr R inv_cs2 = R(3);
  static_for<0, L::q>([&](auto i) {
    constexpr R t = weight<L, R>(i);
    R cu = c_dot<L, i.value>(u);
    cu *= inv_cs2 * inv_cs2;
    R term = R(0);
    static_for<0, 3>([&](auto d) {
      constexpr int cc = L::c(i, d);
      term += ((R(cc) - u[d]) * inv_cs2 + cu * R(cc)) * g[d];
    });
    term *= t;
    term *= force_relax;
    term *= rho;
    f[i] += term;
  });
}

// The same force terms over opposite pairs: with c_opp = -c_i the terms of i
// and opp(i) are t_i (A + B) and t_i (A - B) times force_relax rho, where
// A = 9 (c_i.u)(c_i.F) - 3 u.F and B = 3 c_i.F (reassociated: agrees with the
// reference order to rounding).
template <class L, class R>
OLB_DEV void add_force_paired(R (&f)[L::q], R rho, const R (&u)[3], R force_relax, const R (&g)[3])
{
  const R fr = force_relax * rho;
  const R uf3 = R(3) * (u[0] * g[0] + u[1] * g[1] + u[2] * g[2]);
  f[0] -= uf3 * (weight<L, R>(0) * fr);
  static_for<1, L::half + 1>([&](auto i) {
    constexpr int o = L::opp(i);
    constexpr R t = weight<L, R>(i);
    const R cu = c_dot<L, i.value>(u);
    const R cf = c_dot<L, i.value>(g);
    const R a = R(9) * cu * cf - uf3;
    const R b = R(3) * cf;
    const R k = t * fr;
    f[i] += (a + b) * k;
    f[o] += (a - b) * k;
  });
}

template <class L, class R>
OLB_DEV void add_force(R (&f)[L::q], R rho, const R (&u)[3], R force_relax, const R (&g)[3])
{
#ifdef OLB_B200_EXACT
  add_force_reference<L>(f, rho, u, force_relax, g);
#else
  add_force_paired<L>(f, rho, u, force_relax, g);
#endif
}

// |Pi_neq|^2 for bulk momenta: lbm::computeStress (lbm.h:310-329) and the
// norm of ConcreteTuple::computePiNeqNormSqr (momenta/interface.h:163-172),
// with the reference's double-precision literals kept where they promote.
template <class L, class R>
OLB_DEV R pi_neq_norm_sqr(const R (&f)[L::q], R rho, const R (&u)[3])
{
  R pi[6];
  int k = 0;
  static_for<0, 3>([&](auto a) {
    static_for<a.value, 3>([&](auto b) {
      R s = R(0);
      static_for<0, L::q>([&](auto i) {
        constexpr int cc = L::c(i, a) * L::c(i, b);
        if constexpr (cc == 1) { s += f[i]; }
        else if constexpr (cc == -1) { s += -f[i]; }
      });
      s -= rho * u[a] * u[b];
      if constexpr (a.value == b.value) {
        s -= R(1) / R(3) * (rho - R(1));
      }
      pi[k++] = s;
    });
  });
  R n2 = R(double(pi[0] * pi[0]) + 2. * double(pi[1]) * double(pi[1]) + double(pi[2] * pi[2]));
  n2 = R(double(n2) + (double(pi[2] * pi[2] + pi[3] * pi[3]) + 2. * double(pi[4]) * double(pi[4])
                       + double(pi[5] * pi[5])));
  return n2;
}

// The same norm for the fast build: c_a c_b is even in c, so a population and
// its opposite enter every component of Pi as their sum (half the additions);
// the (rho - 1) term uses the populations' sum delta; the norm is formed in R.
// Algebraically the reference's quantity.
template <class L, class R>
OLB_DEV R pi_neq_norm_sqr_pairs(const R (&f)[L::q], R rho, R delta, const R (&u)[3])
{
  R P[L::half + 1];
  static_for<1, L::half + 1>([&](auto i) { P[i] = f[i] + f[L::opp(i)]; });
  R pi[6];
  static_for<0, 3>([&](auto a) {
    static_for<a.value, 3>([&](auto b) {
      constexpr int k = a.value * 3 - (a.value * (a.value - 1)) / 2 + (b.value - a.value);
      R s = R(0);
      static_for<1, L::half + 1>([&](auto i) {
        constexpr int cc = L::c(i, a) * L::c(i, b);
        if constexpr (cc == 1) { s += P[i]; }
        else if constexpr (cc == -1) { s -= P[i]; }
      });
      s -= rho * u[a] * u[b];
      if constexpr (a.value == b.value) {
        s -= R(1) / R(3) * delta;
      }
      pi[k] = s;
    });
  });
  return pi[0] * pi[0] + pi[3] * pi[3] + pi[5] * pi[5] + R(2) * (pi[1] * pi[1] + pi[2] * pi[2] + pi[4] * pi[4]);
}

// detail::SmagorinskyEffectiveOmega::computeEffectiveOmega
// src/dynamics/collisionLES.h:59-80 (the exact build keeps the reference's
// norm; the fast build uses the pair-summed one)
template <class L, class R>
OLB_DEV R smagorinsky_omega(const R (&f)[L::q], R rho, R delta, const R (&u)[3], R smago_pre, R tau_mol)
{
#ifdef OLB_B200_EXACT
  (void)delta;
  const R pnorm = sqrt(pi_neq_norm_sqr<L>(f, rho, u));
#else
  const R pnorm = sqrt(pi_neq_norm_sqr_pairs<L>(f, rho, delta, u));
#endif
  const R tau_turb = R(0.5) * (sqrt(tau_mol * tau_mol + smago_pre / rho * pnorm) - tau_mol);
  const R tau_eff = tau_mol + tau_turb;
  return R(1) / tau_eff;
}

// collision::Revert  src/dynamics/collision.h:302-309
template <class L, class R>
OLB_DEV void revert(R (&f)[L::q])
{
  static_for<1, L::half + 1>([&](auto i) {
    constexpr int o = L::opp(i);
    const R tmp = f[i];
    f[i] = f[o];
    f[o] = tmp;
  });
}

// Bulk collision dispatch on the compile-time kind.  Returns the cell
// statistic (rho, |u|^2) like the reference's collide().
template <class L, int KIND, class R>
OLB_DEV void collide_bulk(R (&f)[L::q], const DynDevice<R>& p, R& st_rho, R& st_usqr)
{
  R rho, delta, u[3];
  if constexpr (KIND == K_BGK) {
    compute_rho_delta_u<L>(f, rho, delta, u);
    relax_bgk<L>(f, rho, delta, u, p.omega);
    st_rho = rho; st_usqr = norm_sqr(u);
  } else if constexpr (KIND == K_TRT) {
    compute_rho_delta_u<L>(f, rho, delta, u);
    relax_trt<L>(f, rho, delta, u, p.omega, p.omega_minus);
    st_rho = rho; st_usqr = norm_sqr(u);
  } else if constexpr (KIND == K_SMAGORINSKY) {
    compute_rho_delta_u<L>(f, rho, delta, u);
    const R w = smagorinsky_omega<L>(f, rho, delta, u, p.smago_pre, p.tau_mol);
    relax_bgk<L>(f, rho, delta, u, w);
    st_rho = rho; st_usqr = norm_sqr(u);
  } else if constexpr (KIND == K_FORCED_BGK || KIND == K_FORCED_TRT) {
    // forcing::Guo::combined_collision::apply  src/dynamics/forcing.h:53-63
    const R g[3] = {p.force[0], p.force[1], p.force[2]};
    compute_rho_delta_u_forced<L>(f, g, rho, delta, u);
    if constexpr (KIND == K_FORCED_BGK) {
      relax_bgk<L>(f, rho, delta, u, p.omega);
    } else {
      relax_trt<L>(f, rho, delta, u, p.omega, p.omega_minus);
    }
    add_force<L>(f, rho, u, p.force_relax, g);
    st_rho = rho; st_usqr = norm_sqr(u);
  }
}

// ---------------------------------------------------------------------------
// interpolated velocity / pressure boundaries on flat faces

// Sums over the populations in the boundary plane (c_i[dir] == 0) and over
// those along the outward normal (c_i[dir] == orient), each in ascending
// population order: util::populationsContributingToVelocity
// (src/core/util.h:221-229) as velocityBMRho and FixedPressureMomentum use
// them (src/dynamics/momenta/elements.h:54-71, 604-621).
template <class L, class R>
OLB_DEV void bc_sums(const R (&f)[L::q], int dir, int orient, R& on_wall, R& normal)
{
  on_wall = R(0);
  normal = R(0);
  static_for<0, L::q>([&](auto i) {
    constexpr int c0 = L::c(i, 0), c1 = L::c(i, 1), c2 = L::c(i, 2);
    const int cd = dir == 0 ? c0 : (dir == 1 ? c1 : c2);
    if (cd == 0) {
      on_wall += f[i];
    } else if (cd == orient) {
      normal += f[i];
    }
  });
}

// computeRhoU of the exchanged momenta (generic ComputeRhoU,
// src/dynamics/momenta/interface.h:50-58); v = {RHO, VELOCITY x, y, z}:
//   velocity  BasicDirichletVelocityBoundaryTuple (momenta/aliases.h:146-151):
//             u = VELOCITY, rho = velocityBMRho(cell, u) (elements.h:54-71, 325-333)
//   pressure  BasicDirichletPressureBoundaryTuple (momenta/aliases.h:166-171):
//             rho = RHO, u = VELOCITY but u[dir] from the populations
//             (FixedPressureMomentum::computeU, elements.h:596-622)
template <class L, class R>
OLB_DEV void bc_rho_u(const R (&f)[L::q], int kind, int dir, int orient, const R* __restrict__ v, R& rho,
                      R (&u)[3])
{
  R on_wall, normal;
  bc_sums<L>(f, dir, orient, on_wall, normal);
  u[0] = v[1];
  u[1] = v[2];
  u[2] = v[3];
  const R so = R(orient);
  if (!is_pressure(kind)) {
    const R ud = dir == 0 ? u[0] : (dir == 1 ? u[1] : u[2]);
    rho = (R(2) * normal + on_wall + R(1)) / (R(1) + so * ud);
  } else {
    rho = v[0];
    const R un = so * ((R(2) * normal + on_wall + R(1)) / rho - R(1));
    if (dir == 0) {
      u[0] = un;
    } else if (dir == 1) {
      u[1] = un;
    } else {
      u[2] = un;
    }
  }
}

// MixinDynamics::exchange_momenta<...>: the mixin collision (the lattice's
// fluid collision KIND) evaluated with the boundary momenta — BGK
// (collision.h:67-78), TRT (:220-245) or Smagorinsky-BGK (collisionLES.h:59-89,
// whose stress is BulkStress of the same rho and u).
template <class L, int KIND, class R>
OLB_DEV void collide_interpolated(R (&f)[L::q], int kind, const DynDevice<R>* __restrict__ e, int x, int y,
                                  int z, R& st_rho, R& st_usqr)
{
  const R* __restrict__ v = e->bc_values + 4 * size_t(bc_index(e, x, y, z));
  R rho, u[3];
  bc_rho_u<L>(f, kind, e->bc_dir, e->bc_orient, v, rho, u);
  const R delta = rho - R(1);
  if constexpr (KIND == K_TRT) {
    relax_trt<L>(f, rho, delta, u, e->omega, e->omega_minus);
  } else if constexpr (KIND == K_SMAGORINSKY) {
    const R w = smagorinsky_omega<L>(f, rho, delta, u, e->smago_pre, e->tau_mol);
    relax_bgk<L>(f, rho, delta, u, w);
  } else {
    relax_bgk<L>(f, rho, delta, u, e->omega);
  }
  st_rho = rho;
  st_usqr = norm_sqr(u);
}

// equilibrium<DESCRIPTOR>::fromPiToFneq  src/dynamics/lbm.h:225-247
template <class L, int I, class R>
OLB_DEV R from_pi_to_fneq(const R (&pi)[6])
{
  R fneq = R(0);
  static_for<0, 3>([&](auto a) {
    static_for<a.value, 3>([&](auto b) {
      constexpr int k = a.value * 3 - (a.value * (a.value - 1)) / 2 + (b.value - a.value);
      R to_add = R(L::c(I, a) * L::c(I, b));
      if constexpr (a.value == b.value) {
        to_add -= R(1) / R(3);
      } else {
        to_add *= R(2);
      }
      to_add *= pi[k];
      fneq += to_add;
    });
  });
  fneq *= weight<L, R>(I) * R(3) * R(3) / R(2);
  return fneq;
}

// BoundaryHelpers<T,DESCRIPTOR,direction,orientation>::computeStress
// (src/boundary/helper.h:31-80), the stress of momenta::RegularizedBoundaryStress
// (src/dynamics/momenta/elements.h:1667-1673): non-equilibrium parts of the
// populations in the wall plane (c_i[dir] == 0; the rest population counts as
// zero) and, doubled, of those along the outward normal, each set in ascending
// population order.
template <class L, class R>
OLB_DEV void boundary_stress(const R (&f)[L::q], int dir, int orient, R rho, const R (&u)[3], R (&pi)[6])
{
  const R usqr = norm_sqr(u);
  R fneq[L::q];
  static_for<0, L::q>([&](auto i) {
    constexpr int c0 = L::c(i, 0), c1 = L::c(i, 1), c2 = L::c(i, 2);
    const int cd = dir == 0 ? c0 : (dir == 1 ? c1 : c2);
    fneq[i] = R(0);
    if ((cd == 0 && i.value != 0) || cd == orient) {
      fneq[i] = f[i] - feq2<L, i.value>(rho, u, usqr);
    }
  });
  static_for<0, 3>([&](auto a) {
    static_for<a.value, 3>([&](auto b) {
      constexpr int k = a.value * 3 - (a.value * (a.value - 1)) / 2 + (b.value - a.value);
      R sum = R(0);
      static_for<0, L::q>([&](auto i) {
        constexpr int cab = L::c(i, a) * L::c(i, b);
        const int cd = dir == 0 ? L::c(i, 0) : (dir == 1 ? L::c(i, 1) : L::c(i, 2));
        if (cd == 0) sum += R(cab) * fneq[i];
      });
      static_for<0, L::q>([&](auto i) {
        constexpr int cab = L::c(i, a) * L::c(i, b);
        const int cd = dir == 0 ? L::c(i, 0) : (dir == 1 ? L::c(i, 1) : L::c(i, 2));
        if (cd == orient) sum += R(2 * cab) * fneq[i];
      });
      pi[k] = sum;
    });
  });
}

// CombinedRLBdynamics<MIXIN, Regularized{Velocity,Pressure}BoundaryTuple<dir,orient>>
// ::collide (src/dynamics/dynamics.h:419-430; tuples momenta/aliases.h:128-141):
// momenta rho = velocityBMRho, u = VELOCITY (velocity faces) or rho = RHO,
// u = VELOCITY with u[dir] from the populations (pressure faces,
// FixedPressureMomentum::computeU, elements.h:594-616); pi = the regularised
// boundary stress; the populations are rebuilt as feq + fneq(pi), then the
// mixin collides with the same momenta evaluated again on the rebuilt cell.
template <class L, int KIND, class R>
OLB_DEV void collide_local(R (&f)[L::q], int kind, const DynDevice<R>* __restrict__ e, int x, int y, int z,
                           R& st_rho, R& st_usqr)
{
  const R* __restrict__ v = e->bc_values + 4 * size_t(bc_index(e, x, y, z));
  const int dir = e->bc_dir, orient = e->bc_orient;
  R rho, u[3], pi[6];
  bc_rho_u<L>(f, kind, dir, orient, v, rho, u);
  boundary_stress<L>(f, dir, orient, rho, u, pi);
  {
    const R usqr = norm_sqr(u);
    static_for<0, L::q>([&](auto i) { f[i] = feq2<L, i.value>(rho, u, usqr) + from_pi_to_fneq<L, i.value>(pi); });
  }
  bc_rho_u<L>(f, kind, dir, orient, v, rho, u);
  const R delta = rho - R(1);
  if constexpr (KIND == K_TRT) {
    relax_trt<L>(f, rho, delta, u, e->omega, e->omega_minus);
  } else {
    relax_bgk<L>(f, rho, delta, u, e->omega);
  }
  st_rho = rho;
  st_usqr = norm_sqr(u);
}

// velocityBMRho<dir,orient>(cell, u)  src/dynamics/momenta/elements.h:54-71
template <class L, class R>
OLB_DEV R velocity_bm_rho(const R (&f)[L::q], int dir, int orient, const R (&u)[3])
{
  R on_wall, normal;
  bc_sums<L>(f, dir, orient, on_wall, normal);
  const R ud = dir == 0 ? u[0] : (dir == 1 ? u[1] : u[2]);
  return (R(2) * normal + on_wall + R(1)) / (R(1) + R(orient) * ud);
}

// the two normal axes of an edge in the template order <plane, n[(plane+1)%3],
// n[(plane+2)%3]> (src/boundary/setBoundary3D.h:156-197)
OLB_DEV void edge_axes(const int32_t (&n)[3], int& d1, int& d2)
{
  const int plane = n[0] == 0 ? 0 : (n[1] == 0 ? 1 : 2);
  d1 = plane == 2 ? 0 : plane + 1;
  d2 = plane == 0 ? 2 : plane - 1;
}

// InnerEdgeDensity3D (src/dynamics/momenta/elements.h:427-438): the mean of
// velocityBMRho along the edge's two normal axes; InnerCornerDensity3D
// (:400-411): along all three
template <class L, class R>
OLB_DEV R inner_rho(const R (&f)[L::q], int kind, const int32_t (&n)[3], const R (&u)[3])
{
  if (kind == K_VELOCITY_INNER_CORNER) {
    const R rx = velocity_bm_rho<L>(f, 0, n[0], u);
    const R ry = velocity_bm_rho<L>(f, 1, n[1], u);
    const R rz = velocity_bm_rho<L>(f, 2, n[2], u);
    return (rx + ry + rz) / R(3);
  }
  int d1, d2;
  edge_axes(n, d1, d2);
  const R r1 = velocity_bm_rho<L>(f, d1, n[d1], u);
  const R r2 = velocity_bm_rho<L>(f, d2, n[d2], u);
  return (r1 + r2) / R(2);
}

// InnerEdgeStress3D (src/dynamics/momenta/elements.h:1739-1757): populations
// arriving from both walls (c_i = -n on both normal axes) replaced by their
// opposites' non-equilibrium parts; InnerCornerStress3D (:1711-1730): the one
// population along -n (D3Q27 only); then lbm::computeStress (src/dynamics/lbm.h:311-329)
template <class L, class R>
OLB_DEV void inner_stress(const R (&f)[L::q], int kind, const int32_t (&n)[3], R rho, const R (&u)[3],
                          R (&pi)[6])
{
  const R usqr = norm_sqr(u);
  int d1 = 0, d2 = 1;
  if (kind != K_VELOCITY_INNER_CORNER) edge_axes(n, d1, d2);
  R g[L::q];
  static_for<0, L::q>([&](auto i) {
    constexpr int o = L::opp(i);
    constexpr int c0 = L::c(i, 0), c1 = L::c(i, 1), c2 = L::c(i, 2);
    const int ca = d1 == 0 ? c0 : (d1 == 1 ? c1 : c2);
    const int cb = d2 == 0 ? c0 : (d2 == 1 ? c1 : c2);
    const bool unknown = kind == K_VELOCITY_INNER_CORNER ? (c0 == -n[0] && c1 == -n[1] && c2 == -n[2])
                                                          : (ca == -n[d1] && cb == -n[d2]);
    g[i] = unknown ? f[o] - feq2<L, o>(rho, u, usqr) + feq2<L, i.value>(rho, u, usqr) : f[i];
  });
  static_for<0, 3>([&](auto a) {
    static_for<a.value, 3>([&](auto b) {
      constexpr int k = a.value * 3 - (a.value * (a.value - 1)) / 2 + (b.value - a.value);
      R sum = R(0);
      static_for<0, L::q>([&](auto i) { sum += R(L::c(i, a) * L::c(i, b)) * g[i]; });
      sum -= rho * u[a] * u[b];
      if constexpr (a.value == b.value) sum -= R(1) / R(3) * (rho - R(1));
      pi[k] = sum;
    });
  });
}

// CombinedRLBdynamics<MIXIN, InnerEdgeVelocityTuple3D / InnerCornerVelocityTuple3D>
// (src/boundary/localVelocity3D.h:88-101, interpolatedVelocity3D.h:56-67): as
// collide_local with the inner density and stress
template <class L, int KIND, class R>
OLB_DEV void collide_inner_velocity(R (&f)[L::q], const DynDevice<R>* __restrict__ e, int x, int y, int z,
                                    R& st_rho, R& st_usqr)
{
  const R* __restrict__ v = e->bc_values + 4 * size_t(bc_index(e, x, y, z));
  const int kind = e->kind;
  int32_t n[3] = {e->nrm[0], e->nrm[1], e->nrm[2]};
  const R u[3] = {v[1], v[2], v[3]};
  R pi[6];
  R rho = inner_rho<L>(f, kind, n, u);
  inner_stress<L>(f, kind, n, rho, u, pi);
  {
    const R usqr = norm_sqr(u);
    static_for<0, L::q>([&](auto i) { f[i] = feq2<L, i.value>(rho, u, usqr) + from_pi_to_fneq<L, i.value>(pi); });
  }
  rho = inner_rho<L>(f, kind, n, u);
  const R delta = rho - R(1);
  if constexpr (KIND == K_TRT) {
    relax_trt<L>(f, rho, delta, u, e->omega, e->omega_minus);
  } else {
    relax_bgk<L>(f, rho, delta, u, e->omega);
  }
  st_rho = rho;
  st_usqr = norm_sqr(u);
}

// MIXIN::exchange_momenta<FixedVelocityBoundaryTuple> (src/dynamics/momenta/
// aliases.h:188-193) on external edges and corners: BulkDensity and
// u = VELOCITY; the mixin collision on those momenta.
template <class L, int KIND, class R>
OLB_DEV void collide_fixed_velocity(R (&f)[L::q], const DynDevice<R>* __restrict__ e, int x, int y, int z,
                                    R& st_rho, R& st_usqr)
{
  const R* __restrict__ v = e->bc_values + 4 * size_t(bc_index(e, x, y, z));
  R delta = f[0];
  static_for<1, L::q>([&](auto i) { delta += f[i]; });
  const R rho = delta + R(1);
  const R u[3] = {v[1], v[2], v[3]};
  if constexpr (KIND == K_TRT) {
    relax_trt<L>(f, rho, delta, u, e->omega, e->omega_minus);
  } else if constexpr (KIND == K_SMAGORINSKY) {
    const R w = smagorinsky_omega<L>(f, rho, delta, u, e->smago_pre, e->tau_mol);
    relax_bgk<L>(f, rho, delta, u, w);
  } else {
    relax_bgk<L>(f, rho, delta, u, e->omega);
  }
  st_rho = rho;
  st_usqr = norm_sqr(u);
}

// collision of a boundary cell that carries values, by its runtime kind
// (run by boundary_collide_kernel, ahead of the step kernel)
template <class L, int KIND, class R>
OLB_DEV void collide_boundary(R (&f)[L::q], int kind, const DynDevice<R>* __restrict__ e, int x, int y, int z,
                              R& st_rho, R& st_usqr)
{
  if (is_interpolated(kind)) {
    collide_interpolated<L, KIND>(f, kind, e, x, y, z, st_rho, st_usqr);
  } else if (is_local(kind)) {
    if constexpr (KIND == K_BGK || KIND == K_TRT) {
      collide_local<L, KIND>(f, kind, e, x, y, z, st_rho, st_usqr);
    }
  } else if (is_inner(kind)) {
    if constexpr (KIND == K_BGK || KIND == K_TRT) {
      collide_inner_velocity<L, KIND>(f, e, x, y, z, st_rho, st_usqr);
    }
  } else {
    collide_fixed_velocity<L, KIND>(f, e, x, y, z, st_rho, st_usqr);
  }
}

// ---------------------------------------------------------------------------
// BGK / TRT on the scaled 16-bit representation g_i = s_i (f_i - w_i)
//
// 16-bit storage keeps s_i (f_i - w_i), s_i a power of two that depends only
// on the weight class |c_i|^2.  Decoding every population (g_i / s_i) and
// encoding the result (s_i f_i') costs two multiplies per population.  On g
// directly the moments need one multiply per weight class and the relaxation
// none, g_i' = (1 - omega) g_i + omega s_i feq_i, with s_i t_i folded into the
// equilibrium's constants.  Algebraically the same collision; the rounding
// differs well below the 16-bit storage's own.

template <class L>
OLB_HD constexpr int weight_class(int i)
{
  return L::c(i, 0) * L::c(i, 0) + L::c(i, 1) * L::c(i, 1) + L::c(i, 2) * L::c(i, 2);
}

template <class L>
OLB_HD constexpr int first_of_class(int k)
{
  int i = 0;
  while (i < L::q && weight_class<L>(i) != k) ++i;
  return i;
}

template <class L>
OLB_HD constexpr float inv_class_scale(int k)
{
  return first_of_class<L>(k) < L::q ? 1.f / storage_scale<L>(first_of_class<L>(k)) : 0.f;
}

// Arithmetic on one cell (V = float) or on the two cells of a packed 16-bit
// pair at once (V = float2: sm_100's packed FP32 instructions, one instruction
// for both lanes, each lane rounded as its scalar counterpart).
OLB_DEV float v_add(float a, float b) { return a + b; }
OLB_DEV float v_sub(float a, float b) { return a - b; }
OLB_DEV float v_mul(float a, float b) { return a * b; }
OLB_DEV float v_fma(float a, float b, float c) { return fmaf(a, b, c); }
OLB_DEV float v_rcp(float a) { return 1.f / a; }
OLB_DEV float v_sqrt(float a) { return sqrtf(a); }
OLB_DEV float2 v_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as a + (-1) b: the product is exact, so one rounding as in a - b
OLB_DEV float2 v_sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
OLB_DEV float2 v_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
OLB_DEV float2 v_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
OLB_DEV float2 v_rcp(float2 a) { return make_float2(1.f / a.x, 1.f / a.y); }
OLB_DEV float2 v_sqrt(float2 a) { return make_float2(sqrtf(a.x), sqrtf(a.y)); }
// live != 0 ? a : b, per lane
OLB_DEV float v_select(float live, float a, float b) { return live != 0.f ? a : b; }
OLB_DEV float2 v_select(float2 live, float2 a, float2 b)
{
  return make_float2(live.x != 0.f ? a.x : b.x, live.y != 0.f ? a.y : b.y);
}
template <class V> OLB_DEV V v_splat(float x);
template <> OLB_DEV float v_splat<float>(float x) { return x; }
template <> OLB_DEV float2 v_splat<float2>(float x) { return make_float2(x, x); }

// The collisions on g work on the opposite pairs p = 1..half.  The pair's
// representative r is the member whose first nonzero velocity component is
// +1, so every c_r . u starts with a positive term; the pair sum is
// s_p = g_r + g_opp(r) and the difference d_p = g_r - g_opp(r) (s_i = s_opp, so
// the pair shares one scale).
template <class L>
OLB_HD constexpr int pair_rep(int p)
{
  return L::c(p, 0) != 0 ? (L::c(p, 0) > 0 ? p : L::opp(p))
       : L::c(p, 1) != 0 ? (L::c(p, 1) > 0 ? p : L::opp(p))
                         : (L::c(p, 2) > 0 ? p : L::opp(p));
}

// the first pair of weight class k (in pair order), 0 when the class is empty
template <class L>
OLB_HD constexpr int first_pair_of_class(int k)
{
  for (int p = 1; p <= L::half; ++p) {
    if (weight_class<L>(p) == k) return p;
  }
  return 0;
}

// the first pair of weight class k whose velocity has a component along axis
// a, 0 when there is none
template <class L>
OLB_HD constexpr int first_pair_on_axis(int a, int k)
{
  for (int p = 1; p <= L::half; ++p) {
    if (weight_class<L>(p) == k && L::c(pair_rep<L>(p), a) != 0) return p;
  }
  return 0;
}

// the first weight class >= 1 with a pair on axis a (a = -1: any pair)
template <class L>
OLB_HD constexpr int first_class_with_pairs(int a)
{
  for (int k = 1; k < 4; ++k) {
    if (a < 0 ? first_pair_of_class<L>(k) != 0 : first_pair_on_axis<L>(a, k) != 0) return k;
  }
  return 0;
}

// c_r . v with a positive first term (r the pair's representative)
template <class L, int P, class V>
OLB_DEV V rep_dot(const V (&v)[3])
{
  constexpr int r = pair_rep<L>(P);
  constexpr int c0 = L::c(r, 0), c1 = L::c(r, 1), c2 = L::c(r, 2);
  V acc;
  bool first = true;
  auto term = [&](int c, const V& x) {
    if (c == 0) return;
    acc = first ? x : (c > 0 ? v_add(acc, x) : v_sub(acc, x));
    first = false;
  };
  term(c0, v[0]);
  term(c1, v[1]);
  term(c2, v[2]);
  return acc;
}

// Density from g_0 and the pair sums, velocity from the pair differences: one
// multiply by 1/s per weight class; a per-axis sum is kept with the sign of
// its first term folded into that multiplier.
// live: 1 for a fluid lane, 0 for a bounce-back lane, whose velocity is then
// its momentum (no division by a density that its stale populations may not
// give); rinv returns the reciprocal used.
template <class L, class V>
OLB_DEV void scaled_moments(const V& g0, const V (&ps)[L::half + 1], const V (&pd)[L::half + 1], const V& live,
                            V& rho, V& delta, V (&u)[3], V& rinv)
{
  V m[4], j[3][4];
  static_for<1, L::half + 1>([&](auto p) {
    constexpr int k = weight_class<L>(p.value);
    constexpr int r = pair_rep<L>(p.value);
    if constexpr (first_pair_of_class<L>(k) == p.value) {
      m[k] = ps[p];
    } else {
      m[k] = v_add(m[k], ps[p]);
    }
    static_for<0, 3>([&](auto a) {
      constexpr int cc = L::c(r, a);
      if constexpr (cc != 0) {
        constexpr int f = first_pair_on_axis<L>(a, k);
        constexpr int s0 = L::c(pair_rep<L>(f), a);
        if constexpr (f == p.value) {
          j[a][k] = pd[p];
        } else if constexpr (cc == s0) {
          j[a][k] = v_add(j[a][k], pd[p]);
        } else {
          j[a][k] = v_sub(j[a][k], pd[p]);
        }
      }
    });
  });
  delta = v_mul(g0, v_splat<V>(inv_class_scale<L>(0)));
  static_for<1, 4>([&](auto k) {
    if constexpr (first_pair_of_class<L>(k) != 0) {
      delta = v_fma(m[k], v_splat<V>(inv_class_scale<L>(k)), delta);
    }
  });
  static_for<0, 3>([&](auto a) {
    static_for<1, 4>([&](auto k) {
      constexpr int f = first_pair_on_axis<L>(a, k);
      if constexpr (f != 0) {
        constexpr float inv = float(L::c(pair_rep<L>(f), a)) * inv_class_scale<L>(k);
        if constexpr (first_class_with_pairs<L>(a) == k) {
          u[a] = v_mul(j[a][k], v_splat<V>(inv));
        } else {
          u[a] = v_fma(j[a][k], v_splat<V>(inv), u[a]);
        }
      }
    });
  });
  rho = v_add(delta, v_splat<V>(1.f));
  rinv = v_rcp(v_fma(rho, live, v_sub(v_splat<V>(1.f), live)));
  u[0] = v_mul(u[0], rinv);
  u[1] = v_mul(u[1], rinv);
  u[2] = v_mul(u[2], rinv);
}

// BGK / TRT relaxation on g in pair form, with the Guo force term folded in.
// For a pair with representative r, sum s and difference d,
//   g_r' = S + D,  g_opp(r)' = S - D,
//   S = keep s + A,  D = keep' d + B,  keep = (1 - omega)/2,  keep' = (1 - omega')/2
// (omega' = omega_minus for TRT, omega for BGK) with the equilibrium parts of
// A and B (per weight class k = s_i t_i):
//   A = omega k (delta + rho (9/2 (c.u)^2 - 3/2 |u|^2)),  B = 3 omega' k rho (c.u)
// and the Guo term of lbm::addExternalForce (src/dynamics/lbm.h:544-566),
//   t_i (3 (c_i - u).F + 9 (c_i.u)(c_i.F)) force_relax rho,
// which over a pair is Fa +- Fb with Fa = k fr (9 (c.u)(c.F) - 3 u.F) and
// Fb = 3 k fr (c.F), fr = force_relax rho: A += Fa, B += Fb.  Everything that
// depends only on the weight class is formed once per class (the compiler
// shares the products of equal constants), so a pair costs two dot products
// with entries of +-1 and about a dozen FP32 operations.  The same collision
// as relaxing and then adding the force (the rounding differs far below the
// 16-bit storage's own).
template <class L, bool FORCED, class V>
OLB_DEV void relax_scaled(V (&g)[L::q], const V (&ps)[L::half + 1], const V (&pd)[L::half + 1], const V& rho,
                          const V& delta, const V (&u)[3], const V& usqr, const V& omega, const V& omega_b,
                          const V& keep, const V& keep_minus, const V& force_relax, const V (&gf)[3])
{
  const V base = v_fma(v_mul(v_splat<V>(-1.5f), rho), usqr, delta);  // delta + rho e0
  const V rho45 = v_mul(v_splat<V>(4.5f), rho);
  const V rho_odd = v_mul(omega_b, rho);
  V fr = v_splat<V>(0.f), uf3 = v_splat<V>(0.f);
  if constexpr (FORCED) {
    fr = v_mul(force_relax, rho);
    uf3 = v_mul(v_splat<V>(3.f), v_fma(u[2], gf[2], v_fma(u[1], gf[1], v_mul(u[0], gf[0]))));
  }
  {
    constexpr float T = storage_scale<L>(0) * weight<L, float>(0);
    V eq = v_mul(v_mul(omega, v_splat<V>(T)), base);
    if constexpr (FORCED) eq = v_fma(v_mul(v_splat<V>(-T), fr), uf3, eq);
    g[0] = v_fma(v_sub(v_splat<V>(1.f), omega), g[0], eq);
  }
  static_for<1, L::half + 1>([&](auto p) {
    constexpr int r = pair_rep<L>(p.value);
    constexpr int o = L::opp(r);
    constexpr float T = storage_scale<L>(r) * weight<L, float>(r);
    constexpr float K = 3.f * T;
    const V wt = v_mul(omega, v_splat<V>(T));
    const V cu = rep_dot<L, p.value>(u);
    V a0 = v_mul(wt, base);
    V A, B;
    if constexpr (FORCED) {
      const V kf = v_mul(v_splat<V>(T), fr);
      a0 = v_fma(v_mul(v_splat<V>(-1.f), kf), uf3, a0);
      const V cf = rep_dot<L, p.value>(gf);
      A = v_fma(v_mul(wt, rho45), v_mul(cu, cu), v_fma(v_mul(v_splat<V>(9.f), kf), v_mul(cu, cf), a0));
      B = v_fma(v_mul(v_splat<V>(K), rho_odd), cu, v_mul(v_mul(v_splat<V>(3.f), kf), cf));
    } else {
      A = v_fma(v_mul(wt, rho45), v_mul(cu, cu), a0);
      B = v_mul(v_mul(v_splat<V>(K), rho_odd), cu);
    }
    const V S = v_fma(keep, ps[p], A);
    const V D = v_fma(keep_minus, pd[p], B);
    g[r] = v_add(S, D);
    g[o] = v_sub(S, D);
  });
}

// Smagorinsky effective omega from the scaled populations: Pi_ab per weight
// class from the pair sums, one multiply by 1/s per class.
template <class L, class V>
OLB_DEV V smagorinsky_omega_scaled(const V (&ps)[L::half + 1], const V& rho, const V& rinv, const V& delta,
                                   const V (&u)[3], const V& smago_pre, const V& tau_mol)
{
  V pik[6][4];
  static_for<0, 6>([&](auto m) { static_for<0, 4>([&](auto k) { pik[m][k] = v_splat<V>(-0.f); }); });
  static_for<1, L::half + 1>([&](auto p) {
    constexpr int k = weight_class<L>(p.value);
    constexpr int r = pair_rep<L>(p.value);
    static_for<0, 3>([&](auto a) {
      static_for<a.value, 3>([&](auto b) {
        constexpr int m = a.value * 3 - (a.value * (a.value - 1)) / 2 + (b.value - a.value);
        constexpr int cc = L::c(r, a) * L::c(r, b);
        if constexpr (cc == 1) { pik[m][k] = v_add(pik[m][k], ps[p]); }
        else if constexpr (cc == -1) { pik[m][k] = v_sub(pik[m][k], ps[p]); }
      });
    });
  });
  V pi[6];
  static_for<0, 3>([&](auto a) {
    static_for<a.value, 3>([&](auto b) {
      constexpr int m = a.value * 3 - (a.value * (a.value - 1)) / 2 + (b.value - a.value);
      V s = v_splat<V>(-0.f);
      static_for<1, 4>([&](auto k) {
        constexpr float inv = inv_class_scale<L>(k);
        if constexpr (inv != 0.f) { s = v_fma(pik[m][k], v_splat<V>(inv), s); }
      });
      s = v_sub(s, v_mul(v_mul(rho, u[a]), u[b]));
      if constexpr (a.value == b.value) { s = v_sub(s, v_mul(v_splat<V>(1.f / 3.f), delta)); }
      pi[m] = s;
    });
  });
  const V diag = v_fma(pi[5], pi[5], v_fma(pi[3], pi[3], v_mul(pi[0], pi[0])));
  const V off = v_fma(pi[4], pi[4], v_fma(pi[2], pi[2], v_mul(pi[1], pi[1])));
  const V n2 = v_fma(v_splat<V>(2.f), off, diag);
  const V inner = v_fma(v_mul(smago_pre, rinv), v_sqrt(n2), v_mul(tau_mol, tau_mol));
  const V tau_turb = v_mul(v_splat<V>(0.5f), v_sub(v_sqrt(inner), tau_mol));
  return v_rcp(v_add(tau_mol, tau_turb));
}

// Collision constants of the fluid dynamics for the scaled collisions, one
// value per lane: omega (weight of the symmetric equilibrium part), omega_b
// (of the antisymmetric part: omega_minus for TRT, omega for BGK), keep =
// (1 - omega)/2, keep_minus = (1 - omega_b)/2.  A bounce-back lane has omega =
// omega_b = force_relax = 0, keep = 1/2, keep_minus = -1/2 and live = 0: the
// same arithmetic then gives S = s/2, D = -d/2, so g_r' = g_opp, g_opp' = g_r
// and g_0' = g_0 — full-way bounce-back (collision::Revert) up to one FP32
// rounding of the pair's sum and difference (2^-24 of the pair's larger
// member, far below the 16-bit storage's own rounding).  A pass lane
// (keep_minus = +1/2) gives g' = g the same way.
template <class V>
struct ScaledParams {
  V omega, omega_b, keep, keep_minus, force_relax, smago_pre, tau_mol, live;
  V force[3];
};

// Any fluid collision on the scaled 16-bit representation (see above).
template <class L, int KIND, class V>
OLB_DEV void collide_scaled(V (&g)[L::q], const ScaledParams<V>& p, V& st_rho, V& st_usqr)
{
  V ps[L::half + 1], pd[L::half + 1];
  static_for<1, L::half + 1>([&](auto q) {
    constexpr int r = pair_rep<L>(q.value);
    constexpr int o = L::opp(r);
    ps[q] = v_add(g[r], g[o]);
    pd[q] = v_sub(g[r], g[o]);
  });
  V rho, delta, u[3], rinv;
  scaled_moments<L>(g[0], ps, pd, p.live, rho, delta, u, rinv);
  constexpr bool forced = KIND == K_FORCED_BGK || KIND == K_FORCED_TRT;
  V gf[3] = {v_splat<V>(0.f), v_splat<V>(0.f), v_splat<V>(0.f)};
  if constexpr (forced) {
    gf[0] = p.force[0]; gf[1] = p.force[1]; gf[2] = p.force[2];
    const V half = v_splat<V>(0.5f);
    u[0] = v_fma(gf[0], half, u[0]);
    u[1] = v_fma(gf[1], half, u[1]);
    u[2] = v_fma(gf[2], half, u[2]);
  }
  const V usqr = v_fma(u[2], u[2], v_fma(u[1], u[1], v_mul(u[0], u[0])));
  if constexpr (KIND == K_SMAGORINSKY) {
    // the cell's effective omega; a wall or pass lane (live = 0) gets 0 and
    // its own keep_minus
    const V w = v_mul(smagorinsky_omega_scaled<L>(ps, rho, rinv, delta, u, p.smago_pre, p.tau_mol), p.live);
    const V keep = v_mul(v_splat<V>(0.5f), v_sub(v_splat<V>(1.f), w));
    const V keep_minus = v_select(p.live, keep, p.keep_minus);
    relax_scaled<L, false>(g, ps, pd, rho, delta, u, usqr, w, w, keep, keep_minus, v_splat<V>(0.f), gf);
  } else {
    relax_scaled<L, forced>(g, ps, pd, rho, delta, u, usqr, p.omega, p.omega_b, p.keep, p.keep_minus,
                            p.force_relax, gf);
  }
  st_rho = rho;
  st_usqr = usqr;
}

// collision::NguyenLaddCorrection<Revert>  src/dynamics/collision.h:333-346
template <class L, class R>
OLB_DEV void collide_moving_wall(R (&f)[L::q], const DynDevice<R>& p)
{
  revert<L>(f);
  static_for<1, L::q>([&](auto i) {
    f[i] += p.wall_term[i][0];
    f[i] += p.wall_term[i][1];
    f[i] += p.wall_term[i][2];
  });
}

} // namespace olb_b200
