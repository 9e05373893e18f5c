"""Seeded test cases shared by the CPU and GPU tests (geometry + initial state).

Each builder returns an ``oracle.Case`` (per-cell dynamics id + table) and the
initial shifted populations in the logical layout.  Geometries follow the
workloads the reference's configurations describe: a lid-driven cavity with
bounce-back walls and a moving lid, a triply periodic Taylor-Green vortex, a
periodic channel with bounce-back walls and spheres, a channel with a square
cylinder.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def random_state(q, n, dtype, rng, amp_u=0.03, amp_neq=1e-3):
    rho = (1 + 0.01 * rng.standard_normal(n)).astype(dtype)
    u = (amp_u * rng.standard_normal((3, n))).astype(dtype)
    f = O.equilibrium(q, rho, u)
    f += (amp_neq * rng.standard_normal(f.size)).astype(dtype)
    return f


def periodic_case(q, size, kind=O.BGK, omega=1.3, magic=3 / 16, smagorinsky=0.1,
                  force=(1e-4, -2e-5, 3e-5)):
    return O.Case(q=q, size=size, periodic=(1, 1, 1),
                  table=[O.Dynamics(kind, omega=omega, magic=magic, smagorinsky=smagorinsky, force=force)])


def cavity_ids(nx, ny, nz):
    """Cavity as cavity3dBenchmark builds it: walls (id 1) on the box surface,
    the lid (id 2) on the y = ny-1 face interior, fluid (id 0) inside."""
    ids = np.zeros((nx, ny, nz), np.uint8)
    ids[0, :, :] = 1
    ids[-1, :, :] = 1
    ids[:, 0, :] = 1
    ids[:, :, 0] = 1
    ids[:, :, -1] = 1
    ids[1:-1, -1, 1:-1] = 2
    return ids.reshape(-1)


def cavity_case(q, size, omega=1 / 0.692, lid=(0.1, 0.0, 0.0)):
    nx, ny, nz = size
    return O.Case(q=q, size=size, periodic=(0, 0, 0), dyn_id=cavity_ids(nx, ny, nz),
                  table=[O.Dynamics(O.BGK, omega=omega), O.Dynamics(O.BOUNCE_BACK),
                         O.Dynamics(O.BOUNCE_BACK_VELOCITY, wall_u=lid)])


def rest_state(q, n, dtype):
    return O.equilibrium(q, np.ones(n, dtype), np.zeros((3, n), dtype))


def spheres_ids(size, rng, r_min=2.0, r_max=3.5, solid_fraction=0.2, max_tries=20000):
    """Channel periodic in x with bounce-back walls at y/z faces and seeded,
    non-overlapping spheres (id 1 = solid), fluid id 0."""
    nx, ny, nz = size
    solid = np.zeros(size, bool)
    solid[:, 0, :] = solid[:, -1, :] = True
    solid[:, :, 0] = solid[:, :, -1] = True
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    spheres = []
    target = solid_fraction * nx * ny * nz
    tries = 0
    while solid.sum() < target and tries < max_tries:
        tries += 1
        r = rng.uniform(r_min, r_max)
        c = rng.uniform([0, r + 1, r + 1], [nx, ny - r - 1, nz - r - 1])
        if any(np.linalg.norm(c - c2) < r + r2 for c2, r2 in spheres):
            continue
        spheres.append((c, r))
        dx = np.minimum(np.abs(X - c[0]), nx - np.abs(X - c[0]))  # periodic in x
        solid |= dx ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r
    return solid.astype(np.uint8).reshape(-1)


def porous_case(q, size, rng, omega=1.2, magic=3 / 16, g=1e-5):
    ids = spheres_ids(size, rng)
    return O.Case(q=q, size=size, periodic=(1, 0, 0), dyn_id=ids,
                  table=[O.Dynamics(O.FORCED_TRT, omega=omega, magic=magic, force=(g, 0.0, 0.0)),
                         O.Dynamics(O.BOUNCE_BACK)])


def with_force_field(case, dtype, rng, g=1e-4, spread=0.5):
    """The case with a FORCE value per cell: x component g (1 + spread U[-1,1]),
    y and z g spread U[-1,1]/2, rounded to `dtype` (the values a lattice of that
    precision stores), kept as float64 for the oracle."""
    n = case.n
    f = np.empty((3, n))
    f[0] = g * (1 + spread * rng.uniform(-1, 1, n))
    f[1:] = 0.5 * g * spread * rng.uniform(-1, 1, (2, n))
    case.force_field = f.astype(dtype).astype(np.float64)
    return case


def channel_cylinder_case(q, size, omega=1.6, smagorinsky=0.1, side=4):
    """x-periodic channel (bounce-back y/z walls) with a square cylinder
    spanning z; Smagorinsky BGK fluid."""
    nx, ny, nz = size
    ids = np.zeros(size, np.uint8)
    ids[:, 0, :] = ids[:, -1, :] = 1
    ids[:, :, 0] = ids[:, :, -1] = 1
    x0, y0 = nx // 4, ny // 2 - side // 2
    ids[x0:x0 + side, y0:y0 + side, :] = 1
    return O.Case(q=q, size=size, periodic=(1, 0, 0), dyn_id=ids.reshape(-1),
                  table=[O.Dynamics(O.SMAGORINSKY, omega=omega, smagorinsky=smagorinsky),
                         O.Dynamics(O.BOUNCE_BACK)])


def interpolated_channel_case(q, size, mixin=O.BGK, omega=1.6, smagorinsky=0.1, magic=3 / 16,
                              u0=0.05, fluctuation=0.02, rho_out=1.0, side=0, seed=0):
    """Channel with bounce-back walls on the y/z faces, an interpolated
    velocity inlet on the x = 0 face and an interpolated pressure outlet on the
    x = nx-1 face (both over the interior y/z cells, so every boundary cell is a
    flat one), optionally a square cylinder spanning z.  The inlet velocity is
    u0 along x with seeded uniform fluctuations of relative size
    `fluctuation` on every component; the outlet holds rho_out.
    Ids: 0 fluid, 1 wall, 2 inlet (normal -x), 3 outlet (normal +x)."""
    nx, ny, nz = size
    ids = np.zeros(size, np.uint8)
    ids[:, 0, :] = ids[:, -1, :] = 1
    ids[:, :, 0] = ids[:, :, -1] = 1
    ids[0, 1:-1, 1:-1] = 2
    ids[-1, 1:-1, 1:-1] = 3
    if side:
        x0, y0 = nx // 4, ny // 2 - side // 2
        ids[x0:x0 + side, y0:y0 + side, 1:-1] = 1
    rng = np.random.default_rng(seed)
    vals = np.zeros((4,) + tuple(size))
    vals[0] = 1.0
    r = 2 * rng.random((3, ny, nz)) - 1
    vals[1, 0] = u0 * (1 + fluctuation * r[0])
    vals[2, 0] = u0 * fluctuation * r[1]
    vals[3, 0] = u0 * fluctuation * r[2]
    vals[0, -1] = rho_out
    bulk = dict(omega=omega, magic=magic, smagorinsky=smagorinsky)
    table = [O.Dynamics(mixin, **bulk), O.Dynamics(O.BOUNCE_BACK),
             O.Dynamics(O.INTERP_VELOCITY, mixin=mixin, direction=0, orientation=-1, **bulk),
             O.Dynamics(O.INTERP_PRESSURE, mixin=mixin, direction=0, orientation=1, **bulk)]
    return O.Case(q=q, size=size, periodic=(0, 0, 0), dyn_id=ids.reshape(-1), table=table,
                  bc_values=vals.reshape(4, -1))


def local_channel_case(q, size, mixin=O.BGK, omega=1.6, magic=3 / 16, u0=0.05, rho_out=0.995, side=0, seed=0):
    """interpolated_channel_case with local boundaries, as resolvedRock3d and
    microChannel3d set them: a LocalVelocity inlet on the x = 0 face and a
    LocalPressure outlet (density rho_out) on the x = nx-1 face, both over the
    interior y/z cells (flat faces only, the one type LocalPressure takes)."""
    case = interpolated_channel_case(q, size, mixin=mixin, omega=omega, magic=magic, u0=u0, rho_out=rho_out,
                                     side=side, seed=seed)
    case.table[2].kind = O.LOCAL_VELOCITY
    case.table[3].kind = O.LOCAL_PRESSURE
    return case


# DiscreteNormalType (src/geometry/discreteNormals.h:33-39)
FLAT, EXTERNAL_CORNER, INTERNAL_CORNER, EXTERNAL_EDGE, INTERNAL_EDGE = range(5)


def boundary_table(materials, normals, setters, bulk, mixin=O.BGK, velocity=None):
    """Dynamics ids and table of a lattice whose boundary materials are set
    with boundary::set<...> (src/boundary/setBoundary.h:79-157), from the
    discrete normals OpenLB itself computed (oracle.reference_normals):
    one entry per (material, normal type, normal).

    materials: int[nx,ny,nz], 1 = fluid; setters: {material: O.LOCAL_VELOCITY
    | O.INTERP_VELOCITY | O.INTERP_PRESSURE | O.BOUNCE_BACK}; bulk: kwargs of
    the fluid entry; velocity: {material: (ux, uy, uz)} boundary velocity.
    Returns (dyn_id, table, bc_values)."""
    m = np.asarray(materials).reshape(-1)
    n = m.size
    table = [O.Dynamics(mixin, **bulk)]
    key_to_id = {}
    ids = np.zeros(n, np.uint8)
    vals = np.zeros((4, n))
    vals[0] = 1.0
    for cell in range(n):
        mat = int(m[cell])
        if mat == 1:
            continue
        setter = setters[mat]
        if setter == O.BOUNCE_BACK:
            key = (mat, "bb")
            entry = lambda: O.Dynamics(O.BOUNCE_BACK)  # noqa: E731
        else:
            typ = int(normals[0, cell])
            nrm = tuple(int(v) for v in normals[1:, cell])
            if nrm == (0, 0, 0):
                raise ValueError(f"cell {cell} of material {mat} has no discrete normal")
            if typ == FLAT:
                axis = [a for a in range(3) if nrm[a] != 0][0]
                key = (mat, typ, axis, nrm[axis])
                entry = lambda a=axis, o=nrm[axis]: O.Dynamics(  # noqa: E731
                    setter, mixin=mixin, direction=a, orientation=o, **bulk)
            elif typ in (EXTERNAL_EDGE, EXTERNAL_CORNER, INTERNAL_EDGE, INTERNAL_CORNER) and \
                    setter in (O.LOCAL_VELOCITY, O.INTERP_VELOCITY):
                kind = {EXTERNAL_EDGE: O.VELOCITY_EDGE, EXTERNAL_CORNER: O.VELOCITY_CORNER,
                        INTERNAL_EDGE: O.VELOCITY_INNER_EDGE, INTERNAL_CORNER: O.VELOCITY_INNER_CORNER}[typ]
                key = (mat, typ, nrm)
                entry = lambda k=kind, v=nrm: O.Dynamics(  # noqa: E731
                    k, mixin=mixin, normal=v, boundary=setter, **bulk)
            else:
                raise ValueError(f"cell {cell}: normal type {typ} of setter {setter} not covered")
            if velocity and mat in velocity:
                vals[1:, cell] = velocity[mat]
        if key not in key_to_id:
            key_to_id[key] = len(table)
            table.append(entry())
        ids[cell] = key_to_id[key]
    if len(table) > 256:
        raise ValueError("more than 256 entries")
    return ids, table, vals


def local_velocity_cavity_case(q, size, omega=1 / 0.692, lid=(0.1, 0.0, 0.0), mixin=O.BGK):
    """cavity3dBenchmark's default set-up (examples/laminar/cavity3dBenchmark/
    cavity3d.cpp:40-59,71-76): the box surface is material 2 (walls, u = 0)
    except the y = max face, edges and corners included, which is material 3
    (the lid, u = lid); both set with boundary::set<LocalVelocity<T,D,BGK>>.
    Flat faces, external edges and external corners as OpenLB classifies them."""
    nx, ny, nz = size
    mats = np.full(size, 2, np.int32)
    mats[1:-1, 1:-1, 1:-1] = 1
    mats[:, -1, :] = 3
    normals = O.reference_normals(mats, (0, 0, 0), boundary_materials=(2, 3), q=q)
    ids, table, vals = boundary_table(mats, normals, {2: O.LOCAL_VELOCITY, 3: O.LOCAL_VELOCITY},
                                      dict(omega=omega), mixin=mixin, velocity={3: lid})
    return O.Case(q=q, size=size, periodic=(0, 0, 0), dyn_id=ids, table=table, bc_values=vals)


def concave_cavity_case(q, size, omega=1 / 0.692, lid=(0.1, 0.0, 0.0), mixin=O.BGK, setter=O.LOCAL_VELOCITY):
    """cavity3dBenchmark's default set-up with a block standing on the floor:
    the block's surface is a velocity boundary too (u = 0), so OpenLB's
    classification gives flat faces, external edges and corners (the box) and
    internal edges and corners (where the block meets the floor, its top rim).
    Wall cells that touch no fluid cell are bounce-back (material 4)."""
    nx, ny, nz = size
    mats = np.full(size, 2, np.int32)
    mats[1:-1, 1:-1, 1:-1] = 1
    mats[:, -1, :] = 3
    mats[nx // 3:nx // 3 + 4, 1:5, nz // 3:nz // 3 + 4] = 2
    fluid = mats == 1
    near = np.zeros(size, bool)
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                near |= np.roll(fluid, (dx, dy, dz), axis=(0, 1, 2))
    mats[(mats == 2) & ~near] = 4
    normals = O.reference_normals(mats, (0, 0, 0), boundary_materials=(2, 3), q=q)
    ids, table, vals = boundary_table(mats, normals, {2: setter, 3: setter, 4: O.BOUNCE_BACK},
                                      dict(omega=omega), mixin=mixin, velocity={3: lid})
    return O.Case(q=q, size=size, periodic=(0, 0, 0), dyn_id=ids, table=table, bc_values=vals)


def open_inlet_channel_case(q, size, omega=1.6, u0=0.05, mixin=O.BGK, seed=0):
    """Channel whose whole x = 0 face, rim included, is an interpolated
    velocity inlet: its rim cells are external edges and corners of the
    inlet (OuterVelocityEdge/CornerProcessor3D).  Bounce-back walls on the y
    and z faces, an interpolated pressure outlet on the x = nx-1 face interior.
    Inlet velocity u0 along x with seeded 2 % fluctuations."""
    nx, ny, nz = size
    mats = np.full(size, 1, np.int32)
    mats[:, 0, :] = mats[:, -1, :] = 2
    mats[:, :, 0] = mats[:, :, -1] = 2
    mats[0, :, :] = 3
    mats[-1, 1:-1, 1:-1] = 4
    normals = O.reference_normals(mats, (0, 0, 0), boundary_materials=(3, 4), q=q)
    rng = np.random.default_rng(seed)
    r = 2 * rng.random((3, ny, nz)) - 1
    ids, table, vals = boundary_table(mats, normals, {2: O.BOUNCE_BACK, 3: O.INTERP_VELOCITY,
                                                      4: O.INTERP_PRESSURE},
                                      dict(omega=omega), mixin=mixin)
    v = vals.reshape((4,) + tuple(size))
    v[1, 0] = u0 * (1 + 0.02 * r[0])
    v[2, 0] = u0 * 0.02 * r[1]
    v[3, 0] = u0 * 0.02 * r[2]
    return O.Case(q=q, size=size, periodic=(0, 0, 0), dyn_id=ids, table=table, bc_values=v.reshape(4, -1))


def to_abi_table(case):
    """oracle.Case -> openlb_b200 dynamics table (same entries, same ids)."""
    import openlb_b200 as ob
    table = []
    for d in case.table:
        extra = {}
        if d.kind in O.VALUED:
            extra = dict(mixin=d.mixin, direction=d.direction, orientation=d.orientation,
                         normal=tuple(d.normal))
        table.append(ob.Dynamics(kind=d.kind, omega=d.omega, magic=d.magic, smagorinsky=d.smagorinsky,
                                 force=tuple(d.force), wall_u=tuple(d.wall_u), wall_rho=d.wall_rho, **extra))
    return table


def boundary_cells_and_values(case):
    """(cells, values[k, 4]) of the boundary cells that carry values (RHO,
    VELOCITY) of a case, for Lattice.set_boundary_values."""
    kinds = np.array([d.kind for d in case.table])
    cells = np.flatnonzero(np.isin(kinds[case.dyn_id], O.VALUED))
    return cells, case.bc_values[:, cells].T.copy()


def pop_tolerance_violation(q, got, ref, rtol, dtype=np.float64):
    """Max over slots of |got - ref| / (|ref + w_i|): the error relative to the
    unshifted population f_i = (f_i - w_i) + w_i.  NaN slots of ref (values
    that depend on the reference's unspecified padding) are skipped."""
    from openlb_b200.descriptors import descriptor
    w = descriptor(q).w(np.float64)
    g = got.reshape(q, -1).astype(np.float64)
    r = ref.reshape(q, -1).astype(np.float64)
    valid = ~np.isnan(r)
    denom = np.abs(r + w[:, None])
    err = np.where(valid, np.abs(g - r) / denom, 0.0)
    return float(err.max()), float(np.where(valid, np.abs(g - r), 0).max())
