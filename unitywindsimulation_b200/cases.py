"""Seeded case generator: obstacle flags, inflow and solver settings.

Stands in for the reference's voxelizer (BuildingVoxelizer.cs:355-413), which
ray-casts Unity meshes into an ``int[]`` flag array indexed
``z*nx*ny + y*nx + x`` with 1 = solid, keeps a 10-cell building-free margin
near the x/z boundaries (:379) and rotates the domain by the wind direction
(:364).  Here buildings are seeded axis-aligned or rotated boxes rasterised at
cell centres into the same layout.

Axis convention: the reference (and this library) uses y vertical; workload
descriptions written as nx x ny x nz with z vertical map to
(nx, ny_ref, nz_ref) = (nx, nz, ny).

Workloads (synthetic, seeded):
  plain_cube      64 x 32(up) x 48, one 8-cell cube, log inflow u*=0.5 z0=0.1
  urban_block     256 x 96(up) x 192, 48 buildings on a street lattice,
                  u*=0.6 z0=0.3 with 5 % Gaussian inlet perturbation
  batch_directions 16 uneven grids 96..192 x 48..80(up) x 96..160, 8-32
                  buildings each, wind rotated by k * 22.5 degrees
  adjoint_street  128 x 64(up) x 96, 12 soft buildings with continuous heights
  adjoint_batch   8 directions x 256 x 96(up) x 256, 64 soft buildings
  wind_tunnel     100 x 50(up) x 100 on the reference's non-uniform mesh
                  (Assets/Code/Config/WindTunnelBoxConfig.asset)
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import _lib
from .config import default_config
from .soft_mask import SoftBuildings

MARGIN = 10  # building-free cells next to the x and z boundaries (BuildingVoxelizer.cs:379)
KAPPA = 0.41


@dataclasses.dataclass
class Case:
    name: str
    cfg: object                       # WfConfig
    flags: np.ndarray                 # int32, (nz, ny, nx)
    inlet: np.ndarray | None = None   # (nz, ny, 3) float32 X0 plane, None = built-in profile
    steps: int = 1
    seed: int | None = None
    buildings: list = dataclasses.field(default_factory=list)  # (x0, x1, z0, z1, height[, angle])
    soft: SoftBuildings | None = None  # soft building mask (drag field), all cells fluid
    faces: tuple | None = None         # (fx, fy, fz) face positions of a non-uniform grid

    @property
    def n_cells(self) -> int:
        return int(self.cfg.nx) * int(self.cfg.ny) * int(self.cfg.nz)


def log_profile(y_phys, ustar: float, z0: float, kappa: float = KAPPA):
    return ustar / kappa * np.log((np.asarray(y_phys, dtype=np.float64) + z0) / z0)


def inlet_plane(ny: int, nz: int, dx: float, ustar: float, z0: float, kappa: float = KAPPA,
                perturb: float = 0.0, rng: np.random.Generator | None = None) -> np.ndarray:
    """X0 plane (nz, ny, 3): log profile at cell centres (y + 0.5) dx
    (CSSetLogVelBndCond, InitShaderColl.compute:273-285), optionally with a
    multiplicative Gaussian perturbation per inlet face."""
    y = (np.arange(ny, dtype=np.float32) + np.float32(0.5)) * np.float32(dx)
    u = log_profile(y, ustar, z0, kappa).astype(np.float32)
    plane = np.zeros((nz, ny, 3), dtype=np.float32)
    plane[:, :, 0] = u[None, :]
    if perturb:
        rng = rng or np.random.default_rng(0)
        plane[:, :, 0] *= (1.0 + perturb * rng.standard_normal((nz, ny))).astype(np.float32)
    return plane


def cfl_dt(u_max: float, dx: float, cfl: float = 0.5) -> float:
    return float(cfl * dx / u_max)


def remove_isolated_fluid(flags: np.ndarray) -> np.ndarray:
    """Marks solid every fluid cell with no fluid neighbour inside the domain:
    such a cell has a zero pressure diagonal (the reference divides by it,
    FvmColl.compute:2847, PisoColl.compute:255)."""
    f = flags.copy()
    while True:
        fluid = f == 0
        cnt = np.zeros(f.shape, dtype=np.int32)
        for ax in range(3):
            for sh in (1, -1):
                r = np.roll(fluid, sh, axis=ax)
                idx = [slice(None)] * 3
                idx[ax] = 0 if sh == 1 else -1
                r[tuple(idx)] = False
                cnt += r
        iso = fluid & (cnt == 0)
        if not iso.any():
            return f
        f[iso] = 1


def isolated_fluid_count(flags: np.ndarray) -> int:
    return int(((flags == 0) & (remove_isolated_fluid(flags) == 1)).sum())


def rasterise_boxes(nx: int, ny: int, nz: int, boxes, angle_deg: float = 0.0, margin: int = MARGIN) -> np.ndarray:
    """Boxes (x0, x1, z0, z1, h) in cells, rotated by angle_deg about the
    domain centre in the x-z plane, rasterised at cell centres.  Cells within
    `margin` of the x/z boundaries stay fluid.  Returns int32 (nz, ny, nx)."""
    flags = np.zeros((nz, ny, nx), dtype=np.int32)
    xs = np.arange(nx) + 0.5
    zs = np.arange(nz) + 0.5
    X, Z = np.meshgrid(xs, zs)  # (nz, nx)
    cx, cz = nx / 2.0, nz / 2.0
    th = math.radians(angle_deg)
    c, s = math.cos(th), math.sin(th)
    # inverse-rotate cell centres into the building frame
    Xr = cx + (X - cx) * c + (Z - cz) * s
    Zr = cz - (X - cx) * s + (Z - cz) * c
    inside_margin = (X > margin) & (X < nx - margin) & (Z > margin) & (Z < nz - margin)
    for b in boxes:
        x0, x1, z0, z1, h = b[:5]
        h = int(round(h))
        m = (Xr >= x0) & (Xr < x1) & (Zr >= z0) & (Zr < z1) & inside_margin
        if h <= 0 or not m.any():
            continue
        hh = min(h, ny - 1)
        flags[:, :hh, :][np.broadcast_to(m[:, None, :], (nz, hh, nx))] = 1
    return flags


def rasterise_boxes_gpu(nx: int, ny: int, nz: int, boxes, angle_deg: float = 0.0, margin: int = MARGIN,
                        device: int = 0) -> np.ndarray:
    """rasterise_boxes on the GPU (wf_rasterise_boxes): the same flags, bit for
    bit, in a fraction of the time for large grids and many directions."""
    from ctypes import POINTER, c_double, c_int32
    lib = _lib.load()
    b = np.ascontiguousarray([[float(v) for v in bx[:5]] for bx in boxes], dtype=np.float64).reshape(-1)
    out = np.empty((nz, ny, nx), dtype=np.int32)
    st = lib.wf_rasterise_boxes(nx, ny, nz, b.ctypes.data_as(POINTER(c_double)), len(boxes), float(angle_deg),
                                int(margin), int(device), out.ctypes.data_as(POINTER(c_int32)))
    if st != _lib.WF_OK:
        raise RuntimeError(f"wf_rasterise_boxes failed with status {st}")
    return out


def street_lattice_buildings(rng: np.random.Generator, nx: int, nz: int, count: int, fp_lo: int, fp_hi: int,
                             h_lo: float, h_hi: float, block: int = 16, street: int = 2, margin: int = MARGIN,
                             integer_heights: bool = True):
    """`count` buildings placed without overlap, one per lot of a street
    lattice with `block`-cell blocks separated by `street`-cell streets.
    Footprints are uniform in [fp_lo, fp_hi] cells per side, heights uniform
    in [h_lo, h_hi]."""
    pitch = block + street
    lots_x = (nx - 2 * margin - street) // pitch
    lots_z = (nz - 2 * margin - street) // pitch
    lots = [(i, j) for i in range(lots_x) for j in range(lots_z)]
    if count > len(lots):
        raise ValueError(f"{count} buildings do not fit {len(lots)} lots")
    pick = rng.choice(len(lots), size=count, replace=False)
    out = []
    for k in pick:
        i, j = lots[k]
        wx = int(rng.integers(fp_lo, fp_hi + 1))
        wz = int(rng.integers(fp_lo, fp_hi + 1))
        bx = margin + street + i * pitch + int(rng.integers(0, block - wx + 1))
        bz = margin + street + j * pitch + int(rng.integers(0, block - wz + 1))
        h = int(rng.integers(int(h_lo), int(h_hi) + 1)) if integer_heights else float(rng.uniform(h_lo, h_hi))
        out.append((bx, bx + wx, bz, bz + wz, h))
    return out


def _les_piso_cfg(nx, ny, nz, dx, dt, ustar, z0, cs, nv, np_, nc=2):
    return default_config(
        nx=nx, ny=ny, nz=nz, dx=dx, dt=dt, mu=1.5e-5, den=1.0,
        solver_type=_lib.SOLVER_PISO, piso_correctors=nc,
        turbulence=_lib.TURB_SMAGORINSKY, cs=cs,
        vel_iters=nv, pres_iters=np_,
        inflow_type=_lib.INFLOW_LOG, inflow_ustar=ustar, inflow_z0=z0, inflow_kappa=KAPPA,
        wind_speed=0.0,
    )


def plain_cube(nv: int = 50, np_: int = 30, steps: int = 100) -> Case:
    """64 x 32(up) x 48 cells of 0.5 m, one 8-cell cube spanning x 12..20,
    y 0..8, z 20..28; log inflow u* = 0.5, z0 = 0.1; Cs = 0.1; CFL 0.5."""
    nx, ny, nz, dx = 64, 32, 48, 0.5
    ustar, z0 = 0.5, 0.1
    umax = float(log_profile((ny - 0.5) * dx, ustar, z0))
    cfg = _les_piso_cfg(nx, ny, nz, dx, cfl_dt(umax, dx), ustar, z0, 0.1, nv, np_)
    flags = np.zeros((nz, ny, nx), dtype=np.int32)
    flags[20:28, 0:8, 12:20] = 1
    return Case("plain_cube", cfg, flags, None, steps, None, [(12, 20, 20, 28, 8)])


def urban_block(seed: int = 2, nv: int = 50, np_: int = 40, steps: int = 500) -> Case:
    """256 x 96(up) x 192 cells of 0.5 m, 48 buildings (footprints 6-16 cells,
    heights 4-40 cells) on a 16-cell block lattice; inflow u* = 0.6, z0 = 0.3
    with a 5 % multiplicative Gaussian perturbation per inlet face; Cs = 0.12."""
    nx, ny, nz, dx = 256, 96, 192, 0.5
    ustar, z0 = 0.6, 0.3
    rng = np.random.default_rng(seed)
    blds = street_lattice_buildings(rng, nx, nz, 48, 6, 16, 4, 40)
    flags = remove_isolated_fluid(rasterise_boxes(nx, ny, nz, blds))
    inlet = inlet_plane(ny, nz, dx, ustar, z0, perturb=0.05, rng=rng)
    dt = cfl_dt(float(inlet[:, :, 0].max()), dx)
    cfg = _les_piso_cfg(nx, ny, nz, dx, dt, ustar, z0, 0.12, nv, np_)
    return Case("urban_block", cfg, flags, inlet, steps, seed, blds)


def batch_directions(seed: int = 3, n_cases: int = 16, nv: int = 50, np_: int = 30, steps: int = 300):
    """16 cases of uneven size (nx 96..192, ny 48..80 up, nz 96..160, multiples
    of 8), 8-32 buildings (heights 4-30 cells) each, footprints rotated by
    k * 22.5 degrees before rasterising (the domain stays aligned with the
    flow, the buildings rotate)."""
    rng = np.random.default_rng(seed)
    cases = []
    for k in range(n_cases):
        nx = int(rng.integers(12, 25)) * 8
        ny = int(rng.integers(6, 11)) * 8
        nz = int(rng.integers(12, 21)) * 8
        dx = 0.5
        nb = int(rng.integers(8, 33))
        lots = ((nx - 2 * MARGIN - 2) // 18) * ((nz - 2 * MARGIN - 2) // 18)
        blds = street_lattice_buildings(rng, nx, nz, min(nb, lots), 6, 16, 4, 30)
        angle = 22.5 * (k % 16)
        flags = remove_isolated_fluid(rasterise_boxes(nx, ny, nz, blds, angle_deg=angle))
        ustar, z0 = 0.5, 0.1
        umax = float(log_profile((ny - 0.5) * dx, ustar, z0))
        cfg = _les_piso_cfg(nx, ny, nz, dx, cfl_dt(umax, dx), ustar, z0, 0.1, nv, np_)
        cases.append(Case(f"batch_{k:02d}_{angle:g}deg", cfg, flags, None, steps, seed,
                          [b + (angle,) for b in blds]))
    return cases


def batch_small(seed: int = 5, n_cases: int = 16, nv: int = 50, np_: int = 30, steps: int = 300):
    """16 small cases (nx, nz 48..72, ny 24..40 up, multiples of 8; about
    0.1 M cells each) with 1-4 buildings on a 6-cell margin, footprints
    rotated by k * 22.5 degrees: the regime where one case alone leaves most
    of the GPU idle."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_cases):
        nx = int(rng.integers(6, 10)) * 8
        ny = int(rng.integers(3, 6)) * 8
        nz = int(rng.integers(6, 10)) * 8
        dx = 0.5
        lots = ((nx - 2 * 6 - 2) // 18) * ((nz - 2 * 6 - 2) // 18)
        blds = street_lattice_buildings(rng, nx, nz, min(int(rng.integers(1, 5)), lots), 6, 14, 4, ny // 2,
                                        margin=6)
        angle = 22.5 * (k % 16)
        flags = remove_isolated_fluid(rasterise_boxes(nx, ny, nz, blds, angle_deg=angle, margin=6))
        ustar, z0 = 0.5, 0.1
        umax = float(log_profile((ny - 0.5) * dx, ustar, z0))
        cfg = _les_piso_cfg(nx, ny, nz, dx, cfl_dt(umax, dx), ustar, z0, 0.1, nv, np_)
        out.append(Case(f"small_{k:02d}_{angle:g}deg", cfg, flags, None, steps, seed,
                        [b + (angle,) for b in blds]))
    return out


def adjoint_street(seed: int = 4, nv: int = 50, np_: int = 30, steps: int = 200) -> Case:
    """128 x 64(up) x 96 cells of 0.5 m, 12 buildings on a street lattice
    with footprints 6-16 cells and continuous heights in [4, 30] cells, as a
    soft mask (sigmoid of width 1 cell, Brinkman drag 50/dt in solid cells;
    every cell fluid), dt at CFL 0.25.  PISO with turbulence off (the
    adjoint differentiates the laminar step).  Objective patch: the 32 x 32 street region x 48..80,
    z 32..64 at y index 3 (1.5-2.0 m), the last 100 of 200 steps,
    checkpoints every 20 steps."""
    nx, ny, nz, dx = 128, 64, 96, 0.5
    rng = np.random.default_rng(seed)
    blds = street_lattice_buildings(rng, nx, nz, 12, 6, 16, 4, 30, integer_heights=False)
    ustar, z0 = 0.5, 0.1
    umax = float(log_profile((ny - 0.5) * dx, ustar, z0))
    # CFL 0.25 on the inflow maximum: at 0.5 the laminar central-difference
    # step diverges within 20 steps on this layout
    cfg = _les_piso_cfg(nx, ny, nz, dx, cfl_dt(umax, dx, 0.25), ustar, z0, 0.1, nv, np_)
    cfg.turbulence = _lib.TURB_NONE
    soft = SoftBuildings([b[:4] for b in blds], [b[4] for b in blds], chi_max=50.0 / cfg.dt, width=1.0)
    flags = np.zeros((nz, ny, nx), dtype=np.int32)
    return Case("adjoint_street", cfg, flags, None, steps, seed, blds, soft)


ADJOINT_STREET_OBJECTIVE = dict(x0=48, x1=80, z0=32, z1=64, y=3, window=100)
ADJOINT_STREET_CHECKPOINT = 20


def adjoint_batch(seed: int = 6, n_dirs: int = 8, nv: int = 50, np_: int = 40, steps: int = 400):
    """Adjoint at scale: n_dirs wind directions (k * 360/n_dirs degrees; the
    footprints rotate, the domain stays aligned with the flow) over one
    256 x 96(up) x 256 block array of 0.5 m cells with 64 soft buildings
    (footprints 6-16 cells, heights uniform in [6, 40] cells), PISO with
    turbulence off and a constant viscosity of 0.3 m^2/s, nP = 40, dt at
    CFL 0.25, a 400-step window with checkpoints every 25."""
    nx, ny, nz, dx = 256, 96, 256, 0.5
    rng = np.random.default_rng(seed)
    blds = street_lattice_buildings(rng, nx, nz, 64, 6, 16, 6, 40, integer_heights=False)
    ustar, z0 = 0.5, 0.1
    umax = float(log_profile((ny - 0.5) * dx, ustar, z0))
    out = []
    for k in range(n_dirs):
        angle = k * 360.0 / n_dirs
        cfg = _les_piso_cfg(nx, ny, nz, dx, cfl_dt(umax, dx, 0.25), ustar, z0, 0.1, nv, np_)
        cfg.turbulence = _lib.TURB_NONE
        # constant eddy viscosity 0.3 m^2/s in place of the (not
        # differentiated) LES closure: with 1.5e-5 (and with 0.1 for the
        # oblique directions) the central-difference step with 40 pressure
        # sweeps diverges inside the 400-step window on this grid
        cfg.mu = 0.3
        soft = SoftBuildings([b[:4] for b in blds], [b[4] for b in blds], chi_max=50.0 / cfg.dt, width=1.0,
                             angle_deg=angle, margin=MARGIN)
        flags = np.zeros((nz, ny, nx), dtype=np.int32)
        out.append(Case(f"adjoint_batch_{angle:g}deg", cfg, flags, None, steps, seed,
                        [b + (angle,) for b in blds], soft))
    return out


ADJOINT_BATCH_OBJECTIVE = dict(x0=112, x1=144, z0=112, z1=144, y=3, window=200)
ADJOINT_BATCH_CHECKPOINT = 25


def aij_building(nv: int = 100, np_: int = 1000, steps: int = 1) -> Case:
    """The reference's validation case, Assets/Code/Config/AijBuilding0.asset:
    80 x 40 x 40 cells of 1 m, dt 0.04, mu 1.5e-5, SIMPLE, Smagorinsky 0.18,
    log inflow at 10 m/s with the reference's hard-coded kappa 0.4, z0 1,
    href 10, and the hard-coded box of CSInitBoxFlag (x 20..24, y 0..8,
    z 18..22, InitShaderColl.compute:320)."""
    nx, ny, nz = 80, 40, 40
    cfg = default_config(nx=nx, ny=ny, nz=nz, dx=1.0, dt=0.04, mu=1.5e-5, den=1.0,
                         solver_type=_lib.SOLVER_SIMPLE, turbulence=_lib.TURB_SMAGORINSKY, cs=0.18,
                         inflow_type=_lib.INFLOW_LOG, wind_speed=10.0, vel_iters=nv, pres_iters=np_)
    flags = np.zeros((nz, ny, nx), dtype=np.int32)
    flags[18:22, 0:8, 20:24] = 1
    return Case("aij_building", cfg, flags, None, steps, None, [(20, 24, 18, 22, 8)])


def small_case(nx=24, ny=12, nz=16, piso=True, les=True, seed=0, nv=8, np_=12, buildings=2,
               inflow_log=True, compat=0) -> Case:
    """Small seeded case for parity tests (oracle finishes in well under a second)."""
    rng = np.random.default_rng(seed)
    dx = 0.5
    cfg = default_config(nx=nx, ny=ny, nz=nz, dx=dx, mu=1.5e-5, den=1.0,
                         solver_type=_lib.SOLVER_PISO if piso else _lib.SOLVER_SIMPLE, piso_correctors=2,
                         turbulence=_lib.TURB_SMAGORINSKY if les else _lib.TURB_NONE, cs=0.12,
                         vel_iters=nv, pres_iters=np_, compat_flags=compat)
    if inflow_log:
        cfg.inflow_type = _lib.INFLOW_LOG
        cfg.inflow_ustar, cfg.inflow_z0, cfg.inflow_kappa = 0.5, 0.1, KAPPA
        umax = float(log_profile((ny - 0.5) * dx, 0.5, 0.1))
    else:
        cfg.inflow_type = _lib.INFLOW_CONSTANT
        cfg.wind_speed = 3.0
        umax = 3.0
    cfg.dt = cfl_dt(umax, dx)
    flags = np.zeros((nz, ny, nx), dtype=np.int32)
    blds = []
    for _ in range(buildings):
        wx, wz = int(rng.integers(2, 5)), int(rng.integers(2, 5))
        x0 = int(rng.integers(4, max(5, nx - 6 - wx)))
        z0_ = int(rng.integers(3, max(4, nz - 3 - wz)))
        h = int(rng.integers(2, max(3, ny // 2)))
        flags[z0_:z0_ + wz, 0:h, x0:x0 + wx] = 1
        blds.append((x0, x0 + wx, z0_, z0_ + wz, h))
    flags = remove_isolated_fluid(flags)
    return Case(f"small_{nx}x{ny}x{nz}_s{seed}", cfg, flags, None, 1, seed, blds)


def small_soft_case(nx=24, ny=12, nz=16, piso=True, seed=0, nv=6, np_=8, buildings=2) -> Case:
    """Small seeded case with soft buildings (drag field, every cell fluid)
    and turbulence off, for the adjoint tests."""
    base = small_case(nx, ny, nz, piso=piso, les=False, seed=seed, nv=nv, np_=np_, buildings=0)
    rng = np.random.default_rng(1000 + seed)
    fps, hs = [], []
    x = 5
    for _ in range(buildings):
        wx, wz = int(rng.integers(2, 4)), int(rng.integers(3, 6))
        z0_ = int(rng.integers(2, max(3, nz - 2 - wz)))
        fps.append((x, x + wx, z0_, z0_ + wz))
        hs.append(float(rng.uniform(2.0, ny / 2)))
        x += wx + int(rng.integers(3, 6))
    soft = SoftBuildings(fps, hs, chi_max=50.0 / base.cfg.dt, width=1.0)
    return Case(f"small_soft_{nx}x{ny}x{nz}_s{seed}", base.cfg, base.flags, None, 1, seed, [], soft)


def stretched_faces(n: int, dx: float, n_uniform: int, n_side: int, ratio: float = 1.08) -> np.ndarray:
    """Face positions (n + 1, float32) of one axis of the reference's
    non-uniform mesh (InitMeshBuffers, FvmSolverGpu.cs:682-788): n_side cells
    growing by `ratio` towards the lower boundary, n_uniform cells of dx,
    then n - n_uniform - n_side cells towards the upper boundary.  The
    reference sizes the upper side from the lower side's array too
    (:758-762), so that side may not be longer than n_side; it fails there
    with an index error, this raises ValueError.  FP32 throughout, as the
    reference's float arrays."""
    n_upper = n - n_uniform - n_side
    if n_uniform < 0 or n_side < 0 or n_upper < 0 or n_upper > n_side:
        raise ValueError(f"{n} cells cannot be split as {n_side} + {n_uniform} + {n_upper} "
                         f"(the upper side reuses the lower side's {n_side} sizes)")
    d = np.float32(dx)
    r = np.float32(ratio)
    sizes = np.zeros(n_side, dtype=np.float32)
    if n_side > 0:
        sizes[0] = d
        for i in range(1, n_side):
            sizes[i] = np.float32(sizes[i - 1] * r)
    f = np.zeros(n + 1, dtype=np.float32)
    for i in range(1, n_side + 1):                    # largest cell at the boundary
        f[i] = np.float32(f[i - 1] + sizes[n_side - i])
    for i in range(n_side + 1, n_side + n_uniform + 1):
        f[i] = np.float32(f[i - 1] + d)
    for i in range(n_side + n_uniform + 1, n + 1):    # :758-762
        f[i] = np.float32(f[i - 1] + sizes[i - (n_side + n_uniform + 1)])
    return f


def wind_tunnel(nv: int = 800, np_: int = 2000, steps: int = 1) -> Case:
    """The reference's non-uniform grid case, Assets/Code/Config/
    WindTunnelBoxConfig.asset: 100 x 50(up) x 100 cells (physDomainSize
    100 x 50 x 100, gridResX 100, so dx = 1), gridType CollNonUniform with
    the mesh InitMeshBuffers builds (uniform core 50 x 50 x 50, 25 cells per
    side in x and z growing by 1.08, none in y), dt 0.02, mu 1, den 1,
    SIMPLE, no turbulence model, constant inflow at RuntimeConfig.windSpeed
    10 m/s, velocity BCs X0 fixed, Xn zero-gradient, the rest symmetry;
    pressure X0 zero-gradient, Xn fixed, the rest symmetry; velMaxNumIter
    800, presMaxNumIter 2000, and the box of CSInitBoxFlag (x 20..24,
    y 0..8, z 18..22, InitShaderColl.compute:320; solidType Box)."""
    nx, ny, nz = 100, 50, 100
    cfg = default_config(nx=nx, ny=ny, nz=nz, dx=1.0, dt=0.02, mu=1.0, den=1.0,
                         solver_type=_lib.SOLVER_SIMPLE, turbulence=_lib.TURB_NONE,
                         inflow_type=_lib.INFLOW_CONSTANT, wind_speed=10.0, vel_iters=nv, pres_iters=np_)
    vel = {_lib.FACE_X0: _lib.BND_FIXED_VALUE, _lib.FACE_XN: _lib.BND_ZERO_GRAD}
    pres = {_lib.FACE_X0: _lib.BND_ZERO_GRAD, _lib.FACE_XN: _lib.BND_FIXED_VALUE}
    for f in range(6):
        cfg.vel_bc[f] = vel.get(f, _lib.BND_SYMMETRY)
        cfg.pres_bc[f] = pres.get(f, _lib.BND_SYMMETRY)
    flags = np.zeros((nz, ny, nx), dtype=np.int32)
    flags[18:22, 0:8, 20:24] = 1
    faces = (stretched_faces(nx, 1.0, 50, 25), stretched_faces(ny, 1.0, 50, 0), stretched_faces(nz, 1.0, 50, 25))
    return Case("wind_tunnel", cfg, flags, None, steps, None, [(20, 24, 18, 22, 8)], None, faces)


def small_nonuniform_case(nx=16, ny=10, nz=12, log_inflow=False, seed=0, nv=8, np_=12,
                          x_split=(8, 4), les=False) -> Case:
    """Small non-uniform case for parity tests: stretched x (x_split =
    (uniform, per side) cells: 4 + 8 + 4 by default), y (2 + 6 + 2) and z
    (3 + 6 + 3) axes of 0.5 m cores, one box.
    log_inflow=False: the wind-tunnel boundary set with a constant 3 m/s
    inflow; True: the urban set (no-slip ground, symmetry top and sides)
    with a log inflow and no fixed-pressure face (the pressure is
    normalised).  les=True adds the Smagorinsky model (Cs = 0.15), whose
    wall function and LES kernels run with the constant dx, as in the
    reference."""
    rng = np.random.default_rng(seed)
    dx = 0.5
    cfg = default_config(nx=nx, ny=ny, nz=nz, dx=dx, mu=0.01, den=1.0, solver_type=_lib.SOLVER_SIMPLE,
                         turbulence=_lib.TURB_SMAGORINSKY if les else _lib.TURB_NONE, vel_iters=nv,
                         pres_iters=np_)
    if les:
        cfg.cs = 0.15
    if log_inflow:
        cfg.inflow_type = _lib.INFLOW_LOG
        cfg.wind_speed = 4.0
        cfg.inflow_kappa, cfg.inflow_z0, cfg.inflow_href = 0.4, 1.0, 10.0
        cfg.pres_bc[_lib.FACE_XN] = _lib.BND_ZERO_GRAD
    else:
        cfg.inflow_type = _lib.INFLOW_CONSTANT
        cfg.wind_speed = 3.0
        vel = {_lib.FACE_X0: _lib.BND_FIXED_VALUE, _lib.FACE_XN: _lib.BND_ZERO_GRAD}
        pres = {_lib.FACE_X0: _lib.BND_ZERO_GRAD, _lib.FACE_XN: _lib.BND_FIXED_VALUE}
        for f in range(6):
            cfg.vel_bc[f] = vel.get(f, _lib.BND_SYMMETRY)
            cfg.pres_bc[f] = pres.get(f, _lib.BND_SYMMETRY)
    cfg.dt = cfl_dt(6.0, dx)
    flags = np.zeros((nz, ny, nx), dtype=np.int32)
    x0 = int(rng.integers(4, 8))
    z0_ = int(rng.integers(3, 6))
    h = int(rng.integers(2, 5))
    flags[z0_:z0_ + 3, 0:h, x0:x0 + 2] = 1
    faces = (stretched_faces(nx, dx, *x_split), stretched_faces(ny, dx, 6, 2), stretched_faces(nz, dx, 6, 3))
    name = f"small_nu_{nx}x{ny}x{nz}_{'log' if log_inflow else 'const'}{'_les' if les else ''}_s{seed}"
    return Case(name, cfg, flags, None, 1, seed, [(x0, x0 + 2, z0_, z0_ + 3, h)], None, faces)


def apply_case(solver, case: Case) -> None:
    """Reference set-up order: the mesh first (InitMeshBuffers before
    InitVelPresFields, FvmSolverGpu.cs:204-213), flags after the fields
    (FvmSolverController.cs:368-375), then the inlet plane."""
    if case.faces is not None:
        solver.set_face_positions(*case.faces)
        solver.InitVelPresFields()
        solver.SetFixedValueVelBndCond()
    solver.InitFlags(case.flags)
    if case.inlet is not None:
        solver.set_inflow_plane(case.inlet)
    if case.soft is not None:
        c = case.cfg
        solver.set_field(_lib.FIELD_DRAG, case.soft.drag(c.nx, c.ny, c.nz, np.float64).reshape(-1))


WORKLOADS = {
    "plain_cube": plain_cube,
    "urban_block": urban_block,
    "adjoint_street": adjoint_street,
    "aij_building": aij_building,
    "wind_tunnel": wind_tunnel,
}
