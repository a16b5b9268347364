"""Seeded synthetic scenes standing in for the reference's HDF5/PNG scene inputs.

The reference builds scenes from map.h5 / PNG files and a Poisson-disk sampler
(SnapshotManager::PrepareGrid / PopulatePoints, snapshotmanager.cpp:55-270).
These generators produce the same artefacts -- SimParams, the grid status
bytes (100 = modelled water, 0 = land/wall), the current field and an HSSOA in
the reference layout -- from a seed, for the benchmark scene families:

  ice_block   256x128 grid, h=2 m, 200x80-cell rectangle at 2x2 ppc (64,000 points)
  floe_field  4096x2048 grid, h=1 m, 2000 Voronoi floes (70% kept), 4 ppc,
              lognormal(0, 0.3) thickness per floe, Rankine-vortex wind (23.0M points)
  ridging     1024x512 grid, h=2 m, ~1M crushed points driven at 2 m/s against x=0
  random      small grids with randomised state, for parity tests

Particles sit on a 2x2 lattice per cell (sub-cell centres) with uniform jitter
of +-0.25h, then go through the reference's integer-cell conversion
(proxypoint2d.cpp:125-139).  ParticleVolume = h^2/ppc.  The outer ring of two
nodes is wall (status 0): the reference disables points that reach it
(kernels.cuh:254-261).
"""
from dataclasses import dataclass, field

import numpy as np

from . import hssoa as H
from .params import (SimParams, Options, FORCING_COMPAT, FORCING_EXTENDED, WIND_NONE,
                     WIND_UNIFORM, WIND_RANKINE, IDX_VELX, IDX_FE00, IDX_BP00, IDX_JP_INV,
                     IDX_UTILITY, STATUS_CRUSHED)

RHO_ICE = 917.0
RHO_WATER = 1025.0
CD_WATER = 5.5e-3
RHO_AIR = 1.3
CA_AIR = 1.2e-3


@dataclass
class Scene:
    name: str
    prms: SimParams
    status: np.ndarray            # uint8 [G], node = y + x*GridY
    current: np.ndarray           # float64 [2G]: vx block, vy block
    soa: np.ndarray               # float64 [19, capacity]
    n: int
    steps: int
    options: Options = field(default_factory=Options.default)
    seed: int = 0
    info: dict = field(default_factory=dict)

    @property
    def grid_nodes(self) -> int:
        return self.prms.GridXTotal * self.prms.GridYTotal


def base_params(gx, gy, h, dt, frame_steps=100, E=1e9, nu=0.3, rho=RHO_ICE, phi=35.0,
                ppc=4, thickness_ref=1.0) -> SimParams:
    """SimParams for a synthetic scene.  Material values not fixed by the scene
    keep the reference defaults (parameters_sim.cpp:7-55).  Compat water drag:
    waterDragEffectiveQuadratic = rho_w*Cd/(rho_i*thickness_ref), linear = 0."""
    p = SimParams.reset()
    p.GridXTotal, p.GridYTotal = gx, gy
    p.cellsize = h
    p.InitialTimeStep = dt
    p.AnimationFramePeriod = dt * (frame_steps + 0.5)   # int() gives frame_steps
    p.SimulationEndTime = 1e30
    p.YoungsModulus, p.PoissonsRatio, p.IceDensity = E, nu, rho
    p.DP_phi = phi
    p.ParticleVolume = h * h / ppc
    p.sea_water_density = RHO_WATER
    p.waterDragEffectiveLinear = 0.0
    p.waterDragEffectiveQuadratic = RHO_WATER * CD_WATER / (rho * thickness_ref)
    p.InitializationImageSizeX, p.InitializationImageSizeY = gx, gy
    p.DimensionHorizontal = h * (gx - 1)
    p.compute_helper_variables()
    return p


def wall_ring_status(gx, gy, ring=2) -> np.ndarray:
    st = np.full((gx, gy), 100, np.uint8)
    st[:ring, :] = 0
    st[-ring:, :] = 0
    st[:, :ring] = 0
    st[:, -ring:] = 0
    return np.ascontiguousarray(st.reshape(-1))   # index y + x*gy


def uniform_current(gx, gy, vx, vy=0.0) -> np.ndarray:
    G = gx * gy
    c = np.empty(2 * G)
    c[:G] = vx
    c[G:] = vy
    return c


def lattice_points(cells_x, cells_y, h, rng, ppc_side=2, jitter=0.25):
    """Particles of a set of cells (integer arrays of cell corners): ppc_side^2
    per cell at sub-cell centres, jittered uniformly by +-jitter*h.  Output is
    ordered by cell then sub-position."""
    cells_x = np.asarray(cells_x, np.float64)
    cells_y = np.asarray(cells_y, np.float64)
    sub = (np.arange(ppc_side) + 0.5) / ppc_side
    ox, oy = np.meshgrid(sub, sub, indexing="ij")
    ox, oy = ox.reshape(-1), oy.reshape(-1)
    k = len(ox)
    x = (cells_x[:, None] + ox[None, :]).reshape(-1)
    y = (cells_y[:, None] + oy[None, :]).reshape(-1)
    n = len(x)
    x = (x + rng.uniform(-jitter, jitter, n)) * h
    y = (y + rng.uniform(-jitter, jitter, n)) * h
    return x, y, k


def _sort_by_cell(x, y, h, gy, *extra):
    xi = (x / h + 0.5).astype(np.int64)
    yi = (y / h + 0.5).astype(np.int64)
    order = np.argsort(xi * gy + yi, kind="stable")
    return (x[order], y[order]) + tuple(e[order] for e in extra)


def ice_block(seed=1234, forcing=FORCING_COMPAT) -> Scene:
    """256x128 grid, h=2 m, 200x80-cell ice rectangle, 2x2 ppc, jitter +-0.25h
    (64,000 points), thickness 1 m, zero velocity, current 0.1 m/s along +x,
    dt=2e-4 s, 1000 steps.  Extended forcing adds a uniform 10 m/s wind along +x."""
    rng = np.random.default_rng(seed)
    gx, gy, h, dt = 256, 128, 2.0, 2e-4
    p = base_params(gx, gy, h, dt)
    x0, y0 = (gx - 200) // 2, (gy - 80) // 2
    cx, cy = np.meshgrid(np.arange(x0, x0 + 200), np.arange(y0, y0 + 80), indexing="ij")
    x, y, _ = lattice_points(cx.reshape(-1), cy.reshape(-1), h, rng)
    x, y = _sort_by_cell(x, y, h, gy)
    soa = H.init_points(x, y, np.ones(len(x)), h)
    p.nPtsInitial = len(x)
    opts = Options.default(forcing=forcing)
    if forcing == FORCING_EXTENDED:
        opts.wind_kind, opts.wind_u, opts.wind_v = WIND_UNIFORM, 10.0, 0.0
    return Scene("ice_block", p, wall_ring_status(gx, gy), uniform_current(gx, gy, 0.1),
                 soa, len(x), 1000, opts, seed)


def voronoi_floes(gx, gy, n_seeds, keep, rng, margin=3):
    """Per-cell floe id (-1 = open water) from a Voronoi tessellation of the
    cell centres by uniform seeds, keeping a random `keep` fraction of floes."""
    from scipy.spatial import cKDTree
    seeds = np.stack([rng.uniform(0, gx, n_seeds), rng.uniform(0, gy, n_seeds)], 1)
    kept = rng.random(n_seeds) < keep
    tree = cKDTree(seeds)
    cx, cy = np.meshgrid(np.arange(gx), np.arange(gy), indexing="ij")
    cx, cy = cx.reshape(-1), cy.reshape(-1)
    floe = np.full(gx * gy, -1, np.int64)
    inner = (cx >= margin) & (cx < gx - margin - 1) & (cy >= margin) & (cy < gy - margin - 1)
    idx = np.nonzero(inner)[0]
    chunk = 1 << 22
    for s in range(0, len(idx), chunk):
        sl = idx[s:s + chunk]
        _, f = tree.query(np.stack([cx[sl] + 0.5, cy[sl] + 0.5], 1))
        floe[sl] = np.where(kept[f], f, -1)
    return floe, cx, cy, seeds


def floe_field(seed=1235, gx=4096, gy=2048, n_seeds=2000, keep=0.7, forcing=FORCING_EXTENDED,
            max_points=None) -> Scene:
    """4096x2048 grid, h=1 m; 2000 Voronoi floes with 70% kept; 4 ppc with
    +-0.25h jitter; per-floe thickness lognormal(0, 0.3) m; Rankine-vortex wind
    (20 m/s peak at an 800-cell radius, seeded centre); dt=1e-4 s, 200 steps.
    `max_points` keeps whole floes (in random order) until the count is
    reached, for the ~8.4M-point variant."""
    rng = np.random.default_rng(seed)
    h, dt = 1.0, 1e-4
    p = base_params(gx, gy, h, dt)
    floe, cx, cy, seeds = voronoi_floes(gx, gy, n_seeds, keep, rng)
    thick_per_floe = np.exp(rng.normal(0.0, 0.3, n_seeds))
    if max_points is not None:
        ids, counts = np.unique(floe[floe >= 0], return_counts=True)
        order = rng.permutation(len(ids))
        csum = np.cumsum(counts[order] * 4)
        keep_ids = ids[order][csum <= max_points]
        if len(keep_ids) == 0 and len(ids):   # every floe is larger than the cap: keep the smallest
            keep_ids = ids[np.argmin(counts)][None]
        floe = np.where(np.isin(floe, keep_ids), floe, -1)
    ice = floe >= 0
    x, y, k = lattice_points(cx[ice], cy[ice], h, rng)
    thick = np.repeat(thick_per_floe[floe[ice]], k)
    x, y, thick = _sort_by_cell(x, y, h, gy, thick)
    soa = H.init_points(x, y, thick, h)
    p.nPtsInitial = len(x)
    opts = Options.default(forcing=forcing)
    centre = rng.uniform([0.25 * gx, 0.25 * gy], [0.75 * gx, 0.75 * gy])
    opts.wind_kind = WIND_RANKINE
    opts.wind_cx, opts.wind_cy = centre[0] * h, centre[1] * h
    opts.wind_vmax, opts.wind_radius = 20.0, 800.0 * h
    return Scene("floe_field", p, wall_ring_status(gx, gy), uniform_current(gx, gy, 0.1),
                 soa, len(x), 200, opts, seed,
                 info={"floes_kept": int(len(np.unique(floe[ice]))), "n_seeds": n_seeds})


# grid sizes an ensemble scene picks from (cells, smallest that fits its points)
ENSEMBLE_GRIDS = [(128, 128), (256, 128), (256, 256), (512, 256), (512, 512), (1024, 512), (1024, 1024),
                  (2048, 1024)]


def ensemble_scene(seed, target_points, wind_speed, wind_dir, current_speed, current_dir,
                   forcing=FORCING_EXTENDED) -> Scene:
    """One scene of the batched-ensemble workload: floe-field generation rules
    (Voronoi floes, 70% kept, 4 ppc, lognormal thickness) on the smallest grid
    of ENSEMBLE_GRIDS that holds `target_points`, whole floes kept up to that
    count; uniform wind and current of the given speeds and directions."""
    gx, gy = ENSEMBLE_GRIDS[-1]
    for g in ENSEMBLE_GRIDS:
        if g[0] * g[1] * 4 * 0.7 * 0.8 >= target_points:
            gx, gy = g
            break
    n_seeds = max(8, round(gx * gy / 1500))   # floes of ~1500 cells, so whole floes approach the target
    sc = floe_field(seed=seed, gx=gx, gy=gy, n_seeds=n_seeds, forcing=forcing, max_points=target_points)
    sc.options.wind_kind = WIND_UNIFORM
    sc.options.wind_u = float(wind_speed * np.cos(wind_dir))
    sc.options.wind_v = float(wind_speed * np.sin(wind_dir))
    sc.current = uniform_current(gx, gy, float(current_speed * np.cos(current_dir)),
                                 float(current_speed * np.sin(current_dir)))
    sc.name = "ensemble"
    sc.info.update({"target_points": int(target_points), "wind_speed": float(wind_speed),
                    "current_speed": float(current_speed)})
    return sc


def ensemble(n_scenes=96, seed=4242, n_min=10_000, n_max=2_000_000, forcing=FORCING_EXTENDED):
    """Batched-ensemble workload: `n_scenes` independent
    scenes, point counts log-uniform in [n_min, n_max], Voronoi floes as in
    the floe field, grids from 128x128 to 2048x1024 sized to each scene, wind speed
    uniform in 5-25 m/s with a uniform direction, current uniform in
    0-0.3 m/s with a uniform direction."""
    return [ensemble_scene(**spec, forcing=forcing) for spec in ensemble_specs(n_scenes, seed, n_min, n_max)]


def ensemble_specs(n_scenes=96, seed=4242, n_min=10_000, n_max=2_000_000):
    """The draws behind ensemble(): one dict of ensemble_scene arguments per
    scene, cheap to compute, so that ranks can split the scenes by size before
    generating only their own."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        target = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        out.append(dict(seed=seed + 1 + k, target_points=target, wind_speed=rng.uniform(5.0, 25.0),
                        wind_dir=rng.uniform(0, 2 * np.pi), current_speed=rng.uniform(0.0, 0.3),
                        current_dir=rng.uniform(0, 2 * np.pi)))
    return out


def split_by_size(sizes, parts):
    """Scene indices for each of `parts` ranks, largest scenes first onto the
    least-loaded rank, so each rank's point total is about the same."""
    load = [0] * parts
    out = [[] for _ in range(parts)]
    for i in sorted(range(len(sizes)), key=lambda i: -sizes[i]):
        r = min(range(parts), key=lambda r: load[r])
        out[r].append(i)
        load[r] += sizes[i]
    return [sorted(o) for o in out]


def ridging(seed=1236, gx=1024, gy=512, cells_x=500, cells_y=500, h=2.0, dt=2e-4,
            speed=2.0, forcing=FORCING_COMPAT, steps=1000) -> Scene:
    """Compressive ridging scene: a cells_x x cells_y rectangle at 4 ppc
    touching the x=0 wall ring, all points crushed (0x10000, as
    snapshotmanager.cpp:243 marks status-1 ice), moving at `speed` m/s towards
    the wall so the Drucker-Prager return map is active.  Default: 1024x512
    grid, 1M points."""
    rng = np.random.default_rng(seed)
    p = base_params(gx, gy, h, dt)
    y0 = (gy - cells_y) // 2
    cx, cy = np.meshgrid(np.arange(2, 2 + cells_x), np.arange(y0, y0 + cells_y), indexing="ij")
    x, y, _ = lattice_points(cx.reshape(-1), cy.reshape(-1), h, rng)
    x, y = _sort_by_cell(x, y, h, gy)
    n = len(x)
    soa = H.init_points(x, y, np.ones(n), h, crushed=np.ones(n, bool),
                        velocity=(np.full(n, -speed), np.zeros(n)))
    p.nPtsInitial = n
    opts = Options.default(forcing=forcing)
    return Scene("ridging", p, wall_ring_status(gx, gy), uniform_current(gx, gy, -speed),
                 soa, n, steps, opts, seed)


def random_state(seed=7, gx=64, gy=48, h=1.5, dt=1e-4, fill=0.6, ppc_side=2, strain=2e-3,
                 vel=0.5, crushed_frac=0.5, low_jp_frac=0.1, thickness=(0.5, 2.0),
                 forcing=FORCING_COMPAT, capacity=None) -> Scene:
    """Small scene with randomised state for parity tests: random velocities,
    F = I + H with |H| ~ strain, random APIC C, a mix of crushed and intact
    points, some with Jp_inv < 0.1 (return-map case 0), varied thickness."""
    rng = np.random.default_rng(seed)
    p = base_params(gx, gy, h, dt, frame_steps=7)
    cells = [(i, j) for i in range(3, gx - 4) for j in range(3, gy - 4) if rng.random() < fill]
    cells = np.array(cells)
    x, y, k = lattice_points(cells[:, 0], cells[:, 1], h, rng, ppc_side=ppc_side)
    x, y = _sort_by_cell(x, y, h, gy)
    n = len(x)
    thick = rng.uniform(thickness[0], thickness[1], n)
    crushed = rng.random(n) < crushed_frac
    soa = H.init_points(x, y, thick, h, crushed=crushed, capacity=capacity)
    soa[IDX_VELX, :n] = rng.normal(0, vel, n)
    soa[IDX_VELX + 1, :n] = rng.normal(0, vel, n)
    Hm = rng.normal(0, strain, (4, n))
    soa[IDX_FE00:IDX_FE00 + 4, :n] += Hm
    soa[IDX_BP00:IDX_BP00 + 4, :n] = rng.normal(0, vel / h, (4, n))
    jp = rng.uniform(0.5, 1.5, n)
    low = rng.random(n) < low_jp_frac
    jp[low] = rng.uniform(0.02, 0.09, low.sum())
    soa[IDX_JP_INV, :n] = jp
    p.nPtsInitial = n
    cur = np.empty(2 * gx * gy)
    cur[:gx * gy] = rng.normal(0.05, 0.05, gx * gy)
    cur[gx * gy:] = rng.normal(0.0, 0.05, gx * gy)
    opts = Options.default(forcing=forcing)
    if forcing == FORCING_EXTENDED:
        opts.wind_kind, opts.wind_u, opts.wind_v = WIND_UNIFORM, 8.0, -3.0
    return Scene("random", p, wall_ring_status(gx, gy), cur, soa, n, 10, opts, seed)


BUILDERS = {"ice_block": ice_block, "floe_field": floe_field, "ridging": ridging, "random": random_state}
