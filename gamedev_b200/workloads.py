"""Model constants and seeded synthetic swarms for the benchmark configurations.

The reference fixes every constant at compile time in a model's const_defs.cuh and draws its
initial swarm with host samplers (inc/swarm/swarm_host.cuh:51-737).  This module gives each
benchmark configuration its gd_config (the same constants a model directory would hold) and a
deterministic particle array in the reference record layout (position = azimuth, spherical radius,
polar angle; velocity = l_phi, v_r, l_theta; grain diameter; grain count).

Units are cgs: G in cm^3 g^-1 s^-2, the star in grams, R_0 = 1 au, grain sizes are DIAMETERS in
cm (the reference's par_size, const_defs.cuh:200), times in s.  The gas disk is
Sigma = Sigma_0 (R/au)^-1 carrying 100x the dust mass on [1, 100] au, h = 0.05 (R/au)^0.25, so
IDX_P = -1, IDX_Q = -0.5, ASPR_0 = 0.05; STOKES_0 is the Epstein midplane Stokes number of a 1 cm
grain at 1 au.

Config names:
  c0_plain_small   3D, N = 65,536, K = 32, KD search, monodisperse radius 1e-4 cm, coagulation only
  c1_multisize_2d  radial-azimuthal, N = 2^20, K = 64, Morton search, gap at 9-11 au, ring at 30 au,
                   radii log-uniform on [1e-4, 10] cm, fragmentation above 1 m/s
  c3_learned_3d    3D, N = 10^7, K = 64, c0 positions, radii log-uniform on [1e-4, 10] cm
  c4_production_3d as c3, with the full Strang step: drag and gravity, radiation pressure with
                   Poynting-Robertson drag, Ito diffusion and coagulation/fragmentation
  t0_transport_3d  the c4 shapes at N = 65,536 with transport and diffusion but no radiation
  w0_wedge_3d      3D wedge (azimuth [-0.6, 0.6)), N = 65,536, K = 32, KD search, with periodic
                   images
  w1_narrow_2d     radial-azimuthal 0.05 rad wedge, N = 65,536, K = 32, Morton search, with periodic
                   images
  w2_wide_3d       3D 3.8 rad wedge (wider than pi), N = 65,536, K = 32, Morton search: the images
                   the Morton ghost rule keeps
"""

from __future__ import annotations

import math

import numpy as np

from ._lib import GD_KERNEL_CUSTOM, GD_SEARCH_KDTREE, GD_SEARCH_MORTON, config_defaults

AU = 1.495978707e13
MSUN = 1.98847e33
G_CGS = 6.6743e-8
R_IN_AU, R_OUT_AU = 1.0, 100.0
DUST_MASS = 1.0e-4 * MSUN
GAS_TO_DUST = 100.0


def orbital_time() -> float:
    """1 / Omega_K at R_0 = 1 au, the time unit the reference's code-unit constants assume."""
    return math.sqrt(AU ** 3 / (G_CGS * MSUN))


def _base_config(n_k: int, three_d: bool, search: int, v_frag: float, smin: float, smax: float):
    cfg = config_defaults()
    cfg.G, cfg.M_S, cfg.R_0, cfg.S_0 = G_CGS, MSUN, AU, 1.0
    cfg.n_x, cfg.n_y = 64, 64
    cfg.n_z = 32 if three_d else 1
    cfg.x_min, cfg.x_max = -math.pi, math.pi
    cfg.y_min, cfg.y_max = R_IN_AU * AU, R_OUT_AU * AU * (1.0 + 1e-12)
    if three_d:
        cfg.z_min, cfg.z_max = 0.5 * math.pi - 1.0, 0.5 * math.pi + 1.0
    else:
        cfg.z_min = cfg.z_max = 0.5 * math.pi
    gas_mass = GAS_TO_DUST * DUST_MASS
    sigma_0 = gas_mass / (2.0 * math.pi * AU * (R_OUT_AU - R_IN_AU) * AU)
    cfg.sigma_0, cfg.aspr_0, cfg.idx_p, cfg.idx_q = sigma_0, 0.05, -1.0, -0.5
    cfg.const_nu, cfg.alpha = 0, 1.0e-3
    cfg.code_unit = 0
    cfg.rho_0 = 1.0
    cfg.stokes_0 = math.pi * cfg.rho_0 * cfg.S_0 / (4.0 * sigma_0)
    cfg.coag_kernel = GD_KERNEL_CUSTOM
    cfg.n_k = n_k
    cfg.h_search = 1.0
    cfg.v_frag = v_frag
    cfg.col_bath_max = 0.05 * orbital_time()
    cfg.init_smin, cfg.init_smax = smin, smax
    cfg.search = search
    return cfg


CONFIGS = {
    "c0_plain_small": dict(n=65536, k=32, three_d=True, search=GD_SEARCH_KDTREE, v_frag=1.0e30,
                           sizes=("mono", 2.0e-4), radial="loguniform", seed=1),
    "c1_multisize_2d": dict(n=1 << 20, k=64, three_d=False, search=GD_SEARCH_MORTON, v_frag=100.0,
                            sizes=("loguniform", 2.0e-4, 20.0), radial="gap_ring", seed=2),
    "c3_learned_3d": dict(n=10_000_000, k=64, three_d=True, search=GD_SEARCH_KDTREE, v_frag=100.0,
                          sizes=("loguniform", 2.0e-4, 20.0), radial="loguniform", seed=3),
    # the full production step: drag and gravity, radiation pressure with Poynting-Robertson drag
    # through the radial optical depth, Ito diffusion and collisions.  Radiation constants in cgs:
    # a 1 cm grain feels 1e-4 of the star's gravity, its gray opacity is its geometric cross section
    # per mass (1.5 cm^2/g), the force ramps up over one orbit at 1 au
    "c4_production_3d": dict(n=10_000_000, k=64, three_d=True, search=GD_SEARCH_KDTREE, v_frag=100.0,
                             sizes=("loguniform", 2.0e-4, 20.0), radial="loguniform", seed=4,
                             flags=dict(radiation=1, pr_effect=1),
                             run=dict(beta_0=1.0e-4, kappa_0=1.5, t_beta="orbit", c_light=2.99792458e10)),
    # the c4 shapes with the dynamics alone and no radiation field (ssa_transport + diffusion)
    "t0_transport_3d": dict(n=65536, k=64, three_d=True, search=GD_SEARCH_KDTREE, v_frag=100.0,
                            sizes=("loguniform", 2.0e-4, 20.0), radial="loguniform", seed=11),
    # azimuthal wedges (periodic images): a 1.2 rad wedge searched by the KD tree, whose owners
    # beyond ~4 au can reach two images of one particle, and a 0.05 rad sliver searched by the
    # Morton index, where every owner can
    "w0_wedge_3d": dict(n=65536, k=32, three_d=True, search=GD_SEARCH_KDTREE, v_frag=100.0,
                        sizes=("loguniform", 2.0e-4, 20.0), radial="loguniform", seed=7, x_range=(-0.6, 0.6)),
    "w1_narrow_2d": dict(n=65536, k=32, three_d=False, search=GD_SEARCH_MORTON, v_frag=100.0,
                         sizes=("loguniform", 2.0e-4, 20.0), radial="loguniform", seed=8, x_range=(0.0, 0.05)),
    # a 3.8 rad wedge (wider than pi) searched by the Morton index: a rotated image of a particle far
    # from both seams lands among the physical particles, and only the ghost rule keeps it out
    "w2_wide_3d": dict(n=65536, k=32, three_d=True, search=GD_SEARCH_MORTON, v_frag=100.0,
                       sizes=("loguniform", 2.0e-4, 20.0), radial="loguniform", seed=12, x_range=(0.0, 3.8)),
    # a radial-only model in code units with a constant viscosity, radiation pressure, viscous flow and
    # logarithmic output: the settings the other models leave off, so that every branch of the run's
    # parameter file (variables.txt) has a model that writes it
    "v0_radial_units": dict(n=4096, k=16, three_d=False, search=GD_SEARCH_KDTREE, v_frag=100.0,
                            sizes=("loguniform", 2.0e-4, 20.0), radial="loguniform", seed=9, n_x=1,
                            units=dict(const_nu=1, nu=1.0e-5, code_unit=1, reynolds_0=1.0e8),
                            flags=dict(radiation=1, pr_effect=1, visc_flow=1, log_output=1)),
    # radial-polar (no azimuth) with an imported gas density: the last two branches of that file
    "v1_polar_gas": dict(n=4096, k=16, three_d=True, search=GD_SEARCH_KDTREE, v_frag=100.0,
                         sizes=("loguniform", 2.0e-4, 20.0), radial="loguniform", seed=10, n_x=1,
                         flags=dict(importgas=1)),
}


def config(name: str, n: int | None = None, k: int | None = None):
    spec = CONFIGS[name]
    sizes = spec["sizes"]
    smin = sizes[1]
    smax = sizes[1] if sizes[0] == "mono" else sizes[2]
    cfg = _base_config(k or spec["k"], spec["three_d"], spec["search"], spec["v_frag"], smin, smax)
    if "x_range" in spec:
        cfg.x_min, cfg.x_max = spec["x_range"]
    if "n_x" in spec:
        cfg.n_x = spec["n_x"]
    for key, value in spec.get("units", {}).items():
        setattr(cfg, key, value)
    return cfg


# One collision half-operator of a swarm step, in seconds: at the c3/c4 shapes the fastest owner
# expects about two events over it at bath start (its bath-start rate is 0.035 /s; the grain sizes
# span five decades, so a fixed orbital fraction would ask the fastest owners for millions of
# events).  Both benchmark arms use these lengths.
SWARM_HALF_OPERATOR_S = {"c3_learned_3d": 57.0, "c4_production_3d": 57.0}


def swarm_half_operator(name: str) -> float:
    """The half-operator length of a swarm step of workload `name` (0.5/Omega(1 au) where none is
    set)."""
    return SWARM_HALF_OPERATOR_S.get(name, 0.5 * orbital_time())


def run_info(name: str):
    """The model directory's settings outside gd_config (a GdRunInfo): the compile flags
    mod/make_models.py writes for `name` (COLLISION and MULTISIZE; TRANSPORT and DIFFUSION in 3D;
    linear output unless the config asks for others) and the constants those flags bring in.
    variables.txt records them."""
    from ._lib import GdRunInfo

    three_d = CONFIGS[name]["three_d"]
    r = GdRunInfo()
    r.multisize = 1
    r.transport = r.diffusion = int(three_d)
    r.radiation = r.pr_effect = r.visc_flow = r.importgas = r.log_output = 0
    for key, value in CONFIGS[name].get("flags", {}).items():
        setattr(r, key, value)
    r.save_max, r.out_base, r.col_bath_tpb = 10, (10 if r.log_output else 1), 64
    r.metal_z, r.schmidt_x, r.schmidt_r, r.schmidt_z = 1.0e-02, 1.0, 1.0, 1.0
    r.beta_0, r.kappa_0, r.t_beta, r.c_light = 1.0e+01, 1.0, 2.0 * math.pi, 1.0e+04
    r.dt_out, r.dt_max, r.cfl_dyn = 0.5 * orbital_time(), 0.05 * orbital_time(), 0.45
    for key, value in CONFIGS[name].get("run", {}).items():
        setattr(r, key, 2.0 * math.pi * orbital_time() if value == "orbit" else value)
    return r


def _radius_samples(rng, n: int, kind: str) -> np.ndarray:
    if kind == "loguniform":
        return np.exp(rng.uniform(math.log(R_IN_AU), math.log(R_OUT_AU), n))
    # Sigma ~ r^-1 with a x0.1 gap on [9, 11] au and a x5 Gaussian ring at 30 au (width 1 au);
    # equal-mass representatives follow dN/dr ~ r Sigma(r), drawn by inverse CDF on a fine grid
    grid = np.linspace(R_IN_AU, R_OUT_AU, 200_001)
    dens = np.ones_like(grid)
    dens[(grid >= 9.0) & (grid <= 11.0)] *= 0.1
    dens *= 1.0 + 4.0 * np.exp(-0.5 * (grid - 30.0) ** 2)
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (dens[1:] + dens[:-1]) * np.diff(grid))])
    cdf /= cdf[-1]
    return np.interp(rng.uniform(0.0, 1.0, n), cdf, grid)


def particles(name: str, n: int | None = None, seed: int | None = None) -> np.ndarray:
    """Seeded swarm of config `name` as a float64 array [n, 8] in the reference record layout."""
    spec = CONFIGS[name]
    n = int(n or spec["n"])
    rng = np.random.Generator(np.random.PCG64(spec["seed"] if seed is None else seed))
    x_lo, x_hi = spec.get("x_range", (-math.pi, math.pi))
    phi = rng.uniform(0.0, x_hi - x_lo, n)
    r_au = _radius_samples(rng, n, spec["radial"])
    if spec["three_d"]:
        h = 0.05 * r_au ** 0.25
        theta = 0.5 * math.pi + rng.standard_normal(n) * h
    else:
        theta = np.full(n, 0.5 * math.pi)
    sizes = spec["sizes"]
    if sizes[0] == "mono":
        diam = np.full(n, sizes[1])
    else:
        diam = np.exp(rng.uniform(math.log(sizes[1]), math.log(sizes[2]), n))
    grain = math.pi * 1.0 * diam ** 3 / 6.0
    numr = (DUST_MASS / n) / grain
    y = r_au * AU
    R = y * np.sin(theta)
    out = np.empty((n, 8), np.float64)
    out[:, 0] = phi + x_lo  # azimuth in [x_min, x_max)
    out[:, 1] = y
    out[:, 2] = theta
    out[:, 3] = np.sqrt(G_CGS * MSUN * R)  # Keplerian l_phi
    out[:, 4] = 0.0
    out[:, 5] = 0.0
    out[:, 6] = diam
    out[:, 7] = numr
    return out


def c2_batch(swarms: int = 256, seed: int = 5, n_min: int = 1 << 10, n_max: int = 1 << 18):
    """The batched configuration: `swarms` independent 3D swarms with the c0 distributions, sizes
    log-uniform integers on [n_min, n_max], K drawn from {16, 32, 64}, each swarm with its own
    seed.  Returns (cfg, sizes, ks, particles) with particles concatenated swarm by swarm."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = np.floor(np.exp(rng.uniform(math.log(n_min), math.log(n_max + 1), swarms))).astype(np.int64)
    sizes = np.clip(sizes, n_min, n_max)
    ks = rng.choice(np.array([16, 32, 64]), swarms)
    parts = [particles("c0_plain_small", n=int(n), seed=1000 * seed + s) for s, n in enumerate(sizes)]
    cfg = config("c0_plain_small")
    return cfg, [int(v) for v in sizes], [int(v) for v in ks], np.concatenate(parts, axis=0)
