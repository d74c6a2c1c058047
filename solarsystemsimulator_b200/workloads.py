"""Seeded synthetic workloads of the benchmark configurations.

No dataset is involved: every configuration is generated from a seed with
the shapes, sizes and value distributions the configuration states.
"""
from __future__ import annotations

import numpy as np

SEED_STRUCTURE = 20260303   # self-gravitating structure formation


def zeldovich_displacement(ngrid: int, sigma_delta: float, index: float, seed: int):
    """Zel'dovich displacement field psi on an ngrid^3 periodic unit lattice.

    delta_k is a Gaussian random field with P(k) ~ k^index (white noise
    shaped in Fourier space), normalised to rms density contrast
    sigma_delta; psi_k = i k delta_k / k^2 so that delta = -div(psi).
    Returns psi with shape (3, ngrid, ngrid, ngrid)."""
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((ngrid, ngrid, ngrid))
    wk = np.fft.rfftn(white)
    k1 = 2 * np.pi * np.fft.fftfreq(ngrid, d=1.0 / ngrid)
    kr = 2 * np.pi * np.fft.rfftfreq(ngrid, d=1.0 / ngrid)
    kx, ky, kz = np.meshgrid(k1, k1, kr, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = k2 ** (index / 4.0)          # sqrt(P) = k^(index/2) = (k^2)^(index/4)
    amp[0, 0, 0] = 0.0
    dk = wk * amp
    delta = np.fft.irfftn(dk, s=(ngrid,) * 3, axes=(0, 1, 2))
    dk *= sigma_delta / delta.std()
    psi = np.empty((3, ngrid, ngrid, ngrid))
    for c, kc in enumerate((kx, ky, kz)):
        psi[c] = np.fft.irfftn(1j * kc * dk / k2, s=(ngrid,) * 3, axes=(0, 1, 2))
    return psi


def _interp_periodic(field: np.ndarray, q: np.ndarray) -> np.ndarray:
    """Trilinear interpolation of a cell-centred periodic field at q in [0,1)^3."""
    n = field.shape[-1]
    g = q * n - 0.5
    i0 = np.floor(g).astype(np.int64)
    t = g - i0
    out = np.zeros((field.shape[0], len(q)))
    for dx in (0, 1):
        wx = t[:, 0] if dx else 1 - t[:, 0]
        ix = (i0[:, 0] + dx) % n
        for dy in (0, 1):
            wy = t[:, 1] if dy else 1 - t[:, 1]
            iy = (i0[:, 1] + dy) % n
            for dz in (0, 1):
                wz = t[:, 2] if dz else 1 - t[:, 2]
                iz = (i0[:, 2] + dz) % n
                out += field[:, ix, iy, iz] * (wx * wy * wz)
    return out


def structure_formation(n_side: int = 64, n_tracer: int = 524_288, sigma_delta: float = 0.01,
                        index: float = -2.0, seed: int = SEED_STRUCTURE):
    """Self-gravitating structure formation: n_side^3 equal-mass sources in
    the unit cube on a lattice displaced by Zel'dovich displacements from
    P(k) ~ k^index with rms density contrast sigma_delta, cold start (zero
    velocities), plus n_tracer massless tracers drawn uniformly and displaced
    by the same field. Total mass 1.

    Returns dict with pos (n,3), mass (n,), tracer_pos (T,3)."""
    psi = zeldovich_displacement(n_side, sigma_delta, index, seed)
    i = (np.arange(n_side) + 0.5) / n_side
    qx, qy, qz = np.meshgrid(i, i, i, indexing="ij")
    q = np.stack([qx.ravel(), qy.ravel(), qz.ravel()], 1)
    pos = q + np.stack([psi[c].ravel() for c in range(3)], 1)
    rng = np.random.default_rng(seed + 1)
    qt = rng.uniform(0.0, 1.0, (n_tracer, 3))
    tpos = qt + _interp_periodic(psi, qt).T
    n = len(pos)
    return {"pos": pos, "mass": np.full(n, 1.0 / n), "tracer_pos": tpos}


# ------------------------------------------ periodic structure (mesh + MLP)

SEED_PERIODIC = 20260505


def periodic_structure(n_side: int = 128, mesh_n: int = 256, sigma_mesh: float = 0.5, index: float = -2.0,
                       softening: float = 1e-3, seed: int = SEED_PERIODIC, fcc: bool = True):
    """Particle-mesh workload: equal-mass particles (total mass 1, G = 1) in
    the periodic unit box on a lattice displaced by Zel'dovich displacements
    from P(k) ~ k^index normalised to rms density contrast sigma_mesh on the
    n_side^3 lattice (the mesh scale of a mesh twice as fine), wrapped into
    [0, 1); cold start. fcc keeps the lattice sites with i + j + k even (a
    face-centred cubic sublattice, n_side^3 / 2 particles, displaced by the
    same field): n_side = 128 gives the full configuration of 1,048,576
    particles on a 256^3 mesh. fcc = False keeps all n_side^3 sites.

    Returns dict with pos (n,3), vel (n,3), mass (scalar per particle),
    mesh_n, softening."""
    psi = zeldovich_displacement(n_side, sigma_mesh, index, seed)
    g = (np.arange(n_side) + 0.5) / n_side
    qx, qy, qz = np.meshgrid(g, g, g, indexing="ij")
    q = np.stack([qx.ravel(), qy.ravel(), qz.ravel()], 1)
    pos = q + np.stack([psi[c].ravel() for c in range(3)], 1)
    if fcc:
        i, j, k = np.meshgrid(*(np.arange(n_side),) * 3, indexing="ij")
        pos = pos[((i + j + k) % 2 == 0).ravel()]
    pos -= np.floor(pos)
    n = len(pos)
    return {"pos": pos, "vel": np.zeros_like(pos), "mass": 1.0 / n, "mesh_n": mesh_n, "softening": softening}


# ------------------------------------------------ solar system + main belt

SEED_SOLAR_BELT = 20260101
G_AU_DAY = 2.959122e-4            # AU^3 / (Msun day^2) = 4 pi^2 / 365.25^2

# (mass in Msun, semi-major axis in AU) of the eight planets
PLANETS = ((1.6601e-7, 0.3871), (2.4478e-6, 0.7233), (3.0035e-6, 1.0000), (3.2272e-7, 1.5237),
           (9.5479e-4, 5.2034), (2.8589e-4, 9.5371), (4.3662e-5, 19.1913), (5.1514e-5, 30.0690))


def kepler_to_cartesian(a, e, inc, Omega, omega, M, mu):
    """Positions and velocities (3, n) of Keplerian orbits (elliptic),
    eccentric anomaly by Newton iteration."""
    E = M.copy()
    for _ in range(50):
        E = E - (E - e * np.sin(E) - M) / (1 - e * np.cos(E))
    cE, sE = np.cos(E), np.sin(E)
    r = a * (1 - e * cE)
    xp = a * (cE - e)
    yp = a * np.sqrt(1 - e * e) * sE
    n_mean = np.sqrt(mu / a ** 3)
    vxp = -a * n_mean * sE / (1 - e * cE)
    vyp = a * n_mean * np.sqrt(1 - e * e) * cE / (1 - e * cE)
    cO, sO, co, so, ci, si = np.cos(Omega), np.sin(Omega), np.cos(omega), np.sin(omega), np.cos(inc), np.sin(inc)
    R11 = cO * co - sO * so * ci; R12 = -cO * so - sO * co * ci
    R21 = sO * co + cO * so * ci; R22 = -sO * so + cO * co * ci
    R31 = so * si; R32 = co * si
    pos = np.stack([R11 * xp + R12 * yp, R21 * xp + R22 * yp, R31 * xp + R32 * yp])
    vel = np.stack([R11 * vxp + R12 * vyp, R21 * vxp + R22 * vyp, R31 * vxp + R32 * vyp])
    return pos, vel


def solar_system_belt(n_ast: int = 2000, seed: int = SEED_SOLAR_BELT):
    """Sun + 8 planets on circular coplanar orbits (real masses and semi-major
    axes) + n_ast massless asteroids with a ~ U[2.1, 3.3] AU, e ~ U[0, 0.15],
    i ~ U[0, 10 deg], Omega, omega, M ~ U[0, 2 pi). Units AU, day, Msun.
    Returns dict with pos (3, n), vel (3, n), mass, is_ast (n = 9 + n_ast)."""
    rng = np.random.default_rng(seed)
    G = G_AU_DAY
    n = 9 + n_ast
    pos = np.zeros((3, n)); vel = np.zeros((3, n)); mass = np.zeros(n)
    mass[0] = 1.0
    for k, (m, a) in enumerate(PLANETS, start=1):
        th = rng.uniform(0, 2 * np.pi)
        v = np.sqrt(G * (1.0 + m) / a)
        pos[:, k] = (a * np.cos(th), a * np.sin(th), 0.0)
        vel[:, k] = (-v * np.sin(th), v * np.cos(th), 0.0)
        mass[k] = m
    a = rng.uniform(2.1, 3.3, n_ast)
    e = rng.uniform(0.0, 0.15, n_ast)
    inc = rng.uniform(0.0, np.deg2rad(10.0), n_ast)
    Om, om, M = (rng.uniform(0, 2 * np.pi, n_ast) for _ in range(3))
    p, v = kepler_to_cartesian(a, e, inc, Om, om, M, G)
    pos[:, 9:], vel[:, 9:] = p, v
    # the sun at rest in the barycentre of the planets
    ptot = (mass[None, 1:9] * vel[:, 1:9]).sum(1)
    vel[:, 0] = -ptot / mass[0]
    is_ast = np.zeros(n, np.uint8); is_ast[9:] = 1
    return {"pos": pos, "vel": vel, "mass": mass, "is_ast": is_ast, "G": G}


# ------------------------------------------------ asteroid clouds

SEED_CLOUDS = 20260404


def asteroid_clouds(n_per_cloud: int = 40_000, n_clouds: int = 5, seed: int = SEED_CLOUDS):
    """A 1 Msun star, 7 planets (m ~ log-U[1e-6, 1e-3] at 0.4-30 AU) and
    n_clouds Gaussian asteroid clouds (sigma 0.01 AU about random centres at
    1-5 AU, local circular velocity + N(0, 1e-4) AU/day), radii log-U[1e-7,
    1e-5] AU, density 2 g/cm^3. Units AU, day, Msun. 3-D (clouds thin in z)."""
    rng = np.random.default_rng(seed)
    G = G_AU_DAY
    n_ast = n_per_cloud * n_clouds
    n = 8 + n_ast
    pos = np.zeros((3, n)); vel = np.zeros((3, n)); mass = np.zeros(n)
    mass[0] = 1.0
    for k in range(1, 8):
        a = 10 ** rng.uniform(np.log10(0.4), np.log10(30.0))
        m = 10 ** rng.uniform(-6, -3)
        th = rng.uniform(0, 2 * np.pi)
        v = np.sqrt(G * (1.0 + m) / a)
        pos[:, k] = (a * np.cos(th), a * np.sin(th), 0.0)
        vel[:, k] = (-v * np.sin(th), v * np.cos(th), 0.0)
        mass[k] = m
    i0 = 8
    for c in range(n_clouds):
        rc = rng.uniform(1.0, 5.0)
        th = rng.uniform(0, 2 * np.pi)
        cen = np.array([rc * np.cos(th), rc * np.sin(th), 0.0])
        p = cen[:, None] + rng.normal(0, 0.01, (3, n_per_cloud))
        r = np.hypot(p[0], p[1])
        v = np.sqrt(G / r)
        vel[0, i0:i0 + n_per_cloud] = -v * p[1] / r + rng.normal(0, 1e-4, n_per_cloud)
        vel[1, i0:i0 + n_per_cloud] = v * p[0] / r + rng.normal(0, 1e-4, n_per_cloud)
        vel[2, i0:i0 + n_per_cloud] = rng.normal(0, 1e-4, n_per_cloud)
        pos[:, i0:i0 + n_per_cloud] = p
        i0 += n_per_cloud
    rad = 10 ** rng.uniform(-7, -5, n_ast)
    au_cm = 1.495978707e13
    msun_g = 1.98847e33
    mass[8:] = (4.0 / 3.0) * np.pi * (rad * au_cm) ** 3 * 2.0 / msun_g
    radius = np.zeros(n); radius[8:] = rad
    is_ast = np.zeros(n, np.uint8); is_ast[8:] = 1
    return {"pos": pos, "vel": vel, "mass": mass, "radius": radius, "is_ast": is_ast, "G": G}


# ------------------------------------------------ batched small systems

SEED_ENSEMBLE = 20260202
FIGURE8_PERIOD = 6.32591398    # period of the figure-8 choreography (G = m = 1)


def figure8(rng=None, noise: float = 0.0):
    """The Chenciner-Montgomery figure-8 initial conditions of the reference
    (index.html:2464-2490, G = m = 1, unscaled), optionally with N(0, noise)
    velocity perturbations. Returns pos (3, 3), vel (3, 3), mass (3,)."""
    px, py = 0.97000436, 0.24308753
    vx, vy = 0.4662036850, 0.4323657300
    pos = np.array([[-px, px, 0.0], [py, -py, 0.0], [0.0, 0.0, 0.0]])
    vel = np.array([[vx, vx, -2 * vx], [vy, vy, -2 * vy], [0.0, 0.0, 0.0]])
    if noise and rng is not None:
        vel[:2] += rng.normal(0, noise, (2, 3))
    return pos, vel, np.ones(3)


def batched_ensemble(n_systems: int = 4096, n_figure8: int = 512, seed: int = SEED_ENSEMBLE):
    """Independent systems: n_figure8 perturbed figure-8 choreographies (G = 1,
    velocity noise N(0, 1e-3)) and planetary systems of 3-64 bodies (body
    count log-uniform): a 1 Msun star + planets with a ~ log-U[0.05, 30] AU,
    m ~ log-U[1e-7, 1e-3] Msun, e ~ U[0, 0.1], i ~ U[0, 5 deg], random angles
    (G = 4 pi^2, AU/yr). dt = 1e-3 of each system's innermost period.
    Returns a list of dicts (pos (3, n), vel (3, n), mass, G, dt)."""
    rng = np.random.default_rng(seed)
    systems = []
    G_au = 4 * np.pi ** 2
    for s in range(n_systems):
        if s < n_figure8:
            pos, vel, m = figure8(rng, 1e-3)
            systems.append({"pos": pos, "vel": vel, "mass": m, "G": 1.0, "dt": 1e-3 * FIGURE8_PERIOD})
            continue
        n = int(np.round(np.exp(rng.uniform(np.log(3), np.log(64)))))
        n = min(max(n, 3), 64)
        k = n - 1
        a = np.sort(np.exp(rng.uniform(np.log(0.05), np.log(30.0), k)))
        m = np.exp(rng.uniform(np.log(1e-7), np.log(1e-3), k))
        e = rng.uniform(0, 0.1, k)
        inc = rng.uniform(0, np.deg2rad(5.0), k)
        Om, om, M = (rng.uniform(0, 2 * np.pi, k) for _ in range(3))
        p, v = kepler_to_cartesian(a, e, inc, Om, om, M, G_au * (1.0 + m))
        pos = np.concatenate([np.zeros((3, 1)), p], 1)
        vel = np.concatenate([np.zeros((3, 1)), v], 1)
        mass = np.concatenate([[1.0], m])
        vel -= (mass[None] * vel).sum(1, keepdims=True) / mass.sum()
        pos -= (mass[None] * pos).sum(1, keepdims=True) / mass.sum()
        p_in = 2 * np.pi * np.sqrt(a[0] ** 3 / (G_au * (1.0 + m[0])))
        systems.append({"pos": pos, "vel": vel, "mass": mass, "G": G_au, "dt": 1e-3 * p_in})
    return systems
