"""Seeded synthetic inputs with the shapes and value distributions of the benchmark configs.

No public dataset is involved: every config is a synthetic AGN-disk column set built the
way the reference's synthetic disk is (calc_grid, calc_density, calc_temperature in
source/disk.f90:42-129), plus seeded lognormal density perturbations.  All arrays are
float64 in the reference layout (nx, ny, nz) == Fortran (nz, ny, nx).
"""
import math

import numpy as np

Z0, Z1 = -5e15, 5e15
RHO0, H, RHO_FLOOR = 1e-9, 1.496e14, 1e-24
T_MID, SIGMA_T, T_FLOOR = 6.1e4, 2.5e14, 2000.0
FULLY_IONIZED_T = 2e4


def grid(nz, z0=Z0, z1=Z1):
    """calc_grid (disk.f90:48-51): z_i = z0 + (i-1)*dz, dz = (z1-z0)/(nz-1)."""
    dz = (z1 - z0) / (nz - 1)
    return z0 + np.arange(nz, dtype=np.float64) * dz, dz


def log_wavelengths(nw, w0=100.0, w1=1e5):
    """nw log-spaced wavelengths in Angstrom from w0 to w1 (100 A .. 10 um by default)."""
    if nw == 1:
        return np.array([w0])
    return np.logspace(math.log10(w0), math.log10(w1), nw)


def temperature(z, t_mid=T_MID, sigma_t=SIGMA_T, t_floor=T_FLOOR):
    """Gaussian midplane temperature with a floor (calc_temperature semantics with
    isoTemp > midTemp: T = max(midTemp*exp(-z^2/2 sigma^2), floorTemp))."""
    tg = t_mid * np.exp(-0.5 * z * z / (sigma_t * sigma_t))
    return np.where(tg > t_floor, tg, t_floor)


def agn_block(nx, ny, nz, seed=2, rho0=RHO0, sigma_dex=0.3, rho_floor=RHO_FLOOR):
    """Config 'plain FP64 non-grey AGN grid': Gaussian density with a floor times a seeded
    lognormal perturbation of sigma_dex per cell; Gaussian temperature with a 2000 K floor.
    Returns rho, T (nx, ny, nz) and dz."""
    z, dz = grid(nz)
    base = rho0 * np.exp(-0.5 * z * z / (H * H))
    base = np.where(base < rho_floor, rho_floor, base)
    rng = np.random.default_rng(seed)
    pert = 10.0 ** (sigma_dex * rng.standard_normal((nx, ny, nz)))
    rho = base[None, None, :] * pert
    T = np.broadcast_to(temperature(z), (nx, ny, nz)).copy()
    return rho, T, dz


def precision_block(nx, ny, nz, seed=3):
    """Config 'precision form': as agn_block with rho0 drawn log-uniform in [1e-11, 1e-7]."""
    rng = np.random.default_rng(seed)
    rho0 = 10.0 ** rng.uniform(-11.0, -7.0)
    rho, T, dz = agn_block(nx, ny, nz, seed=seed + 1000, rho0=rho0)
    return rho, T, dz, rho0


def grey_isothermal():
    """Config 'plain method, small' == samples/GreyIsothermal: nx=ny=1, nz=10, grey
    sigma=0.4, isothermal 2000 K (isoTemp=midTemp=1 is below the 2000 K floor)."""
    z, dz = grid(10)
    rho = RHO0 * np.exp(-((0.5 * (z * z)) / (H * H)))
    rho = np.where(rho < RHO_FLOOR, RHO_FLOOR, rho)
    T = np.full(10, 2000.0)
    return rho.reshape(1, 1, 10), T.reshape(1, 1, 10), dz


K_CGS, M_U, MU_GAS = 1.380649e-16, 1.66053906660e-24, 0.6


def athena_column(nz, rng, rho0=RHO0, sigma_dex=0.5, t_mid=T_MID, sigma_t=SIGMA_T):
    """One synthetic Athena-style column: density and pressure each Gaussian-stratified times
    a lognormal turbulence of sigma_dex; T = mu m_u p / (rho k) with mu = 0.6 and a 2000 K
    floor (the temperature read_athena.f90 reconstructs from E = p/gamma1 with zero momenta
    and mean_molecular_weight = 0.6).  The pressure scale height combines H and sigma_t so
    that the mean temperature profile is the Gaussian of `temperature`.  Returns rho, T, dz."""
    z, dz = grid(nz)
    g = np.exp(-0.5 * z * z / (H * H))
    rho = np.maximum(rho0 * g, RHO_FLOOR) * 10.0 ** (sigma_dex * rng.standard_normal(nz))
    p0 = rho0 * K_CGS * t_mid / (MU_GAS * M_U)
    pres = p0 * g * np.exp(-0.5 * z * z / (sigma_t * sigma_t)) * 10.0 ** (sigma_dex * rng.standard_normal(nz))
    T = MU_GAS * M_U * pres / (rho * K_CGS)
    T = np.where(T > T_FLOOR, T, T_FLOOR)
    return rho, T, dz


def ragged_batch(ncol=8192, seed=4, nz_range=(64, 2048), nw_range=(32, 1024)):
    """Config 'batching form': ncol independent columns with nz = floor(exp U(ln a, ln b)) and
    nw likewise, each an athena_column; every column's wavelength grid is log_wavelengths(nw),
    one grid per distinct nw.  Returns a dict with per-column nz, nw, dz, wave_off, the packed
    wavelength array, and dense rho, T (concatenated z profiles)."""
    rng = np.random.default_rng(seed)
    nz = np.floor(np.exp(rng.uniform(math.log(nz_range[0]), math.log(nz_range[1]), ncol))).astype(np.int64)
    nw = np.floor(np.exp(rng.uniform(math.log(nw_range[0]), math.log(nw_range[1]), ncol))).astype(np.int64)
    nz = np.clip(nz, nz_range[0], nz_range[1])
    nw = np.clip(nw, nw_range[0], nw_range[1])
    grids, waves, wave_off = {}, [], np.empty(ncol, dtype=np.int64)
    pos = 0
    for i, w in enumerate(nw):
        w = int(w)
        if w not in grids:
            grids[w] = pos
            waves.append(log_wavelengths(w))
            pos += w
        wave_off[i] = grids[w]
    rhos, Ts, dzs = [], [], np.empty(ncol)
    for i in range(ncol):
        r, t, dz = athena_column(int(nz[i]), rng)
        rhos.append(r)
        Ts.append(t)
        dzs[i] = dz
    return {"nz": nz, "nw": nw, "dz": dzs, "wave_off": wave_off, "waves": np.concatenate(waves),
            "rho": np.concatenate(rhos), "T": np.concatenate(Ts)}


SERVING_SIZES = (64, 128, 256, 512)


def serving_stream(n_jobs, rate, seed=5):
    """Config 'serving form': a Poisson stream of n_jobs post-processing jobs at `rate` jobs/s.
    Per job nx = ny drawn from SERVING_SIZES, nz uniform in [128, 1024], nw uniform in
    [64, 512], rho0 log-uniform in [1e-11, 1e-7] (the precision config's construction).
    Returns a list of dicts (arrival_s, nx, ny, nz, nw, rho0, seed)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_jobs))
    jobs = []
    for k in range(n_jobs):
        n = int(rng.choice(SERVING_SIZES))
        jobs.append({"arrival_s": float(t[k] - t[0]), "nx": n, "ny": n, "nz": int(rng.integers(128, 1025)),
                     "nw": int(rng.integers(64, 513)), "rho0": float(10.0 ** rng.uniform(-11.0, -7.0)),
                     "seed": int(rng.integers(1 << 30))})
    return jobs


def job_arrays_device(job, eng, sigma_dex=0.3):
    """rho, T (nx, ny, nz) float64 torch tensors on the engine's device and dz for a
    serving_stream job: the agn_block construction with the job's rho0, generated on the device
    (Engine.disk_inputs_device: the reference's disk model and a Philox-seeded lognormal
    perturbation), so no input crosses PCIe."""
    import torch
    shape = (job["nx"], job["ny"], job["nz"])
    dev = torch.device("cuda", eng.device)
    rho = torch.empty(shape, dtype=torch.float64, device=dev)
    T = torch.empty(shape, dtype=torch.float64, device=dev)
    dz = eng.disk_inputs_device(rho, T, {"rho0": job["rho0"], "sigma_dex": sigma_dex, "seed": job["seed"]})
    return rho, T, dz


def precision_block_device(eng, nx, ny, nz, seed=3):
    """Config 'precision form' generated on the engine's device: rho0 drawn log-uniform in
    [1e-11, 1e-7] as precision_block draws it, the disk and its 0.3 dex lognormal perturbation
    (Philox, keyed by seed + 1000) on the device.  Returns rho, T (torch, (nx, ny, nz)), dz, rho0."""
    import torch
    rng = np.random.default_rng(seed)
    rho0 = 10.0 ** rng.uniform(-11.0, -7.0)
    dev = torch.device("cuda", eng.device)
    rho = torch.empty((nx, ny, nz), dtype=torch.float64, device=dev)
    T = torch.empty((nx, ny, nz), dtype=torch.float64, device=dev)
    dz = eng.disk_inputs_device(rho, T, {"rho0": rho0, "sigma_dex": 0.3, "seed": seed + 1000})
    return rho, T, dz, rho0
