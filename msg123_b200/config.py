"""Seeded synthetic problem generator.

The reference reads its grid, soil parameters, initial head and boundary series
from namelist and binary files (Read_input.f90, Assign_calculation.f90); those
readers are outside this library's path.  This module produces the same arrays
directly, nondimensionalised with the reference's rules:

* len_scal = 10**ceil(log10(max|z|)) (Read_input.f90:1100-1112), held as real(SP);
* lengths are divided by len_scal, alpha and Ss multiplied by it, Ks divided by it,
  all in single precision (Assign_calculation.f90:117,259-260);
* soil parameters are real(SP) (Assign_calculation.f90:19-21);
* pressure head is measured from the cell top, psi = h - cell_top
  (Calc_parameter.f90:45).

Elevations use the bottom of the box as datum.  The named workloads are

* ``box``    : 20x20x50 cells of 0.1 m, homogeneous soil, ponded top (a fixed-head
               layer above the box), free drainage at the bottom, 48 steps of 1800 s.
* ``hetero`` : 256x256x64 cells of 1x1x0.25 m, lognormal Ks from a seeded Gaussian
               random field (exponential covariance), uniform van Genuchten draws,
               hydrostatic start, 20 mm/h rain for 6 h, 96 adaptive steps from 600 s.
* ``large``  : 512x512x96 cells, as ``hetero`` with sigma_lnK = 1.5.
* ``member`` : one ensemble member (random size in [64,160]^2 x [32,48]).
Any workload can be shrunk with ``shape=`` for tests.
"""
from dataclasses import dataclass, field
import math
import numpy as np

F32 = np.float32


@dataclass
class Problem:
    name: str
    nx: int
    ny: int
    nz: int
    sea_top: int
    free_drainage: int
    reta: np.ndarray
    retn: np.ndarray
    resi: np.ndarray
    poro: np.ndarray
    ss: np.ndarray
    ksx: np.ndarray
    ksy: np.ndarray
    ksz: np.ndarray
    cell_top: np.ndarray
    cell_vol: np.ndarray
    dis2face: np.ndarray
    face_area: np.ndarray
    area_r: np.ndarray
    surf_top: np.ndarray
    surf_bott: np.ndarray
    surf_reli: np.ndarray
    surf_parm: np.ndarray
    sea_head: np.ndarray
    head0: np.ndarray
    rech: np.ndarray          # calc_rech per surface cell (volume rate, nondimensional)
    rech_until: float         # seconds; recharge multiplied by rech_after afterwards
    rech_after: float
    nsteps: int
    params: dict = field(default_factory=dict)
    lnk: np.ndarray = None    # ln Ks field (m/s), kept for the learned guess features
    # the unscaled inputs in the units a reference deck holds (deck.write_deck): dx, dy, dz
    # and z_top (m), per-cell float32 alpha (1/m), n, residual and saturated water content,
    # Ss (1/m), Ks x/y/z (m/s), float64 initial heads (m), rain (mm/h) and its duration (h),
    # sea head (m, ponded top)
    phys: dict = None

    @property
    def ncalc(self):
        return self.nx * self.ny * self.nz

    @property
    def ncals(self):
        return self.nx * self.ny


def len_scale(maxabs_z):
    """Read_input.f90:1100-1112 (10**ceil(log10 max|z|)), returned as a float32 value."""
    real_scal = math.log10(maxabs_z)
    ip = int(real_scal)
    ls = 10 ** (ip + 1) if (real_scal - ip) > 0 else 10 ** ip
    return F32(ls)


def default_params(**kw):
    p = dict(
        len_scal=1.0, criteria=1.0e-3, lin_tol=0.0, criteria_rel=0,
        maxout_iter=20, maxinn_iter=10, precon_type=0, ref_quirks=1, precision=0,
        amg_nlevel=10, amg_coarse_max=2000, amg_sweeps=2, amg_lag=0,
        jac_omega=0.67, amg_theta=0.05, smooth_omega=0.67,
        sim_type=0, ini_step=1800.0, inc_fact=1.0, max_step=3600.0, end_time=1.0e30, guess_mode=0, guess_select=1,
        vg_form=0, jv_mode=0,
    )
    p.update(kw)
    return p


def gaussian_field(shape, corr, seed):
    """Zero-mean unit-variance Gaussian random field with (anisotropic) exponential
    covariance exp(-|r/corr|), by spectral synthesis on the periodic grid, with
    shape (nz, ny, nx) and corr = (lz, ly, lx) in cells."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    kz = np.fft.fftfreq(nz) * 2 * np.pi * corr[0]
    ky = np.fft.fftfreq(ny) * 2 * np.pi * corr[1]
    kx = np.fft.rfftfreq(nx) * 2 * np.pi * corr[2]
    k2 = (kz[:, None, None] ** 2) + (ky[None, :, None] ** 2) + (kx[None, None, :] ** 2)
    amp = (1.0 + k2) ** -1.0          # sqrt of the 3D exponential-covariance spectrum (1+k^2)^-2
    noise = rng.standard_normal(shape)
    f = np.fft.irfftn(np.fft.rfftn(noise) * amp, s=shape, axes=(0, 1, 2))
    f -= f.mean()
    f /= f.std()
    return f


def _geometry(nx, ny, nz, dx, dy, dz, ls, extra_top):
    """Uniform box geometry from SP-scaled node coordinates (all DP from SP values)."""
    lsi = F32(1.0) / ls
    ztop_m = nz * dz
    zmax = ztop_m + (dz if extra_top else 0.0)
    # node elevations of the active layers, top first (layer k spans z[k+1]..z[k])
    zn = np.array([(nz - k) * dz for k in range(nz + 1)], dtype=np.float64)
    zs = (zn.astype(F32) * lsi).astype(np.float64)
    dxs = float(F32(dx) * lsi)
    dys = float(F32(dy) * lsi)
    N = nx * ny * nz
    top = np.repeat(zs[:-1], nx * ny)
    bot = np.repeat(zs[1:], nx * ny)
    hz = top - bot
    cell_top = top.copy()
    cell_vol = dxs * dys * hz
    dis = np.empty((6, N))
    area = np.empty((6, N))
    dis[0] = hz * 0.5; dis[5] = hz * 0.5
    dis[1] = dys * 0.5; dis[4] = dys * 0.5
    dis[2] = dxs * 0.5; dis[3] = dxs * 0.5
    area[0] = dxs * dys; area[5] = dxs * dys
    area[1] = dxs * hz; area[4] = dxs * hz
    area[2] = dys * hz; area[3] = dys * hz
    return cell_top, cell_vol, dis.reshape(-1).copy(), area.reshape(-1).copy(), dxs * dys, zmax


def _scaled(v, ls, mode):
    v = np.asarray(v, dtype=F32)
    lsi = F32(1.0) / ls
    if mode == "mul":
        return (v * ls).astype(F32)
    return (v * lsi).astype(F32)


def make_box(shape=(20, 20, 50), d=(0.1, 0.1, 0.1), nsteps=48, **pkw):
    """Homogeneous infiltration box: ponded top (0.05 m), free drainage, psi0 = -10 m."""
    nx, ny, nz = shape
    dx, dy, dz = d
    N = nx * ny * nz
    zmax = nz * dz + dz
    ls = len_scale(zmax)
    cell_top, cell_vol, dis, area, ar, _ = _geometry(nx, ny, nz, dx, dy, dz, ls, True)
    full = lambda v: np.full(N, v, dtype=F32)
    reta = _scaled(full(3.35), ls, "mul")
    ss = _scaled(full(1.0e-5), ls, "mul")
    ks = _scaled(full(9.22e-5), ls, "div")
    lsi = F32(1.0) / ls
    head0 = cell_top + float(F32(-10.0) * lsi)
    top_surface = float(F32(nz * dz) * lsi)
    sea = np.full(nx * ny, float(F32(nz * dz + 0.05) * lsi))
    surf = np.full(nx * ny, top_surface)
    prm = default_params(len_scal=float(ls), criteria=1.0e-8, criteria_rel=1, lin_tol=1.0e-10,
                         maxinn_iter=400, precon_type=0, sim_type=0, ini_step=1800.0, inc_fact=1.0,
                         end_time=1800.0 * nsteps)
    prm.update(pkw)
    phys = dict(dx=dx, dy=dy, dz=dz, z_top=nz * dz, alpha=full(3.35), n=full(2.0), resi=full(0.102),
                ths=full(0.368), ss=full(1.0e-5), ksx=full(9.22e-5), ksy=full(9.22e-5), ksz=full(9.22e-5),
                head0=np.repeat(np.array([(nz - k) * dz for k in range(nz)]), nx * ny) - 10.0,
                rain_mm_h=0.0, rain_hours=0.0, sea_head=nz * dz + 0.05)
    return Problem("box", nx, ny, nz, 1, 1, reta, full(2.0), full(0.102), full(0.368), ss,
                   ks.copy(), ks.copy(), ks.copy(), cell_top, cell_vol, dis, area,
                   np.full(nx * ny, ar), surf, surf.copy(), np.zeros(nx * ny), np.zeros(nx * ny),
                   sea, head0, np.zeros(nx * ny), 1.0e30, 1.0, nsteps, prm, phys=phys)


def make_box1r(shape=(20, 20, 50), nsteps=48, criteria=1.0e-6, **pkw):
    """The box in a form the reference itself can run ("config 1R"): the same ponded sea
    layer on top, but a no-flow bottom (no free drainage), the Eisenstat-Walker linear
    tolerance (lin_tol = 0) and an absolute Newton criterion in metres (criteria_rel = 0),
    i.e. only features the reference's input decks can express."""
    import dataclasses
    p = make_box(shape=shape, nsteps=nsteps)
    prm = dict(p.params, lin_tol=0.0, criteria_rel=0, criteria=criteria)
    prm.update(pkw)
    return dataclasses.replace(p, name="box1r", free_drainage=0, params=prm)


def make_hetero(shape=(256, 256, 64), d=(1.0, 1.0, 0.25), seed=2024, sigma=1.0, corr=(20, 20, 4),
                nsteps=96, wt_depth=None, rain_mm_h=20.0, rain_hours=6.0, **pkw):
    """Heterogeneous block: lnKs GRF, random van Genuchten draws, hydrostatic start."""
    nx, ny, nz = shape
    dx, dy, dz = d
    N = nx * ny * nz
    ls = len_scale(nz * dz)
    cell_top, cell_vol, dis, area, ar, _ = _geometry(nx, ny, nz, dx, dy, dz, ls, False)
    g = gaussian_field((nz, ny, nx), (corr[2], corr[1], corr[0]), seed).reshape(-1)
    lnk = math.log(1.0e-5) + sigma * g
    rng = np.random.default_rng(seed + 1)
    alpha = rng.uniform(1.0, 5.0, N)
    nvg = rng.uniform(1.3, 2.5, N)
    ths = rng.uniform(0.35, 0.45, N)
    reta = _scaled(alpha, ls, "mul")
    ss = _scaled(np.full(N, 1.0e-5), ls, "mul")
    ks = _scaled(np.exp(lnk), ls, "div")
    lsi = F32(1.0) / ls
    if wt_depth is None:                      # 10 m below the top of a 16 m block, scaled with depth
        wt_depth = 0.625 * nz * dz
    hwt = float(F32(nz * dz - wt_depth) * lsi)
    head0 = np.full(N, hwt)
    top_surface = cell_top[: nx * ny].copy()
    rate = float(F32(rain_mm_h * 1.0e-3 / 3600.0) * lsi)
    rech = rate * np.full(nx * ny, ar)
    prm = default_params(len_scal=float(ls), criteria=1.0e-8, criteria_rel=1, lin_tol=0.0,
                         maxinn_iter=100, precon_type=1, ref_quirks=0, amg_coarse_max=128, sim_type=1, ini_step=600.0,
                         max_step=3600.0, end_time=1.0e30)
    prm.update(pkw)
    phys = dict(dx=dx, dy=dy, dz=dz, z_top=nz * dz, alpha=alpha.astype(F32), n=nvg.astype(F32),
                resi=np.full(N, 0.05, dtype=F32), ths=ths.astype(F32), ss=np.full(N, 1.0e-5, dtype=F32),
                ksx=np.exp(lnk).astype(F32), ksy=np.exp(lnk).astype(F32), ksz=np.exp(lnk).astype(F32),
                head0=np.full(N, float(F32(nz * dz - wt_depth))), rain_mm_h=rain_mm_h, rain_hours=rain_hours,
                sea_head=None)
    p = Problem("hetero", nx, ny, nz, 0, 0, reta, nvg.astype(F32), np.full(N, 0.05, dtype=F32),
                ths.astype(F32), ss, ks.copy(), ks.copy(), ks.copy(), cell_top, cell_vol, dis, area,
                np.full(nx * ny, ar), top_surface, top_surface.copy(), np.zeros(nx * ny),
                np.zeros(nx * ny), np.zeros(nx * ny), head0, rech, rain_hours * 3600.0, 0.0,
                nsteps, prm, lnk=lnk.astype(np.float32), phys=phys)
    return p


def member_draw(seed):
    """Shape and lnKs spread of ensemble member `seed` (no fields built):
    nx, ny ~ U{64..160}, nz ~ U{32..48}, sigma_lnK ~ U[0.5, 1.5]."""
    rng = np.random.default_rng(10_000 + seed)
    nx = int(rng.integers(64, 161)); ny = int(rng.integers(64, 161)); nz = int(rng.integers(32, 49))
    sigma = float(rng.uniform(0.5, 1.5))
    return (nx, ny, nz), sigma


def make_member(seed, **pkw):
    """Ensemble member `seed` (member_draw) on the config-2 generator, mixed precision."""
    shape, sigma = member_draw(seed)
    return make_hetero(shape=shape, seed=seed, sigma=sigma, precision=1, **pkw)


def make_config(name, **kw):
    if name == "box":
        return make_box(**kw)
    if name == "box1r":
        return make_box1r(**kw)
    if name == "hetero":
        return make_hetero(**kw)
    if name == "large":
        kw.setdefault("shape", (512, 512, 96))
        kw.setdefault("sigma", 1.5)
        return make_hetero(**kw)
    raise ValueError(f"unknown workload {name!r}")
