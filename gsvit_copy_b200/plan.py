"""Planner: what GSvit's settings/plan layer leaves in SvSet/SvPool, restated.

GSvit turns a parameter file into an SvSet (settings.c) and an SvPool
(init_and_make_plan, plan.c:5442) before the stepping loop starts.  The GPU
driver this package replaces (gpu.c) starts from that state; so does the C
ABI here, through the flat descriptor `fdtd_desc`.  This module builds that
descriptor for the workloads the package is measured and tested on, applying
the planner's own rules, each cited:

  dt                     plan.c:5452
  CPML sigma_opt         settings.c:5151
  material parameters    scan_material, plan.c:3113-3396 (read as float)
  ADE coefficients       calculate_ade_a/bp/c, plan.c:2737-2763
  epsilon/mu scaling     plan.c:4669-4698
  vacuum material 0      plan.c:78-80, plan.c:2418-2422
  sphere voxelisation    plan.c:4376-4387 with is_in_sphere plan.c:2137-2143 (GLfloat)
  voxel box entity       plan.c:4466-4479 (half-open corners)
  VTK index map          load_vtk, plan.c:3877-3958
  TSF generated pulse    write_source, settings.c:443-530
  NFFF spherical area    settings.c:5588-5660
The derived maps (bnds, sourceskip) and all coefficients are computed by the
library itself from this descriptor.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import abi

C0 = 299792458.0
MU0 = 1.256637061435917295e-6
EPS0 = 8.854187817620389850e-12
G_PI = 3.1415926535897932384626433832795028841971693993751


def f32(x: float) -> float:
    """Value after a `fscanf("%f")` into a float, as scan_material reads it."""
    return float(np.float32(x))


def plan_dt(dx: float, dy: float, dz: float, dtmult: float) -> float:
    """plan.c:5452"""
    return 1.0 / C0 / math.sqrt(1.0 / dx / dx + 1.0 / dy / dy + 1.0 / dz / dz) * dtmult


def cpml_sigma_opt(m: int, dx: float) -> float:
    """settings.c:5151 (sigma == -1 in BOUNDARY_* cpml)."""
    return 0.8 * float(m) / (377 * dx)


def _mat(**kw) -> abi.Material:
    m = abi.Material()
    for k, v in kw.items():
        if isinstance(v, (list, tuple)):
            arr = getattr(m, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(m, k, v)
    return m


def vacuum_material() -> abi.Material:
    """mats[0] = mat_vacuum_lintab (plan.c:78-80), scaled by plan.c:4679-4681."""
    return _mat(type=abi.MAT_LINTAB, epsilon=1 * EPS0, mu=1 * MU0, sigma=0.0, sigast=0.0)


def lintab_material(eps_r: float, mu_r: float = 1.0, sigma: float = 0.0, sigast: float = 0.0) -> abi.Material:
    """Type 1 material: scan_material plan.c:3129-3143 (floats), scaling plan.c:4679-4681."""
    return _mat(type=abi.MAT_LINTAB, epsilon=f32(eps_r) * EPS0, mu=f32(mu_r) * MU0,
                sigma=f32(sigma), sigast=f32(sigast))


def pec_material() -> abi.Material:
    """Type 10 material (plan.c:3144-3145); epsilon/mu keep the defaults 1."""
    return _mat(type=abi.MAT_PEC, epsilon=1.0, mu=1.0)


def ade_material(eps_inf: float, sigma: float, omega_p: float, nu: float,
                 poles: Sequence[Sequence[float]], dt: float) -> abi.Material:
    """Type 5 (Drude + two critical points), plan.c:3199-3271.

    poles: two (A, phi, Omega, Gamma) tuples.  Every parameter is rounded to
    float as fscanf("%g") into a float does, then the coefficients follow
    calculate_ade_a / calculate_ade_bp / calculate_ade_c (plan.c:2737-2763)."""
    epsilon, sigma_f, omegap, nu_f = f32(eps_inf), f32(sigma), f32(omega_p), f32(nu)
    m = _mat(type=abi.MAT_ADE, epsilon=epsilon, mu=1.0, sigma=sigma_f, sigast=0.0,
             drude_omega_p=omegap, drude_nu=nu_f)
    # calculate_ade_a, plan.c:2737-2742
    m.ade_a0 = (nu_f * dt - 2) / (nu_f * dt + 2)
    m.ade_a1 = 4 / (nu_f * dt + 2)
    m.ade_a2 = dt * dt * EPS0 * omegap * omegap / (2 * (nu_f * dt + 2))
    for i in range(2):
        a, phi, omega, gamma = (f32(v) for v in poles[i])
        m.cp_a[i], m.cp_phi[i], m.cp_omega[i], m.cp_gamma[i] = a, phi, omega, gamma
        # calculate_ade_bp, plan.c:2745-2752
        den = (omega * omega * dt * dt + (2 + gamma * dt) * (2 + gamma * dt))
        m.ade_bp0[i] = -(omega * omega * dt * dt + (2 - gamma * dt) * (2 - gamma * dt)) / den
        m.ade_bp1[i] = 2 * (4 - (gamma * gamma + omega * omega) * dt * dt) / den
        m.ade_bp2[i] = 2 * EPS0 * a * omega * dt * (omega * dt * math.cos(phi) + (2 - gamma * dt) * math.sin(phi)) / den
        m.ade_bp3[i] = 4 * EPS0 * a * omega * dt * (omega * dt * math.cos(phi) - gamma * dt * math.sin(phi)) / den
        m.ade_bp4[i] = 2 * EPS0 * a * omega * dt * (omega * dt * math.cos(phi) - (2 + gamma * dt) * math.sin(phi)) / den
    # calculate_ade_c, plan.c:2755-2763
    den = (sigma_f * dt / 2 + m.ade_a2 + m.ade_bp4[0] + m.ade_bp4[1] + EPS0 * epsilon)
    m.ade_c0 = dt / den
    m.ade_c1 = 1 / den
    m.ade_c2 = -(m.ade_a2 + m.ade_bp2[0] + m.ade_bp2[1]) / den
    m.ade_c3 = -(sigma_f * dt / 2 + 2 * m.ade_a2 + m.ade_bp3[0] + m.ade_bp3[1] - EPS0 * epsilon) / den
    # plan.c:4690-4693 scales after the coefficients were formed
    m.epsilon = epsilon * EPS0
    m.mu = 1.0 * MU0
    return m


def lorentz_as_cp(eps_s: float, eps_inf: float, omega0: float, delta: float):
    """Single Lorentz pole eps_inf + (eps_s-eps_inf) w0^2/(w0^2 - w^2 - 2 i delta w)
    written as one critical-point term of the type-5 ADE model.

    The CP susceptibility of the ADE scheme is
        chi(w) = A*Omega*[e^{i phi}/(Omega - w - i Gamma) + e^{-i phi}/(Omega + w + i Gamma)]
    (Vial/Chun convention, e^{-i w t}); with phi = 0, Gamma = delta and
    Omega = sqrt(w0^2 - delta^2) this is 2*A*Omega^2/(Omega^2 + Gamma^2 - w^2 - 2 i Gamma w),
    so A = (eps_s - eps_inf) * w0^2 / (2 * Omega^2)."""
    big_omega = math.sqrt(omega0 * omega0 - delta * delta)
    a = (eps_s - eps_inf) * omega0 * omega0 / (2 * big_omega * big_omega)
    return (a, 0.0, big_omega, delta)


def tsf_pulse(nsteps: int, wavelength: float, pulse_width: int, dt: float, amplitude: float) -> np.ndarray:
    """Generated TSF source of type 2 (SRC_PULSE), write_source settings.c:443-530,
    including the %g text round trip of the temporary source file."""
    dampval = 100
    wavefreq = C0 * 2 * G_PI / wavelength
    dpulse = pulse_width * dt
    vals = np.zeros(nsteps)
    for i in range(nsteps):
        v = amplitude * math.sin(wavefreq * dt * float(i))
        if i < dampval:
            v *= (1.0 / float(dampval)) * float(i)
        damp = (float(i) * dt - 4.0 * dpulse) / math.sqrt(2.0) / dpulse
        v *= math.exp(-damp * damp)
        vals[i] = float("%g" % v)
    return vals


def gaussian_pulse(nsteps: int, dt: float, wavelength: float, delay: float, width: float,
                   amplitude: float = 1.0) -> np.ndarray:
    """sin(2 pi c / lambda t) * exp(-((t - delay)/width)^2), t = step*dt; written
    to the waveform file with %.17g so the reference reads the same doubles."""
    t = np.arange(nsteps, dtype=np.float64) * dt
    return amplitude * np.sin(2 * G_PI * C0 / wavelength * t) * np.exp(-((t - delay) / width) ** 2)


def sphere_map(mat: np.ndarray, center, radius, index: int) -> None:
    """Sphere voxelisation without antialiasing, plan.c:4376-4387: cell (i,j,k)
    belongs to the sphere when is_in_sphere(i+0.5f, j+0.5f, k+0.5f) holds in
    GLfloat arithmetic (plan.c:2137-2143)."""
    xres, yres, zres = mat.shape
    c = [np.float32(v) for v in center]
    r = np.float32(radius)
    lo = [int(max(0.0, float(c[a] - r - np.float32(1)))) for a in range(3)]
    hi = [min(float(s), float(c[a] + r + np.float32(1))) for a, s in enumerate((xres, yres, zres))]
    ii = np.arange(lo[0], xres)
    jj = np.arange(lo[1], yres)
    kk = np.arange(lo[2], zres)
    ii = ii[ii < hi[0]]
    jj = jj[jj < hi[1]]
    kk = kk[kk < hi[2]]
    x = (ii.astype(np.float32) + np.float32(0.5))[:, None, None]
    y = (jj.astype(np.float32) + np.float32(0.5))[None, :, None]
    z = (kk.astype(np.float32) + np.float32(0.5))[None, None, :]
    dxv = (x - c[0]) * (x - c[0])
    dyv = (y - c[1]) * (y - c[1])
    dzv = (z - c[2]) * (z - c[2])
    inside = ((dxv + dyv) + dzv) <= (r * r)
    sub = mat[np.ix_(ii, jj, kk)]
    sub[inside] = index
    mat[np.ix_(ii, jj, kk)] = sub


def voxel_box(arr: np.ndarray, p0, p1, value) -> None:
    """Voxel entity: cells i in [p0, p1) on each axis (integer corners)."""
    arr[p0[0]:p1[0], p0[1]:p1[1], p0[2]:p1[2]] = value


def gaussian_height_map(nx: int, ny: int, rms: float, corr_len: float, seed: int) -> np.ndarray:
    """Gaussian-correlated random height map (units of the inputs): seeded white
    noise filtered in Fourier space by a Gaussian of correlation length corr_len,
    rescaled to the requested rms."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((nx, ny))
    kx = np.fft.fftfreq(nx)[:, None]
    ky = np.fft.fftfreq(ny)[None, :]
    filt = np.exp(-(kx * kx + ky * ky) * (math.pi * corr_len) ** 2)
    h = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    h -= h.mean()
    s = h.std()
    return h * (rms / s) if s > 0 else h


def spherical_area(thetares: int, phires: int, radius: int, thetafrom: float, phifrom: float,
                   thetato: float, phito: float, xres: int, yres: int, zres: int):
    """Far points of NFFF_SPHERICAL_AREA, settings.c:5588-5660 (cell units)."""
    pts = []
    for i in range(thetares):
        for j in range(phires):
            th = (thetafrom + float(i) * (thetato - thetafrom) / (thetares - 1)) if thetares > 1 else thetafrom
            ph = (phifrom + float(j) * (phito - phifrom) / (phires - 1)) if phires > 1 else phifrom
            pts.append((int(radius * math.sin(th) * math.cos(ph)) + xres // 2,
                        int(radius * math.sin(th) * math.sin(ph)) + yres // 2,
                        int(radius * math.cos(th)) + zres // 2))
    return np.asarray(pts, dtype=np.int32)


def nfff_istart(points: np.ndarray, dt: float, dx: float, shared: bool) -> np.ndarray:
    """istart of farfield.c:57-102: per point, or the first point's value for a
    whole spherical-area set (individual > 0)."""
    div = C0 * dt / dx
    out = np.zeros(len(points), dtype=np.int32)
    for n, (ri, rj, rk) in enumerate(points):
        v = math.sqrt((ri / div) ** 2 + (rj / div) ** 2 + (rk / div) ** 2) - 500
        out[n] = int(max(0.0, v))
    if shared and len(points):
        out[:] = out[0]
    return out


@dataclass
class Scene:
    """Host-side planned state; `desc()` returns the C descriptor."""
    name: str
    xres: int
    yres: int
    zres: int
    dx: float
    dt: float
    nsteps: int
    matmode: int = abi.MATMODE_FULL
    mats: List[abi.Material] = field(default_factory=list)
    mat: Optional[np.ndarray] = None
    epsilon: Optional[np.ndarray] = None
    sigma: Optional[np.ndarray] = None
    mu: Optional[np.ndarray] = None
    sigast: Optional[np.ndarray] = None
    cpml: Dict[int, tuple] = field(default_factory=dict)      # face -> (depth, m, sigma, kappa, a)
    tsf: Optional[dict] = None
    nfff: Optional[dict] = None
    probes: Optional[np.ndarray] = None
    storage: int = abi.STORE_F32
    design: Optional[dict] = None       # adjoint design region: box=(i0,i1,j0,j1,k0,k1), eps=array of the box
    meta: dict = field(default_factory=dict)

    @property
    def ncells(self) -> int:
        return self.xres * self.yres * self.zres

    def desc(self):
        """Build the ctypes descriptor; returns (desc, keepalive)."""
        keep = []
        d = abi.Desc()
        d.abi_version = abi.ABI_VERSION
        d.xres, d.yres, d.zres = self.xres, self.yres, self.zres
        d.dx = d.dy = d.dz = self.dx
        d.dt = self.dt
        d.nsteps = self.nsteps
        d.matmode = self.matmode
        d.storage = self.storage
        if self.mats:
            arr = (abi.Material * len(self.mats))(*self.mats)
            keep.append(arr)
            d.nmat = len(self.mats)
            d.mats = C.cast(arr, C.POINTER(abi.Material))
        else:
            d.nmat = 0
        for nm, ct in (("mat", C.c_int32), ("epsilon", C.c_float), ("sigma", C.c_float),
                       ("mu", C.c_float), ("sigast", C.c_float)):
            a = getattr(self, nm)
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.int32 if ct is C.c_int32 else np.float32)
                keep.append(a)
                setattr(d, nm, abi.as_ptr(a, ct))
        for f, (depth, m, sigma, kappa, a) in self.cpml.items():
            d.cpml[f].enabled = 1
            d.cpml[f].depth = depth
            d.cpml[f].m = m
            d.cpml[f].sigma = sigma
            d.cpml[f].kappa = kappa
            d.cpml[f].a = a
        if self.tsf:
            t = self.tsf
            d.tsf.enabled = 1
            d.tsf.i0, d.tsf.j0, d.tsf.k0 = t["box"][0]
            d.tsf.in_, d.tsf.jn, d.tsf.kn = t["box"][1]
            for f in range(6):
                d.tsf.skip[f] = int(t.get("skip", [0] * 6)[f])
            d.tsf.skipdepth = t.get("skipdepth", -1)
            d.tsf.theta, d.tsf.phi, d.tsf.psi = t["theta"], t["phi"], t["psi"]
            d.tsf.layered_epsilon = t.get("layered_epsilon", 1.0)
            d.tsf.layered_mu = t.get("layered_mu", 1.0)
            w = np.ascontiguousarray(t["wave"], dtype=np.float64)
            keep.append(w)
            d.tsf.nwave = len(w)
            d.tsf.wave = abi.as_ptr(w, C.c_double)
        if self.nfff:
            f = self.nfff
            d.nfff.enabled = 1
            d.nfff.i0, d.nfff.j0, d.nfff.k0 = f["box"][0]
            d.nfff.in_, d.nfff.jn, d.nfff.kn = f["box"][1]
            for q in range(6):
                d.nfff.skip[q] = 0
            for q, (lo, hi) in f.get("skip", {}).items():
                d.nfff.skip[q] = 1
                d.nfff.skip_lo[q][0], d.nfff.skip_lo[q][1] = lo
                d.nfff.skip_hi[q][0], d.nfff.skip_hi[q][1] = hi
            pts = np.ascontiguousarray(f["points"], dtype=np.int32)
            keep.append(pts)
            d.nfff.npoints = len(pts)
            d.nfff.points = abi.as_ptr(pts, C.c_int32)
            if f.get("istart") is not None:
                ist = np.ascontiguousarray(f["istart"], dtype=np.int32)
                keep.append(ist)
                d.nfff.istart = abi.as_ptr(ist, C.c_int32)
            d.nfff.series = 1 if f.get("series") else 0
            om = np.ascontiguousarray(f.get("omega", np.zeros(0)), dtype=np.float64)
            keep.append(om)
            d.nfff.nfreq = len(om)
            d.nfff.omega = abi.as_ptr(om, C.c_double)
        if self.probes is not None and len(self.probes):
            p = np.ascontiguousarray(self.probes, dtype=np.int32)
            keep.append(p)
            d.nprobes = len(p)
            d.probes = abi.as_ptr(p, C.c_int32)
        if self.design:
            b = self.design["box"]
            e = np.ascontiguousarray(self.design["eps"], dtype=np.float64).reshape(-1)
            keep.append(e)
            d.design.enabled = 1
            d.design.i0, d.design.i1, d.design.j0, d.design.j1, d.design.k0, d.design.k1 = b
            d.design.eps_r = abi.as_ptr(e, C.c_double)
        return d, keep

    def expanded(self) -> "Scene":
        """The same scene with every design cell as a LINTAB material of its
        own (epsilon = eps_r * EPS0 in double precision): the form the
        reference's material table takes, for CPU paths that have no design
        region."""
        if not self.design:
            return self
        import copy
        s = copy.copy(self)
        i0, i1, j0, j1, k0, k1 = self.design["box"]
        eps = np.asarray(self.design["eps"], dtype=np.float64).reshape(i1 - i0, j1 - j0, k1 - k0)
        base = len(self.mats)
        s.mats = list(self.mats) + [_mat(type=abi.MAT_LINTAB, epsilon=float(e) * EPS0, mu=1 * MU0, sigma=0.0, sigast=0.0)
                                    for e in eps.reshape(-1)]
        s.mat = np.array(self.mat, dtype=np.int32, copy=True)
        s.mat[i0:i1, j0:j1, k0:k1] = base + np.arange(eps.size, dtype=np.int32).reshape(eps.shape)
        s.design = None
        return s


def cpml_all(depth: int, m: int, sigma: float, kappa: float, a: float, dx: float) -> Dict[int, tuple]:
    """BOUNDARY_ALL cpml depth m sigma a kappa (settings.c:5137-5162)."""
    s = cpml_sigma_opt(m, dx) if sigma == -1 else sigma
    return {f: (depth, m, s, kappa, a) for f in range(6)}


# ----------------------------------------------------------------- workloads

def sphere_scene(res: int = 100, dx: float = 10e-9, nsteps: int = 1000, radius: float = 20.0,
                 eps_r: float = 2.25, cpml_depth: int = 10, tsf_inset: int = 15,
                 probes=None) -> Scene:
    """Plain FP32 dielectric-sphere scattering: 100^3 cells, dx = 10 nm,
    dt = 0.5 x the 3D Courant limit, 10-cell CPML (m = 3, sigma_opt, kappa 1,
    alpha 0) on all faces, eps_r = 2.25 sphere of radius 20 cells at the centre
    (LINTAB), TSF box inset 15 cells, x-polarised plane wave travelling +z
    (theta = phi = 0, psi = -pi/2 so that gex = +E), 500 nm carrier with a 5 fs
    Gaussian envelope delayed by 15 fs."""
    dt = plan_dt(dx, dx, dx, 0.5)
    s = Scene(name=f"sphere{res}", xres=res, yres=res, zres=res, dx=dx, dt=dt, nsteps=nsteps)
    s.mats = [vacuum_material(), lintab_material(eps_r)]
    s.mat = np.zeros((res, res, res), dtype=np.int32)
    c = res / 2.0
    sphere_map(s.mat, (c, c, c), radius * res / 100.0, 1)
    s.cpml = cpml_all(cpml_depth, 3, -1, 1.0, 0.0, dx)
    lo, hi = tsf_inset, res - tsf_inset
    s.tsf = dict(box=((lo, lo, lo), (hi, hi, hi)), theta=0.0, phi=0.0, psi=-G_PI / 2,
                 wave=gaussian_pulse(max(nsteps, 1) + 1, dt, 500e-9, 15e-15, 5e-15))
    if probes is None:
        h = res // 2
        probes = [(h, h, h + res // 4), (h, h, (res * 12) // 100), ((res * 3) // 10, h, h)]
    s.probes = np.asarray(probes, dtype=np.int32)
    return s


def rough_surface_scene(res: int = 512, zres: Optional[int] = None, dx: float = 5e-9, nsteps: int = 4000,
                        cpml_depth: int = 16, seed: int = 2024, rms: float = 10e-9, corr_len: float = 50e-9,
                        surface_frac: float = 0.5, theta_deg: float = 150.0, wavelength: float = 600e-9,
                        nfff_angles=(91, 181), nfff_wavelengths=(500e-9, 600e-9, 700e-9),
                        dtmult: float = 0.5, tsf_skipdepth: int = 2, tsf_margin: int = 8,
                        nfff_margin: int = 4, yres: Optional[int] = None, material: str = "drude") -> Scene:
    """Rough metal surface: res x yres x zres cells (default 512^3), dx = 5 nm,
    16-cell CPML, the substrate as ADE type 5 below a Gaussian-correlated height
    map (rms 10 nm, correlation 50 nm, seeded FFT-filtered white noise), vacuum
    above; p-polarised TSF plane wave at 30 deg incidence from +z (theta = 150
    deg, phi = 0, psi = 0) with a 600 nm Gaussian pulse; NFFF box between CPML
    and TSF box with far points on a 91 x 181 theta-phi grid and running DFTs at
    500/600/700 nm.  DT_MULT is 0.5 (the value GSvit's dispersive self-tests
    use).  material "drude": silver (eps_inf 3.7, wp 1.38e16 rad/s, gamma
    2.73e13 1/s, no CP poles); "lorentz": one Lorentz pole (eps_s 5, eps_inf 2,
    w0 4e15 rad/s, delta 1e14 1/s) as a critical-point term."""
    xres = res
    yres = yres or res
    zres = zres or res
    dt = plan_dt(dx, dx, dx, dtmult)
    s = Scene(name=f"rough{xres}x{yres}x{zres}", xres=xres, yres=yres, zres=zres, dx=dx, dt=dt, nsteps=nsteps)
    if material == "drude":
        metal = ade_material(3.7, 0.0, 1.38e16, 2.73e13, [(0, 0, 0, 0), (0, 0, 0, 0)], dt)
    elif material == "lorentz":
        metal = ade_material(2.0, 0.0, 0.0, 0.0, [lorentz_as_cp(5.0, 2.0, 4e15, 1e14), (0, 0, 0, 0)], dt)
    else:
        raise ValueError(material)
    s.mats = [vacuum_material(), metal]
    h = gaussian_height_map(xres, yres, rms / dx, corr_len / dx, seed)
    z0 = surface_frac * zres
    surf = z0 + h                                     # in cells
    kk = np.arange(zres, dtype=np.float64)[None, None, :] + 0.5
    s.mat = (kk < surf[:, :, None]).astype(np.int32)  # VTK index map: 1 = metal
    s.cpml = cpml_all(cpml_depth, 3, -1, 1.0, 0.0, dx)
    lo = cpml_depth + tsf_margin
    th = math.radians(theta_deg)
    nw = nsteps + 1
    s.tsf = dict(box=((lo, lo, lo), (xres - lo, yres - lo, zres - lo)), theta=th, phi=0.0, psi=0.0,
                 skip=[0, 0, 0, 0, 1, 0], skipdepth=tsf_skipdepth,
                 wave=gaussian_pulse(nw, dt, wavelength, 3 * 4e-15, 4e-15))
    if nfff_angles:
        nlo = cpml_depth + nfff_margin
        box = ((nlo, nlo, nlo), (xres - nlo, yres - nlo, zres - nlo))
        radius = 10 * max(xres, yres, zres)
        pts = spherical_area(nfff_angles[0], nfff_angles[1], radius, 0.0, 0.0, G_PI / 2, 2 * G_PI,
                             xres, yres, zres)
        s.nfff = dict(box=box, points=pts, istart=nfff_istart(pts, dt, dx, shared=True),
                      omega=np.array([2 * G_PI * C0 / w for w in nfff_wavelengths]))
    s.probes = np.asarray([(xres // 2, yres // 2, min(zres - cpml_depth - 2, int(z0) + 20)),
                           (xres // 2, yres // 2, int(z0) + 2),
                           (xres // 3, yres // 2, int(z0) - 2)], dtype=np.int32)
    s.meta.update(height_map=h, surface_z=z0)
    return s


def batch_scenes(n: int = 48, nsteps: int = 2000, seed: int = 7, sizes_xy=(64, 96, 128, 192), sizes_z=(64, 96, 128),
                 nfff_angles=(10, 19)) -> List[Scene]:
    """Independent rough-surface realisations of uneven size for batched runs:
    x, y drawn from {64, 96, 128, 192} and z from {64, 96, 128}; rms height
    5-20 nm, correlation length 30-100 nm, Drude silver or a single-pole
    Lorentz substrate, incidence 0-60 deg, 8-cell CPML, dx = 5 nm."""
    out = []
    for q, p in enumerate(batch_params(n, seed, sizes_xy, sizes_z)):
        xr, yr, zr = p["shape"]
        s = rough_surface_scene(res=xr, yres=yr, zres=zr, nsteps=nsteps, cpml_depth=8, seed=p["seed"], rms=p["rms"],
                                corr_len=p["corr_len"], theta_deg=p["theta_deg"], tsf_margin=6, material=p["material"],
                                nfff_angles=nfff_angles)
        s.name = f"batch{q}_{xr}x{yr}x{zr}"
        out.append(s)
    return out


def batch_params(n: int = 48, seed: int = 7, sizes_xy=(64, 96, 128, 192), sizes_z=(64, 96, 128)) -> List[dict]:
    """The seeded draws of batch_scenes (shape, surface seed, rms, correlation
    length, incidence, material) without building the scenes."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        xr, yr = int(rng.choice(sizes_xy)), int(rng.choice(sizes_xy))
        zr = int(rng.choice(sizes_z))
        out.append(dict(shape=(xr, yr, zr), seed=int(rng.integers(1 << 30)), rms=float(rng.uniform(5e-9, 20e-9)),
                        corr_len=float(rng.uniform(30e-9, 100e-9)), theta_deg=180.0 - float(rng.uniform(0.0, 60.0)),
                        material="drude" if rng.random() < 0.5 else "lorentz"))
    return out


def shard_instances(cells: Sequence[int], world: int) -> List[List[int]]:
    """Whole instances per rank for a batched run on `world` GPUs (instances
    are independent: no exchange).  Longest processing time first: instances
    by descending cell count (ties by index), each to the rank with the fewest
    cells so far (ties to the lower rank); every rank lists its instances in
    ascending order.  Deterministic, so each rank computes the same split
    without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for q in sorted(range(len(cells)), key=lambda q: (-int(cells[q]), q)):
        r = min(range(world), key=lambda r: (load[r], r))
        out[r].append(q)
        load[r] += int(cells[q])
    return [sorted(o) for o in out]


def selftest_scene(code: str, res: int, nsteps: int) -> Scene:
    """GSvit self-test geometry of make_test (tests.c:93-268) for the TSF +
    CPML + NFFF ids ("31111" electric voxel box with MATMODE_CHECK 1,
    "35011" PEC box): res^3 cells of 1 um, CPML `10 3 -1 0.03 4`, TSF box
    [20, res-20] with theta = phi = pi/2, psi = 0 and the generated pulse
    `2 20e-6 10 5`, NFFF box [16, res-16] and one Ramahi point at res-12."""
    dx = 1e-6
    dt = plan_dt(dx, dx, dx, 1.0)
    s = Scene(name=f"selftest_{res}{code}", xres=res, yres=res, zres=res, dx=dx, dt=dt, nsteps=nsteps)
    p0 = (res // 2 + 10, 30, 30)
    p1 = (res - 30, res - 30, res - 30)
    if code == "31111":       # TEST_MATERIAL_ELECTRIC, matcheck -> ELECTRIC voxel data
        s.matmode = abi.MATMODE_ELECTRIC
        s.epsilon = np.full((res, res, res), np.float32(EPS0), dtype=np.float32)
        s.sigma = np.zeros((res, res, res), dtype=np.float32)
        voxel_box(s.epsilon, p0, p1, np.float32(f32(2.0) * EPS0))
        s.mats = []
    elif code == "35011":     # TEST_MATERIAL_LINTAB_PEC, no matcheck -> FULL
        s.matmode = abi.MATMODE_FULL
        s.mats = [vacuum_material(), pec_material()]
        s.mat = np.zeros((res, res, res), dtype=np.int32)
        voxel_box(s.mat, p0, p1, 1)
    else:
        raise ValueError(code)
    s.cpml = cpml_all(10, 3, -1, 4.0, 0.03, dx)
    s.tsf = dict(box=((20, 20, 20), (res - 20, res - 20, res - 20)), theta=1.57079632679,
                 phi=1.57079632679, psi=0.0, wave=tsf_pulse(nsteps, 20e-6, 10, dt, 5.0))
    pts = np.asarray([(res - 12, res - 12, res - 12)], dtype=np.int32)
    s.nfff = dict(box=((16, 16, 16), (res - 16, res - 16, res - 16)), points=pts,
                  istart=nfff_istart(pts, dt, dx, shared=False), omega=np.zeros(0))
    s.probes = np.zeros((0, 3), dtype=np.int32)
    return s


def small_scene(kind: str, shape=(24, 20, 28), nsteps: int = 40, seed: int = 1) -> Scene:
    """Small mixed scenes for parity tests (odd sizes, every face type)."""
    xr, yr, zr = shape
    dx = 10e-9
    dt = plan_dt(dx, dx, dx, 0.5)
    rng = np.random.default_rng(seed)
    s = Scene(name=f"small_{kind}", xres=xr, yres=yr, zres=zr, dx=dx, dt=dt, nsteps=nsteps)
    s.mats = [vacuum_material(), lintab_material(2.25), lintab_material(4.0, sigma=1e4)]
    s.mat = np.zeros(shape, dtype=np.int32)
    if kind in ("lintab", "full"):
        sphere_map(s.mat, (xr / 2, yr / 2, zr / 2), min(shape) / 4.0, 1)
        s.mat[2:6, 3:9, zr - 9:zr - 4] = 2
    if kind in ("ade", "full"):
        s.mats.append(ade_material(3.7, 0.0, 1.38e16, 2.73e13, [(0.3, -1.2, 3.9e15, 4.5e14), (0.1, 0.5, 2e15, 1e14)], dt))
        idx = len(s.mats) - 1
        hmap = 6 + rng.integers(0, 3, size=(xr, yr))
        for i in range(xr):
            for j in range(yr):
                s.mat[i, j, : hmap[i, j]] = idx
    if kind in ("pec", "full"):
        s.mats.append(pec_material())
        s.mat[xr - 8:xr - 5, 4:8, zr // 2:zr // 2 + 3] = len(s.mats) - 1
    s.cpml = cpml_all(5, 3, -1, 2.0, 0.02, dx)
    s.tsf = dict(box=((7, 7, 9), (xr - 7, yr - 7, zr - 7)), theta=2.4, phi=0.7, psi=0.3,
                 skip=[0, 0, 0, 0, 1, 0] if kind in ("ade", "full") else [0] * 6,
                 skipdepth=1 if kind in ("ade", "full") else -1,
                 wave=gaussian_pulse(nsteps + 1, dt, 20 * dx, 30 * dt, 10 * dt))
    pts = np.asarray([(200, 210, 240), (-150, 40, 260), (30, -180, -220)], dtype=np.int32)
    s.nfff = dict(box=((6, 6, 6), (xr - 6, yr - 6, zr - 6)), points=pts,
                  istart=nfff_istart(pts, dt, dx, shared=False),
                  omega=np.array([2 * G_PI * C0 / 300e-9, 2 * G_PI * C0 / 450e-9]))
    s.probes = np.asarray([(xr // 2, yr // 2, zr // 2), (3, 4, 5), (xr - 2, yr - 3, zr - 2)], dtype=np.int32)
    return s


def cone_objective(scene: Scene, theta_deg: float = 20.0, half_deg: float = 10.0, phi_deg: float = 0.0,
                   nth: int = 9, nph: int = 13, freq: int = 0) -> dict:
    """Far points of a cone of directions within `half_deg` of (theta, phi)
    and their solid-angle weights sin(theta) dtheta dphi, appended to the
    scene's far points; returns the objective {freq, points, weights} (point
    indices into scene.nfff["points"])."""
    f = scene.nfff
    th0, ph0, hw = math.radians(theta_deg), math.radians(phi_deg), math.radians(half_deg)
    ths = np.linspace(max(0.0, th0 - hw), th0 + hw, nth)
    dth = ths[1] - ths[0]
    dphw = hw / max(math.sin(th0), 1e-3)
    phs = np.linspace(ph0 - dphw, ph0 + dphw, nph)
    dph = phs[1] - phs[0]
    n0 = np.array([math.sin(th0) * math.cos(ph0), math.sin(th0) * math.sin(ph0), math.cos(th0)])
    radius = 10 * max(scene.xres, scene.yres, scene.zres)
    pts, w = [], []
    for th in ths:
        for ph in phs:
            n = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
            if math.acos(min(1.0, float(n @ n0))) > hw + 1e-12:
                continue
            pts.append((int(radius * n[0]) + scene.xres // 2, int(radius * n[1]) + scene.yres // 2,
                        int(radius * n[2]) + scene.zres // 2))
            w.append(math.sin(th) * dth * dph)
    old = np.asarray(f["points"], dtype=np.int32).reshape(-1, 3)
    new = np.asarray(pts, dtype=np.int32)
    f["points"] = np.concatenate([old, new]) if len(old) else new
    f["istart"] = nfff_istart(f["points"], scene.dt, scene.dx, shared=False)
    return dict(freq=freq, points=np.arange(len(old), len(old) + len(new), dtype=np.int32),
                weights=np.asarray(w, dtype=np.float64))


def adjoint_scene(shape=(256, 256, 128), dx: float = 10e-9, cpml_depth: int = 12, nsteps: int = 4000,
                  design_shape=(64, 64, 16), seed: int = 5, eps_range=(1.5, 4.0), glass_eps: float = 2.1,
                  glass_cells: int = 20, wavelength: float = 550e-9, margin: int = 4,
                  pulse_delay: float = 15e-15, pulse_width: float = 5e-15, metal_cells: int = 0) -> Scene:
    """Adjoint workload: a design box of per-cell permittivity (seeded uniform
    in eps_range) on a glass slab (eps_r 2.1) inside the TSF box, lit at
    normal incidence (theta = 0, x-polarised) by a 550 nm Gaussian pulse
    (width 5 fs, delay 15 fs by default); NFFF box between the CPML and the TSF box with
    a running DFT at 550 nm.  Default: 256 x 256 x 128 cells of 10 nm, 12-cell
    CPML, 64 x 64 x 16 design cells, 4000 steps, DT_MULT 0.5.  metal_cells > 0
    adds a Drude-silver layer of that many cells at the bottom of the grid
    (inside the z0 CPML and across the x and y slabs): a dispersive problem
    whose adjoint runs through the ADE branch and the CPML inside it."""
    xr, yr, zr = shape
    dt = plan_dt(dx, dx, dx, 0.5)
    s = Scene(name=f"adjoint{xr}x{yr}x{zr}", xres=xr, yres=yr, zres=zr, dx=dx, dt=dt, nsteps=nsteps)
    s.mats = [vacuum_material(), lintab_material(glass_eps)]
    s.mat = np.zeros(shape, dtype=np.int32)
    lo = cpml_depth + margin
    g0 = lo + margin
    gk1 = g0 + glass_cells
    s.mat[g0:xr - g0, g0:yr - g0, g0:gk1] = 1
    if metal_cells > 0:
        s.mats.append(ade_material(3.7, 0.0, 1.38e16, 2.73e13, [(0.0, 0.0, 0.0, 0.0)] * 2, dt))
        s.mat[:, :, :metal_cells] = len(s.mats) - 1
    dxs, dys, dzs = design_shape
    i0, j0 = xr // 2 - dxs // 2, yr // 2 - dys // 2
    box = (i0, i0 + dxs, j0, j0 + dys, gk1, gk1 + dzs)
    if not (i0 > lo and i0 + dxs < xr - lo and j0 > lo and j0 + dys < yr - lo and gk1 + dzs < zr - lo):
        raise ValueError("the design box (and the cells above it) must lie strictly inside the TSF box")
    rng = np.random.default_rng(seed)
    s.design = dict(box=box, eps=rng.uniform(eps_range[0], eps_range[1], size=design_shape))
    s.cpml = cpml_all(cpml_depth, 3, -1, 1.0, 0.0, dx)
    s.tsf = dict(box=((lo, lo, lo), (xr - lo, yr - lo, zr - lo)), theta=0.0, phi=0.0, psi=0.0,
                 skip=[0] * 6, skipdepth=-1,
                 wave=gaussian_pulse(nsteps + 1, dt, wavelength, pulse_delay, pulse_width))
    nlo = cpml_depth + 2
    s.nfff = dict(box=((nlo, nlo, nlo), (xr - nlo, yr - nlo, zr - nlo)), points=np.zeros((0, 3), dtype=np.int32),
                  omega=np.array([2 * G_PI * C0 / wavelength]))
    s.probes = np.asarray([(xr // 2, yr // 2, min(zr - lo - 2, gk1 + dzs + 4))], dtype=np.int32)
    return s

