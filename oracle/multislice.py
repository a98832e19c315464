"""CPU restatement of the reference's plain multislice numerics (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, and only as the
checker. It restates, in numpy, the reference's algorithm for:
  * the spline tables              Atomic_Data::get_atom_coef       src/atomic_data.hpp:1303-1486, 1547-1668
  * the projected-potential splat  eval_cubic_poly / get_bn         src/cpu_fcns.hpp:234-262,1670-1684
  * the transmission function      functor::transmission_function   src/cgpu_fcns.cuh:3072-3086
  * the Fresnel propagator         Propagator::operator()           src/propagator.cuh:34-69
  * the convergent probe           Incident_Wave + exp_i_chi        src/incident_wave.cuh:54-72,
                                                                     src/cgpu_fcns.cuh:1951-1992
  * annular detector sums          sum_square_over_Det              src/cgpu_fcns.cuh:1796-1806
  * the slice loop                 Wave_Function::psi               src/wave_function.cuh:230-252
It runs in float64 (the "FP64 oracle"); `dtype=np.float32` runs the same steps in float32. The
specimen (displaced atoms, slices, thicknesses) is an input: the product's host logic produces it
and is pinned separately against the reference's own dumps.

Parity pinning: tests/golden/ holds outputs of the reference itself (oracle/_ref, the reference's
Multislice<T, e_host> compiled from its sources) for small seeded cases; tests check this module
against them.
"""
from __future__ import annotations

import math

import numpy as np

from oracle import atomic_params

C_POTF = 47.877645145863056
C_PI = 3.141592653589793238463
C_PI2 = 9.869604401089358618834
C_2PI = 6.283185307179586476925
C_HALFPI = 1.570796326794896619231


# ---------------------------------------------------------------------------------------------
# Bessel K0, K1: Abramowitz & Stegun 9.8.1-9.8.8 polynomial approximations (as src/math.cuh:465-630)

np.seterr(over="ignore")  # both branches of np.where are evaluated; the unused one may overflow


def _i0(x):
    ax = np.abs(x)
    y = (x / 3.75) ** 2
    small = 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 + y * (0.360768e-1 + y * 0.45813e-2)))))
    yl = 3.75 / np.maximum(ax, 1e-300)
    large = (np.exp(ax) / np.sqrt(np.maximum(ax, 1e-300))) * (0.39894228 + yl * (0.1328592e-1 + yl * (0.225319e-2 + yl * (
        -0.157565e-2 + yl * (0.916281e-2 + yl * (-0.2057706e-1 + yl * (0.2635537e-1 + yl * (-0.1647633e-1 + yl * 0.392377e-2))))))))
    return np.where(ax < 3.75, small, large)


def _i1(x):
    ax = np.abs(x)
    y = (x / 3.75) ** 2
    small = ax * (0.5 + y * (0.87890594 + y * (0.51498869 + y * (0.15084934 + y * (0.2658733e-1 + y * (0.301532e-2 + y * 0.32411e-3))))))
    yl = 3.75 / np.maximum(ax, 1e-300)
    t = 0.2282967e-1 + yl * (-0.2895312e-1 + yl * (0.1787654e-1 - yl * 0.420059e-2))
    t = 0.39894228 + yl * (-0.3988024e-1 + yl * (-0.362018e-2 + yl * (0.163801e-2 + yl * (-0.1031555e-1 + yl * t))))
    large = t * np.exp(ax) / np.sqrt(np.maximum(ax, 1e-300))
    r = np.where(ax < 3.75, small, large)
    return np.where(x < 0, -r, r)


def bessel_k0(x):
    y = x * x / 4.0
    small = (-np.log(x / 2.0) * _i0(x)) + (-0.57721566 + y * (0.42278420 + y * (0.23069756 + y * (0.3488590e-1 + y * (0.262698e-2 + y * (0.10750e-3 + y * 0.74e-5))))))
    yl = 2.0 / x
    large = (np.exp(-x) / np.sqrt(x)) * (1.25331414 + yl * (-0.7832358e-1 + yl * (0.2189568e-1 + yl * (-0.1062446e-1 + yl * (0.587872e-2 + yl * (-0.251540e-2 + yl * 0.53208e-3))))))
    return np.where(x <= 2.0, small, large)


def bessel_k1(x):
    y = x * x / 4.0
    small = (np.log(x / 2.0) * _i1(x)) + (1.0 / x) * (1.0 + y * (0.15443144 + y * (-0.67278579 + y * (-0.18156897 + y * (-0.1919402e-1 + y * (-0.110404e-2 + y * (-0.4686e-4)))))))
    yl = 2.0 / x
    large = (np.exp(-x) / np.sqrt(x)) * (1.25331414 + yl * (0.23498619 + yl * (-0.3655620e-1 + yl * (0.1504268e-1 + yl * (-0.780353e-2 + yl * (0.325614e-2 + yl * (-0.68245e-3)))))))
    return np.where(x <= 2.0, small, large)


# ---------------------------------------------------------------------------------------------
# Spline tables (src/atomic_data.hpp:1303-1486, 1547-1668)

def lobato_coef(Z):
    cl = np.array(atomic_params.LOBATO_CL[Z - 1], dtype=np.float64)
    cnl = np.array(atomic_params.LOBATO_CNL[Z - 1], dtype=np.float64)
    cnl = np.where(np.abs(cl) <= 1e-13, 0.0, cnl)
    nz = ~((np.abs(cl) <= 1e-13) | (np.abs(cnl) <= 1e-13))
    safe = np.where(nz, cnl, 1.0)
    Vr_cl = np.where(nz, C_POTF * C_PI2 * cl / safe ** 1.5, 0.0)
    Vr_cnl = np.where(nz, C_2PI / np.sqrt(safe), 1.0)
    VR_cl = np.where(nz, 2.0 * C_POTF * C_PI2 * cl / safe ** 1.5, 0.0)
    return Vr_cl, Vr_cnl, VR_cl, Vr_cnl.copy()


def vr_lobato(x, cl, cnl):
    return sum(cl[i] * math.exp(-cnl[i] * x) / x * (2.0 / cnl[i] + x) for i in range(5))


def _gauss_range(pt):
    """Gaussian terms [g0, g1) of potential_type 1-4 (Kirkland's first three terms are Yukawa)."""
    return (3, 6) if pt == 4 else (0, 4 if pt == 1 else 5)


def feg_coef(Z, pt):
    """Vr and VR coefficients of potential_type 1-4: set_Doyle_Peng_neutral_coef and
    set_Kirkland_neutral_coef (src/atomic_data.hpp:1303-1400); unused terms are (0, 1)."""
    Vr_cl, VR_cl = np.zeros(6), np.zeros(6)
    cnl_out = np.ones(6)
    g0, g1 = _gauss_range(pt)
    for j in range(g1):
        cl = atomic_params.FEG_CL[pt - 1][Z - 1][j]
        cnl = 0.0 if abs(cl) <= 1e-13 else atomic_params.FEG_CNL[pt - 1][Z - 1][j] / (1.0 if pt == 4 else 4.0)
        if abs(cl) <= 1e-13 or abs(cnl) <= 1e-13:
            continue
        if j < g0:  # Yukawa
            Vr_cl[j], VR_cl[j], cnl_out[j] = C_POTF * C_PI * cl, C_POTF * C_2PI * cl, C_2PI * math.sqrt(cnl)
        else:
            Vr_cl[j] = C_POTF * cl * (C_PI / cnl) ** 1.5
            VR_cl[j] = C_POTF * C_PI * cl / cnl
            cnl_out[j] = C_PI2 / cnl
    return Vr_cl, cnl_out, VR_cl, cnl_out.copy()


C_2PI2A0 = 10.445539456905012  # 2 pi^2 a0


def ion_coef(Z, q):
    """Vr/VR coefficients of element Z with ionic charge q from Peng's ionic table
    (set_Peng_ions_coef, src/atomic_data.hpp:1489-1543), or None when the table has no entry (the
    atom then uses the neutral coefficients, Atom_Type::charge_to_idx src/types.cuh:4125-4137)."""
    if q == 0:
        return None
    e = atomic_params.PENG_ION.get((Z, 2 * q if q > 0 else -2 * q - 1))
    if e is None or abs(e[0][0]) <= 1e-13 or abs(e[1][0]) <= 1e-13:
        return None
    Vr_cl, VR_cl, cnl_out = np.zeros(6), np.zeros(6), np.ones(6)
    for j in range(5):
        cl = e[0][j]
        cnl = 0.0 if abs(cl) <= 1e-13 else e[1][j] / 4.0
        if abs(cl) <= 1e-13 or abs(cnl) <= 1e-13:
            continue
        Vr_cl[j] = C_POTF * cl * (C_PI / cnl) ** 1.5
        VR_cl[j] = C_POTF * C_PI * cl / cnl
        cnl_out[j] = C_PI2 / cnl
    cl, cnl = q / C_2PI2A0, (C_2PI * 2.0) ** -2
    Vr_cl[5], VR_cl[5], cnl_out[5] = C_POTF * C_PI * cl, C_POTF * C_2PI * cl, C_2PI * math.sqrt(cnl)
    return Vr_cl, cnl_out, VR_cl, cnl_out.copy()


def vr_feg(x, cl, cnl, pt):
    """Vr of potential_type 1-4 (Vr_Doyle/Peng/Kirkland_neutral_*, src/cgpu_fcns.cuh:1023-1070)."""
    g0, g1 = _gauss_range(pt)
    y = sum(cl[i] * math.exp(-cnl[i] * x) / x for i in range(g0))
    return y + sum(cl[i] * math.exp(-cnl[i] * (x * x)) for i in range(g0, g1))


def vr_dvr_projected(R, VR_cl, VR_cnl, pt):
    """VR(R) and dVR/dR (VR_dVR_*_neutral_*, src/cgpu_fcns.cuh:1162-1268)."""
    y = np.zeros_like(R)
    dy = np.zeros_like(R)
    if pt == "ion":
        for i in range(5):
            yt = VR_cl[i] * np.exp(-VR_cnl[i] * (R * R))
            y += yt
            dy += -2 * VR_cnl[i] * R * yt
        y += VR_cl[5] * bessel_k0(VR_cnl[5] * R)
        dy += -VR_cl[5] * VR_cnl[5] * bessel_k1(VR_cnl[5] * R)
        return y, dy
    if pt == 6:
        for i in range(5):
            k0 = bessel_k0(VR_cnl[i] * R)
            k1 = bessel_k1(VR_cnl[i] * R)
            y += VR_cl[i] * (2 * k0 / VR_cnl[i] + R * k1)
            dy += -VR_cl[i] * (VR_cnl[i] * R * k0 + 2 * k1)
        return y, dy
    g0, g1 = _gauss_range(pt)
    for i in range(g0):
        y += VR_cl[i] * bessel_k0(VR_cnl[i] * R)
        dy += -VR_cl[i] * VR_cnl[i] * bessel_k1(VR_cnl[i] * R)
    for i in range(g0, g1):
        yt = VR_cl[i] * np.exp(-VR_cnl[i] * (R * R))
        y += yt
        dy += -2 * VR_cnl[i] * R * yt
    return y, dy


def atom_table(Z, dR_min, Vrl=np.float32(0.015), nR=128, potential_type=6, charge=0):
    """Spline table of element Z (ionic charge `charge`): dict with R_min, R_max, R_tap, tap_cf
    (float64) and R2, c0..c3. An ion's R_min .. tap_cf are its neutral element's
    (src/atomic_data.hpp:1612)."""
    ion = ion_coef(Z, charge)
    if ion is not None:
        t = atom_table(Z, dR_min, Vrl, nR, potential_type)
        return _table_body(t["R_min"], t["R_max"], t["R_tap"], t["tap_cf"], nR, ion[2], ion[3], "ion")
    pt = potential_type
    if pt == 6:
        Vr_cl, Vr_cnl, VR_cl, VR_cnl = lobato_coef(Z)
        vr = lambda x: vr_lobato(x, Vr_cl, Vr_cnl)  # noqa: E731
    else:
        Vr_cl, Vr_cnl, VR_cl, VR_cnl = feg_coef(Z, pt)
        vr = lambda x: vr_feg(x, Vr_cl, Vr_cnl, pt)  # noqa: E731
    A = atomic_params.MASS_NUMBER[Z - 1]
    rn_c = 1.2e-05 * A ** (1.0 / 3.0)
    Vrl = float(Vrl)
    R_min = max(rn_c, float(dR_min))
    R_max = 0.0
    if abs(Vrl) > 1e-13 and abs(Vr_cl[0]) > 1e-13:
        x0, xe = rn_c, 25.0
        fxe = vr(xe) - Vrl
        it = 0
        while True:
            x = 0.5 * (x0 + xe)
            fx = vr(x) - Vrl
            if fx * fxe < 0:
                x0 = x
            else:
                xe, fxe = x, fx
            it += 1
            if not (abs(fx) > 1e-8 and it < 200):
                break
        R_max = x
    R_max = max(R_max, 2.0 * R_min)
    if abs(R_max) <= 1e-13:
        R_max = 1.75 * atomic_params.ATOMIC_RADIUS[Z - 1]
    R_tap = R_min + 0.85 * (R_max - R_min)
    tap_cf = C_HALFPI / (R_max ** 2 - R_tap ** 2)
    return _table_body(R_min, R_max, R_tap, tap_cf, nR, VR_cl, VR_cnl, pt)


def _table_body(R_min, R_max, R_tap, tap_cf, nR, VR_cl, VR_cnl, pt):
    """Knots, tapered VR / dVR and the cubic coefficients (src/atomic_data.hpp:1620-1663)."""
    dlnr = math.log(R_max / R_min) / (nR - 1)
    R = R_min * np.exp(np.arange(nR) * dlnr)
    R2 = R ** 2
    y, dy = vr_dvr_projected(R, VR_cl, VR_cnl, pt)
    dy = 0.5 * dy / R
    x_tap = R_tap ** 2
    t = x_tap < R2
    s, co = np.sin(tap_cf * (R2 - x_tap)), np.cos(tap_cf * (R2 - x_tap))
    dy = np.where(t, dy * co - tap_cf * y * s, dy)
    y = np.where(t, y * co, y)
    idR = 1.0 / (R2[1:] - R2[:-1])
    m = (y[1:] - y[:-1]) * idR
    n = dy[:-1] + dy[1:]
    c2 = np.zeros(nR)
    c3 = np.zeros(nR)
    c2[:-1] = (3.0 * m - n - dy[:-1]) * idR
    c3[:-1] = (n - 2.0 * m) * idR * idR
    return {"R_min": R_min, "R_max": R_max, "R_tap": R_tap, "tap_cf": tap_cf, "R2": R2, "c0": y, "c1": dy,
            "c2": c2, "c3": c3}


# ---------------------------------------------------------------------------------------------
# Physical constants in the reference's float precision (src/cgpu_fcns.cuh:50-145)

def wavelength(E_0, dtype=np.float32):
    E = dtype(E_0)
    return dtype(12.3984244) / np.sqrt(E * (2 * dtype(510.99906) + E))


def vr_factor(E_0, dtype=np.float32):
    E = dtype(E_0)
    gamma = 1 + E / dtype(510.99906)
    return gamma * wavelength(E_0, dtype) / (dtype(47.877645145863056) * np.cos(dtype(0)))


# ---------------------------------------------------------------------------------------------
# Grid helpers (Grid_2d, src/types.cuh:2107-2655)

class Grid:
    def __init__(self, nx, ny, lx, ly, dtype=np.float64):
        self.nx, self.ny = nx, ny
        self.nxh, self.nyh = nx // 2, ny // 2
        f = np.float32
        self.lx, self.ly = f(lx), f(ly)
        self.dRx, self.dRy = f(lx) / f(nx), f(ly) / f(ny)
        self.dgx, self.dgy = f(1) / f(lx), f(1) / f(ly)
        self.dtype = dtype

    def g_shift(self):
        ix = np.arange(self.nx)
        iy = np.arange(self.ny)
        gx = np.where(ix < self.nxh, ix, ix - self.nx).astype(np.float32) * self.dgx
        gy = np.where(iy < self.nyh, iy, iy - self.ny).astype(np.float32) * self.dgy
        return gx.astype(np.float32), gy.astype(np.float32)

    def g2_shift(self):
        gx, gy = self.g_shift()
        return (gx[:, None] * gx[:, None]).astype(np.float32) + (gy[None, :] * gy[None, :]).astype(np.float32)

    def g_max(self):
        return min(np.float32(self.nxh) * self.dgx, np.float32(self.nyh) * self.dgy)


# ---------------------------------------------------------------------------------------------
# Projected potential of one slice (stored, fft-shifted layout [ix, iy])

def projected_potential(grid: Grid, atoms_xy, atoms_Z, atoms_occ, tables, dtype=np.float64):
    """V[ix, iy] = sum_atoms occ * spline(R^2) over each footprint (get_bn, periodic) at
    ind_col_pbc_shift (src/cpu_fcns.hpp:234-262)."""
    nx, ny = grid.nx, grid.ny
    V = np.zeros((nx, ny), dtype=dtype)
    for (x, y), Z, occ in zip(atoms_xy, atoms_Z, atoms_occ):
        t = tables[int(Z)]
        Rm = np.float32(t["R_max"])
        x, y = np.float32(x), np.float32(y)
        ix0 = int(np.floor(np.float32(x - Rm) / grid.dRx))
        ixe = int(np.ceil(np.float32(x + Rm) / grid.dRx))
        iy0 = int(np.floor(np.float32(y - Rm) / grid.dRy))
        iye = int(np.ceil(np.float32(y + Rm) / grid.dRy))
        nxa = 0 if ix0 == ixe else ixe - ix0 + 1
        nya = 0 if iy0 == iye else iye - iy0 + 1
        if nxa == 0 or nya == 0:
            continue
        ix = np.arange(ix0, ix0 + nxa)
        iy = np.arange(iy0, iy0 + nya)
        if dtype == np.float32:
            Rx = (ix.astype(np.float32) * grid.dRx - x).astype(np.float32)
            Ry = (iy.astype(np.float32) * grid.dRy - y).astype(np.float32)
            R2 = (Rx[:, None] * Rx[:, None]).astype(np.float32) + (Ry[None, :] * Ry[None, :]).astype(np.float32)
            R2tab = t["R2"].astype(np.float32)
            cs = [t[k].astype(np.float32) for k in ("c0", "c1", "c2", "c3")]
            R2max = np.float32(Rm * Rm)
        else:
            Rx = ix * float(grid.dRx) - float(x)
            Ry = iy * float(grid.dRy) - float(y)
            R2 = Rx[:, None] ** 2 + Ry[None, :] ** 2
            R2tab = t["R2"]
            cs = [t[k] for k in ("c0", "c1", "c2", "c3")]
            R2max = float(Rm) ** 2
        mask = R2 < R2max
        # unrolled binary search over nR = 128 knots: largest i with R2tab[i] <= R2 (i0 >= 0)
        k = np.clip(np.searchsorted(R2tab, R2, side="right") - 1, 0, len(R2tab) - 2)
        dx = R2 - R2tab[k]
        v = ((cs[3][k] * dx + cs[2][k]) * dx + cs[1][k]) * dx + cs[0][k]
        v = np.where(mask, occ * v, 0.0).astype(dtype)
        jx = (np.mod(ix, nx) + grid.nxh) % nx
        jy = (np.mod(iy, ny) + grid.nyh) % ny
        np.add.at(V, (jx[:, None], jy[None, :]), v)
    return V


def transmission(V, w, dtype=np.float64):
    th = (np.asarray(w, dtype) * V.astype(dtype)).astype(dtype)
    return np.exp(1j * th).astype(np.complex128 if dtype == np.float64 else np.complex64)


def propagator(grid: Grid, lam, dz, dtype=np.float64):
    """P = exp(-i*pi*lambda*dz*g^2)/N on the unshifted FFT grid (propagate, src/cgpu_fcns.cuh:1837)."""
    w = -C_PI * float(lam) * float(dz)
    g2 = grid.g2_shift().astype(np.float64)
    return np.exp(1j * w * g2) / (grid.nx * grid.ny)


def incident_angle(theta, lam, dg_min):
    """set_incident_angle (src/input_multislice.cuh:891-895): the tilt snapped to a whole number of
    Fourier pixels, sin(theta)/lambda = n*dg_min (FP64)."""
    if abs(theta) <= 1e-13:
        return 0.0
    n = np.round(np.sin(theta) / (lam * dg_min))
    return float(np.arcsin(n * lam * dg_min))


def propagate_wave(grid: Grid, lam, psi, z, space=1, gx0=0.0, gy0=0.0):
    """Propagator::operator()(space, gxu, gyu, z, output) on a user wave (src/propagator.cuh:51-103,
    propagate src/cgpu_fcns.cuh:1837-1845): fft2-shift in, FFT, P = exp(-i*pi*lam*z*|g - g0|^2)/N,
    inverse FFT (unnormalised) for real-space output, shift back. |z| <= 1e-5 is isZero
    (src/types.cuh:564-600): the wave itself (real) or FFT2(psi)/N (reciprocal). psi and the
    result are [iy, ix] (MATLAB orientation)."""
    a = np.fft.fftshift(np.asarray(psi, np.complex128).T)
    n = grid.nx * grid.ny
    if abs(float(z)) <= 1e-5:
        out = a if space == 1 else np.fft.fft2(a) / n
    else:
        w = -C_PI * float(lam) * float(z)
        gx, gy = grid.g_shift()
        g2 = (gx.astype(np.float64)[:, None] - gx0) ** 2 + (gy.astype(np.float64)[None, :] - gy0) ** 2
        f = np.fft.fft2(a) * np.exp(1j * w * g2) / n
        out = f if space == 2 else np.fft.ifft2(f) * n
    return np.fft.fftshift(out).T


def probe_fourier(grid: Grid, lam, outer_mrad, inner_mrad, c10, c30_A, beam_x, beam_y, dtype=np.float64):
    """Normalised Fourier-space probe (exp_i_chi + probe, src/cgpu_fcns.cuh:1951-1992 and
    src/gpu_fcns.cuh:1612-1624): aperture * exp(i*(x*gx + y*gy + chi(g)))."""
    f = np.float32
    lam = f(lam)
    g2max = f(f(np.sin(f(f(outer_mrad) * 1e-3))) / lam) ** 2 if outer_mrad > 0 else grid.g_max() ** 2
    g2min = f(f(np.sin(f(f(inner_mrad) * 1e-3))) / lam) ** 2 if inner_mrad > 0 else f(0)
    gx, gy = grid.g_shift()
    g2 = (gx[:, None] * gx[:, None]).astype(f) + (gy[None, :] * gy[None, :]).astype(f)
    ap = (g2min <= g2) & (g2 < g2max)
    xx = float(f(-f(C_2PI) * f(f(beam_x) - f(0.5 * grid.lx))))
    yy = float(f(-f(C_2PI) * f(f(beam_y) - f(0.5 * grid.ly))))
    G2 = g2.astype(np.float64)
    chi = xx * gx.astype(np.float64)[:, None] + yy * gy.astype(np.float64)[None, :]
    chi = chi - C_PI * c10 * float(lam) * G2 - C_PI * c30_A * float(lam) ** 3 / 2.0 * G2 ** 2
    psi = np.where(ap, np.exp(1j * chi), 0.0)
    return psi / np.sqrt(ap.sum())


def multislice(grid: Grid, psi0_real, trans_list, dz_list, lam, out_slices, dtype=np.float64):
    """Slice loop (Wave_Function::psi, src/wave_function.cuh:241-252): transmit, propagate.
    Returns {islice: FFT2(psi)/N after slice islice} for the slices in out_slices."""
    cdt = np.complex128 if dtype == np.float64 else np.complex64
    psi = psi0_real.astype(cdt)
    out = {}
    for k, (T, dz) in enumerate(zip(trans_list, dz_list)):
        psi = psi * T.astype(cdt)
        P = propagator(grid, lam, dz).astype(cdt)
        F = np.fft.fft2(psi) * P
        if k in out_slices:
            out[k] = F.copy()
        psi = np.fft.ifft2(F) * (grid.nx * grid.ny)
        if k == max(out_slices):
            break
    return out, psi


def detector_sum(grid: Grid, psi_hat, g_inner, g_outer):
    """sum_square_over_Det (src/cgpu_fcns.cuh:1796-1806): half-open ring on g2_shift."""
    g2 = grid.g2_shift()
    g2min = np.float32(float(g_inner) ** 2)
    g2max = np.float32(float(g_outer) ** 2)
    m = (g2min <= g2) & (g2 < g2max)
    return float(np.sum(np.abs(psi_hat[m]) ** 2))
