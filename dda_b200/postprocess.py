"""Far-field and cross-section post-processing of the dipole polarisations.

The per-direction sums run on the GPU (dda_far_field); this module restates
the reference's host-side assembly around them:

  grid_angles        GridAngleList (EMSim/AngleList.cpp:71-106): theta-major
                     grid from "start..end/count" specifications in degrees
  scattering_frame   FarFieldCalc::calcEField (DDA/FarFieldCalc.cpp:119-160):
                     direction, perpendicular and parallel vectors per angle
  jones              JonesCalculus::getJonesMatrix (EMSim/JonesCalculus.cpp:74-86)
  cross_sections     PlaneWave::extCross (DDA/Beam.cpp:126-133),
                     AbsCross::absCross (DDA/AbsCross.cpp:28-48) and the
                     efficiencies of outputCrossSections (DDA/DDAMain.cpp:284-304)
"""
import math

import numpy as np

from . import api
from .datafiles import open_out


def parse_angles(spec):
    """'a' or 'start..end/count' in degrees -> (start_rad, step_rad, count)."""
    if ".." not in spec:
        return math.radians(float(spec)), 0.0, 1
    start, rest = spec.split("..")
    end, n = rest.split("/")
    start, end, n = math.radians(float(start)), math.radians(float(end)), int(n)
    step = 0.0 if n <= 1 else (end - start) / (n - 1)
    return start, step, n


def grid_angles(theta_spec="0..180/91", phi_spec="0..360/61"):
    """Theta-major angle grid: angle i has theta index i // nPhi."""
    t0, dt, nt = parse_angles(theta_spec)
    p0, dp, npf = parse_angles(phi_spec)
    i = np.arange(nt * npf)
    return t0 + (i // npf) * dt, p0 + (i % npf) * dp


def scattering_frame(prop, theta, phi, orient=None):
    """Directions n, perpendicular and parallel vectors for each angle, in
    the frame (prop, incPolX = polarisation 2, incPolY = polarisation 1), in
    the particle's coordinates (orient: its ZYZ Euler angles in degrees,
    DDA/FarFieldCalc.cpp:165-170)."""
    pn, py, px, _ = api.beam_frame(prop, orient)
    st, ct = np.sin(theta)[:, None], np.cos(theta)[:, None]
    sp, cp = np.sin(phi)[:, None], np.cos(phi)[:, None]
    n = ct * pn + st * (cp * px + sp * py)
    perp = sp * px - cp * py
    par = -st * pn + ct * (cp * px + sp * py)
    return n, perp, par


def jones(e1, e2, theta, phi, perp, par):
    """Jones matrices [count][2][2] from the far fields e1 (polarisation 1)
    and e2 (polarisation 2), each [count][3] complex."""
    f1par, f1perp = np.einsum("ij,ij->i", e1, par), np.einsum("ij,ij->i", e1, perp)
    f2par, f2perp = np.einsum("ij,ij->i", e2, par), np.einsum("ij,ij->i", e2, perp)
    sp, cp = np.sin(phi), np.cos(phi)
    out = np.empty((len(theta), 2, 2), dtype=np.complex128)
    out[:, 0, 0] = cp * f2par + sp * f1par
    out[:, 0, 1] = sp * f2par - cp * f1par
    out[:, 1, 0] = cp * f2perp + sp * f1perp
    out[:, 1, 1] = sp * f2perp - cp * f1perp
    return out


def jones_far_field(mv, prop, theta, phi, pol=None, orient=None):
    """Jones matrices on an angle grid from the two polarisations of the last
    solve (right-hand sides 0 and 1 of `mv`) or of `pol` ([2][3 nvs])."""
    n, perp, par = scattering_frame(prop, theta, phi, orient)
    e = mv.far_field(n, nrhs=2, pol=pol)  # [count][2][3]
    return jones(e[:, 0, :], e[:, 1, :], theta, phi, perp, par)


def ext_cross_general(params, pol_vec, einc):
    """Cext = 4 pi k sum_i Im(P_i . conj(Einc_i)) over the dipoles: the
    extinction of any incident beam (Beam::extCross, DDA/Beam.cpp:58-67); for
    a plane wave it equals the optical theorem of cross_sections."""
    nvs, nv = params.nvs, params.nv
    p = np.asarray(pol_vec).reshape(3, nvs)[:, :nv]
    e = np.asarray(einc).reshape(3, nvs)[:, :nv]
    return 4 * np.pi * params.wave_num * float(np.sum(np.imag(p * np.conj(e))))


def cross_sections(params, cc, pol_vec, e_forward, prop, pol, einc=None, orient=None):
    """(Cext, Cabs, Qext, Qabs) of one solution: e_forward = far field in the
    propagation direction (in the particle frame: api.beam_frame), cc the
    CoupleConstants of that right-hand side.  einc: the incident field of a
    non-plane beam, whose extinction then comes from ext_cross_general
    (e_forward is not used)."""
    _, p1, p2, _ = api.beam_frame(prop, orient)
    inc = p1 if pol == 1 else p2
    k = params.wave_num
    if einc is not None:
        cext = ext_cross_general(params, pol_vec, einc)
    else:
        cext = -np.dot(np.real(e_forward), inc) * 4 * np.pi / k
    temp1 = k ** 3 * 2 / 3
    multdr = -np.imag(1.0 / cc.cc) - temp1  # [nmat*3]
    nvs, nv = params.nvs, params.nv
    mat = params.geometry.materials.astype(np.int64)
    p = np.asarray(pol_vec).reshape(3, nvs)[:, :nv]
    cabs = 0.0
    for c in range(3):
        cabs += np.sum(multdr[mat * 3 + c] * np.abs(p[c]) ** 2)
    cabs *= 4 * np.pi * k
    a_eq = (3.0 / (4 * np.pi) * nv) ** (1.0 / 3) * params.grid_unit
    norm = 1.0 / (np.pi * a_eq * a_eq)
    return cext, cabs, cext * norm, cabs * norm


def mie(x, m):
    """Mie efficiencies (Qext, Qsca, Qabs) of a homogeneous sphere of size
    parameter x and relative refractive index m: the Bohren-Huffman series
    the reference prints beside the DDA cross sections (EMSim/Mie.cpp:41-174,
    DDA/DDAMain.cpp:431-460).  Downward recurrence for the logarithmic
    derivative, upward for the Riccati-Bessel functions; forward-scattering
    amplitude for Qext."""
    m = complex(m)
    mx = x * m
    xstop = x + 4 * x ** (1.0 / 3) + 2
    nstop = int(xstop)
    nmx = int(max(xstop, abs(mx)) + 15)
    d = np.zeros(nmx, dtype=np.complex128)
    for i in range(nmx - 1, 0, -1):
        d[i - 1] = (i + 1) / mx - 1.0 / (d[i] + (i + 1) / mx)
    psi0, psi1 = math.cos(x), math.sin(x)
    chi0, chi1 = -math.sin(x), math.cos(x)
    xi1 = complex(psi1, -chi1)
    qs = 0.0
    s1 = 0j
    for n in range(nstop):
        rn = n + 1.0
        psi = (2 * rn - 1) * psi1 / x - psi0
        chi = (2 * rn - 1) * chi1 / x - chi0
        xi = complex(psi, -chi)
        a = ((d[n] / m + rn / x) * psi - psi1) / ((d[n] / m + rn / x) * xi - xi1)
        b = ((m * d[n] + rn / x) * psi - psi1) / ((m * d[n] + rn / x) * xi - xi1)
        qs += (2 * rn + 1) * (abs(a) ** 2 + abs(b) ** 2)
        s1 += (2 * rn + 1) / (rn * (rn + 1)) * (a + b) * rn * (rn + 1) / 2
        psi0, psi1 = psi1, psi
        chi0, chi1 = chi1, chi
        xi1 = complex(psi1, -chi1)
    qsca = 2 / (x * x) * qs
    qext = 4 / (x * x) * s1.real
    return qext, qsca, qext - qsca


def mie_amplitudes(x, m, theta):
    """Scattering amplitudes S1(theta), S2(theta) of the sphere of `mie` (the
    Bohren-Huffman series with the angle functions pi_n, tau_n of
    mu = cos theta, as EMSim/Mie.cpp:41-174 evaluates them; phi does not
    enter)."""
    m = complex(m)
    mx = x * m
    mu = np.cos(np.asarray(theta, dtype=np.float64))
    xstop = x + 4 * x ** (1.0 / 3) + 2
    nstop = int(xstop)
    nmx = int(max(xstop, abs(mx)) + 15)
    d = np.zeros(nmx, dtype=np.complex128)
    for i in range(nmx - 1, 0, -1):
        d[i - 1] = (i + 1) / mx - 1.0 / (d[i] + (i + 1) / mx)
    psi0, psi1 = math.cos(x), math.sin(x)
    chi0, chi1 = -math.sin(x), math.cos(x)
    xi1 = complex(psi1, -chi1)
    s1 = np.zeros(mu.shape, dtype=np.complex128)
    s2 = np.zeros(mu.shape, dtype=np.complex128)
    pi0, pi1 = np.zeros(mu.shape), np.ones(mu.shape)
    for n in range(nstop):
        rn = n + 1.0
        psi = (2 * rn - 1) * psi1 / x - psi0
        chi = (2 * rn - 1) * chi1 / x - chi0
        xi = complex(psi, -chi)
        a = ((d[n] / m + rn / x) * psi - psi1) / ((d[n] / m + rn / x) * xi - xi1)
        b = ((m * d[n] + rn / x) * psi - psi1) / ((m * d[n] + rn / x) * xi - xi1)
        fn = (2 * rn + 1) / (rn * (rn + 1))
        pi = pi1
        tau = rn * mu * pi - (rn + 1) * pi0
        s1 += fn * (a * pi + b * tau)
        s2 += fn * (a * tau + b * pi)
        pi1 = ((2 * rn + 1) * mu * pi - (rn + 1) * pi0) / rn
        pi0 = pi
        psi0, psi1 = psi1, psi
        chi0, chi1 = chi1, chi
        xi1 = complex(psi1, -chi1)
    return s1, s2


def mie_jones(x, m, theta, wave_num):
    """Jones matrices [n][2][2] of the Mie far field on the angles `theta`:
    diag(S2, S1) times -1/k, the far-field factor the reference passes
    (DDAMain.cpp:484, EMSim/Mie.cpp:165-172)."""
    s1, s2 = mie_amplitudes(x, m, theta)
    j = np.zeros((len(s1), 2, 2), dtype=np.complex128)
    j[:, 0, 0] = -s2 / wave_num
    j[:, 1, 1] = -s1 / wave_num
    return j


def mueller(j):
    """Mueller matrices [count][4][4] from Jones matrices [count][2][2]
    (MuellerCalculus::computeMuellerMatrix, EMSim/MuellerCalculus.cpp:36-60)."""
    s00, s01, s10, s11 = j[:, 0, 0], j[:, 0, 1], j[:, 1, 0], j[:, 1, 1]
    n = lambda z: np.abs(z) ** 2
    c = np.conj
    m = np.empty((len(j), 4, 4))
    m[:, 0, 0] = (n(s11) + n(s00) + n(s01) + n(s10)) / 2
    m[:, 0, 1] = (-n(s11) + n(s00) - n(s01) + n(s10)) / 2
    m[:, 0, 2] = np.real(s00 * c(s01) + s11 * c(s10))
    m[:, 0, 3] = np.imag(s00 * c(s01) - s11 * c(s10))
    m[:, 1, 0] = (-n(s11) + n(s00) + n(s01) - n(s10)) / 2
    m[:, 1, 1] = (n(s11) + n(s00) - n(s01) - n(s10)) / 2
    m[:, 1, 2] = np.real(s00 * c(s01) - s11 * c(s10))
    m[:, 1, 3] = np.imag(s00 * c(s01) + s11 * c(s10))
    m[:, 2, 0] = np.real(s00 * c(s10) + s11 * c(s01))
    m[:, 2, 1] = np.real(s00 * c(s10) - s11 * c(s01))
    m[:, 2, 2] = np.real(s11 * c(s00) + s01 * c(s10))
    m[:, 2, 3] = np.imag(s00 * c(s11) + s10 * c(s01))
    m[:, 3, 0] = np.imag(s10 * c(s00) + s11 * c(s01))
    m[:, 3, 1] = np.imag(s10 * c(s00) - s11 * c(s01))
    m[:, 3, 2] = np.imag(s11 * c(s00) - s01 * c(s10))
    m[:, 3, 3] = np.real(s11 * c(s00) - s01 * c(s10))
    return m


def store_jones_txt(path, theta, phi, j, store_phi=True):
    """JonesCalculus::storeTxt (EMSim/JonesCalculus.cpp:89-116): angles in
    degrees with two decimals, then s1..s4 = S22, S11, S12, S21 (real, imag);
    `path` may also be a text stream."""
    with open_out(path) as f:
        f.write("#theta " + ("phi " if store_phi else "") + "s1.r s1.i s2.r s2.i s3.r s3.i s4.r s4.i\n")
        for t, p, s in zip(theta, phi, j):
            row = "%.2f " % math.degrees(t)
            if store_phi:
                row += "%.2f " % math.degrees(p)
            vals = (s[1, 1], s[0, 0], s[0, 1], s[1, 0])
            row += " ".join("%.10e %.10e" % (z.real, z.imag) for z in vals)
            f.write(row + "\n")


def store_mueller_txt(path, theta, phi, m, no_phi=False):
    """MuellerCalculus::storeTxt (EMSim/MuellerCalculus.cpp:88-116)."""
    with open_out(path) as f:
        f.write("#theta " + ("" if no_phi else "phi ") + " ".join("s%d%d" % (a, b) for a in range(1, 5)
                                                                  for b in range(1, 5)) + "\n")
        for t, p, e in zip(theta, phi, m):
            row = "%.2f " % math.degrees(t)
            if not no_phi:
                row += "%.2f " % math.degrees(p)
            f.write(row + " ".join("%.10e" % v for v in e.reshape(-1)) + "\n")


def parse_far_field(spec):
    """--far-field FileName=theta,phi[,jones|mueller|both|none][,no-phi]
    (FarFieldOption::parse, DDA/FarFieldCalc.cpp:51-117): (name, theta
    spec, phi spec, store Jones, store Mueller, no-phi)."""
    name, _, rest = spec.rpartition("=")
    if not name and not rest:
        raise ValueError("bad --far-field " + spec)
    if "/" in name:
        raise ValueError("far-field name must not contain '/'")
    parts = rest.split(",")
    if len(parts) < 2:
        raise ValueError("--far-field needs theta and phi: " + spec)
    jones, mueller_, no_phi, have = True, False, False, False
    for o in parts[2:]:
        if o in ("jones", "mueller", "both", "none"):
            if have:
                raise ValueError("more than one of jones/mueller/both/none in " + spec)
            have = True
            jones, mueller_ = {"jones": (True, False), "mueller": (False, True), "both": (True, True),
                               "none": (False, False)}[o]
        elif o == "no-phi":
            no_phi = True
        else:
            raise ValueError("Invalid option '%s' for far field" % o)
    return name, parts[0], parts[1], jones, mueller_, no_phi

