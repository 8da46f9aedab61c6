"""Seeded synthetic inputs in Nebula's formats.

Real cstool ``.mat`` files and measured SEM data are not available, so the
workloads are built from:

* a synthetic material generator that writes the Kieft & Bosch groups read by
  ``source/physics/kieft/elastic.h:120-166`` and
  ``source/physics/kieft/inelastic.h:212-327`` (screened-Rutherford elastic
  scattering blended into a constant acoustic-phonon mean free path below
  100 eV, and a single-pole Drude energy-loss function for the dielectric
  inelastic model), in the reference ``.mat`` HDF5 layout;
* geometry generators (cube, line-space grating, rough surface) writing the
  ``.tri`` triangle format;
* primary-beam generators writing ``.pri`` records, drawn from numpy's
  Philox bit generator.
"""
from __future__ import annotations

import math

import numpy as np

from . import formats
from .h5mat import MatFile

A0_NM = 0.0529177210903          # Bohr radius (nm)
E2_EVNM = 1.439964547            # e^2 / (4 pi eps0) in eV nm
MEC2_EV = 510998.95              # electron rest energy (eV)
AMU_G = 1.66053906660e-24        # atomic mass unit in grams


# ----------------------------------------------------------------------------
# Materials
# ----------------------------------------------------------------------------
def _geomspace(first, last, n):
    """Axis values exactly as ``util::geomspace`` reconstructs them
    (``source/common/util/range.h:271-310``): first * exp(i * step)."""
    step = math.log(last / first) / (n - 1)
    return np.array([first * math.exp(i * step) for i in range(n)], np.float64)


def _linspace(first, last, n):
    step = (last - first) / (n - 1)
    return np.array([first + i * step for i in range(n)], np.float64)


def screening_eta(E, Z):
    """Nigam screening parameter of the screened-Rutherford cross section."""
    tau = E / MEC2_EV
    return 1.7e-5 * Z ** (2.0 / 3.0) / (tau * (tau + 2.0))


def elastic_imfp(E, Z, n_atoms, phonon_imfp):
    """Elastic inverse mean free path (nm^-1).

    Screened Rutherford above 200 eV, a constant acoustic-phonon value below
    100 eV, and log-log interpolation in between (the Kieft & Bosch blend)."""
    E = np.asarray(E, np.float64)
    eta = screening_eta(E, Z)
    sigma = math.pi * (Z * E2_EVNM) ** 2 / (4.0 * E * E * eta * (1.0 + eta))
    sr = n_atoms * sigma
    out = np.where(E >= 200.0, sr, phonon_imfp)
    mid = (E > 100.0) & (E < 200.0)
    if np.any(mid):
        sr200 = n_atoms * math.pi * (Z * E2_EVNM) ** 2 / (4.0 * 200.0 ** 2 * screening_eta(200.0, Z) * (1 + screening_eta(200.0, Z)))
        t = np.log(E[mid] / 100.0) / math.log(2.0)
        out[mid] = np.exp((1 - t) * math.log(phonon_imfp) + t * math.log(sr200))
    return out


def elastic_icdf(E, P, Z):
    """cos(theta) inverse CDF of the screened-Rutherford distribution."""
    eta = screening_eta(np.asarray(E, np.float64), Z)[:, None]
    P = np.asarray(P, np.float64)[None, :]
    return 1.0 + 2.0 * eta - 2.0 * eta * (1.0 + eta) / (P + eta)


def drude_elf(w, wp, gamma):
    """Single-pole Drude energy-loss function Im(-1/eps(w))."""
    return gamma * w * wp * wp / ((wp * wp - w * w) ** 2 + (gamma * w) ** 2)


def inelastic_tables(K, P, wp, gamma, fermi, w_lo, scale):
    """Dielectric IMFP (nm^-1) and omega' inverse CDF (eV) for every energy.

    dIMFP/dw = ELF(w) / (pi a0 K) * ln[(1 + sqrt(1 - w/K)) / (1 - sqrt(1 - w/K))]
    for w between ``w_lo`` and ``K - fermi``."""
    nK, nP = len(K), len(P)
    imfp = np.full(nK, 1e-30)
    icdf = np.full((nK, nP), w_lo)
    for i, k in enumerate(K):
        wmax = k - fermi
        if wmax <= w_lo * 1.0001:
            continue
        w = np.geomspace(w_lo, wmax, 4001)
        x = np.clip(w / k, 0.0, 1.0)
        s = np.sqrt(1.0 - x)
        with np.errstate(divide="ignore"):
            lg = np.log((1.0 + s) / np.maximum(1.0 - s, 1e-300))
        f = drude_elf(w, wp, gamma) / (math.pi * A0_NM * k) * lg * scale
        cum = np.concatenate([[0.0], np.cumsum(0.5 * (f[1:] + f[:-1]) * np.diff(w))])
        if cum[-1] <= 0:
            continue
        imfp[i] = max(cum[-1], 1e-30)
        cdf = cum / cum[-1]
        icdf[i] = np.interp(P, cdf, w)
        icdf[i, 0] = w_lo
        icdf[i, -1] = wmax
    return imfp, icdf


MATERIALS = {
    # name: (Z, atoms/nm^3, A [u], hbar*w_p, gamma, fermi, work function, band gap, phonon loss, density factor)
    "si": (14, 49.94, 28.0855, 16.7, 4.0, 7.8, 4.8, 1.12, 0.063, 1.0),
    "sio2": (10, 66.3, 20.03, 22.0, 4.0, 7.8, 4.8, 9.0, 0.063, 1.0),
    "w": (74, 63.2, 183.84, 25.0, 4.0, 7.8, 4.8, -1.0, 0.063, 8.1),
}


def make_material(path, kind="si", nK=128, nP=256, Kmin=1.0, Kmax=1.0e4, seed=0, penn=True, nW=32, nPq=32):
    """Write a synthetic ``.mat`` file for one of ``MATERIALS``.

    The energy axis is written as the exact ``geomspace`` values the reader
    reconstructs, so the logarithmic-spacing check of
    ``source/io/hdf5_file.cpp:345-351`` passes.  ``seed`` is recorded in the
    file; the tables themselves are deterministic functions of the model
    parameters.  With ``penn`` the file also carries the full Penn groups,
    so the same file serves both inelastic models."""
    Z, n_at, A, wp, gam, fermi, wf, gap, phonon, dens = MATERIALS[kind]
    K = _geomspace(Kmin, Kmax, nK)
    P = _linspace(0.0, 1.0, nP)

    m = MatFile()
    m.set_property_string("name", {"si": "Si-like", "sio2": "SiO2-like", "w": "W-like"}[kind])
    m.set_property_string("cstool_version", "nbx-synthetic-1 (seed %d)" % seed)
    m.set_property_quantity("fermi", fermi, "eV")
    m.set_property_quantity("work_function", wf, "eV")
    m.set_property_quantity("barrier", fermi + wf, "eV")
    if gap >= 0:
        m.set_property_quantity("band_gap", gap, "eV")
    m.set_property_quantity("phonon_loss", phonon, "eV")
    m.set_property_quantity("effective_A", A * AMU_G, "g")
    m.set_property_quantity("density", n_at * dens * A * AMU_G * 1e21, "g/cm^3")

    # Elastic --------------------------------------------------------------
    g = m.group("/kieft/elastic")
    k_el = g.dataset("energy", K, units="eV")
    p_el = g.dataset("probability", P, units="")
    imfp_el = elastic_imfp(K, Z, n_at * dens, phonon_imfp=1.0 * dens)
    d = g.dataset("imfp", (imfp_el * 1e9).astype(np.float32), units="m^-1")   # stored in m^-1
    d.attach_scale(0, k_el)
    d = g.dataset("costheta_icdf", elastic_icdf(K, P, Z).astype(np.float32), units="")
    d.attach_scale(0, k_el)
    d.attach_scale(1, p_el)

    # Inelastic ------------------------------------------------------------
    g = m.group("/kieft/inelastic")
    k_in = g.dataset("energy", K, units="eV")
    p_in = g.dataset("probability", P, units="")
    imfp_in, w0 = inelastic_tables(K, P, wp, gam, fermi, w_lo=0.1, scale=dens)
    d = g.dataset("imfp", imfp_in.astype(np.float32), units="nm^-1")
    d.attach_scale(0, k_in)
    d = g.dataset("w0_icdf", w0.astype(np.float32), units="eV")
    d.attach_scale(0, k_in)
    d.attach_scale(1, p_in)

    # Ionization -------------------------------------------------------------
    g = m.group("/kieft/ionization")
    k_io = g.dataset("energy", K, units="eV")
    p_io = g.dataset("probability", P, units="")
    binding = np.zeros((nK, nP), np.float32)
    binding[:, :] = 5.0                               # valence: < 50 eV
    binding[np.ix_(K > 150.0, P >= 0.97)] = 99.8      # an inner shell
    d = g.dataset("binding_icdf", binding, units="eV")
    d.attach_scale(0, k_io)
    d.attach_scale(1, p_io)
    g.dataset("outer_shells", np.array([100.0, 149.7, 1839.0]), units="eV")

    if penn:
        _write_penn(m, K, P, imfp_in, w0, nW=nW, nPq=nPq)

    m.write(path)
    return path


def q_icdf_table(K, W, Pq):
    """Momentum-transfer inverse CDF (nm^-1) on (K, omega/K, P).

    Between the kinematic limits q-/+ = sqrt(K) -/+ sqrt(K - omega) (in
    units of sqrt(eV), hbar^2 / 2m = 1) the density is taken as 1/q (dipole
    form), floored at 1e-3 sqrt(K); the result is stored in nm^-1 as the
    reference's loader expects (it multiplies by hbar / sqrt(2m) =
    0.19519 nm eV^1/2)."""
    out = np.zeros((len(K), len(W), len(Pq)))
    for i, k in enumerate(K):
        for j, w in enumerate(W):
            om = min(w, 1.0) * k
            q_hi = math.sqrt(k) + math.sqrt(max(k - om, 0.0))
            q_lo = max(math.sqrt(k) - math.sqrt(max(k - om, 0.0)), 1e-3 * math.sqrt(k))
            q_lo = min(q_lo, q_hi)
            out[i, j] = q_lo * (q_hi / q_lo) ** Pq / 0.19519
    return out


def _write_penn(m, K, P, imfp_in, omega_icdf, nW=32, nPq=32, nO=32):
    """Full Penn groups (source/physics/full_penn.h:296-392): /full_penn/imfp
    and /full_penn/omega_icdf from the same dielectric model as the Kieft
    tables, /full_penn/q_icdf on (K, omega/K, P), and the 3-D
    /ionization/binding_icdf on (K, omega/K log-spaced, P) with one inner
    shell (99.8 eV) above 10 % of the omega-cumulative range."""
    g = m.group("/full_penn")
    k_p = g.dataset("energy", K, units="eV")
    p_p = g.dataset("probability", P, units="")
    d = g.dataset("imfp", imfp_in.astype(np.float32), units="nm^-1")
    d.attach_scale(0, k_p)
    d = g.dataset("omega_icdf", omega_icdf.astype(np.float32), units="eV")
    d.attach_scale(0, k_p)
    d.attach_scale(1, p_p)
    W = _linspace(0.0, 1.0, nW)
    Pq = _linspace(0.0, 1.0, nPq)
    w_q = g.dataset("omega_fraction", W, units="")
    p_q = g.dataset("q_probability", Pq, units="")
    d = g.dataset("q_icdf", q_icdf_table(K, W, Pq).astype(np.float32), units="nm^-1")
    d.attach_scale(0, k_p)
    d.attach_scale(1, w_q)
    d.attach_scale(2, p_q)

    g = m.group("/ionization")
    k_i = g.dataset("energy", K, units="eV")
    O = _geomspace(1e-4, 1.0, nO)
    Pb = _linspace(0.0, 1.0, nPq)
    o_i = g.dataset("omega_fraction", O, units="")
    p_i = g.dataset("probability", Pb, units="")
    binding = np.full((len(K), nO, nPq), 5.0, np.float32)          # valence (< 50 eV)
    omega = K[:, None] * O[None, :]
    shell = (omega >= 99.8)[:, :, None] & (Pb >= 0.9)[None, None, :]
    binding[shell] = 99.8
    d = g.dataset("binding_icdf", binding, units="eV")
    d.attach_scale(0, k_i)
    d.attach_scale(1, o_i)
    d.attach_scale(2, p_i)


# ----------------------------------------------------------------------------
# Geometry
# ----------------------------------------------------------------------------
class TriBuilder:
    def __init__(self):
        self.rows = []

    def tri(self, a, b, c, mat_in, mat_out):
        self.rows.append((mat_in, mat_out, (a, b, c)))

    def quad(self, a, b, c, d, mat_in, mat_out):
        """Quad a-b-c-d counter-clockwise seen from the ``mat_out`` side."""
        self.tri(a, b, c, mat_in, mat_out)
        self.tri(a, c, d, mat_in, mat_out)

    def box(self, lo, hi, mat_in, mat_out):
        x0, y0, z0 = lo
        x1, y1, z1 = hi
        q = self.quad
        q((x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1), mat_in, mat_out)  # +z
        q((x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0), mat_in, mat_out)  # -z
        q((x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1), mat_in, mat_out)  # +x
        q((x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0), mat_in, mat_out)  # -x
        q((x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0), mat_in, mat_out)  # +y
        q((x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1), mat_in, mat_out)  # -y

    def array(self):
        out = np.zeros(len(self.rows), formats.TRI_DTYPE)
        for i, (a, b, (p, q, r)) in enumerate(self.rows):
            out[i]["mat_in"] = a
            out[i]["mat_out"] = b
            out[i]["v"] = np.array([p, q, r], np.float64).astype(np.float32)
        return out


def cube_geometry(size=(2000.0, 2000.0, 1000.0), detector_z=10.0, detector_margin=100.0):
    """Axis-aligned block of material 0 with its top face at z=0, vacuum
    around it, and a two-triangle DETECTOR plane above it."""
    sx, sy, sz = size
    b = TriBuilder()
    b.box((-sx / 2, -sy / 2, -sz), (sx / 2, sy / 2, 0.0), 0, formats.VACUUM)
    m = detector_margin
    b.quad((-sx / 2 - m, -sy / 2 - m, detector_z), (sx / 2 + m, -sy / 2 - m, detector_z),
           (sx / 2 + m, sy / 2 + m, detector_z), (-sx / 2 - m, sy / 2 + m, detector_z),
           formats.DETECTOR, formats.DETECTOR)
    return b.array()


def grating_geometry(width=32.0, pitch=64.0, height=50.0, length=2000.0, n_lines=31,
                     depth=1000.0, segment=100.0, detector_z=100.0):
    """Line-space grating: lines along y on a substrate of the same material.

    The solid's outer surface is emitted directly (line tops, trench floors,
    side walls, end faces, substrate sides and bottom); the faces along y are
    split into ``segment``-long pieces (about 5k triangles with the defaults).
    """
    b = TriBuilder()
    half = n_lines * pitch / 2.0
    xs = [(-half + i * pitch + (pitch - width) / 2, -half + i * pitch + (pitch + width) / 2) for i in range(n_lines)]
    y0, y1 = -length / 2, length / 2
    ny = max(1, int(round(length / segment)))
    ys = np.linspace(y0, y1, ny + 1)
    V = formats.VACUUM
    # Profile along x: list of (x_start, x_end, z)
    prof = []
    xcur = -half
    for (a, c) in xs:
        if a > xcur:
            prof.append((xcur, a, 0.0))
        prof.append((a, c, height))
        xcur = c
    if xcur < half:
        prof.append((xcur, half, 0.0))
    for j in range(ny):
        ya, yb = ys[j], ys[j + 1]
        for (a, c, z) in prof:
            b.quad((a, ya, z), (c, ya, z), (c, yb, z), (a, yb, z), 0, V)     # top (+z)
        for (a, c) in xs:
            b.quad((a, ya, 0.0), (a, ya, height), (a, yb, height), (a, yb, 0.0), 0, V)   # -x wall
            b.quad((c, ya, 0.0), (c, yb, 0.0), (c, yb, height), (c, ya, height), 0, V)   # +x wall
    # substrate block sides (z from -depth to 0) and bottom
    b.quad((-half, y0, -depth), (-half, y1, -depth), (half, y1, -depth), (half, y0, -depth), 0, V)   # bottom
    b.quad((half, y0, -depth), (half, y1, -depth), (half, y1, 0.0), (half, y0, 0.0), 0, V)          # +x
    b.quad((-half, y0, -depth), (-half, y0, 0.0), (-half, y1, 0.0), (-half, y1, -depth), 0, V)      # -x
    b.quad((-half, y1, -depth), (-half, y1, 0.0), (half, y1, 0.0), (half, y1, -depth), 0, V)        # +y
    b.quad((-half, y0, -depth), (half, y0, -depth), (half, y0, 0.0), (-half, y0, 0.0), 0, V)        # -y
    # line end caps at y = +-length/2
    for (a, c) in xs:
        b.quad((a, y1, 0.0), (a, y1, height), (c, y1, height), (c, y1, 0.0), 0, V)   # +y
        b.quad((a, y0, 0.0), (c, y0, 0.0), (c, y0, height), (a, y0, height), 0, V)   # -y
    m = 50.0
    b.quad((-half - m, y0 - m, detector_z), (half + m, y0 - m, detector_z),
           (half + m, y1 + m, detector_z), (-half - m, y1 + m, detector_z),
           formats.DETECTOR, formats.DETECTOR)
    return b.array()


def rough_geometry(n=512, size=1000.0, rms=3.0, corr=10.0, depth=1000.0, seed=0, detector_z=50.0):
    """Slab whose top surface is a seeded Gaussian random height field
    (``n`` x ``n`` samples, RMS ``rms`` nm, correlation length ``corr`` nm)."""
    rng = np.random.Generator(np.random.Philox(seed))
    h = rng.standard_normal((n, n))
    dx = size / (n - 1)
    k = np.fft.fftfreq(n, d=dx)
    kk = k[:, None] ** 2 + k[None, :] ** 2
    filt = np.exp(-(math.pi ** 2) * corr ** 2 * kk / 2.0)
    h = np.real(np.fft.ifft2(np.fft.fft2(h) * filt))
    h *= rms / h.std()
    xs = np.linspace(-size / 2, size / 2, n)
    V = formats.VACUUM
    rows = []
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    P = np.stack([X, Y, h], -1).astype(np.float32)
    a = P[:-1, :-1].reshape(-1, 3)
    b_ = P[1:, :-1].reshape(-1, 3)
    c = P[1:, 1:].reshape(-1, 3)
    d = P[:-1, 1:].reshape(-1, 3)
    top = np.zeros(2 * a.shape[0], formats.TRI_DTYPE)
    top["mat_in"] = 0
    top["mat_out"] = V
    top["v"][0::2] = np.stack([a, b_, c], 1)
    top["v"][1::2] = np.stack([a, c, d], 1)
    b = TriBuilder()
    lo, hi = -size / 2, size / 2
    b.quad((lo, lo, -depth), (lo, hi, -depth), (hi, hi, -depth), (hi, lo, -depth), 0, V)
    # side walls follow the height profile along each edge
    for i in range(n - 1):
        x0, x1 = xs[i], xs[i + 1]
        b.quad((x0, lo, -depth), (x1, lo, -depth), (x1, lo, h[i + 1, 0]), (x0, lo, h[i, 0]), 0, V)
        b.quad((x0, hi, -depth), (x0, hi, h[i, -1]), (x1, hi, h[i + 1, -1]), (x1, hi, -depth), 0, V)
        b.quad((lo, x0, -depth), (lo, x0, h[0, i]), (lo, x1, h[0, i + 1]), (lo, x1, -depth), 0, V)
        b.quad((hi, x0, -depth), (hi, x1, -depth), (hi, x1, h[-1, i + 1]), (hi, x0, h[-1, i]), 0, V)
    m = 20.0
    b.quad((lo - m, lo - m, detector_z), (hi + m, lo - m, detector_z), (hi + m, hi + m, detector_z),
           (lo - m, hi + m, detector_z), formats.DETECTOR, formats.DETECTOR)
    return np.concatenate([top, b.array()])


def _quads_to_tris(A, B, C, D, mat_in, mat_out):
    """Triangles (A, B, C), (A, C, D) of quads given as (..., 3) corner arrays,
    counter-clockwise seen from the mat_out side."""
    A, B, C, D = (np.asarray(v, np.float64).reshape(-1, 3) for v in (A, B, C, D))
    out = np.zeros(2 * len(A), formats.TRI_DTYPE)
    out["mat_in"] = mat_in
    out["mat_out"] = mat_out
    out["v"][0::2] = np.stack([A, B, C], 1).astype(np.float32)
    out["v"][1::2] = np.stack([A, C, D], 1).astype(np.float32)
    return out


def _disc(center, ring, mat_in, mat_out, fractions=(0.6, 0.3)):
    """Planar disc bounded by `ring` (holes, n, 3): bands down to inner rings
    at `fractions` of the way from the centre, each with half the points of
    the ring outside it, then a fan round the centre.  With n = 48 no vertex
    is shared by more than 12 triangles, below the octree's split count, so
    the cells round the centre are not split down to the maximum depth (a
    single 48-triangle fan would be).  Counter-clockwise seen from the
    mat_out side when the ring runs so."""
    if ring.shape[1] % (2 ** len(fractions)):
        raise ValueError("ring points must be divisible by %d" % 2 ** len(fractions))
    c = center[:, None, :]
    levels = [ring] + [c + f * (ring[:, ::2 ** (k + 1)] - c) for k, f in enumerate(fractions)]
    tris = []
    for O, I in zip(levels[:-1], levels[1:]):
        o0, o1, o2 = O[:, 0::2], O[:, 1::2], np.roll(O, -2, axis=1)[:, 0::2]
        i1 = np.roll(I, -1, axis=1)
        tris += [np.stack([I, o0, o1], 2), np.stack([I, o1, i1], 2), np.stack([i1, o1, o2], 2)]
    last = levels[-1]
    tris.append(np.stack([np.repeat(c, last.shape[1], 1), last, np.roll(last, -1, axis=1)], 2))
    v = np.concatenate([t.reshape(-1, 3, 3) for t in tris])
    out = np.zeros(len(v), formats.TRI_DTYPE)
    out["mat_in"] = mat_in
    out["mat_out"] = mat_out
    out["v"] = v.astype(np.float32)
    return out


def contact_hole_geometry(n_holes=32, pitch=80.0, radius=20.0, depth=100.0, roughness=2.0, plug_depth=50.0,
                          substrate=500.0, n_theta=48, n_rings=20, detector_z=20.0, seed=0,
                          materials=(0, 1, 2)):
    """Contact-hole array: an ``n_holes`` x ``n_holes`` grid of holes of
    ``radius`` nm (edge roughness up to +-``roughness`` nm, a few seeded
    Fourier modes in angle blended along the depth) through a ``depth`` nm
    film (material ``materials[0]``, SiO2-like) down to plugs (``[1]``,
    W-like, ``plug_depth`` nm) set in the substrate (``[2]``, Si-like).  With
    the defaults 2,506,772 triangles over 2.56 um; a DETECTOR plane sits at
    ``detector_z``.  The surface meshes are conforming: neighbouring cells
    share the vertices of their common edges."""
    film, plug, sub = materials
    V = formats.VACUUM
    rng = np.random.Generator(np.random.Philox(seed))
    H = n_holes * n_holes
    half = n_holes * pitch / 2.0
    idx = np.arange(n_holes)
    cx = (-half + (idx + 0.5) * pitch)
    CX, CY = np.meshgrid(cx, cx, indexing="ij")
    centers = np.stack([CX.ravel(), CY.ravel()], 1)                       # (H, 2)
    # angles: multiples of 360/n_theta, including the square's corners
    theta = 2 * np.pi * np.arange(n_theta) / n_theta
    # edge roughness r(theta, z): modes k = 2..6, top and bottom profiles
    # blended linearly in depth, scaled so the largest excursion is `roughness`
    ks = np.arange(2, 7)

    def profile():
        a = rng.standard_normal((H, len(ks)))
        b = rng.standard_normal((H, len(ks)))
        p = (a[:, :, None] * np.cos(ks[None, :, None] * theta) + b[:, :, None] * np.sin(ks[None, :, None] * theta)).sum(1)
        return p / np.abs(p).max(1, keepdims=True) * roughness

    top_p, bot_p = profile(), profile()
    zs = -depth * np.arange(n_rings + 1) / n_rings                        # 0 .. -depth
    w = (np.arange(n_rings + 1) / n_rings)[None, :, None]
    r = radius + (1 - w) * top_p[:, None, :] + w * bot_p[:, None, :]       # (H, rings+1, n_theta)
    ring = np.stack([centers[:, None, None, 0] + r * np.cos(theta),
                     centers[:, None, None, 1] + r * np.sin(theta),
                     np.broadcast_to(zs[None, :, None], r.shape)], -1)   # (H, rings+1, n_theta, 3)
    parts = []
    # hole walls (film | vacuum inside the hole): normals point to the axis
    A = ring[:, :-1]
    B = np.roll(ring[:, :-1], -1, axis=2)
    Cc = np.roll(ring[:, 1:], -1, axis=2)
    D = ring[:, 1:]
    parts.append(_quads_to_tris(A, B, Cc, D, film, V))
    # square-cell boundary points at the same angles: edge e (right, top,
    # left, bottom) and offset hp * tan(m * step) along it, built from one
    # table of tangents with explicit sign flips so that neighbouring cells
    # compute bit-identical shared vertices
    hp = pitch / 2.0
    if n_theta % 8:
        raise ValueError("n_theta must be a multiple of 8")
    q = n_theta // 8
    T = np.tan(np.arange(q + 1) * (2 * np.pi / n_theta))
    T[q] = 1.0
    sq = np.zeros((n_theta, 2))
    for j in range(n_theta):
        e = ((j + q) // (2 * q)) % 4
        m = j - e * 2 * q
        if m > q:
            m -= n_theta
        off = hp * (np.sign(m) * T[abs(m)])
        sq[j] = ((hp, off), (-off, hp), (-hp, -off), (off, -hp))[e]
    outer = centers[:, None, :] + sq[None, :, :]                          # (H, n_theta, 2)

    def annulus(inner, z, mat_in, mat_out):
        o = np.concatenate([outer, np.full(outer.shape[:2] + (1,), z)], -1)
        return _quads_to_tris(inner, o, np.roll(o, -1, axis=1), np.roll(inner, -1, axis=1), mat_in, mat_out)

    parts.append(annulus(ring[:, 0], 0.0, film, V))                       # film top (normal +z)
    parts.append(annulus(ring[:, -1], -depth, sub, film))                 # film / substrate interface
    bottom = ring[:, -1]
    ctr_b = np.concatenate([centers, np.full((H, 1), -depth)], 1)
    parts.append(_disc(ctr_b, bottom, plug, V))                           # hole floor: plug top
    low = bottom.copy()
    low[..., 2] = -depth - plug_depth
    # plug walls (plug | substrate outside): normals point away from the axis
    parts.append(_quads_to_tris(bottom, low, np.roll(low, -1, axis=1), np.roll(bottom, -1, axis=1), plug, sub))
    ctr_l = np.concatenate([centers, np.full((H, 1), -depth - plug_depth)], 1)
    parts.append(_disc(ctr_l, low[:, ::-1], plug, sub))                   # plug bottom (normal -z)
    # outer box: film and substrate sides, substrate bottom
    b = TriBuilder()
    lo, hi = -half, half
    zb = -depth - substrate
    for z0, z1, m in ((-depth, 0.0, film), (zb, -depth, sub)):
        b.quad((lo, lo, z0), (hi, lo, z0), (hi, lo, z1), (lo, lo, z1), m, V)   # -y
        b.quad((hi, hi, z0), (lo, hi, z0), (lo, hi, z1), (hi, hi, z1), m, V)   # +y
        b.quad((lo, hi, z0), (lo, lo, z0), (lo, lo, z1), (lo, hi, z1), m, V)   # -x
        b.quad((hi, lo, z0), (hi, hi, z0), (hi, hi, z1), (hi, lo, z1), m, V)   # +x
    b.quad((lo, lo, zb), (lo, hi, zb), (hi, hi, zb), (hi, lo, zb), sub, V)     # bottom (normal -z)
    m = 50.0
    b.quad((lo - m, lo - m, detector_z), (hi + m, lo - m, detector_z), (hi + m, hi + m, detector_z),
           (lo - m, hi + m, detector_z), formats.DETECTOR, formats.DETECTOR)
    parts.append(b.array())
    return np.concatenate(parts)


# ----------------------------------------------------------------------------
# Primaries
# ----------------------------------------------------------------------------
def point_beam(n, energy, pos=(0.0, 0.0, 1.0), direction=(0.0, 0.0, -1.0), pixel=(0, 0)):
    r = np.zeros(n, formats.RECORD_DTYPE)
    r["pos"] = pos
    r["dir"] = direction
    r["E"] = energy
    r["px"] = pixel[0]
    r["py"] = pixel[1]
    return r


def scan_beam(nx, ny, per_pixel, energy, spacing=1.0, origin=(-128.0, -128.0), z_start=75.0,
              sigma=1.0, divergence_deg=0.5, seed=0, energies=None, rows=None):
    """Raster scan: ``per_pixel`` primaries per pixel, Gaussian spot focused at
    z=0 (``sigma`` nm) with Gaussian angular divergence, starting at
    ``z_start``.  If ``energies`` is given, each primary's energy is drawn
    uniformly from that list.  ``rows`` restricts the scan to those y rows."""
    rng = np.random.Generator(np.random.Philox(seed))
    rows = range(ny) if rows is None else rows
    py, px = np.meshgrid(np.asarray(list(rows)), np.arange(nx), indexing="ij")
    px = np.repeat(px.ravel(), per_pixel)
    py = np.repeat(py.ravel(), per_pixel)
    n = px.size
    cx = origin[0] + px * spacing + rng.normal(0.0, sigma, n)
    cy = origin[1] + py * spacing + rng.normal(0.0, sigma, n)
    div = math.radians(divergence_deg)
    tx = np.tan(rng.normal(0.0, div, n))
    ty = np.tan(rng.normal(0.0, div, n))
    dirs = np.stack([tx, ty, -np.ones(n)], 1)
    pos = np.stack([cx - tx * z_start, cy - ty * z_start, np.full(n, z_start)], 1)
    if energies is None:
        E = np.full(n, energy)
    else:
        E = np.asarray(energies, np.float64)[rng.integers(0, len(energies), n)]
    return formats.make_records(pos, dirs, E, px, py)


def write_scan_pri(path, nx, ny, per_pixel, energy, rows_per_block=16, seed=0, **scan_kw):
    """Write a raster scan (``scan_beam`` arguments) to a ``.pri`` file,
    ``rows_per_block`` pixel rows at a time, so that a full-size scan (the
    1024 x 1024 x 200 contact-hole scan is 7.5 GB) never sits in memory.
    Block k draws from the Philox stream keyed by (seed, k).  Returns the
    number of primaries written."""
    n = 0
    with open(path, "wb") as f:
        for k, r0 in enumerate(range(0, ny, rows_per_block)):
            recs = scan_beam(nx, ny, per_pixel, energy, seed=[seed, k],
                             rows=range(r0, min(ny, r0 + rows_per_block)), **scan_kw)
            recs.tofile(f)
            n += len(recs)
    return n


# The benchmark scans (line-space grating, rough slab with mixed beam energies,
# contact-hole array): geometry, materials in geometry order, and the raster scan.
SCANS = {
    "grating": dict(geometry=lambda: grating_geometry(), materials=("si",), nx=256, ny=256, per_pixel=100,
                    energy=500.0, energies=None, spacing=1.0, origin=(-128.0, -128.0), z_start=75.0),
    "rough": dict(geometry=lambda: rough_geometry(512), materials=("si",), nx=512, ny=512, per_pixel=20,
                  energy=1000.0, energies=[300.0, 1000.0, 3000.0, 5000.0], spacing=1000.0 / 512,
                  origin=(-500.0, -500.0), z_start=25.0),
    "holes": dict(geometry=lambda: contact_hole_geometry(), materials=("sio2", "w", "si"), nx=1024, ny=1024,
                  per_pixel=200, energy=1000.0, energies=None, spacing=2.5, origin=(-1278.75, -1278.75),
                  z_start=10.0),
}


def write_workload(name, outdir, rows=None, seed=0):
    """Write one benchmark workload as reference-format inputs: ``<name>.tri``,
    one ``<kind>.mat`` per material and ``<name>.pri`` (the first ``rows``
    pixel rows of the scan, all if None).  Returns the paths, ready for
    ``nebula_b200 <tri> <pri> <mat>...``."""
    import os
    w = SCANS[name]
    os.makedirs(outdir, exist_ok=True)
    tri = os.path.join(outdir, name + ".tri")
    formats.write_tri(tri, w["geometry"]())
    mats = [make_material(os.path.join(outdir, k + ".mat"), kind=k) for k in w["materials"]]
    pri = os.path.join(outdir, name + ".pri")
    write_scan_pri(pri, w["nx"], w["ny"] if rows is None else min(rows, w["ny"]), w["per_pixel"], w["energy"],
                   seed=seed, energies=w["energies"], spacing=w["spacing"], origin=w["origin"],
                   z_start=w["z_start"])
    return {"tri": tri, "pri": pri, "mats": mats}


def main(argv=None):
    """python -m nebula_b200.generators {grating,rough,holes} OUTDIR [--rows N] [--seed S]"""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m nebula_b200.generators",
                                 description="write a benchmark workload as .tri/.mat/.pri inputs")
    ap.add_argument("workload", choices=sorted(SCANS))
    ap.add_argument("outdir")
    ap.add_argument("--rows", type=int, default=None, help="first N pixel rows of the scan (default: all)")
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    out = write_workload(args.workload, args.outdir, rows=args.rows, seed=args.seed)
    print(" ".join([out["tri"], out["pri"]] + out["mats"]))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
