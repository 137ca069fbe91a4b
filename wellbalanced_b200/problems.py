"""Seeded initial states of the synthetic workloads (NumPy only, float64).

* ``turbulence_3d`` — 3D decaying turbulence: uniform density and pressure, velocity
  and edge vector potential drawn as Gaussian random fields with a per-mode power
  ``P(k) ~ |k|^-2`` on the integer wavenumbers ``1 <= |k| <= kmax``; the velocity is
  scaled to an rms Mach number and the potential so that the rms of the cell field
  ``|B|`` is ``b_rms``. The field is the discrete curl of the edge potential, so its
  discrete divergence is zero to round-off.
* ``orszag_tang_batch`` — many independent periodic Orszag–Tang instances with seeded
  sizes and seeded field / velocity amplitude factors.
* ``harris_sheet`` — one Harris current sheet ``B_x = tanh(y / w)`` with the density
  ``1 + sech^2(y / w) / beta`` at uniform temperature, and a seeded perturbation of the
  potential over modes 1-16.
* ``multi_blast_3d`` — overpressure spheres placed and sized from a seed.

These are workload definitions, not the reference's data; the reference publishes no
benchmark inputs for the MHD step.
"""

from __future__ import annotations

import numpy as np


def _shell_filter(shape, kmin, kmax, power):
    """sqrt(P(k)) on the half spectrum of a real FFT, zero outside kmin <= |k| <= kmax."""
    axes = [np.fft.fftfreq(n, 1.0 / n) for n in shape[:-1]] + [np.fft.rfftfreq(shape[-1], 1.0 / shape[-1])]
    kk = np.meshgrid(*axes, indexing="ij", sparse=True)
    k = np.sqrt(sum(c * c for c in kk))
    weight = np.zeros(k.shape)
    inside = (k >= kmin) & (k <= kmax)
    weight[inside] = k[inside] ** (power / 2.0)
    return weight, kk


def _random_field(rng, shape, weight, kk, shifts):
    """A real Gaussian random field filtered by ``weight``, sampled at grid + ``shifts``.

    ``shifts`` are offsets in cells along each axis (0 or 0.5), applied as phases.
    """
    from scipy import fft

    noise = rng.standard_normal(shape)
    spectrum = fft.rfftn(noise, workers=-1) * weight
    if any(shifts):
        phase = 0.0
        for k, shift, n in zip(kk, shifts, shape, strict=True):
            if shift:
                phase = phase + 2.0 * np.pi * k * shift / n
        spectrum = spectrum * np.exp(1j * phase)
    return fft.irfftn(spectrum, s=shape, workers=-1)


def _periodic_edge(values, extra):
    """Extend a periodic array by the duplicate last node along each node axis."""
    index = [np.arange(n + e) % n for n, e in zip(values.shape, extra, strict=True)]
    return values[np.ix_(*index)]


def edge_face_fields(ax, ay, az, spacing):
    """Face fields ``B_a = d_b A_c - d_c A_b`` (cyclic) from edge potentials."""
    pot = (ax, ay, az)
    faces = []
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        faces.append(np.diff(pot[c], axis=b) / spacing[b] - np.diff(pot[b], axis=c) / spacing[c])
    return faces


def cell_fields_from_faces(faces):
    out = []
    for a, f in enumerate(faces):
        n = f.shape[a]
        lo = np.take(f, np.arange(0, n - 1), axis=a)
        hi = np.take(f, np.arange(1, n), axis=a)
        out.append(0.5 * (lo + hi))
    return out


def turbulence_3d(n, *, seed=0, kmin=1.0, kmax=8.0, mach=1.0, b_rms=1.0, gamma=5.0 / 3.0,
                  rho=1.0, pressure=1.0):
    """Initial state of the 3D decaying-turbulence workload on ``n^3`` cells of [0,1]^3.

    Returns ``(rho, (u, v, w), p, (ax, ay, az))``: cell arrays ``(n, n, n)`` and edge
    potentials with their periodic duplicate nodes — x-edges ``(n, n+1, n+1)``, y-edges
    ``(n+1, n, n+1)``, z-edges ``(n+1, n+1, n)``.
    """
    rng = np.random.default_rng(seed)
    shape = (n, n, n)
    weight, kk = _shell_filter(shape, kmin, kmax, -2.0)
    velocity = [_random_field(rng, shape, weight, kk, (0.0, 0.0, 0.0)) for _ in range(3)]
    speed = np.sqrt(np.mean(sum(v * v for v in velocity)))
    sound = np.sqrt(gamma * pressure / rho)
    velocity = [v * (mach * sound / speed) for v in velocity]
    shifts = ((0.5, 0.0, 0.0), (0.0, 0.5, 0.0), (0.0, 0.0, 0.5))
    extras = ((0, 1, 1), (1, 0, 1), (1, 1, 0))
    potential = [
        _periodic_edge(_random_field(rng, shape, weight, kk, s), e)
        for s, e in zip(shifts, extras, strict=True)
    ]
    h = 1.0 / n
    cells = cell_fields_from_faces(edge_face_fields(*potential, (h, h, h)))
    size = np.sqrt(np.mean(sum(c * c for c in cells)))
    potential = [a * (b_rms / size) for a in potential]
    return (
        np.full(shape, rho),
        tuple(velocity),
        np.full(shape, pressure),
        tuple(potential),
    )


def conserved_3d(rho, velocity, p, potential, spacing, gamma=5.0 / 3.0, mean_field=(0.0, 0.0, 0.0)):
    """Conserved cell fields (rho, m_x, m_y, m_z, E) of a state with edge potentials."""
    faces = edge_face_fields(*potential, spacing)
    faces = [f + b for f, b in zip(faces, mean_field, strict=True)]
    bx, by, bz = cell_fields_from_faces(faces)
    u, v, w = velocity
    energy = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w) + 0.5 * (bx * bx + by * by + bz * bz)
    return rho, rho * u, rho * v, rho * w, energy


def orszag_tang_sizes(count, *, seed=0, sides=tuple(range(32, 257, 16))):
    """Seeded per-instance sides and (field, velocity) amplitude factors in [0.5, 1.5]."""
    rng = np.random.default_rng(seed)
    n = rng.choice(np.asarray(sides), size=count)
    b_factor = rng.uniform(0.5, 1.5, size=count)
    v_factor = rng.uniform(0.5, 1.5, size=count)
    return n.astype(int), b_factor, v_factor


def orszag_tang_2d(n, b_factor=1.0, v_factor=1.0, gamma=5.0 / 3.0):
    """Orszag–Tang state on ``n^2`` cells of the periodic unit square.

    Returns ``(rho, mx, my, mz, E, bz)`` cell arrays and ``A_z`` at the ``(n+1)^2``
    nodes: density ``25/(36 pi)``, pressure ``5/(12 pi)``, velocity ``v_factor *
    (-sin 2 pi y, sin 2 pi x)``, ``A_z = b_factor * B0 (cos 4 pi x / 4 pi + cos 2 pi y / 2 pi)``.
    """
    h = 1.0 / n
    xc = (np.arange(n) + 0.5) * h
    xn = np.arange(n + 1) * h
    x, y = np.meshgrid(xc, xc, indexing="ij")
    xnn, ynn = np.meshgrid(xn, xn, indexing="ij")
    b0 = b_factor / np.sqrt(4.0 * np.pi)
    az = b0 * (np.cos(4 * np.pi * xnn) / (4 * np.pi) + np.cos(2 * np.pi * ynn) / (2 * np.pi))
    rho = np.full((n, n), 25.0 / (36.0 * np.pi))
    p = np.full((n, n), 5.0 / (12.0 * np.pi))
    u = -v_factor * np.sin(2 * np.pi * y)
    v = v_factor * np.sin(2 * np.pi * x)
    bxf = (az[:, 1:] - az[:, :-1]) / h
    byf = -(az[1:, :] - az[:-1, :]) / h
    bx = 0.5 * (bxf[:-1] + bxf[1:])
    by = 0.5 * (byf[:, :-1] + byf[:, 1:])
    energy = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v) + 0.5 * (bx * bx + by * by)
    zeros = np.zeros((n, n))
    return (rho, rho * u, rho * v, zeros.copy(), energy, zeros.copy()), az


def harris_sheet(nx, ny, *, width=0.05, beta=0.2, amplitude=1e-3, modes=16, seed=0,
                 bounds=((-1.0, 1.0), (-2.0, 2.0))):
    """Callables ``(density, pressure, A_z)`` of one perturbed Harris sheet.

    ``A_z = w ln cosh(y / w)`` gives ``B_x = tanh(y / w)``; the density ``1 + sech^2(y/w) /
    beta`` at uniform temperature ``beta / 2`` gives ``p + B^2 / 2 = const``; the seeded
    perturbation ``amplitude * sum_m a_m cos(2 pi m (x - x0) / Lx + phi_m) * exp(-(y /
    2w)^2)`` over modes 1..``modes`` (normalised so the sum of |a_m| is 1).
    """
    rng = np.random.default_rng(seed)
    (x0, x1), _ = bounds
    lx = x1 - x0
    m = np.arange(1, modes + 1)
    phases = rng.uniform(0.0, 2.0 * np.pi, modes)
    weights = rng.standard_normal(modes)
    weights = weights / np.sum(np.abs(weights))

    def potential(x, y):
        base = width * np.log(np.cosh(y / width))
        wave = 0.0
        for mode, phase, weight in zip(m, phases, weights, strict=True):
            wave = wave + weight * np.cos(2.0 * np.pi * mode * (x - x0) / lx + phase)
        return base + amplitude * wave * np.exp(-((y / (2.0 * width)) ** 2))

    def density(x, y):
        return 1.0 + 1.0 / np.cosh(y / width) ** 2 / beta

    def pressure(x, y):
        return 0.5 * beta * density(x, y)

    return density, pressure, potential


def multi_blast_3d(n, *, seed=0, count=8, background=0.1, inside=10.0, radii=(0.05, 0.1)):
    """Pressure of ``count`` seeded overpressure spheres on ``n^3`` cells of [0,1]^3."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.15, 0.85, size=(count, 3))
    radius = rng.uniform(radii[0], radii[1], size=count)
    h = 1.0 / n
    c = (np.arange(n) + 0.5) * h
    x, y, z = np.meshgrid(c, c, c, indexing="ij")
    p = np.full((n, n, n), background)
    for centre, r in zip(centres, radius, strict=True):
        d2 = (x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2
        p[d2 < r * r] = inside
    return p
