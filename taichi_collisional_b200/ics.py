"""Seeded synthetic initial conditions in Henon units (G = M = 1, E = -1/4), FP64.

The reference reads its particles from 7-column ASCII files (main.cxx:85-128: m x y z vx vy
vz) or HDF5 snapshots; it ships no generator.  These generators make inputs of the shapes
the force evaluation is measured on:

* ``plummer``: Aarseth, Henon & Wielen (1974) sampling of the Plummer sphere, radius
  truncated at ``rmax`` (in Henon units), centred on the centre of mass;
* ``kroupa_masses``: Kroupa (2001) broken power law on [0.08, 100] Msun, dN/dm ~ m^-1.3
  below 0.5 and m^-2.3 above, renormalised to total mass 1;
* ``fractal``: box fractal (Goodwin & Whitworth 2004) of dimension D: 2^3 children per
  generation, each surviving with probability 2^(D-3), positions jittered inside the
  surviving cube, velocities inherited with a Gaussian jitter and scaled to virial ratio Q.
"""
import math

import numpy as np

PLUMMER_SCALE = 3.0 * math.pi / 16.0  # Plummer length scale a in Henon units


def plummer(n, seed, rmax=10.0):
    """Equal-mass Plummer sphere; returns (x, y, z, vx, vy, vz, m) float64 arrays."""
    rng = np.random.default_rng(seed)
    pos = np.empty((n, 3))
    vel = np.empty((n, 3))
    filled = 0
    while filled < n:
        k = n - filled
        x1 = rng.uniform(1e-10, 1.0, size=k)
        r = 1.0 / np.sqrt(x1 ** (-2.0 / 3.0) - 1.0)  # Plummer units (a = 1)
        keep = r * PLUMMER_SCALE < rmax
        r = r[keep]
        k = len(r)
        if k == 0:
            continue
        ct = rng.uniform(-1.0, 1.0, size=k)
        ph = rng.uniform(0.0, 2.0 * math.pi, size=k)
        st = np.sqrt(1.0 - ct * ct)
        p = np.stack([r * st * np.cos(ph), r * st * np.sin(ph), r * ct], axis=1)
        # speed by von Neumann rejection on g(q) = q^2 (1 - q^2)^3.5
        q = np.empty(k)
        todo = np.arange(k)
        while len(todo):
            qq = rng.uniform(0.0, 1.0, size=len(todo))
            yy = rng.uniform(0.0, 0.1, size=len(todo))
            ok = yy < qq * qq * (1.0 - qq * qq) ** 3.5
            q[todo[ok]] = qq[ok]
            todo = todo[~ok]
        v = q * math.sqrt(2.0) * (1.0 + r * r) ** -0.25
        ct = rng.uniform(-1.0, 1.0, size=k)
        ph = rng.uniform(0.0, 2.0 * math.pi, size=k)
        st = np.sqrt(1.0 - ct * ct)
        w = np.stack([v * st * np.cos(ph), v * st * np.sin(ph), v * ct], axis=1)
        pos[filled:filled + k] = p * PLUMMER_SCALE
        vel[filled:filled + k] = w / math.sqrt(PLUMMER_SCALE)
        filled += k
    m = np.full(n, 1.0 / n)
    pos -= (m[:, None] * pos).sum(0) / m.sum()
    vel -= (m[:, None] * vel).sum(0) / m.sum()
    return (pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(),
            vel[:, 0].copy(), vel[:, 1].copy(), vel[:, 2].copy(), m)


def kroupa_masses(n, seed, mlo=0.08, mhi=100.0, mbreak=0.5, a1=1.3, a2=2.3):
    """Kroupa (2001) IMF masses, renormalised so that they sum to 1."""
    rng = np.random.default_rng(seed)

    def seg_int(a, lo, hi):  # integral of m^-a
        return (hi ** (1 - a) - lo ** (1 - a)) / (1 - a)

    # continuity at mbreak: k2 = k1 * mbreak^(a2 - a1)
    w1 = seg_int(a1, mlo, mbreak)
    w2 = mbreak ** (a2 - a1) * seg_int(a2, mbreak, mhi)
    u = rng.uniform(size=n)
    low = rng.uniform(size=n) < w1 / (w1 + w2)

    def inv(a, lo, hi, u):
        return (lo ** (1 - a) + u * (hi ** (1 - a) - lo ** (1 - a))) ** (1.0 / (1 - a))

    m = np.where(low, inv(a1, mlo, mbreak, u), inv(a2, mbreak, mhi, u))
    return m / m.sum()


def plummer_kroupa(n, seed, rmax=10.0):
    x, y, z, vx, vy, vz, _ = plummer(n, seed, rmax)
    m = kroupa_masses(n, seed + 7919)
    cm = np.array([(m * a).sum() for a in (x, y, z)])
    cv = np.array([(m * a).sum() for a in (vx, vy, vz)])
    return (x - cm[0], y - cm[1], z - cm[2], vx - cv[0], vy - cv[1], vz - cv[2], m)


def fractal(n, seed, dim=1.6, q_vir=0.3, potential=None):
    """Cold box fractal.  ``potential(x, y, z, m) -> phi`` (positive convention) is used
    to scale velocities to the virial ratio; without it a sampled direct estimate is used."""
    rng = np.random.default_rng(seed)
    surv = 2.0 ** (dim - 3.0)
    centres = np.zeros((1, 3))
    vels = np.zeros((1, 3))
    half = 1.0
    while len(centres) * surv * 8 < 4 * n or len(centres) < n:
        half *= 0.5
        offs = np.array([[(i >> d & 1) * 2 - 1 for d in range(3)] for i in range(8)], dtype=float) * half
        kids = (centres[:, None, :] + offs[None, :, :]).reshape(-1, 3)
        kv = np.repeat(vels, 8, axis=0) + rng.normal(scale=half, size=(len(kids), 3))
        keep = rng.uniform(size=len(kids)) < surv
        kids, kv = kids[keep], kv[keep]
        kids += rng.uniform(-0.1 * half, 0.1 * half, size=kids.shape)
        centres, vels = kids, kv
        if len(centres) > 64 * n:
            break
    pick = rng.choice(len(centres), size=n, replace=len(centres) < n)
    pos = centres[pick] + rng.uniform(-half, half, size=(n, 3))
    vel = vels[pick] + rng.normal(scale=half, size=(n, 3))
    m = np.full(n, 1.0 / n)
    pos -= pos.mean(0)
    vel -= vel.mean(0)
    x, y, z = pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()
    if potential is not None:
        phi = potential(x, y, z, m)
        w = -0.5 * float((m * phi).sum())
    else:
        k = min(n, 2048)
        idx = rng.choice(n, size=k, replace=False)
        phi = np.zeros(k)
        for c in range(0, n, 1 << 16):
            d = pos[None, c:c + (1 << 16), :] - pos[idx, None, :]
            r = np.sqrt((d * d).sum(-1))
            r[r == 0] = np.inf
            phi += (m[None, c:c + (1 << 16)] / r).sum(1)
        w = -0.5 * float(phi.mean()) * m.sum()
    t = 0.5 * float((m[:, None] * vel * vel).sum())
    vel *= math.sqrt(q_vir * abs(w) / t)
    # rescale to Henon units: E = T + W = -1/4
    e = (q_vir - 1.0) * abs(w)
    s = e / -0.25
    pos *= s
    vel /= math.sqrt(s)
    return (pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(),
            vel[:, 0].copy(), vel[:, 1].copy(), vel[:, 2].copy(), m)
