"""Seeded sets of gold particles of uneven size (the batched-solve workload).

Shapes, each 256-3000 faces, drawn from one ``numpy.random.Generator``:

* spheres: ``trisphere(nv, D)``, D uniform in [10, 60] nm, nv from the
  packaged point sets (284-2446 curved faces);
* rods: cylinder with hemispherical caps (``trirod``), diameter uniform in
  [10, 30] nm, length uniform in [max(30, D + 10), 120] nm, one of four grid
  resolutions (448-1620 flat faces);
* sphere dimers: two ``trisphere(nv, D)`` on the x axis with a gap uniform in
  [1, 5] nm, D uniform in [10, 40] nm (568-2296 faces).

Gold is the Drude metal of the benchmark (eps0 = 10, wp = 9.065 eV,
gamma = 0.0708 eV) inside, the host medium a constant eps outside.  The
resolutions come from small fixed sets so that particles share face counts
and their wavelength sweeps batch together.
"""

import numpy as np

from .geometry import ComParticle, trirod, trisphere
from .materials import EpsConst, EpsDrude

__all__ = ["random_particles", "SPHERE_NV", "ROD_N", "DIMER_NV"]

DRUDE = (10.0, 9.065, 0.0708)
SPHERE_NV = (144, 256, 400, 576, 784, 1024, 1225)
ROD_N = ((17, 9, 13), (21, 11, 17), (25, 13, 21), (31, 16, 25))
DIMER_NV = (144, 256, 400, 576)


def random_particles(count=64, seed=0, eps_host=1.77, kinds=('sphere', 'rod', 'dimer')):
    """``count`` particles: list of (ComParticle, description dict)."""
    rng = np.random.default_rng(seed)
    eps = [EpsConst(eps_host), EpsDrude(*DRUDE)]
    out = []
    for _ in range(count):
        kind = kinds[int(rng.integers(len(kinds)))]
        if kind == 'sphere':
            nv = int(rng.choice(SPHERE_NV))
            d = float(np.round(rng.uniform(10.0, 60.0), 3))
            cp = ComParticle(eps, [trisphere(nv, d)], [[2, 1]], 1)
            desc = {'kind': 'sphere', 'nv': nv, 'diameter': d}
        elif kind == 'rod':
            d = float(np.round(rng.uniform(10.0, 30.0), 3))
            h = float(np.round(rng.uniform(max(30.0, d + 10.0), 120.0), 3))
            n = ROD_N[int(rng.integers(len(ROD_N)))]
            cp = ComParticle(eps, [trirod(d, h, n)], [[2, 1]], 1)
            desc = {'kind': 'rod', 'diameter': d, 'length': h, 'n': list(n)}
        else:
            nv = int(rng.choice(DIMER_NV))
            d = float(np.round(rng.uniform(10.0, 40.0), 3))
            gap = float(np.round(rng.uniform(1.0, 5.0), 3))
            s = trisphere(nv, d)
            c = 0.5 * (d + gap)
            cp = ComParticle(eps, [s.shift([-c, 0.0, 0.0]), s.shift([c, 0.0, 0.0])],
                             [[2, 1], [2, 1]], 1, 2)
            desc = {'kind': 'dimer', 'nv': nv, 'diameter': d, 'gap': gap}
        desc['faces'] = int(cp.n)
        out.append((cp, desc))
    return out
