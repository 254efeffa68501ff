"""Golden Green-function entries, potentials and fields, made by running the
reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_fields.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_fields.py

Output ``golden_fields.npz``:

* trisphere(32, 10) (60 curved faces), Drude gold in vacuum, 550 nm --
  ``CompGreenRet.eval`` (mnpbem/greenfun/compgreen_ret.py:507) of the
  Cartesian derivatives Gp(0, 0), H1p(0, 0), H2p(1, 1); ``eval_block`` of F
  and H1p over columns [10, 25) (compgreen_ret.py:555); ``CompGreenStat`` G, F,
  Gp and H1p (compgreen_stat.py:678); ``BEMRet.potential`` and
  ``BEMRet.field`` (bem_ret.py:1833-1895) of the two-polarisation solution at
  inout 1 and 2.
* the dimer of golden_dimer.npz (two trisphere(144, 10) 2 nm apart, host
  eps 1.77), 600 nm, pol x / dir z: potential and field at inout 1 and 2
  (cross-particle blocks of the region-pair connectivity).

Only ``tests/`` read the output; nothing at run time imports the reference.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MNPBEM_REFERENCE')
    if not root:
        raise SystemExit("give the reference checkout as the first argument or in "
                         "MNPBEM_REFERENCE")
    return root


def _pot(out, pre, pot, inout):
    s = '1' if inout == 1 else '2'
    for name in ('phi', 'phip', 'a', 'ap'):
        key = name[:-1] + s + 'p' if name.endswith('p') else name + s
        out['%s_%s_in%d' % (pre, name, inout)] = np.asarray(getattr(pot, key))


def main(ref_root):
    os.environ.setdefault('NUMBA_CACHE_DIR', '/tmp/numba_cache')
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(HERE, 'mplstub'))
    from mnpbem.geometry.mesh_generators import trisphere
    from mnpbem.geometry.comparticle import ComParticle
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret import BEMRet
    from mnpbem.greenfun.compgreen_stat import CompGreenStat
    from mnpbem.simulation.planewave_ret import PlaneWaveRet

    out = {}
    s = trisphere(32, 10.0)
    cp = ComParticle([EpsConst(1.0), EpsDrude(*DRUDE)], [s], [[2, 1]], 1)
    bem = BEMRet(cp)
    g = bem.g
    enei = 550.0
    out['Gp_00'] = g.eval(0, 0, 'Gp', enei)
    out['H1p_00'] = g.eval(0, 0, 'H1p', enei)
    out['H2p_11'] = g.eval(1, 1, 'H2p', enei)
    out['blkF_00'] = g.eval_block(0, 0, 'F', enei, 10, 25)
    out['blkH1p_00'] = g.eval_block(0, 0, 'H1p', enei, 10, 25)
    gs = CompGreenStat(cp, cp)
    out['stat_G'] = gs.eval('G')
    out['stat_F'] = gs.eval('F')
    out['stat_Gp'] = gs.eval('Gp')
    out['stat_H1p'] = gs.eval('H1p')
    exc = PlaneWaveRet(pol=[[1, 0, 0], [0, 1, 0]], dir=[[0, 0, 1], [0, 0, 1]])
    sig, bem = bem.solve(exc.potential(cp, enei))
    for inout in (1, 2):
        _pot(out, 'sph', bem.potential(sig, inout), inout)
        f = bem.field(sig, inout)
        out['sph_e_in%d' % inout] = np.asarray(f.e)
        out['sph_h_in%d' % inout] = np.asarray(f.h)
    print('sphere done', flush=True)

    s1 = trisphere(144, 10.0).shift([-6.0, 0.0, 0.0])
    s2 = trisphere(144, 10.0).shift([6.0, 0.0, 0.0])
    cpd = ComParticle([EpsConst(1.77), EpsDrude(*DRUDE)], [s1, s2], [[2, 1], [2, 1]], 1, 2)
    bemd = BEMRet(cpd)
    excd = PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sig, bemd = bemd.solve(excd.potential(cpd, 600.0))
    for inout in (1, 2):
        _pot(out, 'dim', bemd.potential(sig, inout), inout)
        f = bemd.field(sig, inout)
        out['dim_e_in%d' % inout] = np.asarray(f.e)
        out['dim_h_in%d' % inout] = np.asarray(f.h)
    print('dimer done', flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_fields.npz'), **out)
    print('wrote golden_fields.npz')


if __name__ == '__main__':
    main(reference_root())
