"""Generate the golden fixtures by running the reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden.py

Needs the reference project importable (pure Python + NumPy/SciPy/Numba);
``tests/golden/mplstub`` stands in for ``matplotlib.path``, which the
reference imports at load time but the BEM path never uses.  Output files:

* ``golden_tiny.npz``   trisphere(32, 10) (60 faces): geometry, near-pair
  matrix, refined coefficients g/f (before and after the closure correction),
  G1/G2/H1/H2 at 550 nm, BEMRet sigma/h at 3 wavelengths, BEMStat sigma.
* ``golden_c0.npz``     trisphere(144, 20) (284 faces), Drude gold in vacuum:
  near-pair lists, a subset of refined coefficients, the 41-wavelength
  extinction/scattering spectrum, sigma/h at 470 nm, BEMStat spectrum.
* ``golden_c1.npz``     trisphere(1444, 40) (2884 faces): near-pair list
  digest, extinction at 3 wavelengths (BEMRet) and BEMStat spectrum points.
* ``golden_rod.npz``    trirod(20, 80, [31, 21, 41]) (2400 flat faces, quads):
  near-pair list digest and one extinction value.

Only ``tests/`` read these files; nothing at run time imports the reference.
"""

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)


def _setup(ref_root):
    os.environ.setdefault('NUMBA_CACHE_DIR', '/tmp/numba_cache')
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(HERE, 'mplstub'))


def _digest(rows, cols, vals):
    h = hashlib.sha256()
    for a in (rows, cols, vals):
        h.update(np.ascontiguousarray(a, dtype=np.int64).tobytes())
    return h.hexdigest()


def main(ref_root):
    _setup(ref_root)
    from mnpbem.geometry.mesh_generators import trisphere, trirod
    from mnpbem.geometry.comparticle import ComParticle
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret import BEMRet
    from mnpbem.bem.bem_stat import BEMStat
    from mnpbem.simulation.planewave_ret import PlaneWaveRet
    from mnpbem.simulation.planewave_stat import PlaneWaveStat
    from mnpbem.greenfun.refine_utils import refinematrix
    from mnpbem.greenfun.greenret_refined import GreenRetRefined

    eps = [EpsConst(1.0), EpsDrude(*DRUDE)]

    def geom(p):
        return dict(pos=p.pos, nvec=p.nvec, tvec1=p.tvec1, tvec2=p.tvec2,
                    area=p.area, bradius=p.bradius())

    def near(p):
        ir = refinematrix(p, p).tocoo()
        order = np.lexsort((ir.col, ir.row))
        return (ir.row[order].astype(np.int64), ir.col[order].astype(np.int64),
                ir.data[order].astype(np.int64))

    # ------------------------------------------------------------ tiny
    s = trisphere(32, 10.0)
    cp = ComParticle(eps, [s], [[2, 1]], 1)
    out = {'n': s.nfaces}
    out.update({'geom_' + k: v for k, v in geom(s).items()})
    r, c, v = near(s)
    out.update(near_rows=r, near_cols=c, near_vals=v)
    raw = GreenRetRefined(s, s, deriv='cart', order=5, RelCutoff=3, AbsCutoff=0)
    out.update(ref_rows=raw.row, ref_cols=raw.col, ref_g=raw.g, ref_f_raw=raw.f)
    bem = BEMRet(cp)
    blk = bem.g.g[0][0].refined
    out.update(ref_f=blk.f)
    enei = 550.0
    G11 = bem.g.eval(0, 0, 'G', enei)
    G22 = bem.g.eval(1, 1, 'G', enei)
    H11 = bem.g.eval(0, 0, 'H1', enei)
    H22 = bem.g.eval(1, 1, 'H2', enei)
    out.update(G1_550=G11, G2_550=G22, H1_550=H11, H2_550=H22)
    exc = PlaneWaveRet(pol=[[1, 0, 0], [0, 1, 0]], dir=[[0, 0, 1], [0, 0, 1]])
    lams = np.array([400.0, 550.0, 700.0])
    out['lams'] = lams
    for i, lam in enumerate(lams):
        sig, bem = bem.solve(exc.potential(cp, lam))
        out['sig1_%d' % i] = sig.sig1
        out['sig2_%d' % i] = sig.sig2
        out['h1_%d' % i] = sig.h1
        out['h2_%d' % i] = sig.h2
        out['ext_%d' % i] = exc.extinction(sig)
        out['sca_%d' % i] = exc.scattering(sig)[0]
    bs = BEMStat(cp)
    exs = PlaneWaveStat([[1, 0, 0]])
    out['stat_F'] = bs.F
    sig, _ = bs.solve(exs.potential(cp, 550.0))
    out['stat_sig_550'] = sig.sig
    np.savez_compressed(os.path.join(HERE, 'golden_tiny.npz'), **out)
    print('tiny done')

    # ------------------------------------------------------------ C0
    s = trisphere(144, 20.0)
    cp = ComParticle(eps, [s], [[2, 1]], 1)
    out = {'n': s.nfaces}
    r, c, v = near(s)
    out.update(near_rows=r, near_cols=c, near_vals=v)
    t0 = time.time()
    bem = BEMRet(cp)
    out['ctor_s'] = time.time() - t0
    blk = bem.g.g[0][0].refined
    sub = np.arange(0, len(blk.row), 23)
    out.update(ref_sub=sub, ref_rows=blk.row[sub], ref_cols=blk.col[sub],
               ref_g=blk.g[sub], ref_f=blk.f[sub])
    exc = PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    lams = np.linspace(400, 800, 41)
    ext, sca = [], []
    t0 = time.time()
    for lam in lams:
        sig, bem = bem.solve(exc.potential(cp, lam))
        ext.append(exc.extinction(sig))
        sca.append(exc.scattering(sig)[0])
        if lam == 470.0:
            out.update(sig1_470=sig.sig1, sig2_470=sig.sig2, h1_470=sig.h1, h2_470=sig.h2)
    out['sweep_s'] = time.time() - t0
    out.update(lams=lams, ext=np.array(ext), sca=np.array(sca))
    bs = BEMStat(cp)
    exs = PlaneWaveStat([[1, 0, 0]])
    sext, ssca = [], []
    for lam in lams[::5]:
        sig, _ = bs.solve(exs.potential(cp, lam))
        sext.append(exs.extinction(sig))
        ssca.append(exs.scattering(sig))
        if lam == 520.0:
            out['stat_sig_520'] = sig.sig
    out.update(stat_lams=lams[::5], stat_ext=np.array(sext), stat_sca=np.array(ssca))
    np.savez_compressed(os.path.join(HERE, 'golden_c0.npz'), **out)
    print('c0 done')

    # ------------------------------------------------------------ C1
    s = trisphere(1444, 40.0)
    cp = ComParticle(eps, [s], [[2, 1]], 1)
    out = {'n': s.nfaces}
    r, c, v = near(s)
    out.update(near_count=len(r), near_self=int((v == 2).sum()), near_digest=_digest(r, c, v))
    t0 = time.time()
    bem = BEMRet(cp)
    out['ctor_s'] = time.time() - t0
    exc = PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    lams = np.array([400.0, 520.0, 800.0])
    ext, sca = [], []
    t0 = time.time()
    for lam in lams:
        sig, bem = bem.solve(exc.potential(cp, lam))
        ext.append(exc.extinction(sig))
        sca.append(exc.scattering(sig)[0])
    out['solve_s'] = (time.time() - t0) / len(lams)
    out.update(lams=lams, ext=np.array(ext), sca=np.array(sca))
    bs = BEMStat(cp)
    exs = PlaneWaveStat([[1, 0, 0]])
    slams = np.array([400.0, 520.0, 800.0])
    sext = []
    for lam in slams:
        sig, _ = bs.solve(exs.potential(cp, lam))
        sext.append(exs.extinction(sig))
    out.update(stat_lams=slams, stat_ext=np.array(sext))
    np.savez_compressed(os.path.join(HERE, 'golden_c1.npz'), **out)
    print('c1 done')

    # ------------------------------------------------------------ rod (flat quads)
    rod = trirod(20.0, 80.0, [31, 21, 41])
    cp = ComParticle(eps, [rod], [[2, 1]], 1)
    out = {'n': rod.nfaces}
    r, c, v = near(rod)
    out.update(near_count=len(r), near_self=int((v == 2).sum()), near_digest=_digest(r, c, v))
    bem = BEMRet(cp)
    exc = PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sig, bem = bem.solve(exc.potential(cp, 650.0))
    out.update(lam=650.0, ext=exc.extinction(sig), sca=exc.scattering(sig)[0])
    np.savez_compressed(os.path.join(HERE, 'golden_rod.npz'), **out)
    print('rod done')


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MNPBEM_REFERENCE')
    if not root:
        raise SystemExit("give the reference checkout as the first argument or in "
                         "MNPBEM_REFERENCE")
    return root


if __name__ == '__main__':
    main(reference_root())
