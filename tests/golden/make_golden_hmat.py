"""Generate the H-matrix / iterative-solver golden fixtures by running the
reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_hmat.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_hmat.py

Output ``golden_hmat.npz`` holds, per case:

* cluster tree (mnpbem/greenfun/clustertree.py): ``ind``, ``cind``, ``son``,
  ``mid``, ``rad``, ``ipart`` and the block partition of
  ``ClusterTree.admissibility`` with the wavenumber-aware criterion of
  mnpbem/greenfun/hmatrix.py:1284 (``row1/col1`` dense, ``row2/col2``
  low-rank, in the reference's dictionary order).  Cases: trisphere(144, 20)
  cleaf 32, trirod(20, 80, [31, 21, 41]) cleaf 64, a two-sphere dimer (two
  trisphere(144, 10), 2 nm gap) cleaf 32; trirod(20, 80, [97, 47, 171])
  (25,152 faces) cleaf 64 is stored as SHA-256 digests of the same arrays.
* ACA of the G(0,0) block matrix of the trirod(20, 80, [31, 21, 41]) rod at
  650 nm, cleaf 64 (mnpbem/greenfun/hmatrix.py:195): rank and relative
  Frobenius error (against the dense matrix) of every low-rank block, U and V
  of the first 12 blocks.
* BEMRetIter (mnpbem/bem/bem_ret_iter.py) sigma/h and extinction for the rod
  at 650 nm with hmatrix=True (cleaf 64, htol 1e-6, preconditioner 'none',
  GMRES tol 1e-6) with the number of operator applications GMRES made, and
  for trisphere(144, 20) at 550 nm with the dense default (hmatrix=False).

Only ``tests/`` read the output; nothing at run time imports the reference.
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


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def _ipart(cp):
    if len(cp.p) <= 1:
        return None
    return np.concatenate([np.full(part.n, i, dtype=np.int64) for i, part in enumerate(cp.p)])


def _tree_case(out, key, cp, cleaf, enei, digest_only=False):
    from mnpbem.greenfun.clustertree import ClusterTree
    from mnpbem.greenfun.hmatrix import make_kaware_fadmiss
    t0 = time.time()
    tree = ClusterTree(cp.pos, cleaf=cleaf, ipart_arr=_ipart(cp))
    adm = tree.admissibility(tree, fadmiss=make_kaware_fadmiss(2.0 * np.pi / enei, eta0=2.5))
    items = list(adm.items())
    row1 = np.array([k[0] for k, v in items if v == 2], dtype=np.int64)
    col1 = np.array([k[1] for k, v in items if v == 2], dtype=np.int64)
    row2 = np.array([k[0] for k, v in items if v == 1], dtype=np.int64)
    col2 = np.array([k[1] for k, v in items if v == 1], dtype=np.int64)
    arrs = dict(ind=tree.ind, cind=tree.cind, son=tree.son, mid=tree.mid, rad=tree.rad,
                ipart=tree.ipart, row1=row1, col1=col1, row2=row2, col2=col2)
    out[key + '_meta'] = np.array([cp.n, cleaf, enei])
    if digest_only:
        for name, a in arrs.items():
            out[key + '_sha_' + name] = np.array(_sha(a))
    else:
        for name, a in arrs.items():
            out[key + '_' + name] = np.asarray(a)
    print(key, 'nodes', tree.son.shape[0], 'dense', len(row1), 'lowrank', len(row2),
          '%.1fs' % (time.time() - t0), flush=True)


def main(ref_root):
    _setup(ref_root)
    from mnpbem.geometry.mesh_generators import trisphere, trirod
    from mnpbem.geometry.comparticle import ComParticle
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret_iter import BEMRetIter
    from mnpbem.simulation.planewave_ret import PlaneWaveRet

    eps = [EpsConst(1.0), EpsDrude(*DRUDE)]
    out = {}

    sph = ComParticle(eps, [trisphere(144, 20.0)], [[2, 1]], 1)
    rod = ComParticle(eps, [trirod(20.0, 80.0, [31, 21, 41])], [[2, 1]], 1)
    s1 = trisphere(144, 10.0).shift([-6.0, 0.0, 0.0])
    s2 = trisphere(144, 10.0).shift([6.0, 0.0, 0.0])
    dimer = ComParticle(eps, [s1, s2], [[2, 1], [2, 1]], 1, 2)
    big = ComParticle(eps, [trirod(20.0, 80.0, [97, 47, 171])], [[2, 1]], 1)

    _tree_case(out, 'sph', sph, 32, 550.0)
    _tree_case(out, 'rod', rod, 64, 650.0)
    _tree_case(out, 'dimer', dimer, 32, 600.0)
    _tree_case(out, 'big', big, 64, 500.0, digest_only=True)

    # ACA of G(0,0) at 650 nm (the inside Green function of the rod)
    enei = 650.0
    bem = BEMRetIter(rod, hmatrix=True, cleaf=64, htol=1e-6, preconditioner='none', tol=1e-6,
                     maxit=200)
    hm = bem.g.eval(0, 0, 'G', enei)
    dense = bem.g.g.eval(0, 0, 'G', enei)
    ranks, us, vs, errs = [], [], [], []
    ind = hm.tree.ind[:, 0]
    for i in range(len(hm.row2)):
        r0, r1 = hm.tree.cind[hm.row2[i]]
        c0, c1 = hm.tree.cind[hm.col2[i]]
        A = dense[np.ix_(ind[r0:r1 + 1], ind[c0:c1 + 1])]
        U, V = hm.lhs[i], hm.rhs[i]
        ranks.append(U.shape[1])
        if i < 12:
            us.append(U.ravel(order='F'))
            vs.append(V.ravel(order='F'))
        errs.append(np.linalg.norm(A - U @ V.T) / np.linalg.norm(A))
    out['aca_rank'] = np.array(ranks, dtype=np.int64)
    out['aca_U'] = np.concatenate(us)
    out['aca_V'] = np.concatenate(vs)
    out['aca_relerr'] = np.array(errs)
    print('aca blocks', len(ranks), 'mean rank', np.mean(ranks), 'max err', max(errs), flush=True)

    # BEMRetIter solves
    exc = PlaneWaveRet(np.array([[1.0, 0.0, 0.0]]), np.array([[0.0, 0.0, 1.0]]))
    count = {'n': 0}
    orig = bem._afun

    def counted(v):
        count['n'] += 1
        return orig(v)

    bem._afun = counted
    t0 = time.time()
    sig, _ = bem.solve(exc.potential(rod, enei))
    out['iter_h_sig1'] = np.asarray(sig.sig1)
    out['iter_h_sig2'] = np.asarray(sig.sig2)
    out['iter_h_h1'] = np.asarray(sig.h1)
    out['iter_h_h2'] = np.asarray(sig.h2)
    out['iter_h_ext'] = np.asarray(exc.extinction(sig))
    out['iter_h_matvecs'] = np.array(count['n'])
    g1 = bem._G1
    out['iter_h_G1_rank'] = np.array([u.shape[1] for u in g1.lhs], dtype=np.int64)
    print('iter hmatrix: matvecs', count['n'], 'ext', out['iter_h_ext'],
          '%.1fs' % (time.time() - t0), flush=True)

    t0 = time.time()
    enei = 550.0
    bemd = BEMRetIter(sph, tol=1e-6)
    sig, _ = bemd.solve(exc.potential(sph, enei))
    out['iter_d_sig1'] = np.asarray(sig.sig1)
    out['iter_d_sig2'] = np.asarray(sig.sig2)
    out['iter_d_h1'] = np.asarray(sig.h1)
    out['iter_d_h2'] = np.asarray(sig.h2)
    out['iter_d_ext'] = np.asarray(exc.extinction(sig))
    print('iter dense: ext', out['iter_d_ext'], '%.1fs' % (time.time() - t0), flush=True)

    np.savez_compressed(os.path.join(HERE, 'golden_hmat.npz'), **out)
    print('wrote golden_hmat.npz')


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MNPBEM_REFERENCE')
    if not root:
        raise SystemExit("give the reference checkout as the first argument or in "
                         "MNPBEM_REFERENCE")
    return root


if __name__ == '__main__':
    main(reference_root())
