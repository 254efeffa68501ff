"""The ACA oracle (oracle/hmat_oracle.py) against the reference's ACA of the
rod's inside Green function at 650 nm (golden_hmat.npz): every block rank
equal, factors equal to rounding."""
import numpy as np

from conftest import golden
from oracle import bem_oracle as bo
from oracle.hmat_oracle import HMatrixOracle
from mnpbem_b200.clustertree import BlockPartition, ClusterTree, make_kaware_fadmiss
from mnpbem_b200.geometry import ComParticle, trirod
from mnpbem_b200.materials import EpsConst, EpsDrude


def test_aca_oracle_matches_reference():
    g = golden('golden_hmat')
    cp = ComParticle([EpsConst(1.0), EpsDrude(10.0, 9.065, 0.0708)],
                     [trirod(20.0, 80.0, (31, 21, 41))], [[2, 1]], 1)
    enei = 650.0
    _, k_in = bo.eps_drude(10.0, 9.065, 0.0708, enei)
    G, _ = bo.RetGreen(cp).GF(k_in)
    tree = ClusterTree(cp.pos, 64)
    part = BlockPartition(tree, make_kaware_fadmiss(2 * np.pi / enei))
    H = HMatrixOracle(G, tree, part, htol=1e-6, kmax=100)
    assert np.array_equal(H.ranks(), g['aca_rank'])
    ou = ov = 0
    for i in range(12):
        m, n, r = part.lowrank[i, 1], part.lowrank[i, 3], g['aca_rank'][i]
        Ur = g['aca_U'][ou:ou + m * r].reshape(m, r, order='F')
        Vr = g['aca_V'][ov:ov + n * r].reshape(n, r, order='F')
        ou += m * r
        ov += n * r
        assert np.abs(H.U[i] - Ur).max() <= 1e-8 * np.abs(Ur).max()
        assert np.abs(H.V[i] - Vr).max() <= 1e-12 * np.abs(Vr).max()
