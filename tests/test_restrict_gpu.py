"""GPU parity of the multi-level trend's compute-or-restrict operators
(csrc/restrict_kernels.cuh through wt_restrict_scalar, wt_restrict_flux and
wt_restrict_u_source) against the CPU oracle (oracle/oracle_restrict.cpp) on
the same seeded child fields and random masks.

The restricted parent flux is compared on the owned edges of every lozenge
bit for bit (FP64 with the reference's operand order, no FMA contraction);
the sub-sampled scalar and the restricted velocity trend exactly."""
import numpy as np
import pytest

from oracle.restrict import Pair
from wavetrisk_hydrostatic_b200 import Grid
from wavetrisk_hydrostatic_b200.grid import halo_edges, halo_nodes
from wavetrisk_hydrostatic_b200.model import WaveletHierarchy

pytestmark = pytest.mark.gpu
NAMES = {"scalar": "scal", "dscalar": "dscal", "flux": "flux", "dvelo": "dvelo"}


def _setup(lmin, lmax, nz):
    G = Grid(lmin, lmax)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    dev = WaveletHierarchy(levels, [np.full(g.NN, -4000.0) for g in levels], nz)
    return levels, dev


def _owned(g, edge):
    own = np.nonzero(g.owned)[0]
    return np.concatenate([own, own + g.NN, own + 2 * g.NN]) if edge else own


@pytest.mark.parametrize("lmin,lmax,nz,masks", [(3, 5, 2, False), (3, 5, 2, True), (4, 6, 1, True)])
def test_restrictions_match_oracle(lmin, lmax, nz, masks):
    levels, dev = _setup(lmin, lmax, nz)
    rng = np.random.default_rng(lmax + 10 * masks)
    for q in range(len(levels) - 1):
        par, chd = levels[q], levels[q + 1]
        orc = Pair(par, chd, nz)
        for which, g in ((0, par), (1, chd)):
            for name in ("scalar", "dscalar", "flux", "dvelo"):
                edge = name in ("flux", "dvelo")
                a = rng.standard_normal((nz, (3 if edge else 1) * g.NN))
                (halo_edges if edge else halo_nodes)(g, a)
                orc.field(which, NAMES[name])[...] = a
                dev.upload(g.level, name, a)
            if masks:
                mn = rng.choice([0, 8, 12, 16, 32], size=g.NN).astype(np.int32)
                me = rng.choice([0, 2, 8, 12, 16], size=3 * g.NN).astype(np.int32)
            else:
                mn = np.full(g.NN, 16, np.int32)
                me = np.full(3 * g.NN, 16, np.int32)
            orc.field(which, "mask_n")[...] = mn
            orc.field(which, "mask_e")[...] = me
            dev.upload(g.level, "mask_n", mn)
            dev.upload(g.level, "mask_e", me)
        assert orc.restrict_flux() == 0
        orc.restrict_scalar()
        orc.restrict_u_source()
        dev.restrict_flux(par.level)
        dev.restrict_scalar(par.level)
        dev.restrict_u_source(par.level)
        o, d = orc.field(0, "flux"), dev.download(par.level, "flux")
        k = _owned(par, True)
        err = np.abs(d[:, k] - o[:, k]).max() / np.abs(o[:, k]).max()
        assert err == 0.0, (par.level, err)
        assert np.array_equal(dev.download(par.level, "scalar"), orc.field(0, "scal"))
        assert np.array_equal(dev.download(par.level, "dvelo"), orc.field(0, "dvelo"))
    assert dev.status() == 0
    dev.close()
