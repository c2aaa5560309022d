"""Neighbour counts on the device (plx_neighbour_counts, the reference's
get_neighbours) against the oracle's all-pairs restatement: bit-identical counts
for the reference's atomistic inputs, for an fcc a = 4.08 A cluster whose
nearest neighbours sit on r0 = 2.885 A, and for the Ag-Au bow-tie of the
benchmark (two metals; the reference's 17-atom Ag-Au inputs carry the
cross-element counts)."""
import os

import numpy as np
import pytest

from oracle import model
from plasmonx_b200 import configs
from plasmonx_b200 import geometry as G
from plasmonx_b200.inputs import Problem, neighbour_counts
from plasmonx_b200.solver import Context, Solver
from tests.conftest import GOLDEN, golden_dirs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def ctx():
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize('name', golden_dirs('atomistic'))
def test_device_counts_match_oracle_on_reference_inputs(ctx, name):
    p = Problem.from_keyword_file(os.path.join(GOLDEN, name, 'input.kw'))
    with Solver(p, ctx=ctx) as sv:
        nb, nn = sv.neighbours, sv.n_neighbours
    nb_o, nn_o = model.get_neighbours(p.coord_ang, p.atom_types, p.znum, len(p.type_names))
    np.testing.assert_array_equal(nn, nn_o)
    np.testing.assert_array_equal(nb, nb_o)


def _device_counts(ctx, ang, types, type_z, r0):
    from plasmonx_b200 import _lib
    n, nt = len(types), len(type_z)
    nb = np.zeros((n, nt), dtype=np.int32)
    nn = np.zeros(n, dtype=np.int32)
    ang = np.ascontiguousarray(ang, dtype=np.float64)
    types = np.ascontiguousarray(types, dtype=np.int32)
    tz = np.ascontiguousarray(type_z, dtype=np.int32)
    r0 = np.asfortranarray(r0, dtype=np.float64).ravel(order='F')
    ctx.check(ctx.lib.plx_neighbour_counts(ctx.h, n, nt, _lib.ptr(ang), _lib.ptr(types, _lib._ip),
                                           _lib.ptr(tz, _lib._ip), _lib.ptr(r0), _lib.ptr(nb, _lib._ip),
                                           _lib.ptr(nn, _lib._ip)))
    return nb.T, nn


def test_fcc_cluster_on_the_cutoff(ctx):
    pts = G.sphere('fcc', 4.08, 12.0)
    types = np.zeros(len(pts), dtype=np.int32)
    z = np.full(len(pts), 47)
    r0 = np.array([[model.R_AG0]])
    nb, nn = _device_counts(ctx, pts, types, [47], r0)
    nb_o, nn_o = model.get_neighbours(pts, types, z, 1)
    np.testing.assert_array_equal(nn, nn_o)
    np.testing.assert_array_equal(nb, nb_o)
    assert nn.max() == 13


def test_bowtie_counts_match_host_counts(ctx):
    p = configs.agau_bowtie(edge=80.0, n_freq=2)
    nb, nn = _device_counts(ctx, p.coord_ang, p.atom_types, p.type_z, p.r0)
    nb_h, nn_h = neighbour_counts(p.coord_ang, p.atom_types, p.znum, len(p.type_names))
    np.testing.assert_array_equal(nn, nn_h)
    np.testing.assert_array_equal(nb, nb_h)
    # each prism counts its own metal (the 10 A gap is wider than r0)
    assert np.all((nb[0] > 0) != (nb[1] > 0))


def test_refuses_bad_input(ctx):
    from plasmonx_b200 import _lib
    with pytest.raises(_lib.PlxError):
        _device_counts(ctx, np.zeros((2, 3)), [0, 1], [47], np.array([[model.R_AG0]]))
