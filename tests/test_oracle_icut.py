"""Illumination cuts: the C++ oracle against the independent numpy
restatement, on small trees built on the CPU in the engine's node layout.
The oracle runs the reference's literal top-down cover loop
(GPU/illumcut.cu:384-440); the numpy restatement and the engine use its
closed form, so agreement here pins that form."""
import numpy as np
import pytest

from mnrt_b200 import gen
from tests import np_restate as R


@pytest.fixture(scope="module", params=[(1500, 8, 11), (2600, 16, 23)])
def tree(request):
    n, leaf, seed = request.param
    ph = gen.photons(n, seed=seed, caustic_frac=0.2)
    nodes, order = R.median_tree(ph.pos, leaf)
    return nodes, ph.pos[order], ph.pow[order]


def test_slots_normals_estimates(oracle_mod, tree):
    nodes, tpos, tpow = tree
    o = oracle_mod.icut(nodes, tpow, use_leafs=True)
    level, first, end, center = R.icut_slots(nodes)
    assert np.array_equal(o["level"], level)
    assert np.array_equal(o["first"], first) and np.array_equal(o["end"], end)
    assert np.array_equal(o["center"].view(np.uint32), center.view(np.uint32))
    normal = R.icut_normals(tpow, first, end)
    assert np.array_equal(o["normal"].view(np.uint32), normal.view(np.uint32))
    est = R.icut_estimate(tpow, first, end, center, normal)
    assert np.array_equal(o["est"].view(np.uint32), est.view(np.uint32))
    # every valid slot below the photon limit has a photon-derived normal on these walls
    valid = level != R.KINV
    assert (np.linalg.norm(normal[valid, :3], axis=1) > 0.99).all()
    # the root covers every photon
    assert first[0] == 0 and end[0] == tpos.shape[0]


@pytest.mark.parametrize("use_leafs,level_emin", [(True, 12), (False, 1), (False, 2), (False, 3), (False, 5), (False, 40)])
def test_coarse_cut(oracle_mod, tree, use_leafs, level_emin):
    nodes, tpos, tpow = tree
    o = oracle_mod.icut(nodes, tpow, use_leafs=use_leafs, level_emin=level_emin)
    coarse, emin = R.icut_coarse(nodes, o["level"], o["est"], use_leafs, level_emin)
    assert np.array_equal(o["coarse"], coarse)
    if emin is not None:
        assert np.array_equal(o["emin"].view(np.uint32), emin.view(np.uint32))
    _assert_covers_every_leaf(nodes, o["level"], coarse)


def _assert_covers_every_leaf(nodes, level, marks):
    """Every leaf has a marked slot on its path to the root (itself included)."""
    slot_parent = {}
    for j in range(nodes.shape[0]):
        for side in range(2):
            sid = 2 * j + side
            _, _, ref, cnt = R._slot(nodes, sid)
            if ref != R.KINV and cnt == 0:
                slot_parent[2 * ref] = sid
                slot_parent[2 * ref + 1] = sid
    for sid in range(2 * nodes.shape[0]):
        _, _, ref, cnt = R._slot(nodes, sid)
        if ref == R.KINV or cnt == 0:
            continue
        s, hit = sid, False
        while True:
            hit = hit or bool(marks[s])
            if s == 0:
                break
            s = slot_parent[s]
        assert hit, sid


@pytest.mark.parametrize("iters,accuracy", [(4, 0.2), (1, 0.05), (8, 0.0)])
def test_final_cut_and_interpolation(oracle_mod, tree, iters, accuracy):
    nodes, tpos, tpow = tree
    o = oracle_mod.icut(nodes, tpow, use_leafs=False, level_emin=4)
    rng = np.random.default_rng(5)
    # stand-in node-centre irradiance: the estimate perturbed, so some nodes pass and some refine
    exact = o["est"] * rng.uniform(0.7, 1.3, size=o["est"].shape).astype(np.float32)
    exact[:, 3] = 0
    fin = oracle_mod.icut_final(nodes, o["coarse"], o["est"], exact, iters, accuracy)
    want = R.icut_final(nodes, o["coarse"], o["est"], exact, iters, accuracy)
    assert np.array_equal(fin, want)
    assert fin.sum() >= o["coarse"].sum() or accuracy > 0
    _assert_covers_every_leaf(nodes, o["level"], fin)
    q = gen.queries(120, seed=9)
    irr, reached = oracle_mod.icut_interp(nodes, fin, o["center"], o["normal"], exact, q.pos, q.nrm, 0.1)
    irr2, reached2 = R.icut_interp(nodes, fin, o["center"], o["normal"], exact, q.pos, q.nrm, 0.1)
    assert np.array_equal(reached, reached2)
    np.testing.assert_allclose(irr, irr2, rtol=1e-12, atol=0)
    assert (reached > 0).mean() > 0.9


def test_caller_normals_replace_the_estimate(oracle_mod, tree):
    nodes, tpos, tpow = tree
    ns = 2 * nodes.shape[0]
    normals = np.zeros((ns, 4), np.float32)
    normals[:, 1] = 1.0   # every slot faces +y: only floor photons are in front
    o = oracle_mod.icut(nodes, tpow, use_leafs=True, normals=normals)
    assert np.array_equal(o["normal"][:, :3], normals[:, :3])
    level, first, end, center = R.icut_slots(nodes)
    est = R.icut_estimate(tpow, first, end, center, normals)
    assert np.array_equal(o["est"].view(np.uint32), est.view(np.uint32))
