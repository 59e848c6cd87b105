"""Crack observables: the oracle's restatement and the product's host-side
mouth selection against the reference's own functions
(tests/golden/crack_obs_w3000.npz)."""
import os

import numpy as np

from oracle import crack as oc

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _g():
    with np.load(os.path.join(HERE, "crack_obs_w3000.npz")) as z:
        return {k: z[k] for k in z.files}


def test_oracle_matches_reference():
    g = _g()
    H = g["H"]
    xu, yu = H[0] / np.linalg.norm(H[0]), H[1] / np.linalg.norm(H[1])
    vx, vy = g["x0"] @ xu, g["x0"] @ yu
    x_min, x_max = vx.min(), vx.max()
    xc = 0.5 * (x_min + x_max)
    up, lo = oc.mouth_groups(vx, vy, xc, float(g["crack_plane_y"]), float(g["half_length"]))
    np.testing.assert_array_equal(up, g["upper"])
    np.testing.assert_array_equal(lo, g["lower"])
    cmod0 = vy[up].mean() - vy[lo].mean()
    for tag in ("0", "1"):
        x = g["x" + tag]
        L, ext = oc.crack_length(x, xu, yu, float(g["crack_plane_y"]), x_min, x_max, xc, float(g["half_length"]),
                                 float(g["threshold"]), int(g["bins"]))
        assert L == float(g["length" + tag]) and abs(ext - float(g["extension" + tag])) < 1e-12
        vyy = x @ yu
        assert abs((vyy[up].mean() - vyy[lo].mean() - cmod0) - float(g["cmod" + tag])) < 1e-12
    np.testing.assert_allclose(oc.project_to_lattice_axes(g["sigma"], H), g["projected"], rtol=1e-13)


def test_host_mouth_selection_matches_reference():
    from simulon_b200.batch import select_mouth_groups
    g = _g()
    H = g["H"]
    xu, yu = H[0] / np.linalg.norm(H[0]), H[1] / np.linalg.norm(H[1])
    vx, vy = g["x0"] @ xu, g["x0"] @ yu
    up, lo = select_mouth_groups(vx, vy, 0.5 * (vx.min() + vx.max()), float(g["crack_plane_y"]),
                                 float(g["half_length"]))
    np.testing.assert_array_equal(up, g["upper"])
    np.testing.assert_array_equal(lo, g["lower"])
