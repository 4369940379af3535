"""The oracle's restatement of the reference's reconstruction (invert_bilinear_sampling and its
helpers, steady_scan.m:290-723) against hand-computed cases: the regulariser, the neighbour
finders' bounds, the push-grid's non-accumulating statements, and the inverse of an undisplaced
sampling."""
import numpy as np

from oracle import reconstruct as rc
from steadyscan_b200 import prep, synth


def test_adjacent_difference_laplacian():
    # 2 x 2 image, vertical pairs weighted vfac: pixels 0 1 (column 0), 2 3 (column 1)
    q = rc.imageadjdiffquadmat(2, 2, 0.5).toarray()
    v = 0.25
    want = np.array([[1 + v, -v, -1, 0], [-v, 1 + v, 0, -1], [-1, 0, 1 + v, -v], [0, -1, -v, 1 + v]])
    np.testing.assert_allclose(q, want)


def test_neighbour_finders_bounds():
    # 3 x 3 template: pixel (row 1, column 1) is i = 5 (1-based); its SE neighbour i = 9 = npixels
    # exists, but the finder's strict "I < npixels" drops it (steady_scan.m:695-699)
    I, Im, M = rc.calc_indices(3, 3)
    k = rc.D  # (1, 1) 0-based: row odd, column odd
    pos = list(I[k]).index(4)
    assert not M[k][pos, 3]          # SE dropped
    assert M[k][pos, 0] and Im[k][pos, 0] == 3  # N is pixel 3
    assert M[k][pos, 2] and Im[k][pos, 2] == 7  # E is pixel 7


def test_pushgrid_statements_do_not_accumulate():
    # two data pixels on the same template square: only the later one stands at each corner
    th = tw = 4
    basex = np.array([[2.25, 2.5]])
    basey = np.array([[2.0, 2.0]])
    tfrac = np.zeros((1, 2))
    pk = np.ones((1, 2), int)
    z = rc.pushgrid_resample(np.array([[10.0, 20.0]]), np.zeros(2), np.zeros(2), basex, basey, tfrac, pk, tw, th)
    # corner (2, 2) (0-based index 1 + 4 * 1 = 5): the second pixel's z / n = 20 * 0.5 / 0.5
    assert np.isclose(z[5], 20.0)


def test_first_guess_at_the_solution_gives_zeros():
    """Undisplaced frames: the push-grid guess is already the solution, the first check finds no
    decrease and the output is the initial candidate, zeros inside the mask (steady_scan.m:359-391)."""
    rng = np.random.default_rng(1)
    n = 16
    tmpl = synth.make_template(n, n, 4, (2.0, 3.0), rng)
    s = prep.init_settings({"nknots": 5}, tmpl, n, n)
    z = np.zeros((5, 1))
    out, mask, its = rc.invert_bilinear_sampling(tmpl[:, :, None].astype(np.float32), z, z, s["basex"], s["basey"],
                                                s["tfrac"], s["prevknotind"], n, n, regfac=1e-6)
    assert its == [1]
    assert np.all(out[:, :, 0][mask[:, :, 0]] == 0)


def test_subpixel_displaced_frames_reconstruct_the_template():
    """Frames sampled bilinearly at a constant sub-pixel displacement, reconstructed with their
    knots: the template inside the mask; the check interval carried from frame to frame
    (round(sqrt(7)) = 3 after a first frame of 7 sweeps)."""
    from scipy.ndimage import map_coordinates
    rng = np.random.default_rng(1)
    n = 24
    tmpl = synth.make_template(n, n, 6, (2.0, 3.0), rng)
    s = prep.init_settings({"nknots": 5}, tmpl, n, n)
    frame = map_coordinates(tmpl, [s["basey"] - 1 + 0.21, s["basex"] - 1 + 0.37], order=1, mode="nearest")
    dx = np.full((5, 3), 0.37)
    dy = np.full((5, 3), 0.21)
    out, mask, its = rc.invert_bilinear_sampling(np.stack([frame] * 3, 2).astype(np.float32), dx, dy, s["basex"],
                                                s["basey"], s["tfrac"], s["prevknotind"], n, n, regfac=1e-4)
    assert its == [7, 9, 9]
    for k in range(3):
        m = mask[:, :, k]
        assert m.sum() > 0.9 * n * n
        assert np.median(np.abs(out[:, :, k][m] - tmpl[m])) < 1e-2 * tmpl.max()
