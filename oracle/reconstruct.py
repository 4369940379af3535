"""CPU restatement of the reference's reconstruction: TEST INFRASTRUCTURE ONLY.

Restates ``invert_bilinear_sampling`` of steady_scan.m:290-404 with ``imageadjdiffquadmat``
(:406-436), ``bilinear_map_linear_constraints`` (:438-499), ``calc_interactions`` (:501-523),
``resample_frame``/``pushgrid`` (:562-599) and ``calc_indices`` with its neighbour finders
(:645-723), keeping the reference's precision classes: the constraints and the regulariser in FP64
(MATLAB's sparse sums), the push-grid first guess and every Gauss-Seidel quantity in FP32 (the
reference's single arrays; a single/double mixed operation is evaluated in single), the energy of
the stopping rule in FP64 from FP32 iterates, with its linear term an FP32 dot product, compared in
FP32. Only tests use it, as the checker of ``ss_reconstruct_frames``.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

A, B, C, D = 0, 1, 2, 3   # colours of the 2 x 2 pattern [A B; C D]
EPS = np.finfo(np.float64).eps


def imageadjdiffquadmat(w: int, h: int, vfac: float = 1.0):
    """GtG with y(:)' GtG y(:) = sum of squared adjacent differences (vertical ones scaled by vfac)."""
    x, y = np.meshgrid(np.arange(1, w + 1), np.arange(1, h + 1))
    x = x.reshape(-1, order="F")
    y = y.reshape(-1, order="F")
    xp = np.concatenate([np.stack([x, x + 1], 1), np.stack([x, x], 1)])
    yp = np.concatenate([np.stack([y, y], 1), np.stack([y, y + 1], 1)])
    keep = np.all((xp <= w) & (yp <= h), axis=1)
    xp, yp = xp[keep], yp[keep]
    npairs = xp.shape[0]
    ind = yp + h * (xp - 1) - 1  # 0-based linear indices of the pair's pixels
    vert = xp[:, 0] == xp[:, 1]
    coef = np.where(vert, vfac, 1.0)
    G = sp.csr_matrix((np.concatenate([coef, -coef]), (np.concatenate([np.arange(npairs)] * 2),
                                                        np.concatenate([ind[:, 0], ind[:, 1]]))),
                      shape=(npairs, w * h))
    return (G.T @ G).tocsr()


def bilinear_map_linear_constraints(data, dxk, dyk, basex, basey, tfrac, prevknotind, tw: int, th: int):
    """wy (npix) and ww (npix x npix) of one frame (steady_scan.m:438-499); knots 1-based indexed."""
    pk = np.asarray(prevknotind).reshape(-1, order="F") - 1
    tf = np.asarray(tfrac, np.float64).reshape(-1, order="F")
    tc = 1 - tf
    x = np.asarray(basex, np.float64).reshape(-1, order="F") + dxk[pk] * tc + dxk[pk + 1] * tf
    y = np.asarray(basey, np.float64).reshape(-1, order="F") + dyk[pk] * tc + dyk[pk + 1] * tf
    m = (x > 1 + EPS) & (x < tw - EPS) & (y > 1 + EPS) & (y < th - EPS)
    x, y = x[m], y[m]
    d = np.asarray(data, np.float64).reshape(-1, order="F")[m]
    xi, yi = np.floor(x), np.floor(y)
    xf, yf = x - xi, y - yi
    base = (yi + th * (xi - 1) - 1).astype(np.int64)  # 0-based index of corner (yi, xi)
    corners = base[:, None] + np.array([0, 1, th, th + 1])[None, :]
    xc, yc = 1 - xf, 1 - yf
    w = np.stack([xc * yc, xc * yf, xf * yc, xf * yf], 1)
    npix = tw * th
    wy = np.bincount(corners.reshape(-1), weights=(w * d[:, None]).reshape(-1), minlength=npix)
    c1 = [0, 0, 0, 0, 1, 1, 1, 2, 2, 3]
    c2 = [0, 1, 2, 3, 1, 2, 3, 2, 3, 3]
    vals = w[:, c1] * w[:, c2]
    off = np.array(c1) != np.array(c2)
    rows = np.concatenate([corners[:, c1].reshape(-1), corners[:, c2][:, off].reshape(-1)])
    cols = np.concatenate([corners[:, c2].reshape(-1), corners[:, c1][:, off].reshape(-1)])
    v = np.concatenate([vals.reshape(-1), vals[:, off].reshape(-1)])
    ww = sp.csr_matrix((v, (rows, cols)), shape=(npix, npix))
    ww.sum_duplicates()
    return wy, ww


def _add_last_wins(a, idx, v):
    """MATLAB's a(idx) = a(idx) + v: the right side reads the old values and, where idx repeats,
    the last occurrence's assignment stands (no accumulation)."""
    last = np.full(a.shape[0], -1, np.int64)
    last[idx] = np.arange(idx.shape[0])  # numpy assigns in order: the last occurrence remains
    sel = last[idx] == np.arange(idx.shape[0])
    a[idx[sel]] = a[idx[sel]] + v[sel]


def pushgrid_resample(data, dxk, dyk, basex, basey, tfrac, prevknotind, tw: int, th: int):
    """resample_frame (steady_scan.m:562-599): FP32 push-grid d / n, NaN where n = 0. pushgrid's
    z(i) = z(i) + v statements do not accumulate repeated indices (the last data point in
    column-major order stands), and they run in the reference's order: z at the corners
    (y, x), (y+1, x), (y, x+1), (y+1, x+1), n at (y+1, x), (y, x+1), (y, x), (y+1, x+1)."""
    pk = np.asarray(prevknotind).reshape(-1, order="F") - 1
    tf = np.asarray(tfrac, np.float64).reshape(-1, order="F")
    tc = 1 - tf
    x = np.asarray(basex, np.float64).reshape(-1, order="F") + dxk[pk] * tc + dxk[pk + 1] * tf
    y = np.asarray(basey, np.float64).reshape(-1, order="F") + dyk[pk] * tc + dyk[pk + 1] * tf
    m = (x >= 1) & (x < tw) & (y >= 1) & (y < th)
    x, y = x[m], y[m]
    d = np.asarray(data).reshape(-1, order="F")[m]
    xi, yi = np.floor(x), np.floor(y)
    xf, yf = x - xi, y - yi
    mi = (yi + th * (xi - 1) - 1).astype(np.int64)
    z = np.zeros(tw * th, np.float32)
    n = np.zeros(tw * th, np.float32)
    d = d.astype(np.float32)
    w00, w10, w01, w11 = (1 - xf) * (1 - yf), (1 - xf) * yf, xf * (1 - yf), xf * yf
    for off, wgt in ((0, w00), (1, w10), (th, w01), (th + 1, w11)):
        _add_last_wins(z, mi + off, wgt.astype(np.float32) * d)
    for off, wgt in ((1, w10), (th, w01), (0, w00), (th + 1, w11)):
        _add_last_wins(n, mi + off, wgt.astype(np.float32))
    with np.errstate(invalid="ignore", divide="ignore"):
        return z / n


def calc_indices(th: int, tw: int):
    """Pixels of each colour and their 8 neighbours N NE E SE S SW W NW (0-based; an absent neighbour
    is index 0 with M false), with the reference's finders' bounds (steady_scan.m:645-723)."""
    npix = th * tw
    ind = np.arange(1, npix + 1)  # 1-based, as the finders
    r = (ind - 1) % th
    c = (ind - 1) // th
    colour = (r % 2) * 2 + (c % 2)  # [A B; C D]
    I, Im, M = [], [], []
    for k in (A, B, C, D):
        i = ind[colour == k]
        cand = [(i - 1, (i - 1) % th != 0),
                (i + th - 1, ((i + th - 1) % th != 0) & (i + th - 1 < npix)),
                (i + th, i + th <= npix),
                (i + th + 1, (i % th != 0) & (i + th + 1 < npix)),
                (i + 1, i % th != 0),
                (i - th + 1, (i % th != 0) & (i - th + 1 > 0)),
                (i - th, i - th > 0),
                (i - th - 1, i - th - 1 > 0)]
        idx = np.stack([np.where(mm, ii, 1) for ii, mm in cand], 1) - 1
        msk = np.stack([mm for _, mm in cand], 1)
        I.append(i - 1)
        Im.append(idx)
        M.append(msk)
    return I, Im, M


def invert_bilinear_sampling(frames, dx_knots, dy_knots, basex, basey, tfrac, prevknotind, th: int, tw: int,
                             regfac: float = 3e-3, aspect: float = 1.0, stop_at=None):
    """data_corrected (th x tw x n, FP32) and mask of a set's frames (steady_scan.m:290-404), the
    error-check interval carried from frame to frame; returns (corrected, mask, iterations).

    ``stop_at`` (sweeps per frame, e.g. those of another implementation) replays the iteration with
    those stopping points instead of the energy rule: every earlier check counts as a decrease. The
    stopping rule compares energies that differ between FP32 summation orders by an ulp near
    convergence; the replay compares the iterates themselves."""
    frames = np.asarray(frames)
    if frames.ndim == 2:
        frames = frames[:, :, None]
    nf = frames.shape[2]
    npix = th * tw
    regmat = imageadjdiffquadmat(tw, th, 1.0 / aspect) * regfac
    I, Im, M = calc_indices(th, tw)
    out = np.full((npix, nf), np.nan, np.float32)
    mask = np.zeros((npix, nf), bool)
    n_iter_error = 1
    iters = []
    for f in range(nf):
        dxk = np.asarray(dx_knots)[:, f].astype(np.float64)
        dyk = np.asarray(dy_knots)[:, f].astype(np.float64)
        wy, ww = bilinear_map_linear_constraints(frames[:, :, f], dxk, dyk, basex, basey, tfrac, prevknotind, tw, th)
        sww = np.asarray(ww.sum(axis=0)).reshape(-1)
        mk = sww > 0
        if not mk.any():
            iters.append(0)
            continue
        iv = pushgrid_resample(frames[:, :, f], dxk, dyk, basex, basey, tfrac, prevknotind, tw, th)
        mk &= ~np.isnan(iv)
        Q = (ww + regmat).tolil()
        dm = sp.diags(mk.astype(np.float64))
        Q = (dm @ Q.tocsr() @ dm).tocsr()
        Lfull = np.where(mk, wy, 0.0)
        Qd = Q.diagonal()
        R, Rm, L = [], [], []
        for k in (A, B, C, D):
            Rk = Qd[I[k]].astype(np.float32)
            Rmk = np.zeros(Im[k].shape, np.float32)
            nz = Rk != 0
            for j in range(8):
                q = np.asarray(Q[I[k][nz], Im[k][nz, j]]).reshape(-1).astype(np.float32)
                Rmk[nz, j] = (q / Rk[nz]) * M[k][nz, j].astype(np.float32)
            with np.errstate(invalid="ignore", divide="ignore"):
                Lk = Lfull[I[k]].astype(np.float32) / Rk
            Lk[~np.isfinite(Lk)] = 0
            R.append(Rk)
            Rm.append(Rmk)
            L.append(Lk)
        Qe = Q[mk][:, mk]
        Le = Lfull[mk].astype(np.float32)
        x = iv.astype(np.float32).copy()
        x[np.isnan(x)] = 0
        xo = np.zeros(npix, np.float32)

        def energy(v):
            vm = v[mk].astype(np.float64)
            return np.float32(vm @ (Qe @ vm) - 2.0 * np.float64(np.dot(Le, v[mk])))

        eo = energy(x)
        it = 0
        while True:
            for k in (A, B, C, D):
                prod = x[Im[k]] * Rm[k]
                s = prod[:, 0].copy()
                for j in range(1, 8):
                    s = s + prod[:, j]
                x[I[k]] = L[k] - s
            it += 1
            if it % n_iter_error == 0:
                if stop_at is not None:
                    if it >= stop_at[f]:
                        break
                    xo = x.copy()
                    continue
                e = energy(x)
                if eo <= e:
                    break
                eo = e
                xo = x.copy()
        n_iter_error = int(max(1, min(10, round_half_away(math.sqrt(np.float32(it))))))
        iters.append(it)
        xo = xo.copy()
        xo[~mk] = np.nan
        out[:, f] = xo
        mask[:, f] = mk
    return out.reshape(th, tw, nf, order="F"), mask.reshape(th, tw, nf, order="F"), iters


def round_half_away(v: float) -> float:
    """MATLAB's int32() rounding: to nearest, halves away from zero."""
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)
