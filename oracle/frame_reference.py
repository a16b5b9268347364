"""CPU restatement of SnapshotManager::PrepareFrameArrays
(simulation/data_manager/snapshotmanager.cpp:623-765 of igorg520b/iceMPM_2d_sp)
in numpy, float64 sums (test infrastructure: the checker of the GPU frame
kernels, never on the product path).

Pinned: tests/test_frame.py checks it against the golden fixture
tests/golden/frame_ridging.npz, the output of the reference function itself
(compiled from the checkout by oracle/refbuild/build_ref.py build_frame, with
stand-ins for the rest of the Model); the reference sums in float32 in point
order, this restatement in float64.  It follows the source line by line:
  * enabled points only (utility without 0x20000);
  * quadratic B-spline weights of the cell-local position (CalculateWeightCoeffs,
    snapshotmanager.cpp:611-620), nodes (x+i)*GridY + (y+j), i, j in -1..1;
  * density += w; mass += w m; vx, vy += w m v; Jpinv, P, Q += w value;
    r, g, b += w * colour channel of point_colors_rgb[point id];
  * count[cell] += 1 (uint8);
  * per node with density > 0: v /= mass, colour /= density, Jpinv = Jpinv /
    density - 1, P, Q /= density;
  * mass_mask = density > 0.1; nodes without the mask or with status != 100
    get density, mass, v, Jpinv, P, Q = 0;
  * rgb = alpha * uint8(clamp(colour, 0, 255)) + (1 - alpha) * water, alpha =
    clamp(density, 0, 1), water = (0x15, 0x1f, 0x2f) (gui/colormap.h:36),
    truncated to uint8;
  * forces_per_region[status >= 100 ? status - 99 : status] += boundary force.
"""
import numpy as np

WATER = np.array([0x15, 0x1f, 0x2f], np.float64)
MAX_REGIONS = 100


def _u32(row):
    return np.ascontiguousarray(row).view(np.uint64).astype(np.uint64) & np.uint64(0xffffffff)


def prepare_frame(prms, soa, n, status, forces_fxfy, colors=None):
    gx, gy = prms.GridXTotal, prms.GridYTotal
    G = gx * gy
    util = _u32(soa[0, :n]).astype(np.uint32)
    cell = _u32(soa[1, :n]).astype(np.uint32)
    pid = _u32(soa[2, :n]).astype(np.uint32)
    en = (util & 0x20000) == 0
    cx = (cell & 0xffff).astype(np.int64)[en]
    cy = (cell >> 16).astype(np.int64)[en]
    x, y = soa[6, :n][en], soa[7, :n][en]
    vx, vy = soa[8, :n][en], soa[9, :n][en]
    jp, P, Q = soa[5, :n][en], soa[3, :n][en], soa[4, :n][en]
    m = prms.ParticleMass * soa[18, :n][en]
    if colors is not None:
        p = pid[en]
        col = np.where(p < len(colors), np.asarray(colors, np.uint32)[np.minimum(p, len(colors) - 1)], 0xffffff)
    else:
        col = np.full(len(cx), 0xffffff, np.uint32)
    rgbp = [((col >> 16) & 0xff).astype(np.float64), ((col >> 8) & 0xff).astype(np.float64),
            (col & 0xff).astype(np.float64)]

    def w3(t):
        return [0.5 * (0.5 - t) ** 2, 0.75 - t * t, 0.5 * (t + 0.5) ** 2]

    wx, wy = w3(x), w3(y)
    ch = {k: np.zeros(G) for k in ("density", "mass", "vx", "vy", "Jpinv", "P", "Q", "r", "g", "b")}
    for a in range(3):
        for b in range(3):
            w = wx[a] * wy[b]
            node = (cx + a - 1) * gy + (cy + b - 1)
            np.add.at(ch["density"], node, w)
            np.add.at(ch["mass"], node, w * m)
            np.add.at(ch["vx"], node, w * m * vx)
            np.add.at(ch["vy"], node, w * m * vy)
            np.add.at(ch["Jpinv"], node, w * jp)
            np.add.at(ch["P"], node, w * P)
            np.add.at(ch["Q"], node, w * Q)
            for k, c in zip(("r", "g", "b"), rgbp):
                np.add.at(ch[k], node, w * c)
    count = np.zeros(G, np.int64)
    np.add.at(count, cx * gy + cy, 1)
    d = ch["density"]
    pos = d > 0
    with np.errstate(divide="ignore", invalid="ignore"):
        ch["vx"][pos] /= ch["mass"][pos]
        ch["vy"][pos] /= ch["mass"][pos]
        for k in ("r", "g", "b", "P", "Q"):
            ch[k][pos] /= d[pos]
        ch["Jpinv"][pos] = ch["Jpinv"][pos] / d[pos] - 1.0
    mask = (d > 0.1).astype(np.uint8)
    st = np.asarray(status, np.uint8)
    off = (mask == 0) | (st != 100)
    alpha = np.clip(d, 0.0, 1.0)
    rgb = np.zeros((G, 3), np.uint8)
    for k, name in enumerate(("r", "g", "b")):
        u8 = np.floor(np.clip(ch[name], 0.0, 255.0))
        rgb[:, k] = np.floor(alpha * u8 + (1.0 - alpha) * WATER[k]).astype(np.uint8)
    for k in ("density", "mass", "vx", "vy", "Jpinv", "P", "Q"):
        ch[k][off] = 0.0
    region = np.where(st >= 100, st.astype(np.int64) - 99, st.astype(np.int64))
    fpr = np.zeros((MAX_REGIONS, 2))
    ok = region < MAX_REGIONS
    np.add.at(fpr[:, 0], region[ok], forces_fxfy[:G][ok])
    np.add.at(fpr[:, 1], region[ok], forces_fxfy[G:2 * G][ok])
    out = dict(ch)
    out.update(rgb=rgb.reshape(-1), mass_mask=mask, count=(count & 0xff).astype(np.uint8),
               forces_per_region=fpr.reshape(-1))
    return out
