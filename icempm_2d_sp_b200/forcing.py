"""Host side of the current and wind forcing (the reference's
WindAndCurrentInterpolator, simulation/data_manager/windandcurrentinterpolator.{h,cpp}).

The reference reads one static current field from the "velocities" dataset of
an HDF5 file (ReadStaticFlowData, windandcurrentinterpolator.cpp:20-63) and
leaves SetTime unfinished (66-70); its Model::Step shows where SetTime would
be called (the commented line at model.cpp:26).  Here a series of current
fields and a series of coarse wind grids, each with the times they hold at,
are kept on the host; SetTime(t) uploads the two frames around t when the
bracket changes (the reference's "return whether data needs to be copied to
GPU") and has the device blend them linearly in time
(icempm_set_forcing_time), the wind also bilinearly in space.
"""
import bisect

import numpy as np


def flow_field_from_image(velocities, prms):
    """ReadStaticFlowData (windandcurrentinterpolator.cpp:20-63): the
    [height, width, 2] float32 velocity image (height = InitializationImageSizeY,
    width = InitializationImageSizeX) cut at ModeledRegionOffsetX/Y into the
    grid's current field, 2 G doubles (vx block, vy block), node j + i*GridY
    taking image pixel (i + ox) + (j + oy)*width."""
    v = np.asarray(velocities)
    w, h = prms.InitializationImageSizeX, prms.InitializationImageSizeY
    if v.ndim != 3 or v.shape != (h, w, 2):
        raise ValueError(f"velocity image must be [{h}, {w}, 2], got {list(v.shape)}")
    gx, gy, ox, oy = prms.GridXTotal, prms.GridYTotal, prms.ModeledRegionOffsetX, prms.ModeledRegionOffsetY
    if ox < 0 or oy < 0 or ox + gx > w or oy + gy > h:
        raise ValueError("the grid does not fit inside the velocity image at the modelled-region offset")
    sub = v[oy:oy + gy, ox:ox + gx, :].astype(np.float32)      # [j, i, c]
    out = np.empty(2 * gx * gy)
    out[:gx * gy] = sub[:, :, 0].T.reshape(-1)                  # node i*gy + j
    out[gx * gy:] = sub[:, :, 1].T.reshape(-1)
    return out


class _Series:
    def __init__(self, times, frames):
        t = [float(x) for x in times]
        if len(t) != len(frames) or not t:
            raise ValueError("a series needs one time per frame and at least one frame")
        if any(b <= a for a, b in zip(t, t[1:])):
            raise ValueError("frame times must increase")
        self.t, self.frames = t, frames
        self.loaded = None

    def bracket(self, time):
        """(k, weight): frames k and k+1 around `time` and the weight of k+1;
        before the first frame or after the last the end frame holds."""
        if len(self.t) == 1 or time <= self.t[0]:
            return 0, 0.0
        if time >= self.t[-1]:
            return len(self.t) - 2, 1.0
        k = bisect.bisect_right(self.t, time) - 1
        return k, (time - self.t[k]) / (self.t[k + 1] - self.t[k])

    def pair(self, k):
        return self.frames[k], self.frames[min(k + 1, len(self.frames) - 1)]


class WindAndCurrentInterpolator:
    """Time series of current fields and wind grids for one context."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.current = None
        self.wind = None
        self.wind_geom = None

    def set_current_series(self, times, fields):
        """Current fields of 2 G doubles (vx block, vy block) at `times` (s)."""
        G = self.ctx.G
        fields = [np.ascontiguousarray(f, np.float64) for f in fields]
        if any(f.size != 2 * G for f in fields):
            raise ValueError(f"each current field must hold {2 * G} values")
        self.current = _Series(times, fields)

    def set_wind_series(self, times, grids, cell, x0=0.0, y0=0.0):
        """Wind grids float32 [rows, cols, 2] (u, v; row along y, column along
        x, spacing `cell` m, sample (r, c) at world (x0 + c cell, y0 + r cell))
        at `times` (s)."""
        grids = [np.asarray(g, np.float32) for g in grids]
        if any(g.ndim != 3 or g.shape[2] != 2 or g.shape != grids[0].shape for g in grids):
            raise ValueError("wind grids must all be [rows, cols, 2]")
        self.wind = _Series(times, grids)
        self.wind_geom = (float(cell), float(x0), float(y0))

    def SetTime(self, t):
        """Upload the frames around time t where the bracket changed and blend
        them on the device; returns whether frames were uploaded."""
        uploaded = False
        tc = tw = 0.0
        if self.current is not None:
            k, tc = self.current.bracket(t)
            if self.current.loaded != k:
                a, b = self.current.pair(k)
                self.ctx.set_flow_frames(a, b)
                self.current.loaded = k
                uploaded = True
        if self.wind is not None:
            k, tw = self.wind.bracket(t)
            if self.wind.loaded != k:
                a, b = self.wind.pair(k)
                self.ctx.set_wind_frames(np.concatenate([a, b], axis=2), *self.wind_geom)
                self.wind.loaded = k
                uploaded = True
        if self.current is not None or self.wind is not None:
            self.ctx.set_forcing_time(tc, tw)
        return uploaded
