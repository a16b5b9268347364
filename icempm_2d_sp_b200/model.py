"""Host-side mirror of icy::Model / GPU_Implementation5 over the C ABI.

icy::Model::Step (simulation/model.cpp:7-78) runs one animation frame:
UpdateEveryNthStep sub-steps (reset grid, P2G, grid update at t = dt*step,
G2P with recordPQ on the frame's first step), then transfer_from_device
(points, error code, disabled count, boundary forces divided by steps*dt),
compaction + re-sort when more than 5% of the points are disabled, and returns
SimulationTime < SimulationEndTime && !error_code.  `Model.Step` keeps that
contract; the sub-steps run on the GPU through icempm_step.  With
prms.SaveSnapshots set, each frame's grid arrays are prepared on the GPU
(icempm_prepare_frame) and handed to a writer thread with the points
(SaveFrameRequest, model.cpp:75 and 104-157).
"""
import numpy as np

from .capi import Context
from .params import SimParams, Options, DISABLED_PTS_PROPORTION_THRESHOLD, N_PTS_ARRAYS
from . import hssoa as H
from .snapshot import SnapshotManager, FrameSaver
from .forcing import WindAndCurrentInterpolator


class Model:
    def __init__(self, prms: SimParams, grid_status, current=None, soa=None, n=0, options: Options = None,
                 capacity=None, title="sim1", output_root=".", point_colors_rgb=None):
        self.prms = prms.copy()
        self.grid_status_buffer = np.ascontiguousarray(grid_status, np.uint8)
        self.current = None if current is None else np.ascontiguousarray(current, np.float64)
        cap = int(capacity if capacity is not None else max(n, 1))
        self.hssoa = soa if soa is not None else H.allocate(cap)
        self.size = int(n)
        self.error_code = 0
        self.disabled_points_count = 0
        self.grid_boundary_forces = np.zeros(2 * self.prms.GridXTotal * self.prms.GridYTotal)
        self.SyncTopologyRequired = True
        self.gpu = Context(self.prms, self.grid_status_buffer, self.current, capacity=cap, options=options)
        self.gpu.upload(self.hssoa, self.size, 0)
        self.snapshot = SnapshotManager(title, output_root)
        self.point_colors_rgb = None if point_colors_rgb is None else np.asarray(point_colors_rgb, np.uint32)
        self.frame = None
        self._saver = None
        self.wac_interpolator = WindAndCurrentInterpolator(self.gpu)

    @classmethod
    def resume(cls, prms: SimParams, grid_status, snapshot_file, current=None, options: Options = None,
               capacity=None, title="sim1", output_root="."):
        """LoadParameterFile with a resume snapshot (model.cpp:196-206): points,
        SimulationStep and SimulationTime from ReadPointsFromSnapshot, point
        colours from point_colors when that file exists."""
        mgr = SnapshotManager(title, output_root)
        soa, n, step, time = mgr.ReadPointsFromSnapshot(snapshot_file, capacity)
        p = prms.copy()
        p.SimulationStep, p.SimulationTime, p.nPtsInitial = step, time, n
        try:
            colors = mgr.ReadPointColors()
        except (RuntimeError, OSError):
            colors = None
        return cls(p, grid_status, current, soa, n, options, capacity=soa.shape[1], title=title,
                   output_root=output_root, point_colors_rgb=colors)

    # Model::Prepare (model.cpp:169-178)
    def Prepare(self):
        self.gpu.update_constants(self.prms)
        self.error_code = 0
        self.gpu.set_current(self.current)

    # Model::Step (model.cpp:7-78)
    def Step(self) -> bool:
        p = self.prms
        self.gpu.clear_force_accumulator()
        nsub = p.UpdateEveryNthStep - (p.SimulationStep % p.UpdateEveryNthStep)
        # time-varying forcing, once per frame at its first sub-step (where
        # the reference's commented wind_interpolator.setTime call sits, model.cpp:26)
        wac = self.wac_interpolator
        if wac.current is not None or wac.wind is not None:
            wac.SetTime(p.InitialTimeStep * p.SimulationStep)
        self.gpu.step(nsub, p.SimulationStep)
        self.transfer_from_device(nsub)
        p.SimulationTime = p.InitialTimeStep * (p.SimulationStep + nsub - 1)
        p.SimulationStep += nsub
        if p.SaveSnapshots:
            self.frame = self.gpu.prepare_frame(nsub, self.point_colors_rgb)
        if self.size and self.disabled_points_count / self.size > DISABLED_PTS_PROPORTION_THRESHOLD:
            self.gpu.sort_compact()
            self.hssoa, self.size = self.gpu.download(self.hssoa)
            self.disabled_points_count = 0
            self.SyncTopologyRequired = True
        if p.SaveSnapshots:
            self.SaveFrameRequest()
        return p.SimulationTime < p.SimulationEndTime and not self.error_code

    # Model::SaveFrameRequest (model.cpp:104-114) and the saver thread (131-157)
    def SaveFrameRequest(self):
        if self._saver is None:
            self._saver = FrameSaver(self.snapshot)
            if self.point_colors_rgb is not None:
                self.snapshot.SavePointColors(self.point_colors_rgb)
        self._saver.request(self.prms, self.hssoa, self.size, self.frame)

    # GPU_Implementation5::transfer_from_device (gpu_implementation5.cpp:188-224)
    def transfer_from_device(self, elapsed_cycles: int):
        if self.gpu.count() > self.hssoa.shape[1]:
            raise RuntimeError("transfer_from_device capacity exceeded")
        self.hssoa, self.size = self.gpu.download(self.hssoa)
        err, dis = self.gpu.status()
        if err:
            self.error_code = err
        self.disabled_points_count = dis
        self.grid_boundary_forces = self.gpu.boundary_forces(elapsed_cycles)

    def close(self):
        try:
            if self._saver is not None:
                self._saver.close()
                self._saver = None
        finally:
            self.gpu.close()
