"""Host-side mirror of icy::Model / GPU_Implementation5 over the C ABI.

icy::Model::Step (simulation/model.cpp:7-78) runs one animation frame:
UpdateEveryNthStep sub-steps (reset grid, P2G, grid update at t = dt*step,
G2P with recordPQ on the frame's first step), then transfer_from_device
(points, error code, disabled count, boundary forces divided by steps*dt),
compaction + re-sort when more than 5% of the points are disabled, and returns
SimulationTime < SimulationEndTime && !error_code.  `Model.Step` keeps that
contract; the sub-steps run on the GPU through icempm_step.
"""
import numpy as np

from .capi import Context
from .params import SimParams, Options, DISABLED_PTS_PROPORTION_THRESHOLD, N_PTS_ARRAYS
from . import hssoa as H


class Model:
    def __init__(self, prms: SimParams, grid_status, current=None, soa=None, n=0, options: Options = None,
                 capacity=None):
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
        self.gpu.step(nsub, p.SimulationStep)
        self.transfer_from_device(nsub)
        p.SimulationTime = p.InitialTimeStep * (p.SimulationStep + nsub - 1)
        p.SimulationStep += nsub
        if self.size and self.disabled_points_count / self.size > DISABLED_PTS_PROPORTION_THRESHOLD:
            self.gpu.sort_compact()
            self.hssoa, self.size = self.gpu.download(self.hssoa)
            self.disabled_points_count = 0
            self.SyncTopologyRequired = True
        return p.SimulationTime < p.SimulationEndTime and not self.error_code

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
        self.gpu.close()
