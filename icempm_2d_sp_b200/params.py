"""SimParams and option structs, mirrored with ctypes.

`SimParams` is field-for-field the reference struct (simulation/parameters_sim.h:36-127);
its x86-64 layout is pinned by tests against offsets extracted from the reference
header.  `reset()` follows SimParams::Reset (parameters_sim.cpp:7-55) and
`compute_helper_variables()` follows ComputeLame/ComputeHelperVariables
(parameters_sim.cpp:122-140).
"""
import ctypes as C

# static constexpr members (parameters_sim.h:39-76)
DISABLED_PTS_PROPORTION_THRESHOLD = 0.05
PI = 3.14159265358979323846
G = 9.8
N_PTS_ARRAYS = 19
N_GRID_ARRAYS = 9

IDX_UTILITY, IDX_CELL, IDX_POINT, IDX_P, IDX_Q, IDX_JP_INV = 0, 1, 2, 3, 4, 5
IDX_POSX, IDX_VELX, IDX_FE00, IDX_BP00, IDX_THICKNESS = 6, 8, 10, 14, 18

GRID_MASS, GRID_PX, GRID_PY, GRID_NX, GRID_NY = 0, 1, 2, 3, 4
GRID_CURRENT_VX, GRID_CURRENT_VY, GRID_FX, GRID_FY = 5, 6, 7, 8

STATUS_CRUSHED = 0x10000
STATUS_DISABLED = 0x20000
STATUS_ERROR = 0x40000

ERR_POINT_POS_NAN = 0x0001
ERR_POINT_VEL_NAN = 0x0002
ERR_POINT_JUMP_CELLS = 0x0004
ERR_POINT_LEFT_AREA = 0x0008
ERR_POINT_BP_NAN = 0x0010
ERR_POINT_FE_NAN = 0x0020
ERR_GRID_P2G_NAN_VEL = 0x0100
ERR_GRID_P2G_NAN_MASS = 0x0200
ERR_GRID_NAN = 0x0400
ERR_FIXED_OVERFLOW = 0x1000
ERR_BARRIER_TIMEOUT = 0x2000

VARIANT_FIXED, VARIANT_FP32, VARIANT_FP64, VARIANT_TEXTBOOK = 0, 1, 2, 3
VARIANTS = {"fixed": VARIANT_FIXED, "fp32": VARIANT_FP32, "fp64": VARIANT_FP64, "textbook": VARIANT_TEXTBOOK}
FORCING_COMPAT, FORCING_EXTENDED = 0, 1
WIND_NONE, WIND_UNIFORM, WIND_RANKINE = 0, 1, 2


class SimParams(C.Structure):
    _fields_ = [
        ("tpb_P2G", C.c_int32), ("tpb_Upd", C.c_int32), ("tpb_G2P", C.c_int32),
        ("nPartitions", C.c_uint32),
        ("nPtsInitial", C.c_int32),
        ("SimulationStartUnixTime", C.c_int64),
        ("InitialTimeStep", C.c_double), ("SimulationEndTime", C.c_double),
        ("AnimationFramePeriod", C.c_double),
        ("SimulationStep", C.c_int32),
        ("SimulationTime", C.c_double),
        ("SaveSnapshots", C.c_bool),
        ("SnapshotPeriod", C.c_int32),
        ("GridXTotal", C.c_int32), ("GridYTotal", C.c_int32),
        ("ModeledRegionOffsetX", C.c_int32), ("ModeledRegionOffsetY", C.c_int32),
        ("InitializationImageSizeX", C.c_int32), ("InitializationImageSizeY", C.c_int32),
        ("DimensionHorizontal", C.c_double),
        ("windDragCoeff_airDensity", C.c_double),
        ("UseWindData", C.c_bool), ("UseCurrentData", C.c_bool),
        ("sea_water_density", C.c_double),
        ("waterDragEffectiveLinear", C.c_double), ("waterDragEffectiveQuadratic", C.c_double),
        ("IceDensity", C.c_double), ("PoissonsRatio", C.c_double), ("YoungsModulus", C.c_double),
        ("IceCompressiveStrength", C.c_double), ("IceTensileStrength", C.c_double),
        ("IceShearStrength", C.c_double), ("IceTensileStrength2", C.c_double),
        ("DP_phi", C.c_double), ("DP_threshold_p", C.c_double),
        ("RidgeFormationCoeff", C.c_double),
        ("cellsize", C.c_double),
        ("ParticleVolume", C.c_double), ("ParticleViewSize", C.c_double),
        ("dt_vol_Dpinv", C.c_double), ("vmax", C.c_double),
        ("lambda_", C.c_double), ("mu", C.c_double), ("kappa", C.c_double),
        ("ParticleMass", C.c_double),
        ("cellsize_inv", C.c_double), ("Dp_inv", C.c_double),
        ("UpdateEveryNthStep", C.c_int32),
    ]

    @classmethod
    def reset(cls) -> "SimParams":
        """Defaults of SimParams::Reset (parameters_sim.cpp:7-55)."""
        p = cls()
        p.nPartitions = 1
        p.UseWindData = False
        p.UseCurrentData = False
        p.SimulationStartUnixTime = 0
        p.DimensionHorizontal = 0
        p.SaveSnapshots = False
        p.SnapshotPeriod = 25
        p.nPtsInitial = 0
        p.windDragCoeff_airDensity = 0.0025 * 1.2
        p.waterDragEffectiveLinear = 0.01
        p.waterDragEffectiveQuadratic = 0.01
        p.InitialTimeStep = 3.e-5
        p.YoungsModulus = 5.e8
        p.ParticleViewSize = 2.5
        p.sea_water_density = 1030
        p.SimulationEndTime = 20000
        p.AnimationFramePeriod = 200
        p.PoissonsRatio = 0.3
        p.IceDensity = 916
        p.SimulationStep = 0
        p.SimulationTime = 0
        p.IceCompressiveStrength = 100e6
        p.IceTensileStrength = 10e6
        p.IceShearStrength = 1e6
        p.IceTensileStrength2 = 10e6
        p.RidgeFormationCoeff = 30
        p.DP_phi = 62
        p.DP_threshold_p = 1e4
        p.tpb_P2G, p.tpb_Upd, p.tpb_G2P = 256, 512, 128
        p.InitializationImageSizeX = p.InitializationImageSizeY = 0
        p.cellsize = 1.0
        p.compute_helper_variables()
        return p

    def compute_lame(self) -> None:
        """SimParams::ComputeLame (parameters_sim.cpp:122-127)."""
        E, nu = self.YoungsModulus, self.PoissonsRatio
        self.lambda_ = E * nu / ((1 + nu) * (1 - 2 * nu))
        self.mu = E / (2 * (1 + nu))
        self.kappa = self.mu * 2. / 3. + self.lambda_

    def compute_helper_variables(self) -> None:
        """SimParams::ComputeHelperVariables (parameters_sim.cpp:129-140)."""
        self.ParticleMass = self.ParticleVolume * self.IceDensity
        self.UpdateEveryNthStep = int(self.AnimationFramePeriod / self.InitialTimeStep)
        self.cellsize_inv = 1. / self.cellsize
        self.Dp_inv = 4. / (self.cellsize * self.cellsize)
        self.dt_vol_Dpinv = self.InitialTimeStep * self.ParticleVolume * self.Dp_inv
        self.vmax = 0.25 * self.cellsize / self.InitialTimeStep
        self.compute_lame()

    def animation_frame_number(self) -> int:
        return self.SimulationStep // self.UpdateEveryNthStep

    def copy(self) -> "SimParams":
        q = SimParams()
        C.memmove(C.byref(q), C.byref(self), C.sizeof(SimParams))
        return q

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class Options(C.Structure):
    """icempm_options_t (include/icempm.h)."""
    _fields_ = [
        ("variant", C.c_int32), ("forcing", C.c_int32), ("sort_every", C.c_int32),
        ("use_graphs", C.c_int32), ("block_threads", C.c_int32), ("warp_reduce", C.c_int32),
        ("device", C.c_int32), ("reserved0", C.c_int32),
        ("water_density", C.c_double), ("water_drag_coeff", C.c_double),
        ("air_density", C.c_double), ("air_drag_coeff", C.c_double),
        ("wind_kind", C.c_int32), ("reserved1", C.c_int32),
        ("wind_u", C.c_double), ("wind_v", C.c_double),
        ("wind_cx", C.c_double), ("wind_cy", C.c_double),
        ("wind_vmax", C.c_double), ("wind_radius", C.c_double),
    ]

    @classmethod
    def default(cls, **kw) -> "Options":
        o = cls()
        o.variant = VARIANT_FIXED
        o.forcing = FORCING_COMPAT
        o.sort_every = 0
        o.use_graphs = 1
        o.block_threads = 0
        o.warp_reduce = 1
        o.device = 0
        o.water_density, o.water_drag_coeff = 1025.0, 5.5e-3
        o.air_density, o.air_drag_coeff = 1.3, 1.2e-3
        o.wind_kind = WIND_NONE
        for k, v in kw.items():
            if k == "variant" and isinstance(v, str):
                v = VARIANTS[v]
            setattr(o, k, v)
        return o
