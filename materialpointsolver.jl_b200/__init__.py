"""B200-native explicit uGIMP MPM step for MaterialPointSolver.jl users.

Host-side mirror of the reference's entry point and structs over the C-ABI
library libmpm_b200.so (hand-written sm_100a CUDA kernels, include/mpm_b200.h).
"""
from .types import (Args2D, Args3D, Grid2D, Grid3D, Particle2D, Particle3D, Property,
                    VBoundary2D, VBoundary3D, UserArgs2D, UserArgs3D, UserGrid2D, UserGrid3D,
                    UserParticle2D, UserParticle3D, UserProperty, UserVBoundary2D,
                    UserVBoundary3D, meshbuilder, jl_range)
from . import workloads
from . import randomfield
from . import surrogate
from . import hdf5
from . import _lib
from .solver import (DeviceModel, host2device, device2host, clean_device, procedure,
                     materialpointsolver, time_sequence, snapshot_path)

build = _lib.build
