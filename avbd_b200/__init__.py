"""B200-native Augmented Vertex Block Descent engine.

A drop-in for the per-step solve of smtobin/avbd (SimulationExecutor::timeStep
/ VBDSolver::solve_Parallel): host code builds a context through the C-ABI of
include/avbd.h and every step runs as hand-written sm_100a kernels.
"""
from .api import (Context, EnergyRegistry, ParticlePool, SimulationContext, SimulationExecutor,  # noqa: F401
                  SimulationParams, VBDSolver)
from ._lib import AvbdError, PRECISION_FP32, PRECISION_FP64  # noqa: F401
