"""xyce_b200 — B200-native MOSFET device-load path of a Xyce-compatible circuit simulator.

The package holds the hot path only: per-instance BSIM4 evaluation and the stamping of F, Q,
dF/dx and dQ/dx into the DAE residual vectors and the CSR Jacobian, as hand-written sm_100a
CUDA kernels behind a C ABI (include/xyce_devload.h), plus the host-side mirror of the
reference's Device interface (``device.Bsim4Device``) and seeded workload generators
(``netlist``).
"""
from .device import (Bsim4Device, Mos1Device, MosfetDevice, ModelCard, SolverFlags, BSIM4_STATE_SLOTS,  # noqa: F401
                     BSIM4_STORE_SLOTS, MOS1_STATE_SLOTS, MOS1_STORE_SLOTS)
from . import netlist  # noqa: F401

__all__ = ["Bsim4Device", "Mos1Device", "MosfetDevice", "ModelCard", "SolverFlags", "netlist", "BSIM4_STATE_SLOTS",
           "BSIM4_STORE_SLOTS", "MOS1_STATE_SLOTS", "MOS1_STORE_SLOTS"]
