"""xyce_b200 — B200-native MOSFET device-load path of a Xyce-compatible circuit simulator.

The package holds the hot path only: per-instance MOSFET (level 1, BSIM3, BSIM4) evaluation and the stamping of F, Q,
dF/dx and dQ/dx into the DAE residual vectors and the CSR Jacobian, as hand-written sm_100a
CUDA kernels behind a C ABI (include/xyce_devload.h), plus the host-side mirror of the
reference's Device interface (``device.Bsim4Device``, ``Bsim3Device``, ``Mos1Device``) and seeded workload generators
(``netlist``).
"""
from .device import (Bsim3Device, Bsim4Device, Mos1Device, MosfetDevice, ModelCard, SolverFlags,  # noqa: F401
                     BSIM3_STATE_SLOTS, BSIM3_STORE_SLOTS, BSIM4_STATE_SLOTS, BSIM4_STORE_SLOTS, MOS1_STATE_SLOTS,
                     MOS1_STORE_SLOTS)
from . import netlist  # noqa: F401

__all__ = ["Bsim3Device", "Bsim4Device", "Mos1Device", "MosfetDevice", "ModelCard", "SolverFlags", "netlist", "BSIM3_STATE_SLOTS",
           "BSIM3_STORE_SLOTS", "BSIM4_STATE_SLOTS", "BSIM4_STORE_SLOTS", "MOS1_STATE_SLOTS", "MOS1_STORE_SLOTS"]
