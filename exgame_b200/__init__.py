"""exgame_b200: a B200-native (sm_100a) implementation of exgame's per-step dynamics path —
all-pairs gravity, the joint force laws and the implicit mid-point Newton step — behind a C ABI
(include/exg.h) with a Python host mirror of the reference's World / Accelerator / Mechanism API.
"""
from . import abi  # noqa: F401
from ._lib import Device, DeviceBatch, DevicePool, DeviceWorld, ExgError, Server, host_bodies, law_lookup, world_footprint  # noqa: F401
