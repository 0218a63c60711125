"""dynamics_b200: B200-native (sm_100a) nonbonded force and integration engine
for the molecular-dynamics library David-OConnor/dynamics.

Layers (all backed by libdynb200.so, C ABI in include/dynb200.h):
  gpu_interface  -- drop-in for the reference's src/gpu_interface.rs
  md             -- device-resident MdState / MdConfig (MdState::step)
  synth          -- seeded synthetic systems of the benchmark shapes
"""
from ._lib import DynError, lib  # noqa: F401

__all__ = ["DynError", "lib"]
