"""B200-native phase retrieval with the speckle.phasing API (dhparks/als_speckle)."""
from . import engine, masking, phasing, synth  # noqa: F401

__all__ = ["phasing", "engine", "masking", "synth"]
