"""SReD block-correlation hot path on NVIDIA B200 (sm_100a).

Drop-in for the 2D global and block repetition maps of SReD
(HenriquesLab/SReD): ``clutils`` and ``utils`` mirror the reference's
``CLUtils`` and ``Utils`` for this path, ``plugins`` its two commands. All
compute runs in ``libsred.so`` (C ABI in ``include/sred.h``).
"""
from . import _lib, clutils, plugins, synth, utils  # noqa: F401
from ._lib import Context, SredError  # noqa: F401

__all__ = ["Context", "SredError", "clutils", "utils", "plugins", "synth"]
