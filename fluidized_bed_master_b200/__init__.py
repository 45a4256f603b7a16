"""B200-native SPH-DEM step engine for SOPHIA_gpu (hojin9908/Fluidized_bed_master).

The product is libsphdem.so (C ABI, include/sphdem.h) built from csrc/;
this package holds its Python binding and the synthetic bed generators.
"""
from .params import DEM, F, SPH, SphdemParams, SphdemStats, reference_params  # noqa: F401


def __getattr__(name):
    if name in ("Engine", "lib", "default_params", "read_solv", "SphdemError"):
        from . import engine

        return getattr(engine, name)
    raise AttributeError(name)
