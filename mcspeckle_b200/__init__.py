"""mcspeckle_b200 - SCMC's Monte Carlo speckle path on B200 (sm_100a).

The walk -> next-event estimation -> accumulation path of cmu-ci-lab/mcspeckle
behind its own interface: `scmc`, `MCfield`, `MCcov` and the interface/
constructors, computed by libscmc_gpu.so (C ABI in include/scmc_gpu.h).
"""
from ._lib import ScmcError, launch_count
from .interface import (HGScatter, boxArea, farFieldSource, invCDF, isotropicScatter, nearFieldSource,
                        tabulatedAmplitudeScatter)
from .fourier_quad import MCfieldFourierQuad, MCfieldFourierQuadOnWave, fq_args
from .hetero import MCCovHetro, MCsampleHetro, hetero_args
from .mc import MCcov, MCfield, MCfieldOnWave, MatlabStyleError, export_records, mc_args, philox_stream, rng
from .formats import load_amplitude_table, load_records, replay_field, save_records
from .postprocess import refocus, sample_from_cov, united_cov
from .scmc_api import ScmcInputError, scmc

__all__ = [
    "scmc", "load_amplitude_table", "load_records", "replay_field", "save_records", "refocus", "sample_from_cov", "united_cov", "MCfield", "MCcov", "MCfieldOnWave", "MCfieldFourierQuad", "MCfieldFourierQuadOnWave", "fq_args", "MCCovHetro", "MCsampleHetro", "hetero_args", "rng", "mc_args", "export_records", "philox_stream",
    "boxArea", "farFieldSource", "nearFieldSource", "isotropicScatter", "HGScatter",
    "tabulatedAmplitudeScatter", "invCDF", "ScmcError", "ScmcInputError", "MatlabStyleError", "launch_count",
]
