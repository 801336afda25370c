"""shtb200 — B200-native scalar and spheroidal/toroidal spherical harmonic transforms.

Python host mirror of SHTnsKit.jl's transform API over the C ABI of
``libshtb200.so`` (``include/shtb200.h``). See ``transforms`` for the API and the
array layout conventions.
"""
from ._lib import ArgumentError, BackendUnavailableError, DimensionMismatch, load  # noqa: F401
from .config import SHTConfig, create_gauss_config, create_gauss_fly_config, gauss_nodes  # noqa: F401
from .transforms import (  # noqa: F401
    CPU, GPU, analysis, analysis_batch, analysis_divvort, analysis_divvort_batch, analysis_into, analysis_qst,
    analysis_qst_batch, analysis_sphtor, analysis_sphtor_batch, divergence_from_spheroidal,
    divergence_from_spheroidal_into, gpu_apply_laplacian, gpu_clear_cache, julia_empty, on_device,
    spheroidal_from_divergence, spheroidal_from_divergence_into, synthesis, synthesis_batch, synthesis_divvort,
    synthesis_divvort_batch, synthesis_into, synthesis_qst, synthesis_qst_batch, synthesis_sphtor,
    synthesis_sphtor_batch, to_device, to_host, toroidal_from_vorticity, toroidal_from_vorticity_into,
    vorticity_from_toroidal, vorticity_from_toroidal_into, LM_index, nlm_calc, pack_lm, unpack_lm,
    synthesis_packed, synthesis_packed_l, analysis_packed, analysis_packed_l, synthesis_packed_batch,
    analysis_packed_batch,
)

__version__ = "0.1.0"
