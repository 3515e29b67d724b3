"""simpler_b200: the refractive radiative transfer photon march of simplEr on B200 (sm_100a).

The compute lives in libsimpler_b200.so (hand-written CUDA behind a C ABI, include/simpler_b200.h);
this package is the Python host side. Every entry point loads the library on first use and raises
if it is missing: there is no CPU fallback.
"""
from . import _lib
from ._lib import SmpError, check_layout, load
from .render import (Plan, adjoint, adjoint_sharded, field_eval, render_sharded, shard_range, field_params, param_count, records_to_arrays, render, render_batch,
                     roi_weights, sources_to_spline, trace_photons, tune_batch_steps, with_field_params)
from .scene import (Setup, bernoulli_texture, config_batch_sweep, config_planewave, config_plain_small, config_sources, config_spline,
                    config_precision, disk_texture)

__all__ = [
    "SmpError", "check_layout", "load", "Plan", "field_eval", "records_to_arrays", "render", "render_batch", "tune_batch_steps",
    "trace_photons", "config_batch_sweep", "config_spline", "config_sources", "adjoint", "field_params", "param_count",
    "roi_weights", "with_field_params", "sources_to_spline", "adjoint_sharded", "render_sharded", "shard_range",
    "Setup", "bernoulli_texture", "config_planewave", "config_plain_small", "config_precision", "disk_texture",
]
