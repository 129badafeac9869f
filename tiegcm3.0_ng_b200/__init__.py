"""B200-native vertical column solvers for TIE-GCM NG.

csrc/        CUDA kernels (sm_100a) and the C ABI, built into libtg_colsolve.so
colsolve.py  Python mirror of the reference interface (trsolv, trsolv_ng,
             blktri, the comp_ng block solve) and of the device/plan API
synth.py     seeded synthetic column systems of the benchmark workloads
dynamics.py  one dynamics_ng step of the column routines on the device
batch.py     builders of the batched (plan) layout for whole workloads
build.py     nvcc build of libtg_colsolve.so
"""
from . import batch, colsolve, dynamics, synth  # noqa: F401
from .colsolve import (TG_OK, TG_EINVAL, TG_EPIVOT, TG_ENONFINITE, TG_ENOCONV, TG_ETIMEOUT,  # noqa: F401
                       TG_ECUDA, TG_ENOMEM, TG_ENODEV, TG_PREC_F64, TG_PREC_F32_REFINE,
                       TG_LAYOUT_COLUMN, TG_LAYOUT_LEVEL, TG_KIND_SCALAR, TG_KIND_BLOCK2,
                       TG_KIND_BLOCK3, TG_FILTER_DT, TG_FILTER_MINOR, TG_FILTER_OPLUS, TgError, Plan, trsolv, trsolv_ng, blktri, comp_blksolve_ng, blksolve, solve_host, dt_ng, dt_ng_dev, minor_ng, minor_ng_dev, comp_ng, comp_ng_dev, comp_diag_ng, comp_diag_ng_dev, comp_post_ng, comp_post_ng_dev, time_filter_ng, time_filter_ng_dev, advec_ng, advec_ng_dev, smooth_ng, smooth_ng_dev, settei_ng, settei_ng_dev, oplus_ng, oplus_ng_dev, oplus_ng_factor_doubles, oplus_ng_factor_dev, oplus_diag_ng, oplus_diag_ng_dev, oplus_ng_solve_dev,
                       trsolv_dev, blksolve_dev, set_refine, set_host_precision, set_tile, set_pipeline, set_prefetch, set_scratch_global, set_cache_hints, set_block_rows, set_block_width, set_stage_levels, set_column_residency, set_assembly_mode, set_walk_prefetch, set_block_scratch_budget, set_scalar_scratch_budget, set_kind_overlap, set_host_pipeline, selftest_wait, selftest_division, selftest_walk, release_buffers, version, ringfilter, ringfilter_dev, filter_o2o, kernel_arch, trsolv_defer, trsolv_flush, dt_diag_ng, dt_diag_ng_dev, minor_diag_ng, minor_diag_ng_dev, dt_ng_post_dev, minor_ng_post_dev, oplus_ng_post_dev)
