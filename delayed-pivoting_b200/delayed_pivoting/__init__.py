"""Python host mirror of the B200 delayed-pivoting LU.

Thin ctypes bindings over ``lib/libdelayed_lu_b200.so`` whose functions keep
the reference's interface (``delayed_lu_cuda/delayed_dgetrf_cuda.hpp``):
same names, argument meaning and error behaviour, so tests read like the
reference's own ``example.cu``.  PyTorch is used only for device memory and
streams.  Nothing here falls back to a CPU implementation: if the CUDA
library is missing, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from .api import (  # noqa: F401
    SUCCESS, INVALID_ARGUMENT, ALLOCATION_FAILED, CUDA_FAILURE, LIBRARY_FAILURE,
    DEVICE_TIMEOUT, POLICY_FULL_PIVOT, POLICY_NONZERO_COLUMN, Options, lib, matgen,
    library_path, delayed_getrf_cuda_device, delayed_getrf_cuda_host,
    delayed_getrf_cuda_native_device, delayed_getrf_cuda_native_host,
    delayed_getrf_cuda_hybrid_device, delayed_getrf_cuda_hybrid_host,
    delayed_getrf_cuda_status_string, getrf_device_ex, getrs_device, gesv_ir_device, IRResult,
    PRECISION_FP64, PRECISION_MIXED_BF16X3, PRECISION_MIXED_BF16X6, getrf_device_noalloc,
    BATCH_MAX_N, BATCH_MAX_NB, BATCH_BUCKETS, BatchOptions, Batch, BatchError, batch_options,
    batch_autotune, batch_tune_save, batch_tune_load, Factor, Server, ServerOptions, Request,
    RequestResult, ServerStats, server_options, server_clock, schur_update_device, gemm_tile, block_solve, mixed_gemm_grid, front_factor, extend_add,
    SytrfOptions, sytrf_device, sytrf_host, sytrf_last_report,
    schur_update_mixed_device, GetrfReport, getrf_last_report, getrf_autotune, getrf_tune_save,
    getrf_tune_load,
)
from .inputs import (  # noqa: F401
    normal_matrix, plant_columns, mt64_nth, planted_matrix, uniform_stream, normal_vector,
    batch_orders, batch_matrix_seed, fill_batch, batch_matrix, symmetric_matrix,
)
