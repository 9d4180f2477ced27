"""tridsolver_b200 — B200-native batched scalar tridiagonal solver.

The product is the C-ABI library lib/libtridsolver_b200.so (sm_100a kernels
behind the reference's tridDmtsvStridedBatch / tridSmtsvStridedBatch (+Inc)
entry points, include/tridsolver.h). This package binds it for Python.
"""

from .api import (  # noqa: F401
    FAMILY_AUTO, FAMILY_HYBRID, FAMILY_LONG, FAMILY_PCR, TridError, TridParams, TridStatus,
    autotune, autotune_reset, describe_plan, ragged_autotune, ragged_table, tridDmtsvRaggedBatch, tridSmtsvRaggedBatch,
    tridDmtsvRaggedBatchSized, tridSmtsvRaggedBatchSized,
    force_plan, force_stream, force_tma, force_systems_per_block, get_blocking, launch_count, on_stream, pivot_status,
    release_scratch, set_tracing,
    set_mixed_mode,
    set_blocking, set_stream, solve, solve_batched_trid, strided_batch, tridDmtsvStridedBatch,
    tridDmtsvStridedBatchAdjoint, tridDmtsvStridedBatchInc, tridDmtsvStridedBatchMixed,
    tridDmtsvStridedBatchRefine,
    tridSmtsvStridedBatch, tridSmtsvStridedBatchAdjoint, tridSmtsvStridedBatchInc)
from ._lib import LIB_PATH, load as load_library  # noqa: F401
