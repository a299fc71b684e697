"""bulk_b200 -- B200-native (sm_100a) device-wide algorithms with the reference's interface.

The compute lives in ``bulk_b200/lib/libbulkb200.so`` (C-ABI declared in
``include/bulk_b200.h``); this package is the host-side mirror over it.
Importing fails when the library is missing: there is no CPU fallback.
"""
from ._lib import BulkError, LIB_PATH, DECLS, lib, check  # noqa: F401
from .algorithms import (  # noqa: F401
    debug_set_fault,
    dtype_tag,
    inclusive_scan,
    merge,
    reduce,
    reduce_by_key,
    stable_sort_by_key,
    workspace_bytes,
    workspace_status,
    workspaces,
)

from .batch import (  # noqa: F401
    BATCH_MAX,
    batch_workspace_bytes,
    inclusive_scan_batch,
    reduce_by_key_batch,
    stable_sort_by_key_batch,
    stable_sort_by_key_copy_batch,
)

__version__ = "1.0.0"
