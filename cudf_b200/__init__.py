"""cudf_b200 -- a B200-native (sm_100a) hash groupby-aggregate engine that is a
drop-in for libcudf's ``cudf::groupby::groupby(keys, null_policy).aggregate``
path.  The compute path is the CUDA library built by ``cudf_b200.build``; there
is no CPU fallback."""
from . import aggregation
from .column import Column, HostStaging, Table
from .batch import BatchGroupBy
from .groupby import GroupBy, GroupByRequest
from .serving import Server
from .types import Kind, NullPolicy, Sorted, TypeId
from .frame import DataFrame
from .io import groupby_parquet, read_parquet, scan_parquet

def _install_tuning():
    """Installs the measured per-size-bucket tuning rules shipped with the
    package, when present (see cudf_b200.autotune)."""
    import os
    from . import autotune
    if os.path.exists(autotune.TUNING_FILE):
        try:
            autotune.load(autotune.TUNING_FILE)
        except Exception:  # the engine library reports itself when it is used
            pass


_install_tuning()

__all__ = ["aggregation", "BatchGroupBy", "Column", "DataFrame", "HostStaging", "Table", "GroupBy", "GroupByRequest",
           "Kind", "NullPolicy", "Server", "Sorted", "TypeId", "groupby_parquet", "read_parquet", "scan_parquet"]
__version__ = "0.1.0"
