"""B200-native drop-in for legate-dataframe's relational hot path.

Same Python surface as the reference for this path:
``legate_dataframe.LogicalTable`` / ``LogicalColumn`` and the ops in
``legate_dataframe.lib.{join,groupby_aggregation,sort,hash_partition}``.
Every op runs hand-written sm_100a kernels through the C ABI of
``libldf_b200.so``; there is no CPU fallback.
"""

from legate_dataframe.lib.core.column import LogicalColumn
from legate_dataframe.lib.core.table import LogicalTable

__all__ = ["LogicalColumn", "LogicalTable"]
__version__ = "0.1.0"
