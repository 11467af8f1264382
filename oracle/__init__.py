"""CPU oracle of the relational hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may import this package, and only as the checker or the timed CPU
baseline.  The product path (``legate_dataframe`` over ``libldf_b200.so``)
never imports it and has no CPU fallback.

* ``oracle.relational``: a numpy restatement of the reference's semantics for
  join / groupby_aggregation / sort / hash_partition, each function citing the
  reference lines it follows.
* ``oracle.arrow_ref``: the reference's own CPU task bodies restated with
  pyarrow (Acero ``hashjoin`` / ``aggregate``, ``sort_indices`` + ``take``),
  i.e. the exact Arrow calls of ``JoinTask::cpu_variant``,
  ``GroupByAggregationTask::cpu_variant`` and ``SortTask::cpu_variant``.  It
  pins the numpy restatement and is the timed CPU baseline.

Pinning: the restatement is checked against the reference's golden vectors
(C++ / Python test files, committed under ``tests/golden/``) and against
``arrow_ref`` on seeded inputs.  Hash-partition bucket ids follow this
project's documented hash (the reference's cudf MURMUR3 bucket ids are not
pinned by any reference test); its parity is by properties.
"""
