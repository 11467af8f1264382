"""Operators of the relational hot path (join, groupby_aggregation, sort, hash_partition)."""
