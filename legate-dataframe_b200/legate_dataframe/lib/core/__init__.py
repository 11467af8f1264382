"""Device-resident column and table types (legate physical layout)."""
