/*
 * ldf_b200.h -- C ABI of the B200-native relational hot path (join, groupby
 * aggregation, sort, local hash partition) of legate-dataframe.
 *
 * Every entry point replaces the libcudf calls made inside one legate GPU task
 * body of the reference.  The task body keeps reading its arguments exactly as
 * it does today (same order, same TaskContext); instead of building cudf views
 * it fills `ldf_column` descriptors straight from the legate physical stores
 * (data, bool-per-row null mask, Rect<1> string ranges + chars) and calls one
 * function below on `ctx.stream()`.
 *
 * Conventions
 *  - Plain C: pointers, sizes, int status.  No cudf/legate/torch types.
 *  - `stream` is a cudaStream_t passed as void*.  All device work is ordered on
 *    it; the only host synchronisation is the read-back of an output row count.
 *  - Inputs are borrowed and read-only.  Outputs are allocated through the
 *    caller's `ldf_allocator` (legate: `legate::create_buffer`-backed, never
 *    cudaMalloc inside a task) and handed back for zero-copy binding.  A NULL
 *    allocator selects stream-ordered cudaMallocAsync/cudaFreeAsync.
 *  - Status: 0 on success; otherwise an LDF_ERR_* code and a message readable
 *    with ldf_b200_last_error() (thread-local).  Host wrappers rethrow them as
 *    std::invalid_argument / std::runtime_error like the reference does.
 */
#ifndef LDF_B200_H
#define LDF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  LDF_OK                   = 0,
  LDF_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
  LDF_ERR_CUDA             = 2, /* LDF_CUDA_TRY failure (utils.hpp:241-245) */
  LDF_ERR_OUT_OF_MEMORY    = 3, /* allocator returned NULL */
  LDF_ERR_UNSUPPORTED      = 4, /* type/aggregation not supported */
  LDF_ERR_TIMEOUT          = 5, /* a bounded device-side wait expired */
  LDF_ERR_INTERNAL         = 6
};

/* ---- column types (Arrow logical types used by the path) ---------------- */
enum {
  LDF_BOOL8   = 1, /* arrow bool, stored one byte per row (legate layout) */
  LDF_INT8    = 2,
  LDF_INT16   = 3,
  LDF_INT32   = 4,
  LDF_INT64   = 5,
  LDF_UINT8   = 6,
  LDF_UINT16  = 7,
  LDF_UINT32  = 8,
  LDF_UINT64  = 9,
  LDF_FLOAT32 = 10,
  LDF_FLOAT64 = 11,
  LDF_STRING  = 12, /* legate string: Rect<1> ranges + int8 chars */
  LDF_TIMESTAMP_US = 13 /* int64 microseconds */
};

/* legate::Rect<1> of a string row: inclusive global [lo, hi] char range. */
typedef struct {
  int64_t lo;
  int64_t hi;
} ldf_range;

/* One column in the legate physical layout (core/column.hpp:454-671).
 *  data       fixed width: `size` values; LDF_STRING: `size` ldf_range
 *  valid      legate null mask, one byte per row, nonzero = valid; NULL when
 *             the column is not nullable
 *  chars      LDF_STRING only: character bytes; global char position p is
 *             chars[p - chars_base]
 */
typedef struct {
  int32_t type;
  int32_t nullable; /* output columns: set by the library; inputs: valid != NULL */
  int64_t size;
  void* data;
  uint8_t* valid;
  char* chars;
  int64_t chars_base;
  int64_t num_chars;
} ldf_column;

/* Device memory for outputs and scratch (legate TaskMemoryResource,
 * core/allocator.cu:27-81). `allocate` returns NULL on failure. */
typedef struct {
  void* ctx;
  void* (*allocate)(void* ctx, size_t nbytes, void* stream);
  void (*deallocate)(void* ctx, void* ptr, size_t nbytes, void* stream);
} ldf_allocator;

/* ---- join --------------------------------------------------------------- */
enum { LDF_JOIN_INNER = 0, LDF_JOIN_LEFT = 1, LDF_JOIN_FULL = 2, LDF_JOIN_SEMI = 3, LDF_JOIN_ANTI = 4 };

/* Hash join: build on `rhs`, probe with `lhs`; the output holds the lhs_out
 * columns followed by the rhs_out columns.  LEFT makes every rhs output column
 * nullable, FULL every output column (join.cpp:348-383).  `out` has
 * n_lhs_out + n_rhs_out entries and is filled by the call.
 * Replaces cudf_join + cudf::gather in JoinTask::gpu_variant (join.cu:32-155);
 * semantics of JoinTask::cpu_variant (join.cpp:168-228). */
int ldf_b200_join(const ldf_column* lhs, int32_t lhs_ncols,
                  const ldf_column* rhs, int32_t rhs_ncols,
                  const int32_t* lhs_keys, const int32_t* rhs_keys, int32_t nkeys,
                  int32_t join_type, int32_t nulls_equal,
                  const int32_t* lhs_out, int32_t n_lhs_out,
                  const int32_t* rhs_out, int32_t n_rhs_out,
                  ldf_column* out, const ldf_allocator* alloc, void* stream);

/* ---- groupby aggregation ------------------------------------------------ */
enum {
  LDF_AGG_SUM            = 0,
  LDF_AGG_MIN            = 1,
  LDF_AGG_MAX            = 2,
  LDF_AGG_COUNT          = 3,
  LDF_AGG_COUNT_ALL      = 4,
  LDF_AGG_MEAN           = 5,
  LDF_AGG_COUNT_DISTINCT = 6,
  LDF_AGG_PRODUCT        = 7,
  LDF_AGG_VARIANCE       = 8,
  LDF_AGG_STDDEV         = 9
};
/* arrow::compute::CountOptions::CountMode */
enum { LDF_COUNT_ONLY_VALID = 0, LDF_COUNT_ONLY_NULL = 1, LDF_COUNT_ALL = 2 };

typedef struct {
  int32_t in_col;     /* input column (ignored for COUNT_ALL) */
  int32_t kind;       /* LDF_AGG_* */
  int32_t count_mode; /* LDF_COUNT_* for COUNT / COUNT_DISTINCT */
  int32_t out_type;   /* output LDF_* type (the Arrow hash_<kind> result type) */
} ldf_aggregation;

/* Hash groupby: output = key columns then one column per aggregation, in
 * request order; null keys form a group (null_policy::INCLUDE).  Output row
 * order is unspecified.  Replaces the cudf::groupby call in
 * GroupByAggregationTask::gpu_variant (groupby_aggregation.cu:90-167);
 * semantics of the Acero hash_* aggregations (groupby_aggregation.cpp:41-94).
 * Input buffers may also be host memory (pinned, or pageable at lower copy
 * speed): such columns are copied to the device inside the call on a side
 * stream, keys first, and each pass starts as soon as the columns it reads
 * have arrived; the host buffers must stay valid until `stream` has passed
 * the end of the call. */
int ldf_b200_groupby_aggregation(const ldf_column* table, int32_t ncols,
                                 const int32_t* keys, int32_t nkeys,
                                 const ldf_aggregation* aggs, int32_t naggs,
                                 ldf_column* out, const ldf_allocator* alloc, void* stream);

/* ---- sort --------------------------------------------------------------- */
/* Stable lexicographic sort of the whole table on `keys`.  `nulls_at_end`
 * applies to every key regardless of direction (sort.cu:309-323).
 * `limit` = INT64_MIN for none, >0 head, <0 tail (sort.cu:275-291).
 * The sort is always stable, so `stable` only documents the request.
 * Replaces cudf::(stable_)sort_by_key in SortTask::gpu_variant (sort.cu:325-330). */
int ldf_b200_sort(const ldf_column* table, int32_t ncols,
                  const int32_t* keys, const uint8_t* ascending, int32_t nkeys,
                  int32_t nulls_at_end, int32_t stable, int64_t limit,
                  ldf_column* out, const ldf_allocator* alloc, void* stream);

/* ---- local hash partition ---------------------------------------------- */
/* Reorder the table so that rows of bucket b (= hash(keys) % nparts) are
 * contiguous, buckets in order, input order kept inside a bucket.
 * `offsets` (host, nparts + 1 entries) receives the bucket start offsets and
 * the total.  Replaces cudf::hash_partition + cudf::split in
 * task::repartition_by_hash (core/repartition_by_hash.cu:296-310). */
int ldf_b200_hash_partition(const ldf_column* table, int32_t ncols,
                            const int32_t* keys, int32_t nkeys, int32_t nparts,
                            ldf_column* out, int64_t* offsets,
                            const ldf_allocator* alloc, void* stream);

/* ---- distinct ------------------------------------------------------------ */
/* One row per distinct combination of the `keys` columns; `out` receives
 * every column of `table` (ncols entries), whole rows of one representative
 * input row per group (for non-key columns "any value is possible").  Null
 * keys form one group.  Output row order is unspecified.  Replaces
 * cudf::distinct in DistinctTask::gpu_variant (stream_compaction.cu:45-76);
 * semantics of legate::dataframe::distinct (stream_compaction.cpp:121-150). */
int ldf_b200_distinct(const ldf_column* table, int32_t ncols,
                      const int32_t* keys, int32_t nkeys,
                      ldf_column* out, const ldf_allocator* alloc, void* stream);

/* ---- Arrow buffers -> legate layout (on the device) ------------------------ */
/* An Arrow bitmap (validity, or boolean values) -> one byte per row (1 = bit
 * set), the legate null-mask / bool layout: out[i] = bit (bit_offset + i) of
 * `bits` (LSB first).  Device pointers; `bits` holds at least
 * (bit_offset + n + 7) / 8 bytes.  The converse of bitmask_to_bools
 * (null_mask.cu:98-113), used on the column copy of
 * PhysicalColumn::from_arrow (column.cpp:86-122). */
int ldf_b200_arrow_bits_to_bytes(const uint8_t* bits, int64_t bit_offset, int64_t n,
                                 uint8_t* out, void* stream);
/* Arrow string offsets (offset_bytes 4 or 8; n + 1 entries) -> n legate
 * ranges: ranges[i] = {offsets[i], offsets[i + 1] - 1}, inclusive global
 * char positions; the chars copied from position offsets[0] on get
 * chars_base = offsets[0].  Device pointers.  As offsets_to_ranges
 * (ranges.cu:109-138). */
int ldf_b200_arrow_offsets_to_ranges(const void* offsets, int32_t offset_bytes, int64_t n,
                                     ldf_range* ranges, void* stream);

/* ---- CSV text -> columns, parsed on the device --------------------------- */
/* Replaces cudf::io::read_csv in CSVRead::gpu_variant (csv.cu:53-139) with
 * the conversions of the reference's Arrow reader (CSVRead::cpu_variant,
 * csv.cpp:58-130).  `text` (device) holds one file's `nbytes` bytes.
 * Records end at '\n', "\r\n" or a lone '\r' outside quotes; empty records
 * are skipped; `skip_first` skips the first record (the header).  A field
 * that starts with '"' is quoted up to the next lone '"' ("" is one quote;
 * terminators inside quotes belong to the field; characters after the
 * closing quote are kept).  Every record must have as many fields as the
 * first.  Output column j is field `fields[j]` converted to `types[j]`:
 * LDF_BOOL8 ("1/True/TRUE/true", "0/False/FALSE/false"), the integer types
 * (decimal, or 0x-hex bit patterns; spaces and tabs trimmed), LDF_FLOAT32/64
 * (correctly rounded; "inf"/"infinity" any case), LDF_STRING (valid UTF-8).
 * Fields equal to one of the `n_nulls` spellings in `nulls` (NUL-separated,
 * `nulls_bytes` bytes in all; host memory) are nulls, and then every output
 * column has a null mask; with no spellings no column has one.  A value that
 * does not convert fails with LDF_ERR_INVALID_ARGUMENT and the record's line.
 * At most 64 output columns and 1024 fields per record. */
int ldf_b200_csv_read(const uint8_t* text, int64_t nbytes, char delimiter, int32_t skip_first,
                      const int32_t* fields, const int32_t* types, int32_t ncols,
                      const char* nulls, int32_t nulls_bytes, int32_t n_nulls,
                      ldf_column* out, int64_t* nrows, const ldf_allocator* alloc, void* stream);

/* ---- Parquet pages -> columns, decoded on the device ------------------------ */
/* Replaces cudf::io::read_parquet in ParquetRead::gpu_variant
 * (parquet.cu:48-101).  The caller walks the file's metadata and page headers
 * (Thrift, small) and passes one entry per page; the pages' bytes are decoded
 * on the device from `file` (the whole file, in device memory).  Flat columns
 * only (max repetition level 0, max definition level 0 or 1). */
enum { LDF_PQ_DICT_PAGE = 0, LDF_PQ_DATA_V1 = 1, LDF_PQ_DATA_V2 = 2 };
enum { LDF_PQ_UNCOMPRESSED = 0, LDF_PQ_SNAPPY = 1 };
/* Parquet physical types used (the values of the format's Type enum) */
enum { LDF_PQ_BOOLEAN = 0, LDF_PQ_INT32 = 1, LDF_PQ_INT64 = 2, LDF_PQ_FLOAT = 4, LDF_PQ_DOUBLE = 5,
       LDF_PQ_BYTE_ARRAY = 6 };
typedef struct {
  int64_t offset;       /* first byte of the page's payload in `file` (after its header) */
  int64_t compressed;   /* payload bytes in the file */
  int64_t uncompressed; /* payload bytes once decompressed */
  int64_t row0;         /* data pages: first row of the page in its column */
  int32_t num_values;   /* values in the page, nulls included */
  int32_t kind;         /* LDF_PQ_* page kind */
  int32_t encoding;     /* Parquet Encoding of the values (0 PLAIN, 2/8 dictionary indices) */
  int32_t codec;        /* LDF_PQ_UNCOMPRESSED / LDF_PQ_SNAPPY */
  int32_t levels_bytes; /* v2 data pages: definition-level bytes at the payload's start, never compressed */
  int32_t dict;         /* data pages: index of the chunk's dictionary page in `pages`, -1 none */
  int32_t column;       /* output column */
  int32_t reserved;
} ldf_parquet_page;
/* Columns: `physical[j]` (LDF_PQ_*), output type `types[j]` (the integer
 * types narrow INT32/INT64 values), `nullable[j]` (max definition level 1),
 * `nrows` rows each.  Outputs are nullable exactly when `nullable[j]`. */
/* The page table of column chunks, from their page headers (Thrift compact
 * protocol) in host memory: chunk k spans `chunk_bytes[k]` bytes of
 * `file_host` from `chunk_start[k]` (its dictionary page, else its first data
 * page), holds rows from `chunk_row0[k]` of output column
 * `chunk_column[k]`, with codec `chunk_codec[k]` (LDF_PQ_*) and physical type
 * `chunk_physical[k]`.  With `pages` NULL only *npages is set (the count);
 * otherwise at most `max_pages` entries are written.  Pages the decoder
 * cannot take (another encoding, repetition levels) fail with
 * LDF_ERR_UNSUPPORTED.  Host memory only; no device work. */
int ldf_b200_parquet_pages(const uint8_t* file_host, int64_t file_bytes, const int64_t* chunk_start,
                           const int64_t* chunk_bytes, const int64_t* chunk_row0, const int32_t* chunk_column,
                           const int32_t* chunk_codec, const int32_t* chunk_physical, int32_t nchunks,
                           ldf_parquet_page* pages, int32_t max_pages, int32_t* npages);
int ldf_b200_parquet_decode(const uint8_t* file, int64_t file_bytes,
                            const ldf_parquet_page* pages, int32_t npages,
                            const int32_t* physical, const int32_t* types, const int32_t* nullable,
                            int32_t ncols, int64_t nrows,
                            ldf_column* out, const ldf_allocator* alloc, void* stream);

/* ---- test hook: a bounded wait that runs out ------------------------------ */
/* No counterpart in the reference (its waits are inside libcudf).  Runs the
 * library's look-back scan kernel as one block that takes the second tile of
 * a two-tile input, so its look-back waits on a predecessor status word that
 * nothing writes.  The wait ends after `spin_limit` polls (1 .. the
 * library's own limit of 2^22) and the call returns LDF_ERR_TIMEOUT, the
 * status every op returns when one of its bounded device-side waits expires;
 * the context stays usable.  Scratch comes from `alloc` (NULL: stream-ordered
 * cudaMallocAsync). */
int ldf_b200_test_stalled_lookback(uint32_t spin_limit, const ldf_allocator* alloc, void* stream);

/* ---- hash partition without device allocation ----------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory themselves -- a task body running concurrently with other tasks on the
 * same GPU, where cudaMalloc synchronizes the device and can deadlock with
 * them, or a host whose device memory is all handed to its own pool.  Same
 * result as ldf_b200_hash_partition, for fixed-width columns, at most
 * LDF_B200_NOALLOC_MAX_ROWS rows and at most 256 buckets; larger inputs are
 * rejected with LDF_ERR_INVALID_ARGUMENT.  The caller passes the output
 * buffers in `out` (out[j].data: rows x width bytes; out[j].valid: rows bytes
 * for a nullable input column); the call fills them and sets the other
 * fields.  All scratch is one fixed array (about 5 MiB) in the library's
 * device image, held by every GPU that loads the library until the process
 * exits; no cudaMalloc/cudaFree or allocating library routine is called.  The
 * first call on a device looks up the array's device address, so make that
 * first call before any stream capture; the address is kept for the life of
 * the process, so do not call this again on a device after a cudaDeviceReset
 * of it.  Each call synchronizes `stream` twice: the bucket counts and the
 * wait status are read back to the host.  Every call shares the array: calls
 * whose work overlaps on the GPU race and must be serialized. */
#define LDF_B200_NOALLOC_MAX_ROWS (1 << 20)
int ldf_b200_hash_partition_noalloc(const ldf_column* table, int32_t ncols,
                                    const int32_t* keys, int32_t nkeys, int32_t nparts,
                                    ldf_column* out, int64_t* offsets, void* stream);

/* ---- batched execution of many small joins / groupbys ------------------- */
/* No counterpart in the reference (its ops run one task launch per op).  A
 * batch of requests whose inputs are already on the device runs as ONE replay
 * of a CUDA graph captured at engine creation: descriptor upload from mapped
 * pinned memory, three persistent kernels (table init, build/aggregate,
 * probe/emit) over a work list of row tiles of all requests, and the download
 * of per-request output row counts and overflow flags.
 *
 * kind LDF_BATCH_GROUPBY: int64 keys k1[n], value v1[n] (vtype int64 or
 *   float64, optional 1-byte validity vvalid).  Output o0 = key (int64), o1 =
 *   SUM of the valid values (int64 wrapping, or float64 correctly rounded from
 *   an exact fixed-point sum), o2 = COUNT of the valid values (int64).  A group
 *   whose values are all null has o2 = 0 (its SUM is null).  The hash table
 *   takes (cap + 1) x 3 words (int64) or (cap + 1) x 8 words (float64).
 * kind LDF_BATCH_INNER_JOIN: probe k1[n]/v1[n] (int64 key/payload), build
 *   k2[m]/v2[m]; output rows (o0 = lhs key, o1 = lhs payload, o2 = rhs key,
 *   o3 = rhs payload).  The multimap takes cap x 2 words, cap > m.
 * Output row order is unspecified; every output column holds out_cap rows.
 * A request whose table or output overflows its reservation, or whose float
 * values fall outside the exact fixed-point range (|x| < 2^95 and x = 0 or
 * |x| >= 2^-44), is flagged in `overflow` and must be re-run on the per-op
 * path.  Requests of one batch must not share table or output memory. */
enum { LDF_BATCH_GROUPBY = 0, LDF_BATCH_INNER_JOIN = 1 };
enum { LDF_BATCH_INT64 = 0, LDF_BATCH_FLOAT64 = 1 };

typedef struct {
  int32_t kind;            /* LDF_BATCH_* */
  int32_t vtype;           /* groupby value type: LDF_BATCH_INT64 / LDF_BATCH_FLOAT64 */
  int64_t n, m;            /* rows of k1/v1 and of k2/v2 */
  const int64_t* k1;
  const void* v1;
  const int64_t* k2;
  const int64_t* v2;
  const uint8_t* vvalid;   /* groupby value validity (1 byte per row) or NULL */
  uint64_t* table;         /* device scratch of the hash table */
  uint64_t cap;            /* hash table slots (>= 2) */
  void* o0; void* o1; void* o2; void* o3;
  int64_t out_cap;         /* rows reserved in each output column */
} ldf_batch_request;

/* Create an engine for batches of up to max_reqs requests and max_items row
 * tiles of tile_rows rows per kernel; the kernels run ctas_per_sm CTAs per SM
 * on `stream`. */
int ldf_b200_batch_create(int32_t max_reqs, int32_t max_items, int64_t tile_rows,
                          int32_t ctas_per_sm, void* stream, void** engine);
/* Enqueue one batch (asynchronous; the request array is copied). */
int ldf_b200_batch_run(void* engine, const ldf_batch_request* reqs, int32_t nreq);
/* Wait for the last batch; out_rows / overflow receive max_reqs entries. */
int ldf_b200_batch_wait(void* engine, uint64_t* out_rows, int32_t* overflow);
int ldf_b200_batch_destroy(void* engine);

/* ---- utilities ---------------------------------------------------------- */
/* Message of the last failed call on this thread ("" if none). */
const char* ldf_b200_last_error(void);
/* Library version string. */
const char* ldf_b200_version(void);
/* Release the buffers of an output column produced by this library. */
int ldf_b200_free_column(ldf_column* col, const ldf_allocator* alloc, void* stream);

/* ---- instrumentation (no counterpart in the reference; used by the bench) */
/* Number of kernels this library has launched in the process. */
unsigned long long ldf_b200_launch_count(void);
/* Bracket every later launch with CUDA events on its stream (on != 0). */
void ldf_b200_profile_enable(int on);
/* Per-kernel "name launches total_ms" lines; returns the full text length. */
int ldf_b200_profile_report(char* buf, size_t len, int reset);

#ifdef __cplusplus
}
#endif

#endif /* LDF_B200_H */
