// Stand-in declarations of the task-side API that legate-dataframe's GPU task
// bodies use.  legate, rmm, Arrow and the legate-dataframe headers are not
// installed here, so these declarations restate, one by one, the members that
// task_bodies.cpp calls, with the signatures the reference's headers and call
// sites give them (cited per item).  Nothing is defined: the translation unit
// is only type-checked (g++ -fsyntax-only), which catches drift between the
// task bodies and both the reference's interfaces and include/ldf_b200.h.
#pragma once

#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <optional>
#include <string>
#include <utility>
#include <vector>

// ---- Arrow (the types the task arguments carry; utils.cpp:30-139) ---------
namespace arrow {
struct Type {
  enum type {
    BOOL,
    INT8,
    INT16,
    INT32,
    INT64,
    UINT8,
    UINT16,
    UINT32,
    UINT64,
    FLOAT,
    DOUBLE,
    STRING,
    LARGE_STRING,
    TIMESTAMP
  };
};
class DataType {
 public:
  Type::type id() const;
};
namespace compute {
class FunctionOptions {
 public:
  virtual ~FunctionOptions();
};
class CountOptions : public FunctionOptions {  // groupby_aggregation.cpp:58-71 reads `mode`
 public:
  enum CountMode { ONLY_VALID, ONLY_NULL, ALL };
  CountMode mode;
};
}  // namespace compute
}  // namespace arrow

// ---- Arrow's Parquet metadata reader (parquet.cpp:459-468 opens files with
// it; the column-chunk members are those of Arrow's parquet/metadata.h) -----
namespace arrow::io {
class ReadableFile {
 public:
  static std::shared_ptr<ReadableFile> Open(const std::string& path);  // through ARROW_RESULT at parquet.cpp:459
};
}  // namespace arrow::io
namespace parquet {
struct Type {  // the Parquet physical types (Thrift enum Type): the values of LDF_PQ_*
  enum type { BOOLEAN = 0, INT32 = 1, INT64 = 2, INT96 = 3, FLOAT = 4, DOUBLE = 5, BYTE_ARRAY = 6, FIXED_LEN_BYTE_ARRAY = 7 };
};
struct Compression {
  enum type { UNCOMPRESSED, SNAPPY, GZIP, BROTLI, ZSTD, LZ4, LZ4_FRAME, LZO, BZ2 };
};
class ColumnChunkMetaData {
 public:
  bool has_dictionary_page() const;
  int64_t dictionary_page_offset() const;
  int64_t data_page_offset() const;
  int64_t total_compressed_size() const;
  Compression::type compression() const;
  Type::type type() const;
};
class RowGroupMetaData {
 public:
  int64_t num_rows() const;  // parquet.cpp:468
  std::unique_ptr<ColumnChunkMetaData> ColumnChunk(int i) const;
};
class FileMetaData {
 public:
  int num_row_groups() const;  // parquet.cpp:463
  std::unique_ptr<RowGroupMetaData> RowGroup(int i) const;
};
class ParquetFileReader {
 public:
  static std::unique_ptr<ParquetFileReader> Open(std::shared_ptr<arrow::io::ReadableFile> source);  // parquet.cpp:460
  std::shared_ptr<FileMetaData> metadata() const;  // parquet.cpp:461
};
}  // namespace parquet

// ---- rmm (TaskMemoryResource is an rmm device_memory_resource) -------------
namespace rmm {
class cuda_stream_view {
 public:
  cuda_stream_view(cudaStream_t stream);
};
}  // namespace rmm

// ---- legate (members used by the reference's column.cu:44-120, utils.hpp:214) --
namespace legate {
template <int DIM>
class Point {
 public:
  Point(int64_t coord);  // column.cu:66 passes a row count where a Point<1> is taken
  int64_t operator[](int dim) const;
};
template <int DIM>
class Rect {
 public:
  Point<DIM> lo, hi;
  std::size_t volume() const;
};
template <typename T, int DIM = 1>
class Buffer {
 public:
  T* ptr(const Point<DIM>& p) const;
  void destroy();
};
template <typename T, int DIM>
class AccessorRO {
 public:
  const T* ptr(const Point<DIM>& p) const;
};
class PhysicalStore {
 public:
  bool is_unbound_store() const;                                                // column.cu:65
  void bind_untyped_data(Buffer<int8_t, 1>& buffer, const Point<1>& extents) const;  // column.cu:66
  void bind_empty_data() const;                                                 // parquet.cu:201
  template <int DIM>
  Rect<DIM> shape() const;                                                      // utils.hpp:221
  template <typename T, int DIM, bool VALIDATE_TYPE = true>
  AccessorRO<T, DIM> read_accessor() const;
  template <typename T, int DIM>
  Buffer<T, DIM> create_output_buffer(const Point<DIM>& extents, bool bind_buffer) const;  // utils.hpp:218
};
class StringPhysicalArray;
class PhysicalArray {
 public:
  bool nullable() const;                          // column.cu:53
  PhysicalStore data() const;                     // column.cu:65
  PhysicalStore null_mask() const;                // column.cu:54
  StringPhysicalArray as_string_array() const;    // column.cu:105
};
class StringPhysicalArray {
 public:
  PhysicalArray ranges() const;  // column.cu:108
  PhysicalArray chars() const;   // column.cu:109
};
}  // namespace legate

// ---- legate-dataframe --------------------------------------------------------
namespace legate::dataframe {

enum class JoinType : int32_t { INNER = 0, LEFT, FULL, SEMI, ANTI };  // join.hpp:25

class MemAlloc {  // core/allocator.cuh:30-56
 public:
  MemAlloc();
  MemAlloc(MemAlloc&& other) noexcept;
  bool valid() const noexcept;
  std::size_t nbytes() const noexcept;
  legate::Buffer<int8_t>& buffer() noexcept;
};

class TaskMemoryResource {  // core/allocator.cuh:76-115
 public:
  // the public entry points of rmm::mr::device_memory_resource, which
  // forward to the do_allocate / do_deallocate overrides (allocator.cu:27-52)
  void* allocate(std::size_t bytes, rmm::cuda_stream_view stream);
  void deallocate(void* ptr, std::size_t bytes, rmm::cuda_stream_view stream);
  MemAlloc* find_buffer(const void* base_ptr);  // allocator.cuh:90
};

class TaskContext {  // core/task_context.hpp:42-110
 public:
  const int rank;
  const int nranks;
  TaskMemoryResource* mr();
  cudaStream_t stream();
};

namespace task {
class PhysicalColumn {  // core/column.hpp:454-671
 public:
  PhysicalColumn(PhysicalColumn&& other)                 = default;
  PhysicalColumn(const PhysicalColumn& other)            = delete;
  PhysicalColumn& operator=(const PhysicalColumn& other) = delete;
  std::size_t num_rows() const;
  bool nullable() const;
  std::shared_ptr<arrow::DataType> arrow_type() const;
  bool is_partitioned() const;
  void bind_empty_data() const;
  // The one addition the integration makes to column.hpp: access to the
  // private `legate::PhysicalArray array_` (column.hpp:663), which the task
  // bodies read and bind without converting the null mask or the ranges.
  legate::PhysicalArray& physical_array();
  const legate::PhysicalArray& physical_array() const;
};

class PhysicalTable {  // core/table.hpp:348-626
 public:
  int32_t num_columns() const;
  bool is_partitioned() const;
  std::vector<PhysicalColumn> release();  // table.hpp:563
};
}  // namespace task

namespace argument {
template <typename T>
T get_next_input(TaskContext& ctx);  // table.hpp:664 (PhysicalTable)
template <typename T>
T get_next_output(TaskContext& ctx);  // table.hpp:677 (PhysicalTable)
template <typename T>
T get_next_scalar(TaskContext& ctx);  // task_argument.hpp:126
template <typename T>
std::vector<T> get_next_scalar_vector(TaskContext& ctx);  // task_argument.hpp:148
void get_parallel_launch_task(TaskContext& ctx);         // task_argument.hpp:281
}  // namespace argument

[[nodiscard]] std::pair<size_t, size_t> evenly_partition_work(size_t work_size, size_t rank,
                                                              size_t nranks);  // utils.hpp:156

namespace task {
// The rank's files and their row groups (parquet.cpp:60-93)
std::pair<std::vector<std::string>, std::vector<std::vector<int>>> find_files_and_row_groups(
  const std::vector<std::string>& file_paths, const std::vector<size_t>& ngroups_per_file, size_t from_row_group,
  size_t num_row_groups);
}  // namespace task

}  // namespace legate::dataframe
