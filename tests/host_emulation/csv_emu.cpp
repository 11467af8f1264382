// Host emulation of the CSV reader's per-record device code
// (legate-dataframe_b200/csrc/csv.cu): the quoting automaton, the field walk
// and every conversion (integers, hex, booleans, correctly rounded floats,
// strings with quotes, null spellings, UTF-8 checks) compiled as host C++.
// The test that builds it (tests/test_csv_emulated.py) extracts those
// sections from the CUDA source; this file supplies the CUDA built-ins and a
// sequential driver that splits the records with the same automaton.
//
// Input (stdin): one line "delim skip_first ncols n_nulls", then ncols lines
// "field type", then n_nulls lines (null spellings, possibly empty), then the
// CSV text up to EOF.  Output: "rows R", then per column one line per row:
// "N" (null) or the value ("I <int64>", "U <uint64>", "F <hex bits>",
// "S <hex bytes>"); or "error <code> <record>".
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <string>
#include <vector>

#include "ldf_b200.h"

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)
struct uint4 { unsigned x, y, z, w; };
static inline int __clzll(long long x) { return x == 0 ? 64 : __builtin_clzll((unsigned long long)x); }
static inline unsigned long long __umul64hi(unsigned long long a, unsigned long long b)
{
  return (unsigned long long)(((unsigned __int128)a * b) >> 64);
}
template <typename T> static inline T atomicMin(T* p, T v) { T o = *p; if (v < o) *p = v; return o; }
template <typename T> static inline T atomicAdd(T* p, T v) { T o = *p; *p = o + v; return o; }
struct dim3 { unsigned x; };
static dim3 threadIdx{0}, blockIdx{0}, blockDim{1}, gridDim{1};

#include "pow5_table.inc"

namespace ldf {
using std::max;
#include "csv_sections.inc"
}  // namespace ldf

using namespace ldf;

static std::string read_all(FILE* f)
{
  std::string s;
  char buf[1 << 16];
  size_t k;
  while ((k = fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, k);
  return s;
}

static std::string next_line(const std::string& s, size_t& pos)
{
  size_t e = s.find('\n', pos);
  std::string l = s.substr(pos, e - pos);
  pos = e + 1;
  return l;
}

int main()
{
  const std::string in = read_all(stdin);
  size_t pos = 0;
  int delim, skip_first, ncols, n_nulls;
  sscanf(next_line(in, pos).c_str(), "%d %d %d %d", &delim, &skip_first, &ncols, &n_nulls);
  static CsvParams P;
  memset(&P, 0, sizeof(P));
  for (int f = 0; f < kCsvMaxFields; ++f) P.col_of_field[f] = -1;
  static const int widths[] = {0, 1, 1, 2, 4, 8, 1, 2, 4, 8, 4, 8, 16, 8};
  for (int j = 0; j < ncols; ++j) {
    int f, t;
    sscanf(next_line(in, pos).c_str(), "%d %d", &f, &t);
    P.col_of_field[f] = (int16_t)j;
    P.nfield_map      = std::max(P.nfield_map, f + 1);
    P.types[j]        = t;
    P.widths[j]       = widths[t];
  }
  P.n_null = n_nulls;
  int o    = 0;
  for (int k = 0; k < n_nulls; ++k) {
    const std::string sp = next_line(in, pos);
    P.null_off[k]        = o;
    memcpy(P.null_chars + o, sp.data(), sp.size());
    o += (int)sp.size();
    P.null_chars[o++] = 0;
  }
  P.null_off[n_nulls] = o;
  const std::string text = in.substr(pos);
  const int64_t n        = (int64_t)text.size();
  std::vector<uint8_t> tb(text.begin(), text.end());
  tb.resize(n + 16, 0);
  P.text  = tb.data();
  P.n     = n;
  P.delim = delim;
  P.ncols = ncols;
  // records: the automaton over the whole text, one state
  std::vector<int64_t> term;
  uint32_t st = kFs;
  for (int64_t i = 0; i < n; ++i) {
    const uint32_t cls = byte_class(tb[i], i + 1 < n ? tb[i + 1] : 0, i + 1 < n, (uint8_t)delim);
    uint32_t eol;
    st = fsm_step(st, cls, eol);
    if (eol) term.push_back(i);
  }
  std::vector<std::pair<int64_t, int64_t>> rec;
  const int64_t nrec = n > 0 ? (int64_t)term.size() + 1 : 0;
  for (int64_t i = 0; i < nrec; ++i) {
    const int64_t s = i == 0 ? 0 : term[i - 1] + 1;
    int64_t e       = i < (int64_t)term.size() ? term[i] : n;
    if (i < (int64_t)term.size() && tb[e] == '\n' && e > s && tb[e - 1] == '\r') --e;
    rec.push_back({s, e});
  }
  int64_t first = -1;
  for (int64_t i = 0; i < nrec && first < 0; ++i)
    if (rec[i].second > rec[i].first) first = i;
  int nfields = first >= 0 ? walk_fields(P.text, rec[first].first, rec[first].second, (uint8_t)delim,
                                         [](int, int64_t, int64_t) {})
                           : 0;
  std::vector<int64_t> rows_of(nrec, -1);
  int64_t rows = 0;
  for (int64_t i = 0; i < nrec; ++i) {
    if (rec[i].second <= rec[i].first || (skip_first && i == first)) continue;
    rows_of[i] = rows++;
  }
  std::vector<std::vector<uint8_t>> data(ncols);
  for (int j = 0; j < ncols; ++j) data[j].assign(std::max<int64_t>(rows, 1) * P.widths[j], 0);
  std::vector<std::vector<uint8_t>> valid(ncols, std::vector<uint8_t>(std::max<int64_t>(rows, 1), 1));
  std::vector<std::vector<int64_t>> ssrc(ncols, std::vector<int64_t>(std::max<int64_t>(rows, 1)));
  std::vector<std::vector<int64_t>> slen(ncols, std::vector<int64_t>(std::max<int64_t>(rows, 1)));
  std::vector<DeferredFloat> deferred(kCsvMaxDeferred);
  unsigned int ndeferred = 0;
  static CsvOut O;
  memset(&O, 0, sizeof(O));
  for (int j = 0; j < ncols; ++j) {
    O.data[j]    = data[j].data();
    O.valid[j]   = n_nulls > 0 ? valid[j].data() : nullptr;
    O.str_src[j] = ssrc[j].data();
    O.str_len[j] = slen[j].data();
  }
  O.deferred  = deferred.data();
  O.ndeferred = &ndeferred;
  unsigned long long err = ~0ull;
  for (int64_t i = 0; i < nrec; ++i) {
    if (rows_of[i] < 0) continue;
    const int64_t row = rows_of[i];
    const int got     = walk_fields(P.text, rec[i].first, rec[i].second, (uint8_t)delim, [&](int f, int64_t b, int64_t e) {
      if (f >= P.nfield_map) return;
      const int k = P.col_of_field[f];
      if (k >= 0) convert_field(P, O, P.text, 0, i, row, k, b, e, &err);
    });
    if (got != nfields) csv_error(&err, i, 0, kErrFields);
  }
  if (err == ~0ull && ndeferred > 0) csv_exact_float_kernel(P, O, ndeferred, &err);
  if (err != ~0ull) {
    printf("error %llu %lld\n", err & 0xff, (long long)(err >> 16));
    return 0;
  }
  printf("rows %lld\n", (long long)rows);
  for (int j = 0; j < ncols; ++j) {
    const int t = P.types[j];
    for (int64_t r = 0; r < rows; ++r) {
      if (n_nulls > 0 && !valid[j][r]) {
        printf("N\n");
        continue;
      }
      uint64_t v = 0;
      if (t != LDF_STRING) memcpy(&v, data[j].data() + r * P.widths[j], P.widths[j]);
      if (t == LDF_STRING) {
        printf("S ");
        const int64_t s = ssrc[j][r], len = slen[j][r];
        std::vector<uint8_t> out;
        if (s & kQuotedBit) {
          Unquote u(P.text, s & ~kQuotedBit, n);
          uint8_t c;
          for (int64_t k = 0; k < len && u.next(c); ++k) out.push_back(c);
        } else {
          out.assign(P.text + s, P.text + s + len);
        }
        for (uint8_t c : out) printf("%02x", c);
        printf("\n");
      } else if (t == LDF_FLOAT32 || t == LDF_FLOAT64) {
        printf("F %llx\n", (unsigned long long)(t == LDF_FLOAT32 ? (v & 0xffffffffull) : v));
      } else if (t == LDF_INT8 || t == LDF_INT16 || t == LDF_INT32 || t == LDF_INT64) {
        const int w = P.widths[j] * 8;
        const int64_t sv = w == 64 ? (int64_t)v : ((int64_t)(v << (64 - w)) >> (64 - w));
        printf("I %lld\n", (long long)sv);
      } else {
        printf("U %llu\n", (unsigned long long)v);
      }
    }
  }
  return 0;
}
