/* Neumaier-compensated float sums of contiguous row segments.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of float SUM / MEAN at full size):
 * the rows of every group are laid out contiguously (group-sorted), segment
 * s is rows [off[s], off[s + 1]).  Null rows (valid[r] == 0) are skipped, as
 * Acero's hash_sum / hash_mean skip them (cpp/src/groupby_aggregation.cpp:
 * 41-94 names those kernels).  Each segment is summed in input order with
 * Neumaier's compensated summation (Neumaier 1974, "Rundungsfehleranalyse
 * einiger Verfahren zur Summation endlicher Summen"), whose error is at most
 * about one rounding of the result for the group sizes checked here.
 */
#include <math.h>
#include <stdint.h>

static void segsum(const double* xd, const float* xf, const uint8_t* valid, const int64_t* off, int64_t nseg,
                   double* out, int64_t* nvalid)
{
  for (int64_t s = 0; s < nseg; ++s) {
    double sum = 0.0, comp = 0.0;
    int64_t cnt = 0, nonfinite = 0;
    double plain = 0.0;
    for (int64_t r = off[s]; r < off[s + 1]; ++r) {
      if (valid && !valid[r]) continue;
      const double x = xd ? xd[r] : (double)xf[r];
      ++cnt;
      if (!isfinite(x)) nonfinite = 1;
      plain += x;
      const double t = sum + x;
      if (fabs(sum) >= fabs(x)) comp += (sum - t) + x;
      else comp += (x - t) + sum;
      sum = t;
    }
    out[s]    = nonfinite ? plain : sum + comp;
    nvalid[s] = cnt;
  }
}

void ldf_oracle_segsum_f64(const double* x, const uint8_t* valid, const int64_t* off, int64_t nseg, double* out,
                           int64_t* nvalid)
{
  segsum(x, 0, valid, off, nseg, out, nvalid);
}

void ldf_oracle_segsum_f32(const float* x, const uint8_t* valid, const int64_t* off, int64_t nseg, double* out,
                           int64_t* nvalid)
{
  segsum(0, x, valid, off, nseg, out, nvalid);
}
