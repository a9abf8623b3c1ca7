// bq_io.cu -- the binary-dump file format of the reference's samples
// (samples/common/IO.h:27-70): a size_t (8-byte, little-endian on the
// supported hosts) element count N, then N raw elements.  Point files
// written by the reference's generator hold vec_t<double,D>; loading them
// as float points is convert<float,D> (IO.h:62-68), an element-wise
// double->float conversion (round to nearest).
//
// Host code only: these calls touch no GPU.
#include <cstdio>

#include "bq_internal.cuh"

namespace bq {
namespace {

struct File {
  FILE *f;
  explicit File(FILE *p) : f(p) {}
  ~File()
  {
    if (f) fclose(f);
  }
};

int read_count(FILE *f, uint64_t *count)
{
  uint64_t n = 0;
  if (fread(&n, sizeof(n), 1, f) != 1) return set_error(BQ_ERR_INVALID_ARGUMENT, "file is shorter than its count");
  *count = n;
  return BQ_OK;
}

} // namespace
} // namespace bq

using namespace bq;

extern "C" {

int bq_load_binary(const char *path, size_t itemBytes, void *out, uint64_t capacity, uint64_t *count)
{
  if (!path || !count || itemBytes == 0) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL path/count or zero item size");
  File f(fopen(path, "rb"));
  if (!f.f) return set_error(BQ_ERR_INVALID_ARGUMENT, "could not open the file");
  uint64_t n = 0;
  BQ_TRY(read_count(f.f, &n));
  *count = n;
  if (!out) return BQ_OK;
  if (n > capacity) return set_error(BQ_ERR_INVALID_ARGUMENT, "the file holds more elements than the capacity");
  if (n && fread(out, itemBytes, n, f.f) != n) return set_error(BQ_ERR_INVALID_ARGUMENT, "file is shorter than its count says");
  return BQ_OK;
}

int bq_save_binary(const char *path, const void *data, uint64_t count, size_t itemBytes)
{
  if (!path || (count && !data) || itemBytes == 0)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL path/data or zero item size");
  File f(fopen(path, "wb"));
  if (!f.f) return set_error(BQ_ERR_INVALID_ARGUMENT, "could not create the file");
  if (fwrite(&count, sizeof(count), 1, f.f) != 1 || (count && fwrite(data, itemBytes, count, f.f) != count))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "write failed");
  return BQ_OK;
}

int bq_load_points_f64_as_f32(const char *path, int dims, float *out, uint64_t capacity, uint64_t *count)
{
  if (!path || !count || dims < 1 || dims > 4) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL path/count or bad dims");
  File f(fopen(path, "rb"));
  if (!f.f) return set_error(BQ_ERR_INVALID_ARGUMENT, "could not open the file");
  uint64_t n = 0;
  BQ_TRY(read_count(f.f, &n));
  *count = n;
  if (!out) return BQ_OK;
  if (n > capacity) return set_error(BQ_ERR_INVALID_ARGUMENT, "the file holds more points than the capacity");
  double buf[4 * 1024];
  const uint64_t per = 1024;
  for (uint64_t i = 0; i < n; i += per) {
    const uint64_t m = n - i < per ? n - i : per;
    if (fread(buf, sizeof(double) * dims, m, f.f) != m)
      return set_error(BQ_ERR_INVALID_ARGUMENT, "file is shorter than its count says");
    for (uint64_t j = 0; j < m * dims; j++) out[i * dims + j] = (float)buf[j];
  }
  return BQ_OK;
}

} // extern "C"
