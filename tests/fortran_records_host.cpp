/* Host build of the Fortran record writer (fortran_records.h) for the CPU tests. */
#include <cstddef>
#include <cstdio>

#include "fortran_records.h"

/* Appends one record to the file at path (created if absent); 0 on success. */
extern "C" int append_fortran_record(const char *path, const unsigned char *data, size_t bytes, size_t max_sub) {
  FILE *fp = fopen(path, "ab");
  if (!fp) return 1;
  const bool ok = oco::write_fortran_record(fp, data, bytes, max_sub);
  return (fclose(fp) == 0 && ok) ? 0 : 1;
}
