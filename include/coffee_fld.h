/* coffee_fld.h -- raw little-endian field file ("*.fld").
 *
 * One fixed 80-byte header followed by `nfields` arrays of
 * dims[0]*dims[1]*dims[2] elements of `elem_size` bytes each, every array in
 * the reference's multi_array order (index i + j*dims[0] + k*dims[0]*dims[1],
 * src/data/multi_array_impl.hpp:81-91 of the reference), guard cells
 * included.  The field order is E0 E1 E2 B0 B1 B2 P, optionally followed by
 * auxiliary arrays (J0 J1 J2 divE divB, or the LSRK accumulators of a
 * snapshot).
 *
 * The reference stores fields in HDF5 (src/utils/data_exporter.cpp:134-259);
 * HDF5 is not available to this project, so this plain format carries the
 * same arrays for parity fixtures, snapshots and the oracle driver.
 * Header-only; C and C++.
 */
#ifndef COFFEE_FLD_H
#define COFFEE_FLD_H

#include <stdint.h>
#include <stdio.h>
#include <string.h>

#ifdef __cplusplus
#include <vector>
#endif

#define COFFEE_FLD_MAGIC "COFFEEF1"

typedef struct fld_header {
  char magic[8];      /* "COFFEEF1" */
  int32_t version;    /* 1 */
  int32_t elem_size;  /* 4 (float) or 8 (double) */
  int32_t nfields;
  int32_t flags;      /* bit 0: arrays after the 7th are LSRK accumulators */
  int32_t dims[3];    /* including guard cells */
  int32_t guard[3];
  uint32_t crc32;     /* CRC-32 (IEEE) of the payload, 0 = not checked */
  uint32_t reserved;
  double time;
  int64_t step;
  int64_t reserved2;
} fld_header;

#ifdef __cplusplus
static_assert(sizeof(fld_header) == 80, "fld_header must be 80 bytes");
#endif

/* CRC-32 (IEEE 802.3, reflected, polynomial 0xEDB88320), bitwise form. */
static inline uint32_t fld_crc32_update(uint32_t crc, const void* data,
                                        size_t len) {
  const unsigned char* p = (const unsigned char*)data;
  crc = ~crc;
  for (size_t i = 0; i < len; ++i) {
    crc ^= p[i];
    for (int b = 0; b < 8; ++b) crc = (crc >> 1) ^ (0xEDB88320u & (0u - (crc & 1u)));
  }
  return ~crc;
}

static inline void fld_header_init(fld_header* h, int elem_size, int nfields,
                                   const int dims[3], const int guard[3]) {
  memset(h, 0, sizeof(*h));
  memcpy(h->magic, COFFEE_FLD_MAGIC, 8);
  h->version = 1;
  h->elem_size = elem_size;
  h->nfields = nfields;
  for (int i = 0; i < 3; ++i) {
    h->dims[i] = dims[i];
    h->guard[i] = guard ? guard[i] : 0;
  }
}

/* Write header + nfields arrays of n elements each; the header's crc32 is
 * recomputed over the arrays.  Returns 1 on success. */
static inline int fld_write(const char* path, const fld_header* h_in,
                            const void* const* arrays, size_t n) {
  fld_header h = *h_in;
  uint32_t crc = 0;
  for (int a = 0; a < h.nfields; ++a)
    crc = fld_crc32_update(crc, arrays[a], n * (size_t)h.elem_size);
  h.crc32 = crc;
  FILE* f = fopen(path, "wb");
  if (!f) return 0;
  if (fwrite(&h, sizeof(h), 1, f) != 1) { fclose(f); return 0; }
  for (int a = 0; a < h.nfields; ++a)
    if (fwrite(arrays[a], (size_t)h.elem_size, n, f) != n) { fclose(f); return 0; }
  return fclose(f) == 0;
}

#ifdef __cplusplus
/* Read a whole file into a header and a contiguous payload buffer. */
static inline bool fld_read(const char* path, fld_header* h,
                            std::vector<char>* payload) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  if (fread(h, sizeof(*h), 1, f) != 1 || memcmp(h->magic, COFFEE_FLD_MAGIC, 8) != 0) {
    fclose(f);
    return false;
  }
  const size_t n = (size_t)h->dims[0] * h->dims[1] * h->dims[2];
  const size_t bytes = n * (size_t)h->elem_size * (size_t)h->nfields;
  payload->resize(bytes);
  const bool ok = fread(payload->data(), 1, bytes, f) == bytes;
  fclose(f);
  return ok;
}
#endif

#endif /* COFFEE_FLD_H */
