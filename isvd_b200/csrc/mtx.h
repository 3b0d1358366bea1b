// Matrix Market files: the dense and coordinate real formats of the reference's data/*.mtx and
// demo/cdemo.c:51-73 (there read through the NIST mmio library and isvd_?Fget).
#pragma once

#include <cstddef>

namespace isvdb {

struct MtxInfo {
  bool coordinate = false;  // "coordinate" (triplets) or "array" (dense, column-major values)
  int field = 0;            // 0 real, 1 integer, 2 pattern
  int symmetry = 0;         // 0 general, 1 symmetric, 2 skew-symmetric
  long long m = 0, n = 0, entries = 0;
};

// Reads the header (and, with a != nullptr, the values) of a Matrix Market file into the m x n
// matrix a: ordera 'C' a[i + j * lda], 'R' a[i * lda + j].  Entries a coordinate file omits are
// zero; symmetric files are mirrored (skew-symmetric with the sign flipped).  Values are parsed
// in parallel on the host threads.  Failures throw isvdb::Error(kErrArgument) naming the reason.
template <class T>
MtxInfo mtx_read(const char *path, T *a, long long lda, char ordera);

// Writes a as "matrix array real general" (column-major values, the shortest decimal form that
// reads back to the same value).
template <class T>
void mtx_write(const char *path, long long m, long long n, const T *a, long long lda, char ordera);

}  // namespace isvdb
