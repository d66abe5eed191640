// Device primitives of libtapas_b200 (scan, radix sort), issued on ctx->stream.
#pragma once
#include "common.cuh"

namespace tb {

// out[i] = sum(in[0..i)); *d_total (device, may be null) = sum(in).  n <= 4096^2.
int scan_exclusive(tapas_b200_ctx *ctx, const int32_t *in, int32_t *out, int64_t n,
                   int32_t *d_total);

// Stable LSD radix sort on key bits [begin_bit, end_bit).  Keys (and values,
// if vals is non-null) are sorted between the two buffers; on return `keys`
// and `vals` point at the sorted data (the pointers are swapped per pass).
int radix_sort(tapas_b200_ctx *ctx, uint64_t *&keys, uint64_t *&keys_alt, uint32_t *&vals,
               uint32_t *&vals_alt, int64_t n, int begin_bit, int end_bit);

}  // namespace tb
