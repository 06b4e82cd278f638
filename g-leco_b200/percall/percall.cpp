// percall.cpp -- the plain per-call form of a request stream: one libglc call per request, in
// order, on one stream, issued from C++ (the loop a caller writes without the server).  The
// serving benchmark times it against the server on the same requests and the same GPU.
#include <cstdint>

#include "glc.h"

extern "C" __attribute__((visibility("default"))) int percall_run(
    glc_ctx* ctx, glc_column* const* cols, int32_t nreq, const int32_t* kind, const int32_t* col,
    const int64_t* first, const int64_t* count, const uint64_t* positions, const uint64_t* out, glc_stream stream) {
  for (int32_t i = 0; i < nreq; i++) {
    glc_status st;
    if (kind[i] == GLC_REQ_LOOKUP)
      st = glc_random_access(ctx, cols[col[i]], GLC_SRC_PACKED, (const int32_t*)(uintptr_t)positions[i], count[i],
                             (void*)(uintptr_t)out[i], 0, 0, stream);
    else
      st = glc_decompress_range(ctx, cols[col[i]], GLC_SRC_PACKED, first[i], count[i], (void*)(uintptr_t)out[i], 0,
                                stream);
    if (st != GLC_OK) return (int)st;
  }
  return 0;
}
