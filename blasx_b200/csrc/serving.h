// serving.h -- request queue, admission and continuous batching of host GEMM
// calls from many threads (no counterpart in the reference, whose GEMM path
// is not re-entrant: blas/blasx_tile_resource.c:13-26).
#pragma once

#include "runtime.h"

namespace bx {
namespace serve {

// True while the serving loop runs; host calls are then routed through it.
bool active();

// Queues a host GEMM and blocks until it completed (or failed). Returns a
// blasx status; the call statistics of the calling thread are filled.
int submit(const Gemm &g);

}  // namespace serve
}  // namespace bx
