// tile_engine.h -- out-of-core execution of a host GEMM through the HBM tile
// cache, and the stream drain shared by the host pipelines.
#pragma once

#include <vector>

#include "runtime.h"
#include "staging.h"

namespace bx {

// Waits for the context's three streams when it goes out of scope. Declared
// after a call's device buffers and host pins, it runs before they are freed
// or unregistered, so that an early error return does neither while a copy
// or kernel of the call is still in flight. On the success path the streams
// are already idle.
struct StreamDrain {
    Context *c;
    ~StreamDrain() {
        if (!c) return;
        cudaStreamSynchronize(c->h2d);
        cudaStreamSynchronize(c->compute);
        cudaStreamSynchronize(c->d2h);
    }
};

// Bytes spanned by a column-major rows x cols matrix with leading dimension ld.
size_t host_extent(int64_t ld, int64_t rows, int64_t cols, size_t es);

// Host GEMM through tile x tile operand tiles cached in an HBM arena of
// `budget` bytes (policy: 0 Belady, 1 LRU). Synchronous. With ws_bytes > 0
// every K-step runs on the emulated (Ozaki) path in precision mode `mode`,
// on a scratch of ws_bytes carved from the same budget; otherwise on the
// native kernels. A symmetric or Hermitian operand stored as one triangle
// (Gemm::a_form / b_form of SYMM, HEMM) is read from its stored triangle tile
// by tile.
int tiled_host_gemm(const Gemm &g, Context *c, size_t budget, int tile, int policy,
                    size_t ws_bytes = 0, int mode = 0);

// The smallest budget tiled_host_gemm accepts for tile edge T and a step
// scratch of ws_bytes: the C tiles and two operand tiles beside the scratch.
size_t tiled_min_bytes(DType dt, int T, size_t ws_bytes);

// Frees the arena (blasx_finalize).
void release_tile_arena();

}  // namespace bx
