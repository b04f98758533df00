// profile.h -- optional per-phase timing with CUDA events recorded on the
// stream a phase is launched on (enabled with blasx_profile_enable).
#pragma once

#include "runtime.h"

namespace bx {
namespace prof {

enum Phase : int {
    kSlice = 0,        // emulated path: stats, decision, scaling and slicing
    kResidueGemm = 1,  // emulated path: INT8 tcgen05 residue GEMMs
    kReconstruct = 2,  // emulated path: CRT reconstruction + epilogue
    kNative = 3,       // native FP64 / complex128 / FP32 kernel
    kNumPhases = 4
};

bool enabled();
// Records an event on `s` and returns its handle (nullptr when disabled).
cudaEvent_t mark(cudaStream_t s);
// Adds the interval [a, b] to `phase` once both events have completed.
void span(int phase, cudaEvent_t a, cudaEvent_t b);

}  // namespace prof
}  // namespace bx
