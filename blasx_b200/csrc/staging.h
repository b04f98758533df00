// staging.h -- host memory of a host GEMM call: pinned by the caller, staged
// through pinned bounce buffers, or registered for the call.
//
// A BLAS caller usually passes pageable memory, which the copy engines cannot
// read. The reference registers it for every call (blas/dgemm.c:88-121,
// cudaHostRegister of A, B and C); for a 16384^3 DGEMM that costs ~0.65 s,
// five times the copies themselves. A call here instead marks its pageable
// operands as staged (HostPin::pin) and routes its copies through copy2d:
//   host -> device  the calling thread packs a piece of the region (at most
//                   one bounce buffer) into a free buffer of the inbound ring,
//                   with several threads, and enqueues the buffer's DMA on the
//                   stream; the buffer is reused once that DMA has completed;
//   device -> host  the DMA into a buffer of the outbound ring is enqueued on
//                   the stream and a copy-out thread, once it has completed,
//                   unpacks the piece into the destination and frees the
//                   buffer.
// So packing overlaps the DMA of the previous piece and unpacking overlaps the
// device work that follows. HostPin::finish (and its destructor) waits for the
// call's copy-outs: the results are in host memory when the call returns.
// Copies whose host side is not staged go straight to cudaMemcpy2DAsync.
#pragma once

#include <atomic>
#include <cstddef>
#include <utility>
#include <vector>

#include "runtime.h"

namespace bx {

// The host ranges of one call. Staged ranges belong to the calling thread
// while the object lives (calls nest: the innermost one that holds a range
// stages it); registered ranges are unregistered on destruction.
struct HostPin {
    std::vector<void *> regs;
    std::vector<std::pair<const char *, size_t>> staged;
    HostPin *outer = nullptr;  // the thread's enclosing call with staged ranges
    bool linked = false;
    std::atomic<int> pending{0};   // copy-outs not yet unpacked
    std::atomic<int> error{BLASX_OK};
    // Leaves memory the device can copy directly (pinned, device) alone;
    // stages pageable memory (registers it when staging is switched off or
    // the range cannot be staged).
    int pin(const void *p, size_t bytes);
    // Waits for the call's copy-outs; returns a blasx status.
    int finish();
    // How the call's host memory was copied: 0 directly (pinned by the
    // caller), 1 staged, 2 registered for the call.
    int mode() const { return !staged.empty() ? 1 : (!regs.empty() ? 2 : 0); }
    HostPin() = default;
    HostPin(const HostPin &) = delete;
    HostPin &operator=(const HostPin &) = delete;
    ~HostPin();
};

// cudaMemcpy2DAsync with a blasx status: height rows of width bytes, pitches
// in bytes, on stream s; staged when the host side lies in a range the
// calling thread's HostPin staged.
int copy2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t height,
           cudaMemcpyKind kind, cudaStream_t s);

// Frees the bounce buffers (blasx_finalize); later calls allocate them again.
void release_staging();

}  // namespace bx
