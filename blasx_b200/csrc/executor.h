// executor.h -- the serving loop's persistent tile executor.
//
// One kernel, one CTA of 256 threads per SM, runs the work of every request
// the serving loop has in flight: the tiles of native FP64 / complex128
// (DMMA) and FP32 / complex64 (SIMT) requests, and every stage of emulated
// requests -- row statistics, the modulus decision, the int8 slices, the
// INT8 residue GEMM tiles on the tcgen05 tensor cores, the CRT
// reconstruction. The scheduler thread publishes tasks into a ring in pinned
// host memory while the kernel runs; CTAs claim them in publication order
// (one device-memory counter), run them, and mark each one done in pinned
// host memory. A request's next stage is published once its current stage
// has completed, so tasks never wait on one another on the device. Every
// wait of the kernel is bounded: a CTA with no task to claim for a while
// (or told to stop) exits, and the kernel ends when all of them have; the
// scheduler launches it again when tasks are pending.
#pragma once

#include "runtime.h"

namespace bx {
namespace exec {

class Executor;

// Creates the executor for `slots` request slots (its ring, device tables
// and stream) on the current device. Returns a blasx status.
int create(int slots, Executor **out);
void destroy(Executor *e);

// Whether the executor runs request g (its operands, C and, for the emulated
// path, its scratch already on the device): every GEMM of the serving loop
// except those whose operands are stored as one triangle (SYMM, HEMM) or
// whose output is Hermitian (HERK, HER2K).
bool supports(const Gemm &g);

// Prepares slot `slot` for the device-resident request g (emulated: on the
// scratch ws of ozaki_scratch_bytes bytes, precision mode `mode`): builds
// its descriptor and enqueues the descriptor's copy to the device on stream
// s (the request's own stream, after its operand copies). The request's
// first stage is published by start() once that stream has reached this
// point.
int prepare(Executor *e, int slot, const Gemm &g, bool emulated, int mode, void *ws, cudaStream_t s);
// Publishes the first stage of the prepared request in `slot`.
int start(Executor *e, int slot);
// Advances the request in `slot`: when all tasks of its current stage are
// done, publishes the next stage. Returns 1 when the request's device work
// is complete (C holds the result), 0 while it is still running, or a
// negative value when the device reported an error (a bounded wait that ran
// out: the request's C is undefined).
int advance(Executor *e, int slot);
// The path the request in `slot` took: 1 native, 2 emulated, 4 native
// fallback chosen on the device; and its modulus count (emulated).
void path_of(Executor *e, int slot, int *path, int *moduli);
// Launches the kernel when tasks are pending and it is not running.
int pump(Executor *e);
// True when nothing is published that has not completed.
bool idle(Executor *e);
// Asks the kernel to exit at its next claim and waits for it (bounded by the
// tasks it is running).
int stop(Executor *e);
// Statistics: kernel launches and tasks run since creation.
void counters(Executor *e, long long *launches, long long *tasks);

}  // namespace exec
}  // namespace bx
