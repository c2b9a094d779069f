// ctx_hooks.hpp — what the batch engine (batch.cu) uses of a single-solve
// context (capi.cu) to run an instance with the Coulomb mean field: the
// context's whole loop, captured in one CUDA graph, launched on the
// context's own stream beside the batch's chunk graphs.
#pragma once
#include <stdint.h>

#include "../../include/edus_b200.h"
#include "host/problem.hpp"

namespace edus {

// Launch the whole run of a fresh constant-dt context without waiting.
int ctx_start_async(edus_ctx* c);
// Whether that run has ended (then its device error word is checked).
int ctx_poll(edus_ctx* c, bool* done);
// Wait for the run to end.
int ctx_wait(edus_ctx* c);
// Device memory the context holds, and an upper bound of it before creation.
size_t ctx_device_bytes(const edus_ctx* c);
int64_t ctx_footprint_estimate(const Problem& P);
// CUDA-event time of the context's last run (ms).
double ctx_last_ms(const edus_ctx* c);
// Register a context whose whole run ctx_start_async launched (the server
// creates and starts Coulomb contexts on a thread of its own) as a running
// instance of the batch; the batch takes ownership. EDUS_ENOMEM when no slot
// is free (the context is left to the caller then).
int batch_adopt_context(edus_batch* b, edus_ctx* ctx, const Problem& P, int64_t tag, int32_t* slot);
// Whether any class of the batch has tiles to advance, and a non-blocking
// retirement of the Coulomb contexts whose run has ended (the server's loop
// must not wait on one while requests arrive).
bool batch_has_tiles(const edus_batch* b);
int batch_poll_contexts(edus_batch* b);

}  // namespace edus
