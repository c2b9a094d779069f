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

}  // namespace edus
