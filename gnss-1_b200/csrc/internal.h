// internal.h -- library-internal entry points shared by the translation
// units of libgnss_b200.so (not part of the C ABI).
#pragma once
#include <cstddef>

#include "gnss_b200.h"

// Members a batched step launch holds at most.
constexpr int GNSS_BATCH_MAX = 16;

// Bytes of step scratch one member of a batch needs (the fused step's
// intermediates of the context's geometry).
size_t gnss_batch_scratch_bytes(const gnss_ctx *ctx);

// Whether a context's kernel choices allow batched steps: the register z
// kernel and x / y lengths with register passes (64 .. 512).
bool gnss_batch_supported(const gnss_ctx *ctx);

// One fused step of n members of one geometry (grid, precision, scalar count,
// the CN/AB2 scheme, drift coefficient) in one launch per stage.  Member m's
// state and history fields lie m * member_bytes after state0's and hist0's;
// its scratch lies m * scratch_bytes after `scratch` (scratch_bytes >=
// gnss_batch_scratch_bytes, a multiple of 256).  Each member keeps its own
// update coefficients (Reynolds and Schmidt numbers, time step) and FP64 mean
// line; the kernel options of ctxs[0] apply to all.  Each member's result is
// bit-identical to gnss_step on it alone.
gnss_status gnss_step_batch(gnss_ctx *const *ctxs, int n, const gnss_fields *state0, const gnss_fields *hist0,
                            size_t member_bytes, void *scratch, size_t scratch_bytes, int euler, void *stream);
