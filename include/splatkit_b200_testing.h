/* splatkit-b200 test hooks: the library's error paths made to fire without a GPU fault.
 *
 * The reference's renderer keeps its previous world when an upload fails
 * (metal/frame/MetalFrameCompute.mm:113-139), latches a GPU failure for good
 * (metal/presentation/MetalFrameLoop.h:51-55, engine/src/engine/SplatEngine.cpp:517-536), and this
 * library bounds every device wait (a look-back that never sees its predecessor gives up, records
 * the error and lets the frame finish). These hooks make each of those happen on purpose: a
 * failure made on the host (a faked allocation failure, a faked CUDA status) or a device wait that
 * runs out because a status word is never published. None of them faults, traps or hangs a GPU.
 * They exist for tests; a production caller has no use for them.
 */
#ifndef SPLATKIT_B200_TESTING_H
#define SPLATKIT_B200_TESTING_H

#include "splatkit_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The next `count` device allocations of this library (any context) fail as if the device were
 * out of memory; 0 clears the count. Allocations that reuse a large enough buffer are not
 * allocations and do not count. */
void sk_testing_fail_device_allocations(uint32_t count);

/* The next CUDA status `ctx` checks reads as `cuda_error` (a cudaError_t value) instead of its
 * own: a stand-in for a failing CUDA call. An error other than out-of-memory latches the context
 * failed, as a real one would (sk_gpu_failed, SK_E_DEVICE from every later call). */
sk_status sk_testing_fail_next_check(sk_context* ctx, int32_t cuda_error);

/* In the next frame `ctx` draws, tile `tile` (4096 keys per tile) of the depth sort's first pass
 * publishes none of its look-back status words. The tiles after it wait for them until their
 * bounded waits run out, record the error and finish: that frame reports SK_E_TIMEOUT (and
 * stats.device_error) and its order is wrong; the frame after it is drawn normally. A tile at or
 * past the frame's last does nothing. */
sk_status sk_testing_withhold_sort_status(sk_context* ctx, uint32_t tile);

#ifdef __cplusplus
}
#endif

#endif /* SPLATKIT_B200_TESTING_H */
