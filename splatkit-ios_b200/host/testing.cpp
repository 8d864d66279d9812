// The test hooks of include/splatkit_b200_testing.h: each sets a one-shot state the library's own
// paths read (DeviceBuffer::allocate, Context::check, the depth sort's launch arguments).
#include "../../include/splatkit_b200_testing.h"

#include "context.h"

extern "C" {

void sk_testing_fail_device_allocations(uint32_t count) { sk::gTestFailedAllocations.store(count); }

sk_status sk_testing_fail_next_check(sk_context* handle, int32_t cuda_error) {
  auto* ctx = reinterpret_cast<sk::Context*>(handle);
  if (!ctx || cuda_error == 0) return SK_E_INVALID;
  ctx->testInjectedError = static_cast<cudaError_t>(cuda_error);
  return SK_OK;
}

sk_status sk_testing_withhold_sort_status(sk_context* handle, uint32_t tile) {
  auto* ctx = reinterpret_cast<sk::Context*>(handle);
  if (!ctx || tile == 0xffffffffu) return SK_E_INVALID;
  ctx->testWithheldTile = tile + 1;
  return SK_OK;
}

}  // extern "C"
