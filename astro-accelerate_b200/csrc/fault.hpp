// fault.hpp -- host-side failure injection for tests: after
// arm_injected_failure(n), the n-th CUDA result checked by a pipeline or a
// batch engine reads as a failure ("injected failure"), whatever the call
// returned.  The GPU is not involved: the call itself ran normally, so the
// error paths (status codes, messages, releasing what was allocated) are
// exercised without a fault.
#pragma once

namespace aab200 {

void arm_injected_failure(long long n); // n <= 0 disarms
bool injected_failure_now();            // true once, at the n-th call
long long injected_failure_countdown();

} // namespace aab200
