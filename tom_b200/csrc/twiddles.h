// Per-length twiddle tables tw[m] = exp(-2 pi i m / L), built on the host in
// double precision and kept on each device for the life of the process.
#pragma once
#include <cuda_runtime.h>

namespace tg {
// Device pointer to the table for length L on the current device (nullptr on
// failure).  Safe to call from several host threads.
template <typename C> const C* twiddle_table(int L);
}  // namespace tg
