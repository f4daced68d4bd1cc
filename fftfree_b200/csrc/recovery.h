// recovery.h -- host-side emulation of the reference recovery path
// (enable_backup with an outer WorkerPool): dropout decisions, restore
// observer calls, retries and range splitting, decided on the host so no
// GPU work is ever made to fail.
#pragma once

#include <cstddef>
#include <vector>

namespace ffb {

// Frames per column batch of fft_execute_batched (fft_cffi.cpp:754-758).
size_t recovery_batch_frames(size_t N);

// Runs the coordinator over `frames` frames of one batch; `raw` receives 1
// for frames left in their restored (untransformed) state.
void run_recovery_coordinator(size_t frames, std::vector<char>* raw);

}  // namespace ffb
