// queue_split.cu -- the split-form instantiation of the persistent batch
// kernel (fft_queue.cuh), in its own translation unit so that the two forms
// compile in parallel.
#define MCFFT_QUEUE_KERNEL
#include "fft_queue.cuh"

namespace mcfft {

const void* queue_fn_split() { return reinterpret_cast<const void*>(&fft_queue<true>); }

}  // namespace mcfft
