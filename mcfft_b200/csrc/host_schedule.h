// Chunk schedule of mcfftExecHost (host only, no CUDA).
//
// A single-shape plan is cut into runs of whole transforms: lengths 1, 2,
// 4, .. rising to B (the largest power of two with B transforms in at most
// the target bytes of input, default 32 MiB), runs of B, the rest in powers
// of two, and the rising lengths again in reverse.  Short first and last
// chunks shorten the time only one copy direction is busy (the first copy
// in, the last copy out); long middle chunks keep the per-chunk cost small.
#pragma once

#include <cstdint>
#include <vector>

namespace mcfft {

// B: the largest power of two with B <= batch and B * per_bytes <= target.
inline int64_t host_chunk_big(int64_t batch, int64_t per_bytes, int64_t target) {
  int64_t big = 1;
  while (2 * big <= batch && 2 * big * per_bytes <= target) big *= 2;
  return big;
}

// Chunk lengths (transforms per chunk, in order); they sum to `batch`.
inline std::vector<int64_t> host_schedule(int64_t batch, int64_t big) {
  std::vector<int64_t> head, mid;
  int64_t rem = batch;
  for (int64_t s = 1; s < big && rem >= 2 * s; s *= 2) {
    head.push_back(s);
    rem -= 2 * s;
  }
  for (; rem >= big; rem -= big) mid.push_back(big);
  for (int64_t s = big; s >= 1; s /= 2)
    if (rem >= s) {
      mid.push_back(s);
      rem -= s;
    }
  std::vector<int64_t> out = head;
  out.insert(out.end(), mid.begin(), mid.end());
  out.insert(out.end(), head.rbegin(), head.rend());
  return out;
}

}  // namespace mcfft
