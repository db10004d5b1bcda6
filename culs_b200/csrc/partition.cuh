// Disjoint SM partitions of one GPU for engines that run at once.
//
// The served mode runs several batches at once, each on an engine of its
// own.  Sharing the SMs through the block scheduler alone, a batch's short
// kernels wait behind the other batches' persistent dataflow kernels (their
// blocks hold SMs for a whole stage).  A partition is a green context over
// a disjoint set of SMs with a stream of its own: kernels launched into
// that stream run on those SMs only, so a batch of small jobs is never
// queued behind a large batch's critical path.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace culs {

struct SmPartition {
    void *green = nullptr;          // the green context (CUgreenCtx)
    cudaStream_t stream = nullptr;  // a non-blocking stream of that context
    int sms = 0;                    // SMs it runs on
};

// Splits the SMs of `device` into n disjoint partitions as evenly as the
// hardware's SM groups allow (the SMs the split leaves over go to the last
// partition).  Returns false, with the reason in *why and nothing created,
// when the driver cannot (no green context support, or fewer SM groups than
// n).
bool make_sm_partitions(int device, int n, std::vector<SmPartition> &out, std::string *why);

// Destroys the partitions' streams and green contexts; every engine that
// used one must be gone.
void destroy_sm_partitions(std::vector<SmPartition> &parts);

}  // namespace culs
