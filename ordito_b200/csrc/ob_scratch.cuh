// Stream-ordered scratch memory for one call: each take() is one pool allocation on the call's
// stream, released in stream order (after the call's kernels) when the object goes out of scope.
#pragma once

#include <cuda_runtime.h>

#include "ob_internal.cuh"

namespace ob {

class Scratch {
  public:
    explicit Scratch(cudaStream_t stream) : stream_(stream) {}
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
    ~Scratch() {
        for (int i = 0; i < count_; ++i) cudaFreeAsync(blocks_[i], stream_);
    }

    // Returns `n` elements of T, or nullptr (and commit() fails) when the allocation is refused.
    template <typename T>
    T* take(size_t n) {
        if (status_ != OB_OK || count_ == kMax) {
            if (status_ == OB_OK) status_ = fail(OB_ERR_INVALID, "scratch: too many buffers");
            return nullptr;
        }
        void* p = nullptr;
        cudaError_t e = pool_malloc(&p, sizeof(T) * (n == 0 ? 1 : n), stream_);
        if (e != cudaSuccess) {
            cudaGetLastError();
            status_ = cuda_status(e, "scratch allocation");
            return nullptr;
        }
        blocks_[count_++] = p;
        return static_cast<T*>(p);
    }

    // OB_OK when every take() succeeded.
    int commit() const { return status_; }

  private:
    static constexpr int kMax = 32;
    cudaStream_t stream_;
    void* blocks_[kMax] = {};
    int count_ = 0;
    int status_ = OB_OK;
};

}  // namespace ob
