/*
 * Device memory pool of a context.  Task state is one block per task;
 * creating and destroying tasks at serving rates must not pay a cudaMalloc
 * and cudaFree (each of which can synchronise the device) per task.
 *
 * Blocks are 256-byte multiples.  A freed block goes to a free list keyed by
 * size and is reused by the next request of the same size, or of a size at
 * most twice smaller; other requests are carved from 256 MiB chunks, and
 * requests over 64 MiB get a chunk of their own.  Chunks are returned to
 * CUDA only when the context is destroyed.  Not thread-safe: a context has a
 * single owning host thread.
 */
#ifndef SLSF_POOL_H
#define SLSF_POOL_H

#include <cuda_runtime.h>

#include <cstddef>
#include <map>
#include <utility>
#include <vector>

namespace slsf {

class DevicePool {
   public:
    static constexpr size_t kChunk = size_t(256) << 20;
    static constexpr size_t kLarge = size_t(64) << 20;

    cudaError_t allocate(size_t bytes, void** out) {
        bytes = round(bytes);
        auto it = free_.lower_bound(bytes);
        if (it != free_.end() && it->first <= 2 * bytes) {
            *out = it->second;
            /* keep the remainder of a larger block usable */
            const size_t rest = it->first - bytes;
            void* tail = static_cast<char*>(it->second) + bytes;
            free_.erase(it);
            if (rest) free_.emplace(rest, tail);
            return cudaSuccess;
        }
        if (bytes > kLarge) {
            void* p = nullptr;
            cudaError_t e = cudaMalloc(&p, bytes);
            if (e != cudaSuccess) return e;
            chunks_.push_back(p);
            *out = p;
            return cudaSuccess;
        }
        if (bytes > left_) {
            if (left_) free_.emplace(left_, cur_);
            void* p = nullptr;
            cudaError_t e = cudaMalloc(&p, kChunk);
            if (e != cudaSuccess) {
                left_ = 0;
                return e;
            }
            chunks_.push_back(p);
            cur_ = static_cast<char*>(p);
            left_ = kChunk;
        }
        *out = cur_;
        cur_ += bytes;
        left_ -= bytes;
        return cudaSuccess;
    }

    void free(void* p, size_t bytes) {
        if (p) free_.emplace(round(bytes), p);
    }

    void release() {
        for (void* p : chunks_) cudaFree(p);
        chunks_.clear();
        free_.clear();
        cur_ = nullptr;
        left_ = 0;
    }

   private:
    static size_t round(size_t b) { return (b + 255) & ~size_t(255); }
    std::vector<void*> chunks_;
    std::multimap<size_t, void*> free_;
    char* cur_ = nullptr;
    size_t left_ = 0;
};

}  // namespace slsf

#endif /* SLSF_POOL_H */
