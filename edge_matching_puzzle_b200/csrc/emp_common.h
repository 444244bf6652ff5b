// Shared host helpers of the C ABI: error reporting, device buffers, handles.
#pragma once

#include "emp_b200.h"
#include "emp_model.h"

#include <cuda_runtime.h>

#include <string>
#include <utility>

namespace emp {

std::string& last_error();
void clear_error();
emp_status fail(emp_status status, const std::string& message);
emp_status cuda_fail(cudaError_t e, const char* what);
// Makes `device` current (-1: keep the current one) and reports its ordinal.
emp_status select_device(int device, int* ordinal);

// Owning device allocation (move-only).
struct DeviceBuffer {
    void* p = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept
    {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n)
    {
        release();
        bytes = n;
        return n ? cudaMalloc(&p, n) : cudaSuccess;
    }
    // Keeps the allocation when it holds n bytes already (cudaFree synchronises
    // the whole device, which would stall work queued on other streams).
    cudaError_t reserve(size_t n) { return n <= bytes && p ? cudaSuccess : alloc(n); }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

}  // namespace emp

struct emp_puzzle_t {
    emp::PuzzleModel model;
    std::vector<uint32_t> order;
    std::vector<emp::LevelPlan> plan;
    emp::DeviceTables tables;
    uint32_t extra_count = 0;
};

#define CUDA_TRY(expr)                                       \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return emp::cuda_fail(e_, #expr); \
    } while (0)

#define EMP_TRY(expr)                       \
    do {                                    \
        emp_status s_ = (expr);             \
        if (s_ != EMP_OK) return s_;        \
    } while (0)
