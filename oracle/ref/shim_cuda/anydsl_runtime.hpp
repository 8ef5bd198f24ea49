/* Device-memory stand-in for the AnyDSL runtime's buffer API (anydsl::Array, anydsl::copy,
 * anydsl_copy; ray_queue.h:46-53,77-80,277,292 and scene.cpp:10-188) for the build of the
 * reference that takes its traversal from libimbart (libref_imbart.so): arrays of
 * Platform::Cuda live in GPU memory (cudaMalloc) as under the real runtime, host arrays in
 * host memory, and copies go through cudaMemcpy with unified addressing. Found ahead of
 * oracle/ref/shim/anydsl_runtime.hpp on that build's include path. TEST INFRASTRUCTURE ONLY. */
#ifndef IMBART_REF_ANYDSL_SHIM_HPP
#define IMBART_REF_ANYDSL_SHIM_HPP
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>

// The five CUDA runtime calls the shim makes, declared here rather than through
// cuda_runtime.h, whose global float3/float4 types would clash with the reference's own
// (the harness sources use namespace imba). Error and copy-kind enums are passed as int.
extern "C" {
int cudaMalloc(void** ptr, size_t size);
int cudaFree(void* ptr);
int cudaMemset(void* ptr, int value, size_t count);
int cudaMemcpy(void* dst, const void* src, size_t count, int kind);
const char* cudaGetErrorString(int error);
}

namespace anydsl {
constexpr int kCudaMemcpyDefault = 4;   // cudaMemcpyDefault: direction from unified addressing

enum class Platform { Host = 0, Cuda = 1 };
struct Device {
    int id;
    explicit Device(int i = 0) : id(i) {}
};

inline void check_cuda(int e, const char* what) {
    if (e != 0) {
        std::fprintf(stderr, "anydsl shim: %s: %s\n", what, cudaGetErrorString(e));
        std::abort();
    }
}

template <typename T>
class Array {
public:
    Array() : data_(nullptr), size_(0), gpu_(false) {}
    explicit Array(int64_t size) : Array(Platform::Host, Device(0), size) {}
    Array(Platform p, Device, int64_t size) : data_(nullptr), size_(size), gpu_(p == Platform::Cuda) {
        if (size <= 0) return;
        if (gpu_) {
            check_cuda(cudaMalloc((void**)&data_, sizeof(T) * size), "cudaMalloc");
            check_cuda(cudaMemset(data_, 0, sizeof(T) * size), "cudaMemset");
        } else {
            data_ = new T[size];
            std::memset((void*)data_, 0, sizeof(T) * size);
        }
    }
    Array(const Array&) = delete;
    Array& operator=(const Array&) = delete;
    Array(Array&& o) : data_(o.data_), size_(o.size_), gpu_(o.gpu_) { o.data_ = nullptr; o.size_ = 0; }
    Array& operator=(Array&& o) {
        std::swap(data_, o.data_);
        std::swap(size_, o.size_);
        std::swap(gpu_, o.gpu_);
        return *this;
    }
    ~Array() {
        if (gpu_) cudaFree(data_);
        else delete[] data_;
    }
    T* data() { return data_; }
    const T* data() const { return data_; }
    int64_t size() const { return size_; }
    int32_t device() const { return gpu_ ? 1 : 0; }
    T& operator[](int64_t i) { return data_[i]; }
    const T& operator[](int64_t i) const { return data_[i]; }
    T* begin() { return data_; }
    T* end() { return data_ + size_; }
    const T* begin() const { return data_; }
    const T* end() const { return data_ + size_; }
    bool on_gpu() const { return gpu_; }

private:
    T* data_;
    int64_t size_;
    bool gpu_;
};

template <typename T>
void copy(const Array<T>& src, Array<T>& dst, int64_t size) {
    if (size > 0) check_cuda(cudaMemcpy((void*)dst.data(), (const void*)src.data(), sizeof(T) * size, kCudaMemcpyDefault),
                             "cudaMemcpy");
}
}  // namespace anydsl

inline void anydsl_copy(int32_t, const void* src, int64_t off_src, int32_t, void* dst, int64_t off_dst, int64_t size) {
    if (size > 0)
        anydsl::check_cuda(cudaMemcpy((char*)dst + off_dst, (const char*)src + off_src, size, anydsl::kCudaMemcpyDefault),
                           "cudaMemcpy");
}
#endif
