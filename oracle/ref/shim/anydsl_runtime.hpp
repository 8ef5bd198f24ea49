/* Host-memory stand-in for the AnyDSL runtime's buffer API used by the reference
 * (anydsl::Array, anydsl::copy, anydsl_copy; ray_queue.h:46-53,77-80,277,292 and
 * scene.cpp:10-188). Every platform, including Platform::Cuda, is plain host memory: the
 * oracle harness runs the reference's GPU code path on the CPU, with the oracle traversal
 * behind the traversal_gpu entry points. TEST INFRASTRUCTURE ONLY. */
#ifndef IMBART_REF_ANYDSL_SHIM_HPP
#define IMBART_REF_ANYDSL_SHIM_HPP
#include <cstdint>
#include <cstring>
#include <utility>

namespace anydsl {
enum class Platform { Host = 0, Cuda = 1 };
struct Device {
    int id;
    explicit Device(int i = 0) : id(i) {}
};

template <typename T>
class Array {
public:
    Array() : data_(nullptr), size_(0) {}
    explicit Array(int64_t size) : Array(Platform::Host, Device(0), size) {}
    Array(Platform, Device, int64_t size) : data_(nullptr), size_(size) {
        if (size > 0) {
            data_ = new T[size];
            std::memset((void*)data_, 0, sizeof(T) * size);
        }
    }
    Array(const Array&) = delete;
    Array& operator=(const Array&) = delete;
    Array(Array&& o) : data_(o.data_), size_(o.size_) { o.data_ = nullptr; o.size_ = 0; }
    Array& operator=(Array&& o) {
        std::swap(data_, o.data_);
        std::swap(size_, o.size_);
        return *this;
    }
    ~Array() { delete[] data_; }
    T* data() { return data_; }
    const T* data() const { return data_; }
    int64_t size() const { return size_; }
    int32_t device() const { return 0; }
    T& operator[](int64_t i) { return data_[i]; }
    const T& operator[](int64_t i) const { return data_[i]; }
    T* begin() { return data_; }
    T* end() { return data_ + size_; }
    const T* begin() const { return data_; }
    const T* end() const { return data_ + size_; }

private:
    T* data_;
    int64_t size_;
};

template <typename T>
void copy(const Array<T>& src, Array<T>& dst, int64_t size) {
    std::memcpy((void*)dst.data(), (const void*)src.data(), sizeof(T) * size);
}
}  // namespace anydsl

inline void anydsl_copy(int32_t, const void* src, int64_t off_src, int32_t, void* dst, int64_t off_dst, int64_t size) {
    std::memcpy((char*)dst + off_dst, (const char*)src + off_src, size);
}
#endif
