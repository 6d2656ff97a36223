/* concurrent_vector.h -- TEST INFRASTRUCTURE ONLY.
 * Minimal stand-in for MSVC's Parallel Patterns Library header that the reference includes
 * (pic_simulator.cpp:4): a mutex-guarded std::vector with the members InitializeParticles uses
 * (pic_simulator.cpp:529-547).  Used only when compiling the reference CPU path for the oracle. */
#pragma once
#include <mutex>
#include <vector>

namespace concurrency {
template <class T>
class concurrent_vector {
  public:
    void push_back(const T& value)
    {
        std::lock_guard<std::mutex> lock(mutex_);
        data_.push_back(value);
    }
    size_t size() const { return data_.size(); }
    typename std::vector<T>::const_iterator begin() const { return data_.begin(); }
    typename std::vector<T>::const_iterator end() const { return data_.end(); }

  private:
    std::vector<T> data_;
    std::mutex mutex_;
};
}  // namespace concurrency
