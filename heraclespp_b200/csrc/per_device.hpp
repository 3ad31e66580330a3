// per_device.hpp -- launch properties cached once per device.
//
// Kernel attributes such as the dynamic shared-memory opt-in
// (cudaFuncAttributeMaxDynamicSharedMemorySize) belong to one device, and so
// do occupancy answers.  A process may hold handles on several devices
// (hcl_config.device) and call the library from several threads, so each
// launcher keeps one PerDevice cache: the first call on a device runs `make`
// with that device current and stores its answer under the cache's lock;
// later calls on that device read it back.  Plain C++ (no CUDA types), so the
// host test suite compiles it on its own.
#pragma once

#include <map>
#include <mutex>

namespace hcl {

class PerDevice {
public:
    // The value for device `dev`: make() on the first call for that device
    // (under the lock, so two threads never both configure one device), the
    // stored value afterwards.
    template <class F>
    int get(int dev, F&& make)
    {
        std::lock_guard<std::mutex> lock(m_);
        const auto it = v_.find(dev);
        if (it != v_.end()) {
            return it->second;
        }
        const int x = make();
        v_.emplace(dev, x);
        return x;
    }

    // number of devices configured so far
    int devices()
    {
        std::lock_guard<std::mutex> lock(m_);
        return (int)v_.size();
    }

private:
    std::mutex m_;
    std::map<int, int> v_;
};

} // namespace hcl
