// Host check of hcl::PerDevice (heraclespp_b200/csrc/per_device.hpp): one
// value per device id, computed once per device even when many threads ask at
// the same time.  Built and run by tests/test_per_device.py.
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>

#include "per_device.hpp"

int main()
{
    hcl::PerDevice cache;
    std::atomic<int> calls[4] = {};
    std::vector<std::thread> pool;
    std::atomic<int> wrong{0};
    for (int t = 0; t < 16; ++t) {
        pool.emplace_back([&, t] {
            for (int rep = 0; rep < 200; ++rep) {
                const int dev = (t + rep) % 4;
                const int v = cache.get(dev, [&] {
                    calls[dev].fetch_add(1);
                    return 100 + dev;
                });
                if (v != 100 + dev) {
                    wrong.fetch_add(1);
                }
            }
        });
    }
    for (auto& th : pool) {
        th.join();
    }
    int bad = wrong.load();
    for (int d = 0; d < 4; ++d) {
        if (calls[d].load() != 1) {
            std::printf("device %d configured %d times\n", d, calls[d].load());
            ++bad;
        }
    }
    if (cache.devices() != 4) {
        std::printf("%d devices cached\n", cache.devices());
        ++bad;
    }
    std::printf(bad ? "FAIL\n" : "OK\n");
    return bad ? 1 : 0;
}
