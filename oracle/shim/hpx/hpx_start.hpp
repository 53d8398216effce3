// Test infrastructure (oracle build only): runtime start/stop entry points of
// the HPX shim.  "--hpx:threads=N" sets the pool size; other arguments are
// ignored.
#pragma once

#include <hpx/future.hpp>

#include <cstring>

namespace hpx
{

inline bool start(std::nullptr_t, int argc, char **argv)
{
    unsigned n = 0;
    for (int i = 0; i < argc && argv != nullptr; ++i)
    {
        if (argv[i] == nullptr)
        {
            continue;
        }
        const char *prefix = "--hpx:threads=";
        if (std::strncmp(argv[i], prefix, std::strlen(prefix)) == 0)
        {
            n = static_cast<unsigned>(std::atoi(argv[i] + std::strlen(prefix)));
        }
    }
    shim::pool::instance().request_threads(n);
    shim::pool::instance().ensure_started(n);
    return true;
}

template <typename F>
void post(F &&f)
{
    shim::pool::instance().submit(std::function<void()>(std::forward<F>(f)));
}

inline int finalize() { return 0; }

inline int stop()
{
    shim::pool::instance().shutdown();
    return 0;
}

}  // namespace hpx
