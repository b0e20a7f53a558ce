// Host phase timers of the library, printed to stderr when STZ_TRACE is set.
#pragma once
#include <chrono>
#include <cstdio>
#include <cstdlib>

namespace stz {

// Host phase timer, printed to stderr when STZ_TRACE is set.
struct Trace {
    const char* name;
    std::chrono::steady_clock::time_point t0;
    bool on;
    explicit Trace(const char* n) : name(n), on(std::getenv("STZ_TRACE") != nullptr)
    {
        if (on) t0 = std::chrono::steady_clock::now();
    }
    ~Trace()
    {
        if (on)
            std::fprintf(stderr, "[stz] %-28s %8.3f ms\n", name,
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
};

// Lap timer: mark(name) prints the time since the previous mark (STZ_TRACE).
struct Lap {
    const char* scope;
    std::chrono::steady_clock::time_point t;
    bool on;
    explicit Lap(const char* s) : scope(s), on(std::getenv("STZ_TRACE") != nullptr)
    {
        if (on) t = std::chrono::steady_clock::now();
    }
    void mark(const char* what)
    {
        if (!on) return;
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[stz] %s: %-24s %8.3f ms\n", scope, what,
                     std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

}  // namespace stz
