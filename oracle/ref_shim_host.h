/*
 * Test infrastructure: force-included (g++ -include) when the reference's
 * host sources are compiled into oracle/_ref/.  Leaves the sources untouched:
 *  - src/model/netgen.cpp:16 calls std::swap on two vector<bool> proxies;
 *    libstdc++ 13 defines that overload only as a hidden friend, so it is
 *    declared here at namespace scope to make the qualified call resolve.
 *  - src/model/netgen.cpp:47 seeds std::mt19937 from system_clock::now();
 *    system_clock is mapped to a clock whose now() returns MGB_REF_MT_SEED
 *    so that generation is reproducible.
 */
#pragma once
#include <vector>
#include <chrono>
#include <random>
#include <cstdlib>
#include <cstdint>
#include <ctime>
#include <queue>
#include <unordered_map>
#include <unordered_set>
#include <algorithm>
#include <cmath>
#include <fstream>
#include <iostream>
#include <string>
#include <utility>
#include <array>
#include <memory.h>

namespace std {
void swap(std::_Bit_reference a, std::_Bit_reference b) noexcept;
namespace chrono {
struct mgb_seed_clock {
    struct tp {
        struct d {
            unsigned long c;
            unsigned long count() const { return c; }
        } v;
        d time_since_epoch() const { return v; }
    };
    static tp now()
    {
        const char* s = getenv("MGB_REF_MT_SEED");
        tp t;
        t.v.c = s ? strtoul(s, nullptr, 10) : 5489UL;
        return t;
    }
};
}  // namespace chrono
}  // namespace std
#define system_clock mgb_seed_clock
