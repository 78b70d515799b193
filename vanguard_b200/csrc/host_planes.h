// Host-side passes over whole state planes, shared by the grid and batch entry points: the checks of planes a
// kernel variant does not carry (they must hold a constant) and the fills of those planes on download.
//
// They sit inside vg_solve's copy-in and copy-out, next to DMA copies that move a 4096^2 plane in a few
// milliseconds, while one host thread streams it several times slower; so each pass is split over up to 16
// threads of at least 1 Mi elements, and callers run them while their copies are in flight.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <thread>
#include <vector>

namespace vg {
namespace host {

template <class F>
inline void parallel(long n, F f) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const long nt = std::max(1L, std::min<long>(std::min(hw, 16u), n >> 20));
    if (nt == 1) {
        f(0L, n);
        return;
    }
    std::vector<std::thread> th;
    for (long t = 0; t < nt; t++) th.emplace_back(f, n * t / nt, n * (t + 1) / nt);
    for (auto& x : th) x.join();
}

// Whether any element of the given planes differs from val (NaN differs).
inline bool any_differs(const std::vector<const double*>& ps, double val, long n) {
    std::atomic<bool> found{false};
    for (const double* p : ps)
        parallel(n, [&](long lo, long hi) {
            for (long i = lo; i < hi && !found.load(std::memory_order_relaxed); i += 4096) {
                const long e = std::min(hi, i + 4096);
                bool d = false;
                for (long k = i; k < e; k++) d |= !(p[k] == val);
                if (d) found.store(true, std::memory_order_relaxed);
            }
        });
    return found.load();
}

inline void fill_plane(double* p, double val, long n) {
    parallel(n, [&](long lo, long hi) { std::fill(p + lo, p + hi, val); });
}

// NaN into the `constant` planes (bit r: plane r) of every cell whose `carried` planes hold a non-finite value.
inline void mark_nonfinite(double* planes, long n, int nref, unsigned carried, unsigned constant) {
    parallel(n, [&](long lo, long hi) {
        for (long i = lo; i < hi; i++) {
            bool bad = false;
            for (int r = 0; r < nref; r++)
                if (carried >> r & 1u) bad |= !std::isfinite(planes[(long)r * n + i]);
            if (bad)
                for (int r = 0; r < nref; r++)
                    if (constant >> r & 1u) planes[(long)r * n + i] = std::numeric_limits<double>::quiet_NaN();
        }
    });
}

}  // namespace host
}  // namespace vg
