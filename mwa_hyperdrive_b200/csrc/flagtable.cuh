// Sorted 16-bit index lists passed in a launch's parameters (no device
// table, nothing allocated): flagged chanblocks and tiles, which the
// reference indexes with u16 / usize below 65536.
#pragma once

#include <algorithm>
#include <vector>

namespace hdc {

template <int CAP>
struct FlagTable {
    int n;
    unsigned short v[CAP];  // ascending
};

// #{k : tab.v[k] <= x} (binary search over the parameter bank)
template <int CAP>
__device__ __forceinline__ int flag_count_le(const FlagTable<CAP>& tab, int x) {
    int lo = 0, hi = tab.n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((int)tab.v[mid] <= x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Host: sort and check a flag list against [0, limit) (no repeats); returns
// the sorted list or an empty optional-like flag via ok.
inline std::vector<int> sorted_flags(const int* h, int n, int limit, bool* ok) {
    std::vector<int> fl(h, h + n);
    std::sort(fl.begin(), fl.end());
    *ok = true;
    for (int k = 0; k < n; k++)
        if (fl[k] < 0 || fl[k] >= limit || (k > 0 && fl[k] == fl[k - 1])) *ok = false;
    return fl;
}

}  // namespace hdc
