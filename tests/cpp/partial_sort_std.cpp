// The real std::partial_sort with the reference's key-only KeyPair ordering
// (include/Type.h:449-452), to pin the oracle's and the kernel's emulation.
#include <algorithm>
#include <vector>

struct Pair {
    float key;
    int payload;
    bool operator<(const Pair &o) const { return key < o.key; }
};

extern "C" void std_partial_sort_f32(float *keys, int *payload, int m, int n)
{
    std::vector<Pair> v(n);
    for (int i = 0; i < n; ++i) v[i] = {keys[i], payload[i]};
    std::partial_sort(v.begin(), v.begin() + m, v.end());
    for (int i = 0; i < n; ++i) {
        keys[i] = v[i].key;
        payload[i] = v[i].payload;
    }
}
