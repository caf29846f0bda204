// Compares the restated introsort of detnqs_b200/csrc/refsort.cuh with
// libstdc++'s std::sort (the algorithm behind the reference's
// std::ranges::sort(row, std::greater{}, &Entry::w), hb_table.cpp:133) on
// seeded inputs with many ties.  Prints "ok <cases>" or the first mismatch.
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

#include "../detnqs_b200/csrc/refsort.cuh"

struct Entry {
    uint64_t k;
    uint32_t v;
};

int main() {
    std::mt19937_64 rng(20240611);
    const int sizes[] = {0, 1, 2, 3, 15, 16, 17, 18, 31, 32, 33, 63, 100, 257, 1000, 4099,
                         20000, 100000};
    int cases = 0;
    for (int n : sizes)
        for (int distinct : {1, 2, 3, 7, 50, 1000000})
            for (int pattern = 0; pattern < 4; ++pattern) {
                std::vector<Entry> e(n);
                for (int i = 0; i < n; ++i) {
                    uint64_t key = rng() % (uint64_t)distinct;
                    if (pattern == 1) key = (uint64_t)(i % distinct);          // ascending runs
                    if (pattern == 2) key = (uint64_t)((n - i) % distinct);    // descending runs
                    if (pattern == 3) key = (i & 1) ? 5 : key;                 // half equal
                    e[i] = {0x3c00000000000000ull + key, (uint32_t)i};
                }
                std::vector<uint64_t> k(n);
                std::vector<uint32_t> v(n);
                for (int i = 0; i < n; ++i) { k[i] = e[i].k; v[i] = e[i].v; }
                std::vector<Entry> h = e;
                std::vector<uint64_t> hk = k;
                std::vector<uint32_t> hv = v;
                dnq::refsort::sort(dnq::refsort::Seq{k.data(), v.data()}, n);
                // the heapsort fallback alone: std::partial_sort(first, last, last)
                std::sort(e.begin(), e.end(),
                          [](const Entry& x, const Entry& y) { return x.k > y.k; });
                std::partial_sort(h.begin(), h.end(), h.end(),
                                  [](const Entry& x, const Entry& y) { return x.k > y.k; });
                dnq::refsort::heap_sort(dnq::refsort::Seq{hk.data(), hv.data()}, 0, n);
                for (int i = 0; i < n; ++i)
                    if (hk[i] != h[i].k || hv[i] != h[i].v) {
                        std::printf("heap mismatch n=%d distinct=%d pattern=%d at %d\n", n,
                                    distinct, pattern, i);
                        return 1;
                    }
                for (int i = 0; i < n; ++i)
                    if (k[i] != e[i].k || v[i] != e[i].v) {
                        std::printf("mismatch n=%d distinct=%d pattern=%d at %d\n", n, distinct,
                                    pattern, i);
                        return 1;
                    }
                ++cases;
            }
    std::printf("ok %d\n", cases);
    return 0;
}
