// refsort.cuh -- the order in which the reference leaves tied heat-bath
// weights.
//
// The reference sorts each heat-bath row with
// std::ranges::sort(row, std::greater{}, &Entry::w) (hb_table.cpp:133),
// which libstdc++ implements as std::sort: an unstable introsort, so entries
// of equal weight end in an order set by the algorithm's steps.  This file
// restates that algorithm from its published description (Musser's
// introsort, in the arrangement libstdc++ uses):
//   * ranges longer than 16 elements are split by an unguarded Hoare
//     partition around the median of (first+1, middle, last-1), moved to
//     first; the right part is sorted as its own range, the left part
//     continues;
//   * a range that has used up 2*floor(log2 n) levels is heap-sorted
//     (make_heap, then repeated pop_heap with the hole-sifting adjust_heap);
//   * a final insertion sort runs over the whole range: guarded over the
//     first 16 elements, unguarded after them.
// Elements are (key, val) pairs, comp(x, y) = key_x > key_y (keys are the
// bits of nonnegative doubles, which order like the doubles).  The code
// compiles for host and device; a CPU test compares it with std::sort on
// inputs full of ties.  The index guards below never change a result of a
// correct introsort; they only keep a wrong input in bounds.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define DNQ_HD __host__ __device__
#else
#define DNQ_HD
#endif

namespace dnq {
namespace refsort {

constexpr int64_t kThreshold = 16;

struct Seq {
    uint64_t* k;
    uint32_t* v;
    DNQ_HD void swap(int64_t x, int64_t y) const {
        const uint64_t tk = k[x]; k[x] = k[y]; k[y] = tk;
        const uint32_t tv = v[x]; v[x] = v[y]; v[y] = tv;
    }
    DNQ_HD void move(int64_t to, int64_t from) const { k[to] = k[from]; v[to] = v[from]; }
    DNQ_HD bool comp(int64_t x, int64_t y) const { return k[x] > k[y]; }
};

DNQ_HD inline int floor_log2(int64_t n) {
    int lg = 0;
    while (n > 1) { n >>= 1; ++lg; }
    return lg;
}

// Sift the hole at `hole` down to a leaf, then push (vk, vv) up from there.
DNQ_HD inline void adjust_heap(const Seq& s, int64_t f, int64_t hole, int64_t len, uint64_t vk,
                               uint32_t vv) {
    const int64_t top = hole;
    int64_t second = hole;
    while (second < (len - 1) / 2) {
        second = 2 * (second + 1);
        if (s.comp(f + second, f + second - 1)) --second;
        s.move(f + hole, f + second);
        hole = second;
    }
    if ((len & 1) == 0 && second == (len - 2) / 2) {
        second = 2 * (second + 1);
        s.move(f + hole, f + second - 1);
        hole = second - 1;
    }
    int64_t parent = (hole - 1) / 2;
    while (hole > top && s.k[f + parent] > vk) {
        s.move(f + hole, f + parent);
        hole = parent;
        parent = (hole - 1) / 2;
    }
    s.k[f + hole] = vk;
    s.v[f + hole] = vv;
}

DNQ_HD inline void heap_sort(const Seq& s, int64_t f, int64_t l) {
    const int64_t len = l - f;
    if (len >= 2) {
        for (int64_t parent = (len - 2) / 2;; --parent) {
            adjust_heap(s, f, parent, len, s.k[f + parent], s.v[f + parent]);
            if (parent == 0) break;
        }
    }
    for (int64_t last = l; last - f > 1;) {
        --last;
        const uint64_t vk = s.k[last];
        const uint32_t vv = s.v[last];
        s.move(last, f);
        adjust_heap(s, f, 0, last - f, vk, vv);
    }
}

DNQ_HD inline void median_to_first(const Seq& s, int64_t r, int64_t a, int64_t b, int64_t c) {
    if (s.comp(a, b)) {
        if (s.comp(b, c)) s.swap(r, b);
        else if (s.comp(a, c)) s.swap(r, c);
        else s.swap(r, a);
    } else if (s.comp(a, c)) {
        s.swap(r, a);
    } else if (s.comp(b, c)) {
        s.swap(r, c);
    } else {
        s.swap(r, b);
    }
}

// Partition [f, l) around the median moved to f; returns the cut.
DNQ_HD inline int64_t partition_pivot(const Seq& s, int64_t f, int64_t l) {
    const int64_t mid = f + (l - f) / 2;
    median_to_first(s, f, f + 1, mid, l - 1);
    int64_t lo = f + 1, hi = l;
    for (;;) {
        while (lo < l && s.comp(lo, f)) ++lo;
        --hi;
        while (hi > f && s.comp(f, hi)) --hi;
        if (!(lo < hi)) return lo;
        s.swap(lo, hi);
        ++lo;
    }
}

// Move element `last` left past every element it compares before (stops at
// `floor`, which a correct introsort never reaches through the comparison).
DNQ_HD inline void linear_insert(const Seq& s, int64_t last, int64_t floor) {
    const uint64_t vk = s.k[last];
    const uint32_t vv = s.v[last];
    int64_t next = last - 1;
    while (next >= floor && vk > s.k[next]) {
        s.move(last, next);
        last = next;
        --next;
    }
    s.k[last] = vk;
    s.v[last] = vv;
}

DNQ_HD inline void insertion_sort(const Seq& s, int64_t f, int64_t l) {
    if (f == l) return;
    for (int64_t i = f + 1; i != l; ++i) {
        if (s.comp(i, f)) {
            const uint64_t vk = s.k[i];
            const uint32_t vv = s.v[i];
            for (int64_t t = i; t > f; --t) s.move(t, t - 1);
            s.k[f] = vk;
            s.v[f] = vv;
        } else {
            linear_insert(s, i, f);
        }
    }
}

// Sorts s[0, n).
DNQ_HD inline void sort(const Seq& s, int64_t n) {
    if (n <= 0) return;
    // Pending right-hand ranges of the introsort loop with their remaining
    // depth.  Popping a range of depth d pushes ranges of depths d-1, d-2,
    // ... in that order, so the stack holds strictly decreasing depths and
    // never more than 2*floor(log2 n) + 1 <= 127 entries.
    int64_t st_f[128], st_l[128];
    int st_d[128];
    int top = 1;
    st_f[0] = 0;
    st_l[0] = n;
    st_d[0] = 2 * floor_log2(n);
    while (top > 0) {
        --top;
        const int64_t f = st_f[top];
        int64_t l = st_l[top];
        int depth = st_d[top];
        while (l - f > kThreshold) {
            if (depth == 0) {
                heap_sort(s, f, l);
                break;
            }
            --depth;
            const int64_t cut = partition_pivot(s, f, l);
            if (top < 128) {
                st_f[top] = cut;
                st_l[top] = l;
                st_d[top] = depth;
                ++top;
            }
            l = cut;
        }
    }
    if (n > kThreshold) {
        insertion_sort(s, 0, kThreshold);
        for (int64_t i = kThreshold; i != n; ++i) linear_insert(s, i, 0);
    } else {
        insertion_sort(s, 0, n);
    }
}

}  // namespace refsort
}  // namespace dnq
