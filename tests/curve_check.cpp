// Host build of the query-order keys of csrc/device/curves.cuh (the device qualifiers
// defined away), checked for the Hilbert curve's defining properties: on every block of
// cells aligned to its size the indices are one contiguous range, distinct, and
// consecutive indices are face-adjacent cells.  Prints one JSON object.
#define __device__
#define __forceinline__ inline
#include "device/curves.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <utility>
#include <vector>

namespace {

struct Result {
    long blocks = 0, bad_range = 0, bad_step = 0, bad_unique = 0;
};

// the cells of one aligned block of side `side` at `base`, in index order; morton: the
// Morton code instead, as a control that the checks tell the curves apart
template <int D>
void check_block(const uint32_t (&base)[D], uint32_t side, Result &r, bool morton = false) {
    std::vector<std::pair<uint32_t, std::vector<uint32_t>>> cells;
    uint32_t n = 1;
    for (int k = 0; k < D; ++k) n *= side;
    for (uint32_t i = 0; i < n; ++i) {
        std::vector<uint32_t> c(D);
        uint32_t rest = i;
        for (int k = 0; k < D; ++k) {
            c[k] = base[k] + rest % side;
            rest /= side;
        }
        uint32_t key;
        if (morton)
            key = D == 3 ? (gqd::spread3(c[0]) << 2) | (gqd::spread3(c[1]) << 1) | gqd::spread3(c[D - 1])
                         : (gqd::spread2(c[0]) << 1) | gqd::spread2(c[D - 1]);
        else
            key = D == 3 ? gqd::hilbert3(c[0], c[1], c[D - 1]) : gqd::hilbert2(c[0], c[D - 1]);
        cells.push_back({key, c});
    }
    std::sort(cells.begin(), cells.end());
    ++r.blocks;
    if (cells.back().first - cells.front().first + 1 != n) ++r.bad_range;
    for (size_t i = 1; i < cells.size(); ++i) {
        if (cells[i].first == cells[i - 1].first) ++r.bad_unique;
        long step = 0;
        for (int k = 0; k < D; ++k) step += std::labs((long)cells[i].second[k] - (long)cells[i - 1].second[k]);
        if (step != 1) ++r.bad_step;
    }
}

}  // namespace

int main() {
    Result r3, r2;
    // 3D: 1024 cells per axis; blocks of 16^3 and 8^3 at the corners, the centre and
    // pseudo-random aligned places
    uint32_t s = 12345;
    auto next = [&s]() {
        s = s * 1103515245u + 12345u;
        return s >> 8;
    };
    for (uint32_t side : {16u, 8u}) {
        const uint32_t fixed[][3] = {{0, 0, 0}, {1024 - side, 1024 - side, 1024 - side}, {512, 512, 512},
                                     {0, 1024 - side, 512}};
        for (const auto &b : fixed) {
            const uint32_t base[3] = {b[0], b[1], b[2]};
            check_block<3>(base, side, r3);
        }
        for (int t = 0; t < 40; ++t) {
            const uint32_t base[3] = {next() % (1024 / side) * side, next() % (1024 / side) * side,
                                      next() % (1024 / side) * side};
            check_block<3>(base, side, r3);
        }
    }
    // 2D: 32768 cells per axis; blocks of 64^2 and 256^2
    for (uint32_t side : {64u, 256u}) {
        const uint32_t fixed[][2] = {{0, 0}, {32768 - side, 32768 - side}, {16384, 16384}, {0, 32768 - side}};
        for (const auto &b : fixed) {
            const uint32_t base[2] = {b[0], b[1]};
            check_block<2>(base, side, r2);
        }
        for (int t = 0; t < 20; ++t) {
            const uint32_t base[2] = {next() % (32768 / side) * side, next() % (32768 / side) * side};
            check_block<2>(base, side, r2);
        }
    }
    Result m3;
    {
        const uint32_t base[3] = {512, 512, 512};
        check_block<3>(base, 16, m3, true);
    }
    // the whole 2D curve at 15 bits cannot be enumerated here; its top level can: the
    // four 16384^2 quadrants take the four quarters of the index range, each once
    uint32_t quarter_seen = 0;
    for (uint32_t qx = 0; qx < 2; ++qx)
        for (uint32_t qy = 0; qy < 2; ++qy) quarter_seen |= 1u << (gqd::hilbert2(qx * 16384, qy * 16384) >> 28);
    std::printf("{\"blocks3\": %ld, \"bad_range3\": %ld, \"bad_step3\": %ld, \"bad_unique3\": %ld, "
                "\"blocks2\": %ld, \"bad_range2\": %ld, \"bad_step2\": %ld, \"bad_unique2\": %ld, \"quarters2\": %u, "
                "\"morton_bad_step3\": %ld}\n",
                r3.blocks, r3.bad_range, r3.bad_step, r3.bad_unique, r2.blocks, r2.bad_range, r2.bad_step,
                r2.bad_unique, quarter_seen, m3.bad_step);
    return 0;
}
