// Host-side checks of the SIMT grouped-GEMM tile tables (csrc/simt_tiles.hpp),
// compiled and run by test_simt_tiles_cpu.py.  Prints "ok" or the first failure.
#include <cstdio>
#include <random>
#include <vector>

#include "simt_tiles.hpp"

namespace {

int failures = 0;

void expect(bool ok, const char* what, int trial) {
    if (!ok && failures++ == 0) std::printf("FAIL %s (trial %d)\n", what, trial);
}

// Every complex column of the first m members exactly once; no tile wider
// than the width or crossing its group's columns.
bool covers(const skb::SimtTileTable& t, int tiles, const std::vector<int>& gc, const std::vector<int>& gf,
            std::uint64_t perMember, std::uint64_t m, int width, bool virtualColumns) {
    std::vector<int> seen(m * perMember, 0);
    for (int i = 0; i < tiles; ++i) {
        const int g = t.group[i], per = gc[g];
        if (t.count[i] < 1 || t.count[i] > width || t.per[i] != per || t.first[i] != gf[g]) return false;
        for (int c = 0; c < t.count[i]; ++c) {
            std::uint64_t col;
            if (virtualColumns) {
                const int v = t.column[i] + c;
                if (v >= static_cast<int>(m) * per) return false;
                const int member = v / per;
                col = member * perMember + gf[g] + (v - member * per);
            } else {
                col = static_cast<std::uint64_t>(t.column[i] + c);
                const std::uint64_t within = col % perMember;
                if (within < static_cast<std::uint64_t>(gf[g]) || within >= static_cast<std::uint64_t>(gf[g] + per))
                    return false;
            }
            if (col >= seen.size()) return false;
            ++seen[col];
        }
    }
    for (const int s : seen)
        if (s != 1) return false;
    return true;
}

}  // namespace

int main() {
    const int width = 32;
    std::mt19937 rng(7);
    for (int trial = 0; trial < 300; ++trial) {
        const int groups = 1 + static_cast<int>(rng() % 60);
        const int fields = std::vector<int>{1, 2, 3, 4, 7, 8, 15}[rng() % 7];
        const std::uint64_t members = 1 + rng() % 8;
        std::vector<int> gc(groups), gf(groups);
        int first = 0;
        for (int g = 0; g < groups; ++g) {
            const int modes = 1 + static_cast<int>(rng() % 12);
            gc[g] = modes * fields;
            gf[g] = first;
            first += gc[g];
        }
        const std::uint64_t perMember = static_cast<std::uint64_t>(first);
        // Member tiles: one table, prefixes for every member count.
        std::vector<int> prefix;
        const auto full = skb::simt_tiles(gc, gf, perMember, members, width, false, &prefix);
        expect(prefix.size() == members && prefix.back() == static_cast<int>(full.group.size()), "prefix size", trial);
        for (std::uint64_t m = 1; m <= members; ++m) {
            expect(covers(full, prefix[m - 1], gc, gf, perMember, m, width, false), "member tiles cover", trial);
            const auto own = skb::simt_tiles(gc, gf, perMember, m, width, false);
            expect(static_cast<int>(own.group.size()) == prefix[m - 1], "member prefix length", trial);
            for (int i = 0; i < prefix[m - 1] && i < static_cast<int>(own.group.size()); ++i)
                expect(own.group[i] == full.group[i] && own.column[i] == full.column[i] &&
                           own.count[i] == full.count[i],
                       "member prefix equals the table of fewer members", trial);
            // Virtual tiles: a table per count, never more tiles than member tiles.
            const auto v = skb::simt_tiles(gc, gf, perMember, m, width, true);
            expect(covers(v, static_cast<int>(v.group.size()), gc, gf, perMember, m, width, true),
                   "virtual tiles cover", trial);
            expect(v.group.size() <= static_cast<std::size_t>(prefix[m - 1]), "virtual tiles are fewer", trial);
            // Launch order: member of the first column nondecreasing.
            for (std::size_t i = 1; i < v.group.size(); ++i)
                expect(v.column[i - 1] / v.per[i - 1] <= v.column[i] / v.per[i], "virtual member-major order", trial);
        }
    }
    // The fill rule: 15 fields of the K^2 groups stay member tiles, 4 targets
    // go virtual (group sizes of two, four and six modes), one member never.
    const std::vector<int> modes{2, 4, 6, 4, 2, 6, 4, 8};
    auto columns = [&](int fields) {
        std::vector<int> gc;
        for (const int m : modes) gc.push_back(m * fields);
        return gc;
    };
    expect(!skb::simt_virtual_tiles(columns(15), 8, width), "15 fields member tiles", -1);
    expect(skb::simt_virtual_tiles(columns(4), 8, width), "4 targets virtual tiles", -1);
    expect(!skb::simt_virtual_tiles(columns(4), 1, width), "one member: member tiles", -1);
    if (failures == 0) std::printf("ok\n");
    return failures == 0 ? 0 : 1;
}
