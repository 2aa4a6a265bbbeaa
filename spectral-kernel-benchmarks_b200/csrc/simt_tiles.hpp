// Tile tables of the SIMT grouped vertical GEMM (host side, no CUDA; the
// numberings are described at GroupTiles in vertical.hpp).
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <vector>

namespace skb {

struct SimtTileTable {
    std::vector<int> group, column, count, per, first;
};

// Virtual tiles over each group's member-concatenated columns when member
// tiles of `width` columns would run under 90 % full and the plan has several
// members; member tiles otherwise.
inline bool simt_virtual_tiles(const std::vector<int>& groupColumns, std::uint64_t members, int width) {
    std::uint64_t used = 0, padded = 0;
    for (const int n : groupColumns) {
        used += static_cast<std::uint64_t>(n);
        padded += (static_cast<std::uint64_t>(n) + width - 1) / width * width;
    }
    return members > 1 && used < 0.9 * static_cast<double>(padded);
}

// Tiles covering `members` members, launched member-major (by the member of a
// tile's first column, then group), as consecutive CTAs then stream through
// one member's operands; virtual tiles of a group still run on across
// members.  groupColumns / groupFirst: complex columns per member of each
// group and the group's first column within a member; perMember: columns per
// member.  memberPrefix (member tiles only, optional): memberPrefix[m - 1] =
// tiles of the first m members, which are a prefix of the table.
inline SimtTileTable simt_tiles(const std::vector<int>& groupColumns, const std::vector<int>& groupFirst,
                                std::uint64_t perMember, std::uint64_t members, int width, bool virtualColumns,
                                std::vector<int>* memberPrefix = nullptr) {
    std::vector<std::array<std::uint64_t, 3>> order;  // (member, group, first column in the group's list)
    for (std::uint64_t gi = 0; gi < groupColumns.size(); ++gi) {
        const auto per = static_cast<std::uint64_t>(groupColumns[gi]);
        if (virtualColumns) {
            for (std::uint64_t c = 0; c < members * per; c += width) order.push_back({c / per, gi, c});
        } else {
            for (std::uint64_t mm = 0; mm < members; ++mm)
                for (std::uint64_t c = 0; c < per; c += width) order.push_back({mm, gi, mm * per + c});
        }
    }
    std::sort(order.begin(), order.end());
    SimtTileTable t;
    for (const auto& o : order) {
        const std::uint64_t mm = o[0], gi = o[1], c = o[2];
        const auto per = static_cast<std::uint64_t>(groupColumns[gi]);
        t.group.push_back(static_cast<int>(gi));
        if (virtualColumns) {
            t.column.push_back(static_cast<int>(c));
            t.count.push_back(static_cast<int>(std::min<std::uint64_t>(width, members * per - c)));
        } else {
            const std::uint64_t within = c - mm * per;
            t.column.push_back(static_cast<int>(mm * perMember + static_cast<std::uint64_t>(groupFirst[gi]) + within));
            t.count.push_back(static_cast<int>(std::min<std::uint64_t>(width, per - within)));
        }
        t.per.push_back(groupColumns[gi]);
        t.first.push_back(groupFirst[gi]);
    }
    if (memberPrefix != nullptr && !virtualColumns) {
        memberPrefix->assign(members, 0);
        for (const auto& o : order) ++(*memberPrefix)[o[0]];
        for (std::uint64_t mm = 1; mm < members; ++mm) (*memberPrefix)[mm] += (*memberPrefix)[mm - 1];
    }
    return t;
}

}  // namespace skb
