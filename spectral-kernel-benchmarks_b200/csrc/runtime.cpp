#include "runtime.hpp"

#include "columns_warp.hpp"
#include "simt_tiles.hpp"

#include <algorithm>
#include <array>
#include <cstring>

#include "util.hpp"

namespace skb {

void throw_cuda(cudaError_t err, const char* what) {
    const int code = err == cudaErrorMemoryAllocation ? -4 : -2;
    throw Error(code, std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")");
}

void DeviceBuffer::allocate(size_t bytes) {
    release();
    if (bytes == 0) return;
    check_cuda(cudaMalloc(&ptr_, bytes), "cudaMalloc");
    bytes_ = bytes;
}

void DeviceBuffer::release() noexcept {
    if (ptr_ != nullptr) cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
}

void DeviceBuffer::upload(const void* src, size_t bytes, cudaStream_t stream) {
    if (bytes > bytes_) throw Error(-1, "upload larger than the device buffer");
    if (stream == nullptr) {
        check_cuda(cudaMemcpy(ptr_, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    } else {
        check_cuda(cudaMemcpyAsync(ptr_, src, bytes, cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync H2D");
    }
}

int sm_count() {
    int device = 0, count = 0;
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    return count;
}

size_t element_bytes(Precision p) { return p == Precision::f64 ? sizeof(double) : sizeof(float); }

DeviceBuffer upload_real_table(const std::vector<double>& values, Precision p) {
    if (p == Precision::f64) return upload_vector(values);
    std::vector<float> f(values.begin(), values.end());
    return upload_vector(f);
}

namespace {
std::uint64_t active_columns(const std::vector<RetainedMode>& modes) {
    std::uint64_t active = 0;
    for (const auto& m : modes) active = std::max<std::uint64_t>(active, m.kx + 1);
    return active;
}
}  // namespace

HorizontalPlan::HorizontalPlan(const Workload& w, Precision p, bool pruned, std::uint64_t maxPlanes)
    : w_(w), p_(p), maxPlanes_(maxPlanes) {
    validate_workload(w);
    if (!supported_length(static_cast<long long>(w.nx)) || !supported_length(static_cast<long long>(w.ny)))
        throw Error(-2, "unsupported: the cuda provider transforms power-of-two Nx and Ny in [2, 1024]; got " +
                            std::to_string(w.nx) + "x" + std::to_string(w.ny));
    const auto planStart = Clock::now();
    const auto modes = retained_modes(w);
    modeCount_ = modes.size();
    if (pruned && modes.empty()) throw Error(-1, "pruned provider: the workload retains no modes");
    keep_ = static_cast<int>(pruned ? active_columns(modes) : w.nxHalf());
    const auto columnsForTables = pruned ? static_cast<std::uint64_t>(keep_) : w.nxHalf();
    const auto tables = column_tables(w, modes, columnsForTables);
    const auto twHalf = twiddle_table(std::max<std::uint64_t>(1, w.nx / 2));
    const auto twFull = twiddle_table(w.nx);
    const auto twCol = twiddle_table(w.ny);
    planningSeconds = seconds_since(planStart);

    const auto allocStart = Clock::now();
    twHalf_ = upload_real_table(twHalf, p);
    twFull_ = upload_real_table(twFull, p);
    twCol_ = upload_real_table(twCol, p);
    cellMap_ = upload_vector(tables.cellMap);
    gatherMap_ = upload_vector(tables.gatherMap);
    colStart_ = upload_vector(tables.colStart);
    colKy_ = upload_vector(tables.colKy);
    colMode_ = upload_vector(tables.colMode);
    modeKx_ = upload_vector(tables.modeKx);
    modeKy_ = upload_vector(tables.modeKy);
    modeConj_ = upload_vector(tables.modeConj);
    const size_t binBytes = static_cast<size_t>(w.ny) * keep_ * maxPlanes * 2 * element_bytes(p);
    bins_.allocate(binBytes);
    {
        // Per-column band of the retained cells, and whether it is exact.
        std::vector<int> band(static_cast<size_t>(keep_), -1);
        for (int kx = 0; kx < keep_; ++kx)
            for (std::uint64_t ky = 0; ky < w.ny; ++ky)
                if (tables.cellMap[kx * w.ny + ky] >= 0)
                    band[kx] = std::max(band[kx], static_cast<int>(std::min<std::uint64_t>(ky, w.ny - ky)));
        bandExact_ = true;
        for (int kx = 0; kx < keep_ && bandExact_; ++kx)
            for (std::uint64_t ky = 0; ky < w.ny; ++ky) {
                const bool cell = tables.cellMap[kx * w.ny + ky] >= 0;
                const bool inBand = static_cast<int>(std::min<std::uint64_t>(ky, w.ny - ky)) <= band[kx];
                if (cell != inBand) {
                    bandExact_ = false;
                    break;
                }
            }
        band_ = upload_vector(band);
    }
    allocationSeconds = seconds_since(allocStart);
    persistentBytes = twHalf_.bytes() + twFull_.bytes() + twCol_.bytes() + cellMap_.bytes() + gatherMap_.bytes() +
                      colStart_.bytes() +
                      colKy_.bytes() + colMode_.bytes() + modeKx_.bytes() + modeKy_.bytes() + modeConj_.bytes();
    scratchBytes = bins_.bytes();
}

ModeTables HorizontalPlan::tables() const {
    return {cellMap_.get<int>(), colStart_.get<int>(), colKy_.get<int>(), colMode_.get<int>(), gatherMap_.get<int>()};
}

void HorizontalPlan::forward_rows(const void* real, std::uint64_t planes, cudaStream_t s) const {
    if (planes > maxPlanes_) throw Error(-1, "plane count exceeds the plan's scratch");
    check_cuda(launch_rows_forward(p_, static_cast<int>(w_.nx), static_cast<int>(w_.ny),
                                   static_cast<long long>(planes), keep_, real, scratch(planes), twHalf_.get(),
                                   twFull_.get(), s),
               "row r2c kernel");
}

void HorizontalPlan::forward_columns(const ViewSet& views, double scale, cudaStream_t s) const {
    const auto planes = static_cast<std::uint64_t>(views.count) * w_.nz;
    if (planes > maxPlanes_) throw Error(-1, "plane count exceeds the plan's scratch");
    check_cuda(launch_columns_gather(p_, static_cast<int>(w_.ny), static_cast<int>(w_.nz), keep_, scratch(planes),
                                     views, tables(), scale, twCol_.get(), s),
               "column c2c + retention kernel");
}

void HorizontalPlan::inverse_columns(const ViewSet& views, cudaStream_t s) const {
    const auto planes = static_cast<std::uint64_t>(views.count) * w_.nz;
    if (planes > maxPlanes_) throw Error(-1, "plane count exceeds the plan's scratch");
    check_cuda(launch_columns_embed(p_, static_cast<int>(w_.ny), static_cast<int>(w_.nz), keep_, views, tables(),
                                    scratch(planes), twCol_.get(), s),
               "embedding + column c2c kernel");
}

void HorizontalPlan::inverse_columns_into(const ViewSet& views, DenseBins out, cudaStream_t s, int zStride) const {
    if (out.kxStride != keep_) throw Error(-1, "bin array must hold keep() columns per row");
    const int nz = static_cast<int>(w_.nz);
    if (zStride == 0) zStride = nz;
    if (p_ == Precision::f32 && columns_warp_supported(static_cast<long long>(w_.ny))) {
        check_cuda(launch_columns_embed_warp(static_cast<int>(w_.ny), nz, zStride, keep_, views, tables(), out,
                                             twCol_.get(), s),
                   "warp embedding + column c2c kernel");
        return;
    }
    if (zStride != nz) throw Error(-3, "padded bin planes need the FP32 warp column kernels");
    check_cuda(launch_columns_embed(p_, static_cast<int>(w_.ny), static_cast<int>(w_.nz), keep_, views, tables(), out,
                                    twCol_.get(), s),
               "embedding + column c2c kernel");
}

void HorizontalPlan::forward_columns_from(DenseBins in, const ViewSet& views, double scale, cudaStream_t s,
                                          int zStride) const {
    if (in.kxStride != keep_) throw Error(-1, "bin array must hold keep() columns per row");
    const int nz = static_cast<int>(w_.nz);
    if (zStride == 0) zStride = nz;
    if (p_ == Precision::f32 && columns_warp_supported(static_cast<long long>(w_.ny))) {
        check_cuda(launch_columns_gather_warp(static_cast<int>(w_.ny), nz, zStride, keep_, in, views, tables(), scale,
                                              twCol_.get(), s),
                   "warp column c2c + retention kernel");
        return;
    }
    if (zStride != nz) throw Error(-3, "padded bin planes need the FP32 warp column kernels");
    check_cuda(launch_columns_gather(p_, static_cast<int>(w_.ny), static_cast<int>(w_.nz), keep_, in, views,
                                     tables(), scale, twCol_.get(), s),
               "column c2c + retention kernel");
}

void HorizontalPlan::inverse_columns_band(DenseBins bins, int slots, int zStride, cudaStream_t s) const {
    if (!bandExact_ || p_ != Precision::f32 || !columns_warp_supported(static_cast<long long>(w_.ny)))
        throw Error(-3, "band column stage needs FP32, an exact retained band and Ny in [32, 512]");
    check_cuda(launch_columns_inverse_band(static_cast<int>(w_.ny), static_cast<int>(w_.nz), zStride, slots, keep_,
                                           bins, band_.get<int>(), twCol_.get(), bandFormInverse_, s),
               "band inverse column kernel");
}

void HorizontalPlan::forward_columns_band(DenseBins bins, int slots, double scale, int zStride, cudaStream_t s) const {
    if (!bandExact_ || p_ != Precision::f32 || !columns_warp_supported(static_cast<long long>(w_.ny)))
        throw Error(-3, "band column stage needs FP32, an exact retained band and Ny in [32, 512]");
    check_cuda(launch_columns_forward_band(static_cast<int>(w_.ny), static_cast<int>(w_.nz), zStride, slots, keep_,
                                           bins, band_.get<int>(), scale, twCol_.get(), bandFormForward_, s),
               "band forward column kernel");
}

void HorizontalPlan::inverse_rows(void* real, std::uint64_t planes, cudaStream_t s) const {
    if (planes > maxPlanes_) throw Error(-1, "plane count exceeds the plan's scratch");
    check_cuda(launch_rows_inverse(p_, static_cast<int>(w_.nx), static_cast<int>(w_.ny),
                                   static_cast<long long>(planes), keep_, scratch(planes), real, twHalf_.get(),
                                   twFull_.get(), s),
               "row c2r kernel");
}

void HorizontalPlan::forward(const void* real, std::uint64_t planes, const ViewSet& views, double scale,
                             cudaStream_t s) const {
    if (planes != static_cast<std::uint64_t>(views.count) * w_.nz)
        throw Error(-1, "field views must cover every real plane");
    forward_rows(real, planes, s);
    forward_columns(views, scale, s);
}

void HorizontalPlan::inverse(const ViewSet& views, void* real, cudaStream_t s) const {
    inverse_columns(views, s);
    inverse_rows(real, static_cast<std::uint64_t>(views.count) * w_.nz, s);
}

void HorizontalPlan::forward_dense(const void* real, void* wvm, std::uint64_t planes, cudaStream_t s) const {
    if (keep_ != static_cast<int>(w_.nxHalf())) throw Error(-3, "dense transform requested from a pruned plan");
    const DenseBins out{wvm, static_cast<long long>(planes), static_cast<long long>(w_.nxHalf())};
    check_cuda(launch_rows_forward(p_, static_cast<int>(w_.nx), static_cast<int>(w_.ny),
                                   static_cast<long long>(planes), keep_, real, out, twHalf_.get(), twFull_.get(), s),
               "row r2c kernel");
    check_cuda(launch_columns_dense(p_, -1, static_cast<int>(w_.ny), keep_, static_cast<long long>(planes), out, out,
                                    twCol_.get(), s),
               "column c2c kernel");
}

void HorizontalPlan::inverse_dense(const void* wvm, void* real, std::uint64_t planes, cudaStream_t s) const {
    if (keep_ != static_cast<int>(w_.nxHalf())) throw Error(-3, "dense transform requested from a pruned plan");
    if (planes > maxPlanes_) throw Error(-1, "plane count exceeds the plan's scratch");
    const DenseBins in{const_cast<void*>(wvm), static_cast<long long>(planes), static_cast<long long>(w_.nxHalf())};
    check_cuda(launch_columns_dense(p_, +1, static_cast<int>(w_.ny), keep_, static_cast<long long>(planes), in,
                                    scratch(planes), twCol_.get(), s),
               "column c2c kernel");
    check_cuda(launch_rows_inverse(p_, static_cast<int>(w_.nx), static_cast<int>(w_.ny),
                                   static_cast<long long>(planes), keep_, scratch(planes), real, twHalf_.get(),
                                   twFull_.get(), s),
               "row c2r kernel");
}

void HorizontalPlan::gather_dense(const void* wvm, std::uint64_t planes, const ViewSet& views, double scale,
                                  cudaStream_t s) const {
    const DenseBins in{const_cast<void*>(wvm), static_cast<long long>(planes), static_cast<long long>(w_.nxHalf())};
    check_cuda(launch_gather_dense(p_, static_cast<int>(w_.ny), static_cast<int>(w_.nz),
                                   static_cast<long long>(modeCount_), modeKx_.get<int>(), modeKy_.get<int>(),
                                   modeConj_.get<unsigned char>(), in, views, scale, s),
               "retention kernel");
}

void HorizontalPlan::embed_dense(const ViewSet& views, void* wvm, std::uint64_t planes, cudaStream_t s) const {
    if (keep_ != static_cast<int>(w_.nxHalf())) throw Error(-3, "dense embedding requested from a pruned plan");
    const DenseBins out{wvm, static_cast<long long>(planes), static_cast<long long>(w_.nxHalf())};
    check_cuda(launch_embed_dense(p_, static_cast<int>(w_.ny), static_cast<int>(w_.nz), keep_, views, tables(), out,
                                  s),
               "embedding kernel");
}

VerticalPlan::VerticalPlan(GemmPrecision p, int rowsOut, int inner, const std::vector<ModeGroup>& groups,
                           std::uint64_t fields, std::uint64_t members, const std::vector<double>& natural)
    : p_(p), R_(rowsOut), S_(inner) {
    if (groups.empty() || fields == 0 || members == 0) throw Error(-1, "Vertical GEMM requires groups and fields.");
    const auto matrixElems = static_cast<std::uint64_t>(rowsOut) * inner;
    if (natural.size() != groups.size() * matrixElems && natural.size() != matrixElems)
        throw Error(-1, "Vertical GEMM matrix family size does not match the groups.");
    const bool common = natural.size() == matrixElems && groups.size() > 1;
    std::uint64_t expected = 0;
    for (const auto& g : groups) {
        if (g.count == 0 || g.first != expected) throw Error(-1, "Vertical GEMM groups must be nonempty and contiguous.");
        expected += g.count;
    }
    const std::uint64_t perMember = expected * fields;
    if (members * perMember > static_cast<std::uint64_t>(INT32_MAX)) throw Error(-1, "too many GEMM columns");
    columns_ = members * perMember;
    members_ = members;
    memberColumns_ = static_cast<long long>(perMember);
    const std::uint64_t groupsCount = common ? 1 : groups.size();

    if (p == GemmPrecision::tf32x3 || p == GemmPrecision::bf16x3) {
        if (!tc_gemm_supported(rowsOut, inner))
            throw Error(-2, "unsupported: tensor-core GEMM needs the padded group matrix and two data stages in "
                            "227 KB of shared memory (R=" + std::to_string(rowsOut) + ", S=" + std::to_string(inner) +
                            ")");
        // FP32 matrices (one, if common to all groups) -> the kernel's
        // operand images, split into TF32 hi/lo or BF16 h/m/l and swizzled
        // once here.
        std::vector<float> f(natural.begin(), natural.end());
        const DeviceBuffer staged = upload_vector(f);
        const int images = static_cast<int>(groupsCount);
        imageStride_ = common ? 0 : static_cast<long long>(tc_gemm_image_bytes(rowsOut, inner));
        matrices_.allocate(static_cast<size_t>(images) * tc_gemm_image_bytes(rowsOut, inner));
        check_cuda(tc_gemm_build_images(staged.get<float>(), images, rowsOut, inner,
                                        p == GemmPrecision::bf16x3 ? 1 : 0, matrices_.get(), nullptr),
                   "tensor-core GEMM operand images");
        check_cuda(cudaStreamSynchronize(nullptr), "tensor-core GEMM operand images");
        std::vector<int> gc(groups.size()), gf(groups.size());
        for (std::uint64_t gi = 0; gi < groups.size(); ++gi) {
            gc[gi] = static_cast<int>(groups[gi].count * fields);
            gf[gi] = static_cast<int>(groups[gi].first * fields);
        }
        groupColumnsHost_ = gc;
        build_units(tc_gemm_unit_tiles());
        groupColumns_ = upload_vector(gc);
        groupFirst_ = upload_vector(gf);
        error_.allocate(sizeof(int));
        check_cuda(cudaMemset(error_.get(), 0, sizeof(int)), "cudaMemset");
        return;
    }

    // SIMT forms read the transposed matrices At[g][s][r].
    std::vector<double> At(groupsCount * matrixElems);
    for (std::uint64_t g = 0; g < groupsCount; ++g)
        for (int r = 0; r < rowsOut; ++r)
            for (int s = 0; s < inner; ++s)
                At[g * matrixElems + static_cast<std::uint64_t>(s) * rowsOut + r] =
                    natural[g * matrixElems + static_cast<std::uint64_t>(r) * inner + s];
    const int width = gemm_tile_columns(p);
    std::vector<int> gc(groups.size()), gf(groups.size());
    for (std::uint64_t gi = 0; gi < groups.size(); ++gi) {
        gc[gi] = static_cast<int>(groups[gi].count * fields);
        gf[gi] = static_cast<int>(groups[gi].first * fields);
    }
    groupColumnsHost_ = gc;
    // Member tiles unless they would run under 90 % full in a plan of several
    // members; then virtual tiles over each group's member-concatenated columns
    // (measured at 512², Nz 129, 8 members, FP64: forward 6.1 -> 4.5 ms with 4
    // targets, the two-family GEMMs 23.2 / 11.3 -> 21.9 / 4.6 ms; the 15-field
    // inverse, 94 % full as member tiles, ran 17.0 ms as member tiles and 20.4
    // as virtual ones).  Member tiles: one table whose prefixes serve smaller
    // member counts; virtual tiles: one table per member count.
    virtualTiles_ = simt_virtual_tiles(gc, members, width);
    const std::uint64_t tables = virtualTiles_ ? members : 1;
    tileTables_.resize(tables);
    tilePrefix_.assign(members, 0);
    for (std::uint64_t ti = 0; ti < tables; ++ti) {
        const std::uint64_t m = virtualTiles_ ? ti + 1 : members;
        const SimtTileTable h = simt_tiles(gc, gf, perMember, m, width, virtualTiles_, &tilePrefix_);
        TileTable& t = tileTables_[ti];
        t.group = upload_vector(h.group);
        t.column = upload_vector(h.column);
        t.count = upload_vector(h.count);
        t.per = upload_vector(h.per);
        t.first = upload_vector(h.first);
        t.tiles = static_cast<int>(h.group.size());
        if (virtualTiles_) tilePrefix_[m - 1] = t.tiles;
    }
    matrixStride_ = common ? 0 : static_cast<long long>(matrixElems);
    if (p == GemmPrecision::f64) {
        matrices_ = upload_vector(At);
    } else {
        std::vector<float> f(At.begin(), At.end());
        matrices_ = upload_vector(f);
    }
    groupColumns_ = upload_vector(gc);
    groupFirst_ = upload_vector(gf);
}

// Units: runs of up to tiles * 64 virtual (member, column) pairs of one
// group, largest first so the long units start early.  One table per active
// member count so partial batches launch only their units.
void VerticalPlan::build_units(int tiles) {
    if (tiles < 1) throw Error(-1, "work units need at least one tile");
    struct Unit {
        int g, col, count;
    };
    int device = 0, sms = 0;
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    const int span = tiles * 64;
    std::vector<UnitTable> tables;
    for (std::uint64_t active = 1; active <= members_; ++active) {
        // A group's units (runs of <= `tiles` M-tiles of its member columns)
        // go to one CTA, so the CTA loads the group's operand image once; a
        // group with more than a CTA's share of the work is cut into pieces of
        // at most that share.  Pieces are dealt largest first to the CTA with
        // the least work so far (one tile of work per piece stands for its
        // image load), and each CTA walks its units as one contiguous range.
        struct Piece {
            std::vector<Unit> units;
            long long work = 0;
        };
        const int groups = static_cast<int>(groupColumnsHost_.size());
        long long totalTiles = 0;
        int unitCount = 0;
        for (int gi = 0; gi < groups; ++gi) {
            const int total = static_cast<int>(active) * groupColumnsHost_[gi];
            totalTiles += (total + 63) / 64;
            unitCount += (total + span - 1) / span;
        }
        const int ctas = std::max(1, std::min(unitCount, sms > 0 ? sms : 148));
        const long long share = std::max<long long>(tiles, (totalTiles + ctas - 1) / ctas);
        std::vector<Piece> pieces;
        for (int gi = 0; gi < groups; ++gi) {
            const int total = static_cast<int>(active) * groupColumnsHost_[gi];
            Piece cur;
            for (int col = 0; col < total; col += span) {
                const Unit u{gi, col, std::min(span, total - col)};
                const long long t = (u.count + 63) / 64;
                if (!cur.units.empty() && cur.work + t > share) {
                    cur.work += 1;
                    pieces.push_back(std::move(cur));
                    cur = Piece{};
                }
                cur.units.push_back(u);
                cur.work += t;
            }
            if (!cur.units.empty()) {
                cur.work += 1;
                pieces.push_back(std::move(cur));
            }
        }
        std::vector<int> order(pieces.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = static_cast<int>(i);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return pieces[a].work > pieces[b].work; });
        std::vector<std::vector<int>> owned(ctas);
        // Least-loaded CTA by a min-heap of (load, cta).
        std::vector<std::pair<long long, int>> heap;
        for (int c = 0; c < ctas; ++c) heap.push_back({0, c});
        auto greater = [](const std::pair<long long, int>& a, const std::pair<long long, int>& b) { return a > b; };
        std::make_heap(heap.begin(), heap.end(), greater);
        for (const int pi : order) {
            std::pop_heap(heap.begin(), heap.end(), greater);
            auto& least = heap.back();
            owned[least.second].push_back(pi);
            least.first += pieces[pi].work;
            std::push_heap(heap.begin(), heap.end(), greater);
        }
        std::vector<int> ug, uc, un, first{0};
        for (int c = 0; c < ctas; ++c) {
            for (const int pi : owned[c])
                for (const Unit& u : pieces[pi].units) {
                    ug.push_back(u.g);
                    uc.push_back(u.col);
                    un.push_back(u.count);
                }
            first.push_back(static_cast<int>(ug.size()));
        }
        UnitTable table;
        table.units = static_cast<int>(ug.size());
        table.ctas = ctas;
        table.group = upload_vector(ug);
        table.column = upload_vector(uc);
        table.count = upload_vector(un);
        table.first = upload_vector(first);
        tables.push_back(std::move(table));
    }
    unitTables_ = std::move(tables);
    unitTiles_ = tiles;
}

void VerticalPlan::set_unit_tiles(int tiles) {
    if (!tensor_core()) throw Error(-3, "work-unit size applies to the tensor-core forms only");
    if (tiles != unitTiles_) build_units(tiles);
}

std::uint64_t VerticalPlan::persistentBytes() const {
    std::uint64_t units = 0;
    for (const auto& t : unitTables_) units += t.group.bytes() + t.column.bytes() + t.count.bytes() + t.first.bytes();
    for (const auto& t : tileTables_)
        units += t.group.bytes() + t.column.bytes() + t.count.bytes() + t.per.bytes() + t.first.bytes();
    return matrices_.bytes() + units +
           groupColumns_.bytes() + groupFirst_.bytes() + error_.bytes();
}

void VerticalPlan::execute(ComplexOperand in, ComplexOperand out, cudaStream_t s, std::uint64_t members,
                           const BinBoundary* inBins, const BinBoundary* outBins) const {
    if (members == 0) members = members_;
    if (members > members_) throw Error(-1, "more ensemble members than the plan was built for");
    if (tensor_core()) {
        if (in.im != nullptr || out.im != nullptr)
            throw Error(-3, "the tensor-core GEMM form takes interleaved complex operands");
        const UnitTable& table = unitTables_[members - 1];
        TcGemmArgs a{};
        a.B = matrices_.get<unsigned char>();
        a.imageStride = imageStride_;
        a.R = R_;
        a.S = S_;
        a.NP = (R_ + 15) / 16 * 16;
        a.KCH = (S_ + 31) / 32;
        a.unitGroup = table.group.get<int>();
        a.unitColumn = table.column.get<int>();
        a.unitCount = table.count.get<int>();
        a.units = table.units;
        a.ctaFirst = table.first.get<int>();
        a.ctas = table.ctas;
        a.groupColumns = groupColumns_.get<int>();
        a.groupFirst = groupFirst_.get<int>();
        a.memberColumns = memberColumns_;
        a.in = static_cast<const float2*>(in.re);
        a.out = static_cast<float2*>(out.re);
        a.error = error_.get<int>();
        a.expireWaitForTest = expireWaitForTest_ ? 1 : 0;
        a.kind = p_ == GemmPrecision::bf16x3 ? 1 : 0;
        if (inBins != nullptr) a.inBins = *inBins;
        if (outBins != nullptr) a.outBins = *outBins;
        check_cuda(launch_tc_gemm(a, s), "tensor-core grouped vertical GEMM kernel");
        return;
    }
    // SIMT tiles of the table for this member count; cell-addressed operands
    // decompose a tile column's global plan column into (member, mode, field)
    // with the plan's columns per member.
    const TileTable& table = tileTables_[virtualTiles_ ? members - 1 : 0];
    const GroupTiles t{table.group.get<int>(), table.column.get<int>(), table.count.get<int>(), table.per.get<int>(),
                       table.first.get<int>(), tilePrefix_[members - 1], memberColumns_, matrixStride_,
                       virtualTiles_};
    BinBoundary ib, ob;
    if (inBins != nullptr) {
        ib = *inBins;
        ib.memberColumns = memberColumns_;
    }
    if (outBins != nullptr) {
        ob = *outBins;
        ob.memberColumns = memberColumns_;
    }
    check_cuda(launch_grouped_gemm(p_, R_, S_, matrices_.get(), t, in, out, s, inBins ? &ib : nullptr,
                                   outBins ? &ob : nullptr),
               "grouped vertical GEMM kernel");
}

void VerticalPlan::check_device_error() const {
    if (error_.bytes() == 0) return;
    int flag = 0;
    check_cuda(cudaMemcpy(&flag, error_.get(), sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
    if (flag != 0) throw Error(-2, "tensor-core GEMM: a bounded device wait expired (MMA completion not observed)");
}

}  // namespace skb
