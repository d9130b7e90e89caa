// Host code: the sweep's tiles (tiles.h).
#include <algorithm>
#include <cmath>
#include <numeric>

#include "luna_b200.h"
#include "tiles.h"

namespace luna {

std::string build_sweep_tiles(int dim, int64_t n_cells, const double* positions, const double* box, const int32_t* start,
                              const int32_t* list, const int32_t* owner, const int32_t* neighbour, SweepTiles& out) {
    const int64_t N = n_cells;
    auto neighbour_of = [&](int32_t e) -> int32_t {  // the list entry's other cell (~f: a face the cell does not own)
        const int32_t f = e >= 0 ? e : ~e;
        return e >= 0 ? neighbour[f] : owner[f];
    };
    for (int64_t c = 0; c < N; ++c)
        if (start[c + 1] - start[c] + 1 > kBigTileRows)
            return "cell " + std::to_string(c) + " has " + std::to_string(start[c + 1] - start[c]) + " faces; the sweep stages at most " +
                   std::to_string(kBigTileRows - 1) + " neighbours of a cell";

    std::vector<std::pair<uint64_t, int32_t>> keyed(static_cast<size_t>(N));
    for (int64_t c = 0; c < N; ++c) keyed[c] = {morton_key(dim, positions + dim * c, box), static_cast<int32_t>(c)};
    std::sort(keyed.begin(), keyed.end());

    // Greedy cut along the Morton order: a cell joins the open tile while the tile has room for it and for the new
    // staged rows it brings (itself and its neighbours not yet staged).
    std::vector<std::vector<int32_t>> tile_cells, tile_rows;
    std::vector<int32_t> mark(static_cast<size_t>(N), -1);
    std::vector<int32_t> cells, rows, added;
    int32_t open = 0;
    auto touch_cell = [&](int32_t c) {
        added.clear();
        auto touch = [&](int32_t j) {
            if (mark[j] != open) {
                mark[j] = open;
                added.push_back(j);
            }
        };
        touch(c);
        for (int32_t k = start[c]; k < start[c + 1]; ++k) touch(neighbour_of(list[k]));
    };
    auto close = [&]() {
        tile_cells.push_back(cells);
        tile_rows.push_back(rows);
        cells.clear();
        rows.clear();
        ++open;
    };
    for (const auto& kc : keyed) {
        const int32_t c = kc.second;
        touch_cell(c);
        if (!cells.empty() && (static_cast<int>(cells.size()) == kTileCells || rows.size() + added.size() > static_cast<size_t>(kTileRows))) {
            for (int32_t j : added) mark[j] = -1;
            close();
            touch_cell(c);
        }
        cells.push_back(c);
        rows.insert(rows.end(), added.begin(), added.end());
    }
    if (!cells.empty()) close();

    // Tiles within the row budget first, then the single cells that need more.
    std::vector<int64_t> tile_order;
    for (size_t t = 0; t < tile_cells.size(); ++t)
        if (tile_rows[t].size() <= static_cast<size_t>(kTileRows)) tile_order.push_back(static_cast<int64_t>(t));
    out.normal_tiles = static_cast<int64_t>(tile_order.size());
    for (size_t t = 0; t < tile_cells.size(); ++t)
        if (tile_rows[t].size() > static_cast<size_t>(kTileRows)) tile_order.push_back(static_cast<int64_t>(t));
    out.tiles = static_cast<int64_t>(tile_order.size());

    const int64_t threads = out.tiles * kTileCells, slices = threads / 32;
    out.order.assign(static_cast<size_t>(threads), -1);
    out.slice_base.assign(static_cast<size_t>(slices + 1), 0);
    out.stage_start.assign(static_cast<size_t>(out.tiles + 1), 0);
    out.stage_cells.clear();
    out.normal_rows = out.big_rows = 0;
    auto length = [&](int32_t c) { return start[c + 1] - start[c]; };
    for (int64_t u = 0; u < out.tiles; ++u) {
        std::vector<int32_t>& tc = tile_cells[static_cast<size_t>(tile_order[u])];
        std::stable_sort(tc.begin(), tc.end(), [&](int32_t a, int32_t b) { return length(a) > length(b); });
        for (size_t k = 0; k < tc.size(); ++k) out.order[u * kTileCells + static_cast<int64_t>(k)] = tc[k];
        for (int s = 0; s < kTileCells / 32; ++s) {
            int longest = 0;
            for (int l = 0; l < 32; ++l) {
                const int32_t c = out.order[u * kTileCells + 32 * s + l];
                if (c >= 0) longest = std::max(longest, length(c));
            }
            const int64_t slice = u * (kTileCells / 32) + s;
            out.slice_base[slice + 1] = out.slice_base[slice] + longest;
        }
        // staged rows: the tile's cells in thread order, then the halo by cell index
        std::vector<int32_t> halo;
        for (int32_t j : tile_rows[static_cast<size_t>(tile_order[u])]) mark[j] = -2;
        for (int32_t c : tc) mark[c] = -3;
        for (int32_t j : tile_rows[static_cast<size_t>(tile_order[u])])
            if (mark[j] == -2) halo.push_back(j);
        std::sort(halo.begin(), halo.end());
        out.stage_cells.insert(out.stage_cells.end(), tc.begin(), tc.end());
        out.stage_cells.insert(out.stage_cells.end(), halo.begin(), halo.end());
        const int rows_here = static_cast<int>(tc.size() + halo.size());
        out.stage_start[u + 1] = out.stage_start[u] + rows_here;
        int& most = u < out.normal_tiles ? out.normal_rows : out.big_rows;
        most = std::max(most, rows_here);
    }

    // Each entry's neighbour as a row of its tile's staged cells.
    const size_t slots = static_cast<size_t>(out.slice_base[slices]) * 32;
    out.local.assign(slots > 0 ? slots : 1, 0u);
    std::vector<int32_t>& row_of = mark;  // reused: the staged row of a cell within the tile being filled
    for (int64_t u = 0; u < out.tiles; ++u) {
        const int32_t s0 = out.stage_start[u], s1 = out.stage_start[u + 1];
        for (int32_t r = s0; r < s1; ++r) row_of[out.stage_cells[r]] = r - s0;
        for (int k = 0; k < kTileCells; ++k) {
            const int64_t t = u * kTileCells + k;
            const int32_t c = out.order[t];
            if (c < 0) continue;
            const int64_t slot0 = static_cast<int64_t>(out.slice_base[t >> 5]) * 32 + (t & 31);
            for (int32_t e = 0; e < length(c); ++e)
                out.local[static_cast<size_t>(slot0 + 32 * static_cast<int64_t>(e))] = static_cast<uint32_t>(row_of[neighbour_of(list[start[c] + e])]);
        }
    }
    return std::string();
}

std::string build_tile_faces(int64_t n_cells, int64_t n_faces, int64_t tiles, const int32_t* order, const int32_t* start, const int32_t* list,
                             const int32_t* owner, const int32_t* neighbour, TileFaces& out) {
    const int64_t N = n_cells, F = n_faces;
    if (F >= kCrossing) return "too many faces for the fused pass";
    std::vector<int32_t> tile_of(static_cast<size_t>(N), -1);
    for (int64_t t = 0; t < tiles; ++t)
        for (int k = 0; k < kTileCells; ++k) {
            const int32_t c = order[t * kTileCells + k];
            if (c < 0) continue;
            if (c >= N || tile_of[c] >= 0) return "a cell out of range or in two tiles";
            tile_of[c] = static_cast<int32_t>(t);
        }
    for (int64_t i = 0; i < N; ++i)
        if (tile_of[i] < 0) return "a cell in no tile";
    // every list entry must be its face's owner's (owned) or neighbour's (not owned) entry
    for (int64_t i = 0; i < N; ++i)
        for (int32_t k = start[i]; k < start[i + 1]; ++k) {
            const int32_t e = list[k], f = e >= 0 ? e : ~e;
            if ((e >= 0 ? owner[f] : neighbour[f]) != i) return "a list entry its face's owner or neighbour does not match";
        }
    std::vector<int32_t> xindex(static_cast<size_t>(F), -1), slot_of(static_cast<size_t>(F), -1);
    out.xface.clear();
    for (int64_t f = 0; f < F; ++f)
        if (tile_of[owner[f]] != tile_of[neighbour[f]]) {
            xindex[f] = static_cast<int32_t>(out.xface.size());
            out.xface.push_back(static_cast<int32_t>(f));
        }
    out.tstart.assign(static_cast<size_t>(tiles) + 1, 0);
    out.tface.clear();
    out.max_slots = 0;
    for (int64_t t = 0; t < tiles; ++t) {
        const size_t base = out.tface.size();
        for (int k = 0; k < kTileCells; ++k) {
            const int32_t c = order[t * kTileCells + k];
            if (c < 0) continue;
            for (int32_t j = start[c]; j < start[c + 1]; ++j) {
                const int32_t e = list[j];
                if (e < 0 || xindex[e] >= 0) continue;
                slot_of[e] = static_cast<int32_t>(out.tface.size() - base);
                out.tface.push_back(e);
            }
        }
        const size_t slots = out.tface.size() - base;
        if (slots >= static_cast<size_t>(kCrossing)) return "too many faces in a tile";
        out.max_slots = std::max(out.max_slots, static_cast<int>(slots));
        out.tstart[t + 1] = static_cast<int32_t>(out.tface.size());
    }
    out.eslot.resize(static_cast<size_t>(2 * F));
    for (int64_t k = 0; k < 2 * F; ++k) {
        const int32_t e = list[k], f = e >= 0 ? e : ~e;
        const int32_t v = xindex[f] >= 0 ? (kCrossing | xindex[f]) : slot_of[f];
        if (v < 0) return "an interior face without its owner's entry";
        out.eslot[k] = e >= 0 ? v : ~v;
    }
    return std::string();
}

}  // namespace luna

namespace luna {
// The library's error report (luna_last_error), defined with the other entry points.
luna_status report_error(luna_status s, const std::string& what);
}  // namespace luna

extern "C" {

LUNA_API luna_status luna_mesh_tiles(const luna_mesh_desc* mesh, int64_t counts[6], int32_t* order, int32_t* slice_base, int32_t* stage_start,
                                     int32_t* stage_cells, uint32_t* local) {
    if (!mesh || !counts) return luna::report_error(LUNA_EINVAL, "luna_mesh_tiles: null argument");
    if (mesh->on_device) return luna::report_error(LUNA_EINVAL, "luna_mesh_tiles: the mesh arrays must be host pointers");
    if (mesh->dim != 2 && mesh->dim != 3) return luna::report_error(LUNA_EINVAL, "luna_mesh_tiles: dim must be 2 or 3");
    if (mesh->n_cells <= 0 || mesh->n_faces < 0 || !mesh->cell_face_start || !mesh->positions || (mesh->n_faces > 0 && (!mesh->cell_face || !mesh->owner || !mesh->neighbour)))
        return luna::report_error(LUNA_EINVAL, "luna_mesh_tiles: mesh arrays missing");
    for (int a = 0; a < mesh->dim; ++a)
        if (!(mesh->box[a] > 0)) return luna::report_error(LUNA_EINVAL, "luna_mesh_tiles: box sides must be positive");
    luna::SweepTiles t;
    const std::string why = luna::build_sweep_tiles(mesh->dim, mesh->n_cells, mesh->positions, mesh->box, mesh->cell_face_start, mesh->cell_face,
                                                    mesh->owner, mesh->neighbour, t);
    if (!why.empty()) return luna::report_error(LUNA_EINVAL, "mesh: " + why);
    counts[0] = t.tiles;
    counts[1] = t.normal_tiles;
    counts[2] = static_cast<int64_t>(t.stage_cells.size());
    counts[3] = static_cast<int64_t>(t.local.size());
    counts[4] = t.normal_rows;
    counts[5] = t.big_rows;
    if (order) std::copy(t.order.begin(), t.order.end(), order);
    if (slice_base) std::copy(t.slice_base.begin(), t.slice_base.end(), slice_base);
    if (stage_start) std::copy(t.stage_start.begin(), t.stage_start.end(), stage_start);
    if (stage_cells) std::copy(t.stage_cells.begin(), t.stage_cells.end(), stage_cells);
    if (local) std::copy(t.local.begin(), t.local.end(), local);
    return LUNA_OK;
}

}  // extern "C"
