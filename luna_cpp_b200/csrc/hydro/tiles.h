// The sweep's tiles: groups of up to kTileCells cells close in space, each with the set of cells its lists reach (its
// own cells, then the halo), which one block stages into shared memory before it walks the lists. Built on the host
// once per mesh (a static mesh: once; a moving mesh: after each remesh).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace luna {

constexpr int kTileCells = 128;  // cells (threads) of a tile: one block
constexpr int kTileRows = 416;   // staged rows a tile may use (39 KB of shared memory); a cell alone needing more gets a
                                 // tile of its own, swept by a second launch with more shared memory
constexpr int kBigTileRows = 2360;  // the most rows one block can stage (227 KB); a mesh with a larger list is refused

struct SweepTiles {
    std::vector<int32_t> order;        // [tiles * kTileCells]: the cell of each thread, -1 for an idle one
    std::vector<int32_t> slice_base;   // [tiles * kTileCells / 32 + 1]: each warp's first slot, in slots of 32 entries
    std::vector<int32_t> stage_start;  // [tiles + 1]
    std::vector<int32_t> stage_cells;  // the staged cells of each tile: its own cells in thread order, then the halo
    std::vector<uint32_t> local;       // [slots]: each entry's neighbour as a row of its tile's staged cells
    int64_t tiles = 0, normal_tiles = 0;  // tiles [normal_tiles, tiles) are single cells needing > kTileRows rows
    int normal_rows = 0, big_rows = 0;    // the most staged rows in a tile of each kind
};

// Cells in Morton order of their generators, cut greedily into tiles of at most kTileCells cells and kTileRows
// staged rows; within a tile, cells by list length (longest first), so a warp's lists have nearly one length.
// Returns an empty string, or why the mesh cannot be tiled.
std::string build_sweep_tiles(int dim, int64_t n_cells, const double* positions, const double* box, const int32_t* start,
                              const int32_t* list, const int32_t* owner, const int32_t* neighbour, SweepTiles& out);

}  // namespace luna
