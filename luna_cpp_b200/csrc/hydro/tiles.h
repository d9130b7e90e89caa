// The sweep's tiles: groups of up to kTileCells cells close in space, each with the set of cells its lists reach (its
// own cells, then the halo), which one block stages into shared memory before it walks the lists. Built on the host
// once per mesh (a static mesh: once; a moving mesh: after each remesh).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "luna_b200.h"

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

// The Morton key of a generator: its cell on a 2^b grid of the box per axis (b = 21 in 3D, 32 in 2D), bits
// interleaved with axis 0 lowest.
__host__ __device__ inline uint64_t morton_key(int dim, const double* x, const double* box) {
    const int bits = dim == 3 ? 21 : 32;
    const double cells = static_cast<double>(uint64_t(1) << bits);
    uint64_t key = 0;
    for (int a = 0; a < dim; ++a) {
        double u = x[a] / box[a];
        u -= floor(u);  // generators may sit anywhere in their periodic image
        uint64_t q = static_cast<uint64_t>(u * cells);
        const uint64_t top = (uint64_t(1) << bits) - 1;
        if (q > top) q = top;
        for (int b = 0; b < bits; ++b) key |= ((q >> b) & 1u) << (dim * b + a);
    }
    return key;
}

// Cells in Morton order of their generators, cut greedily into tiles of at most kTileCells cells and kTileRows
// staged rows; within a tile, cells by list length (longest first), so a warp's lists have nearly one length.
// Returns an empty string, or why the mesh cannot be tiled.
std::string build_sweep_tiles(int dim, int64_t n_cells, const double* positions, const double* box, const int32_t* start,
                              const int32_t* list, const int32_t* owner, const int32_t* neighbour, SweepTiles& out);

// The faces of the tiles for the fused flux-and-update pass of a static mesh (geometry.cuh::k_tile_flux_update): a face
// whose two cells share a tile is an interior face of that tile, solved by the tile's block into shared memory; a face
// between two tiles is a crossing face, solved once by its own pass into a flux row in HBM. Each list entry names its
// face's flux: an interior slot s of its cell's tile, or kCrossing | the crossing index; ~ of that for a face the cell
// does not own (the list's own encoding).
constexpr int32_t kCrossing = 1 << 30;
struct TileFaces {
    std::vector<int32_t> tstart;  // [tiles + 1]: each tile's interior faces in tface
    std::vector<int32_t> tface;   // the interior faces, tile by tile: the tile's cells in thread order, each cell's owned
                                  // entries in list order
    std::vector<int32_t> xface;   // the crossing faces, in face order
    std::vector<int32_t> eslot;   // [2F]: each list entry's flux
    int max_slots = 0;            // the most interior faces of a tile
};
// From the sweep's tiles (order [tiles * kTileCells]) and the mesh's lists; an empty string, or why the plan cannot be
// made (a cell in no tile or in two, a list entry its face's owner or neighbour does not match).
std::string build_tile_faces(int64_t n_cells, int64_t n_faces, int64_t tiles, const int32_t* order, const int32_t* start, const int32_t* list,
                             const int32_t* owner, const int32_t* neighbour, TileFaces& out);

// The same tiles cut on the device from a device mesh, for a mesh that is rebuilt every step (the moving mesh's
// remesh): the cells of a tile are 128 consecutive cells of the Morton order (no greedy cut), within a tile by list
// length, longest first; a tile staging more than kTileRows rows goes with the single-cell tiles of the host cut to the
// second launch. The sweep's results do not depend on the tiling (the staged rows are copies of HBM rows).
struct DeviceTilePlan {
    int64_t tiles = 0, normal_tiles = 0, staged = 0, slots = 0;
    int normal_rows = 0, big_rows = 0;
    bool fits = false;  // false: a tile needs more than the block can sort or stage (use the host cut)
};
class DeviceTiler;
DeviceTiler* device_tiler_create();
void device_tiler_destroy(DeviceTiler* t);
// Plans the tiles (synchronises on s for their sizes); the mesh arrays must stay valid until device_tiles_fill.
luna_status device_tiles_plan(DeviceTiler* t, int dim, int64_t n, const double* pos, const double* box, const int32_t* start,
                              const int32_t* list, const int32_t* owner, const int32_t* neighbour, cudaStream_t s, DeviceTilePlan* plan);
// Writes the planned tiles: order [tiles * kTileCells], slice_base [tiles * kTileCells / 32 + 1], stage_start
// [tiles + 1], stage_cells [staged], local [slots] (as SweepTiles).
luna_status device_tiles_fill(DeviceTiler* t, int32_t* order, int32_t* slice_base, int32_t* stage_start, int32_t* stage_cells, uint32_t* local,
                              cudaStream_t s);

}  // namespace luna
