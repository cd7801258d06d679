// Halo tiles of the fused member-stage kernels (mpsw_fused.cuh).
//
// A tile owns a run of K consecutive cells of the internal (Hilbert) order and the edges whose
// lower-numbered cell is among them.  The fused kernel of a tangent-linear or adjoint RK stage
// computes every intermediate it needs for its owned cells and edges inside one thread block,
// on a halo of neighbouring cells, edges and vertices around them, so the stage reads its
// member inputs once and writes only its outputs: no intermediate row goes to HBM.
//
// Each tile numbers its entities locally (16-bit indices) in nested layers: the owned entities
// first, then each ring the stage's phases need, so a phase works on a prefix of a local
// space.  cnt[] holds the prefix sizes (TileLayer), the records give each local entity's
// neighbours as local indices (kNoLocal where the neighbour is not in the tile, which the
// builder checks no phase reads), and g*[] its internal index.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "mpsw_internal.h"
#include "mpsw_setup.h"

namespace mpsw {

constexpr uint16_t kNoLocal = 0xFFFF;

// Prefix sizes of a tile's local spaces (TileLayer, mpsw_internal.h):
//   tangent linear: E_OWN owned edges | E_MID = E1 (owned + their edgesOnEdge) | E_ALL inputs
//                   C_OWN owned cells | C_KE = owned + cells of owned edges | C_MID = C1 (cells
//                   of E1) | C_ALL inputs;  V_ALL = vertices of C1 and E1
//   adjoint:        E_OWN | E_MID = EA (edges whose pv_edge / thickness-flux adjoints are formed)
//                   | E_ALL;  C_OWN | C_KE | C_MID = CB (cells whose pv_cell adjoint is formed)
//                   | C_ALL;  V_ALL = vertices of the owned cells and edges

// Record strides (16-bit words): edge c1 c2 v1 v2 eoe[10] + 2 pad; cell es[6] vs[6] nb[6] + 6
// pad; vertex es[3] cs[3] + 2 pad.
constexpr int kERec = 16, kCRec = 24, kVRec = 8;

struct TileSetHost {
  int K = 0, ntiles = 0;
  int max_cnt[kTileCounts] = {};            // largest count of each layer over the tiles
  std::vector<int> cnt;                     // [ntiles][kTileCounts]
  std::vector<int> off;                     // [ntiles][3] first edge / cell / vertex of ge / gc / gv
  std::vector<int> ge, gc, gv;              // internal index of each local entity, tile after tile
  std::vector<unsigned char> blob;          // the tiles' blobs (BlobSection), each 16-byte aligned
  std::vector<long long> blob_off;          // [ntiles] byte offset of each tile's blob
  size_t smem[4] = {0, 0, 0, 0};            // shared memory of the stage's block, 4 / 8 / 16 / 32 members
};

// Build the tangent-linear (adjoint = false) or adjoint tiles for a mesh with at most 6 edges
// per cell and 10 edgesOnEdge, with their blobs (coefficients formed in FP64 from the mesh and
// rounded to FP32).  Each tile owns a run of consecutive cells of the internal order, as long as
// its block's shared memory with M members per chunk stays within `budget` bytes and at most
// `kmax` cells.  Returns an empty string or the problem found (a cell whose halo alone exceeds
// the budget, or a phase that would read outside its tile).
std::string build_tiles(const BuiltMesh &m, size_t budget, int kmax, int M, bool adjoint, TileSetHost *out);

}  // namespace mpsw
