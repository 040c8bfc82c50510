// Zincblende conventional cell: in-cell site positions (units of a) and the
// four-neighbour map {di, dj, dk, site} per site, in the order of
// Cell::Initialize / Cell::nnmap (nemo3d/src/base/Cell.c:185-210, 599-715).
// The order is part of the vector layout contract, so it is carried over.
#pragma once

#include <cstdint>

namespace tbgpu {

static __constant__ double c_site_pos[8][3] = {
    {0, 0, 0},           {0, -0.5, -0.5},       {-0.5, -0.5, 0},
    {-0.5, 0, -0.5},     {-0.25, -0.25, -0.25}, {-0.25, -0.75, -0.75},
    {-0.75, -0.75, -0.25}, {-0.75, -0.25, -0.75}};

static __constant__ int8_t c_nnmap[8][4][4] = {
    {{0, 0, 0, 4}, {1, 0, 1, 7}, {1, 1, 0, 6}, {0, 1, 1, 5}},
    {{0, 0, 0, 5}, {0, 0, 0, 4}, {1, 0, 0, 6}, {1, 0, 0, 7}},
    {{0, 0, 0, 4}, {0, 0, 0, 6}, {0, 0, 1, 5}, {0, 0, 1, 7}},
    {{0, 0, 0, 4}, {0, 0, 0, 7}, {0, 1, 0, 5}, {0, 1, 0, 6}},
    {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 0, 2}, {0, 0, 0, 3}},
    {{0, 0, 0, 1}, {0, -1, 0, 3}, {0, 0, -1, 2}, {0, -1, -1, 0}},
    {{0, 0, 0, 2}, {0, -1, 0, 3}, {-1, 0, 0, 1}, {-1, -1, 0, 0}},
    {{0, 0, 0, 3}, {0, 0, -1, 2}, {-1, 0, 0, 1}, {-1, 0, -1, 0}}};

// c_rev_slot[m][n]: for site m and its neighbour slot n, the slot of the
// neighbour's list that points back across the same bond (derived from the
// map above).  Every bond is stored once, in the cation's slot; an anion
// reads that block, transposed, through this table.
#define TBGPU_REV_SLOT_TABLE                                 \
  {{0, 3, 3, 3}, {0, 1, 2, 2}, {2, 0, 2, 1}, {3, 0, 1, 1}, \
   {0, 1, 0, 0}, {0, 2, 2, 3}, {1, 3, 2, 2}, {1, 3, 3, 1}}
static __constant__ int8_t c_rev_slot[8][4] = TBGPU_REV_SLOT_TABLE;
// the same table for host code
constexpr int8_t kRevSlot[8][4] = TBGPU_REV_SLOT_TABLE;

}  // namespace tbgpu
