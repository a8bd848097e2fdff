// Level-set wall classification of one Cartesian patch: the cell layers next
// to the zero level of a signed-distance field G, their normalised G
// gradients and, for the inner (G < 0) layers, the 8-point mirror-point
// donors of the slip-wall boundary condition.
//
// Host code, run once per geometry.  Restates LevelSetObject::extractBCellLayers
// (levelsetobject.cpp:83-388) step by step so that the layer lists, gradients
// and donor tables equal the reference's (compile with -ffp-contract=off):
//   g_eps = (g_max - g_min) * 1e-7                      levelsetobject.cpp:108-117
//   layer 0: a face neighbour of the other sign, tested with the eps-guarded
//            products (neighbour order k-1, k+1, j-1, j+1, i-1, i+1,
//            CartesianPatch::cellOverFaceNeighbours, cartesianpatch.cpp:55-96)
//                                                       levelsetobject.cpp:119-155
//   inner layer 0 replaced by deeper neighbours where G > -min_rel * (spread of
//   the neighbours' G) / 2                              levelsetobject.cpp:157-222
//   further layers: unmarked face neighbours of the layer below with G < 0
//   (inner) or G > 0 (outer)                            levelsetobject.cpp:237-292
//   gradient: central differences (one-sided at the patch edge), normalised
//                                                       CartesianPatch::computeNablaVar,
//                                                       cartesianpatch.cpp:1592-1657
//   mirror point x_c - 2 G grad(G) and its trilinear donors in the same patch,
//   fixed to 8 entries; cells whose mirror point leaves the donor zone are
//   dropped                                             levelsetobject.cpp:294-369
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "dn_overlap.h"

namespace dn {

struct LayerCell {
  uint64_t cell;
  double g;            // level-set value
  double grad[3];      // normalised gradient of G
  uint64_t donor[8];   // mirror-point donors (inner layers only)
  double weight[8];
};

struct LevelSetLayers {
  std::vector<std::vector<LayerCell>> inner;   // [layer][cell]
  std::vector<std::vector<LayerCell>> outer;
  int64_t replaced = 0;                        // inner layer-0 cells replaced by deeper ones
};

// Classifies one patch.  Returns false with a message on invalid input or
// where the reference stops with a BUG.
bool classify_levelset(const OverlapPatch& patch, const double* G, int num_inner, int num_outer,
                       double min_inner_rel_dist, LevelSetLayers& out, std::string& err);

} // namespace dn
