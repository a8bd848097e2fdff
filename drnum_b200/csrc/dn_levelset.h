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

// The reference's GPU level-set path (GPU_CartesianLevelSetBC, with
// StoredLevelSet and CompressibleLsSlip; gpu_cartesianlevelsetbc.h:106-125,
// 129-229, 414-487):
//   - every cell with G < 0 is deactivated (its constructor, :106-125);
//   - such a cell with a G >= 0 cell within two cells (the 5x5x5 box the
//     search walks, limited at the patch edges, :150-202) is a boundary cell
//     whose kernel writes nothing (its state-writing part is commented out,
//     :358-410, and it is launched on the other list, :509);
//   - every other G < 0 cell ("inside") is replaced after each stage by the
//     weighted mean of the cells of its (edge-limited) box whose G is larger,
//     weight |d . grad G| / |d| (:414-487), grad G by central differences
//     (one-sided at the patch edge, :78-93).
struct LsInsideCell {
  uint64_t cell;
  std::vector<uint64_t> nbr;   // averaged neighbours, in the kernel's loop order (di, dj, dk)
  std::vector<double> w;       // their weights
};

struct LevelSetGpu {
  std::vector<uint64_t> below;           // cells with G < 0, ascending
  std::vector<LsInsideCell> inside;      // inside cells, ascending
};

// Classifies one patch for the GPU level-set path.  Returns false with a
// message where the reference stops with a BUG (a G < 0 cell whose search
// box reaches, at twice its offset, beyond the patch: gpu_cartesianlevelsetbc.h:170-179).
bool classify_levelset_gpu(const OverlapPatch& patch, const double* G, LevelSetGpu& out, std::string& err);

} // namespace dn
