// Overlap set-up between Cartesian patches: receiving (seek) cells, donor
// cells and trilinear weights, in the form the reference hands to its donor
// copy (Patch::buildDonorTransferData, patch.cpp:128-218).
//
// Host code, run once per grid.  The tables are built with the reference's
// floating-point steps so that indices are identical and weights equal bit
// for bit (compile with -ffp-contract=off):
//   region bounds          CartesianPatch::buildRegions       cartesianpatch.cpp:314-390
//   cell spacing, centres  CartesianPatch::computeDeltas      cartesianpatch.cpp:160-212
//                          CartesianPatch::xyzCell            cartesianpatch.h:267-273
//   receiving cells        CartesianPatch::extractSeekCells   cartesianpatch.cpp:393-491
//                          Patch::compactReceiveCellLists     patch.cpp:466-484
//   receiver -> donor frame CoordTransform concatenate/transform (math/coordtransform.h:105-165)
//                          for axis-aligned patches: x_d = x_r + (o_r - o_d)
//   1-D coefficients       CartesianPatch::linearCCInterpolCoeffs   cartesianpatch.cpp:1053-1162
//   8-point weights        CartesianPatch::computeCCDataInterpolCoeffs_V1  cartesianpatch.cpp:1166-1299
//   weight clean-up        WeightedSet::Unify / EliminateBelowEps / adjustWeightSumShift
//                          (weightedset.h:374-404, 569-619)
//   donor order            PatchGrid::computeDependencies     patchgrid.cpp:119-268 (ascending
//                          patch index; patches that serve no receiving cell are dropped)
//   multi-donor average    Patch::finalizeDependencies        patch.cpp:319-465,
//                          InterCoeffWS::adjust2Average       intercoeffws.h:233-242
//   padding to a stride    InterCoeffPad::build               intercoeffpad.h:139-170
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "drnum_b200.h"

namespace dn {

struct OverlapPatch {
  int n[3];            // cells per axis
  double origin[3];    // lower corner, inertial frame
  double d[3];         // cell spacing
  int seek[6];         // seek layers imin, imax, jmin, jmax, kmin, kmax
  int add_protect;     // additional protected layers
};

// Donor tables of one receiving patch, laid out like the reference's
// concatenated direct-transfer arrays.
struct DonorTables {
  std::vector<uint64_t> rec_unique;        // receiving cells with at least one donor, ascending
  std::vector<int32_t> donor_patch;        // donor patch per donor (ascending patch index)
  std::vector<int64_t> num_receivers;      // receiving cells served per donor
  std::vector<int32_t> stride;             // padded contributions per receiving cell, per donor
  std::vector<uint64_t> rec_concat;        // receiving cell per (donor, receiver), donors concatenated
  std::vector<uint64_t> donor_idx;         // donor cell per (donor, receiver, contribution)
  std::vector<double> weight;              // weight per (donor, receiver, contribution)
  int64_t no_donor = 0;                    // seek cells that found no donor (dropped)
};

// Builds the tables of every patch.  Returns false with a message when a
// patch description is invalid.
bool build_overlap(const std::vector<OverlapPatch>& patches, std::vector<DonorTables>& out, std::string& err);

// Cell-centred trilinear interpolation weights of point xyz (patch frame)
// inside the donor zone of patch p (CartesianPatch::computeCCDataInterpolCoeffs_V1,
// cartesianpatch.cpp:1166-1299).  Returns 1 with the weights, 0 outside the
// donor zone, -1 where the reference stops with a BUG.  *pad_index (when
// given and some weight was dropped) receives the index the reference's
// fixed-size transfer pads with.
int cc_interpolation_weights(const OverlapPatch& p, const double xyz[3], std::vector<std::pair<size_t, double>>& ws,
                             size_t* pad_index);

// Cell spacing of a patch description: length/n where a length is given
// (CartesianPatch::computeDeltas, cartesianpatch.cpp:160-165), else dx/dy/dz.
void desc_spacing(const struct dn_patch_desc& d, double out[3]);

// Overlap description of a patch description.
OverlapPatch overlap_patch(const struct dn_patch_desc& d);

// Exchange lists of a patch grid sharded over ranks (patch p on rank
// owner[p]).  For every peer q of `rank`: recv = the donor cells of patches
// of q that the donor tables of this rank's receiving patches read, send =
// the donor cells of this rank's patches that q's receiving patches read;
// each as (patch, cell) pairs, unique, ascending by patch then cell, so that
// both sides of a pair of ranks derive the same order independently.
struct Exchange {
  int rank = 0, world = 1;
  std::vector<std::vector<int32_t>> send_patch, recv_patch;   // [peer][item]
  std::vector<std::vector<uint64_t>> send_cell, recv_cell;
  // device copies (allocated on first use by the context that packs/unpacks)
  int device = -1;
  std::vector<void*> dev;
};

bool build_exchange(const std::vector<DonorTables>& tables, const int32_t* owner, int rank, int world,
                    Exchange& ex, std::string& err);

} // namespace dn

struct dn_overlap {
  std::vector<dn::DonorTables> tables;
};

struct dn_exchange {
  dn::Exchange ex;
};
