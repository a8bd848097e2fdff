// Overlap set-up between Cartesian patches (see dn_overlap.h for the
// reference steps each part restates).  Compiled with -ffp-contract=off: the
// weights must round exactly like the reference's.
#include "dn_overlap.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <utility>

namespace dn {

namespace {

// Donor zone and geometry of one patch, derived once.
struct Zone {
  int n[3];
  size_t first[3], afterlast[3];   // donor zone [first, afterlast) per axis
  double d[3];                     // spacing
  double cc_min[3];                // centre of cell 0 (0.5 * d)
  double origin[3];
  double lo[3], hi[3];             // bounding box, inertial frame
};

Zone make_zone(const OverlapPatch& p)
{
  Zone z;
  for (int a = 0; a < 3; ++a) {
    const int s_lo = p.seek[2 * a], s_hi = p.seek[2 * a + 1];
    // protected layers = seek + additional, none on a side without seek layers
    const int prot_lo = s_lo == 0 ? 0 : s_lo + p.add_protect;
    const int prot_hi = s_hi == 0 ? 0 : s_hi + p.add_protect;
    z.n[a] = p.n[a];
    z.first[a] = (size_t)prot_lo;
    z.afterlast[a] = (size_t)(p.n[a] - prot_hi);
    z.d[a] = p.d[a];
    z.cc_min[a] = 0.5 * p.d[a];
    z.origin[a] = p.origin[a];
    z.lo[a] = p.origin[a];
    z.hi[a] = p.origin[a] + p.n[a] * p.d[a];
  }
  return z;
}

// One axis of the cell-centred interpolation: sectors 0..4 of the donor zone,
// reference cell and linear coefficient.  Returns 1 inside the donor zone,
// 0 outside (sectors 0 and 4), -1 where the reference stops with a BUG (a
// donor zone narrower than two cells, or a coefficient outside [-eps, 1+eps];
// cartesianpatch.cpp:1146-1158).
int linear_coeff(double s_test, size_t first, size_t afterlast, double ds, size_t num,
                 size_t& cell_ref, double& coeff)
{
  const double rs = s_test / ds;
  const double rs0 = (double)(float)first;
  const double rs1 = rs0 + 0.5;
  const double rs2 = (double)(float)afterlast - 0.5;
  const double rs3 = rs2 + 0.5;
  if (rs < rs0) return 0;
  long lc;
  if (rs < rs1) {                        // lower half cell: all weight on `first`
    lc = (long)first;
    coeff = 0.0;
  } else if (rs < rs2) {                 // interior
    lc = long(rs - 0.5 + (double)(float)num) - (long)num;
    if (lc == (long)first - 1) lc = (long)first;
    else if (lc == (long)afterlast - 1) lc = (long)afterlast - 2;
    else if (lc < -1 || lc > (long)afterlast - 1) return -1;
    const double rs_ref = 0.5 + (double)(float)(size_t)lc;
    coeff = rs - rs_ref;
  } else if (rs < rs3) {                 // upper half cell: all weight on `afterlast - 1`
    lc = (long)afterlast - 2;
    coeff = 1.0;
  } else {
    return 0;
  }
  const double eps = 1.e-5;
  if (lc < (long)first || lc > (long)afterlast - 2 || coeff < -eps || coeff > 1. + eps) return -1;
  cell_ref = (size_t)lc;
  return 1;
}

typedef std::pair<size_t, double> Contrib;

// 8-point trilinear weights of point (x, y, z) (donor frame) in donor zone
// `dz`, cleaned like the reference: merge equal indices in sorted order, drop
// |w| < 10*eps, shift so the weights sum to one.  Returns 1 (weights), 0 (the
// point is outside the donor zone) or -1 (see linear_coeff).
int donor_weights(const Zone& dz, const double xyz[3], std::vector<Contrib>& ws, size_t* pad_index = nullptr)
{
  size_t ref[3];
  double c[3];
  for (int a = 0; a < 3; ++a) {
    const int in = linear_coeff(xyz[a], dz.first[a], dz.afterlast[a], dz.d[a], (size_t)dz.n[a], ref[a], c[a]);
    if (in != 1) return in;
  }
  const double x = c[0], y = c[1], z = c[2];
  double w[8];
  w[0] = (1. - x) * (1. - y) * (1. - z);
  w[1] = (1. - x) * (1. - y) * z;
  w[2] = (1. - x) * y * (1. - z);
  w[3] = (1. - x) * y * z;
  w[4] = x * (1. - y) * (1. - z);
  w[5] = x * (1. - y) * z;
  w[6] = x * y * (1. - z);
  w[7] = x * y * z;
  size_t up[3];
  for (int a = 0; a < 3; ++a) {
    up[a] = ref[a] + 1;
    if (up[a] + 1 > (size_t)dz.n[a]) up[a] = ref[a];   // flat axis
  }
  const size_t nj = (size_t)dz.n[1], nk = (size_t)dz.n[2];
  auto idx = [&](size_t i, size_t j, size_t k) { return i * nj * nk + j * nk + k; };
  ws.clear();
  ws.emplace_back(idx(ref[0], ref[1], ref[2]), w[0]);
  ws.emplace_back(idx(ref[0], ref[1], up[2]), w[1]);
  ws.emplace_back(idx(ref[0], up[1], ref[2]), w[2]);
  ws.emplace_back(idx(ref[0], up[1], up[2]), w[3]);
  ws.emplace_back(idx(up[0], ref[1], ref[2]), w[4]);
  ws.emplace_back(idx(up[0], ref[1], up[2]), w[5]);
  ws.emplace_back(idx(up[0], up[1], ref[2]), w[6]);
  ws.emplace_back(idx(up[0], up[1], up[2]), w[7]);

  // merge: sort (index, weight) pairs, add weights of equal indices in order
  std::sort(ws.begin(), ws.end());
  size_t keep = 0;
  for (size_t it = 1; it < ws.size(); ++it) {
    if (ws[it].first == ws[keep].first) ws[keep].second += ws[it].second;
    else ws[++keep] = ws[it];
  }
  ws.resize(keep + 1);
  // drop small weights (absolute threshold 10 * 1e-5), erasing in place:
  // the slot just past the shortened list then holds the last entry before
  // the final erase, which the reference's fixed-size transfer reads as its
  // padding index (WeightedSet::tranferToFixedArrays, weightedset.h:655-659)
  const double eps = 10 * 1.e-5;
  size_t it = 0;
  while (it < ws.size()) {
    double t = ws[it].second;
    if (t < 0.) t = -t;
    if (t < eps) {
      if (pad_index) *pad_index = ws.back().first;
      ws.erase(ws.begin() + (long)it);
    } else {
      ++it;
    }
  }
  // shift to a weight sum of one
  if (!ws.empty()) {
    double sum = 0.;
    for (const Contrib& cw : ws) sum += cw.second;
    const double corr = (1. - sum) / (double)ws.size();
    for (Contrib& cw : ws) cw.second += corr;
  }
  return 1;
}

bool boxes_touch(const Zone& a, const Zone& b)
{
  for (int ax = 0; ax < 3; ++ax) {
    const double tol = 0.5 * (a.d[ax] > b.d[ax] ? a.d[ax] : b.d[ax]);
    if (a.hi[ax] + tol < b.lo[ax] || b.hi[ax] + tol < a.lo[ax]) return false;
  }
  return true;
}

struct Entry {
  size_t ll;                 // position in the receiving-cell list
  size_t cell;               // receiving cell
  std::vector<Contrib> ws;
};

size_t setup_threads();
bool receiver_tables(size_t r, const std::vector<OverlapPatch>& patches, const std::vector<Zone>& zones,
                     DonorTables& t, std::string& err);

} // namespace

int cc_interpolation_weights(const OverlapPatch& p, const double xyz[3], std::vector<std::pair<size_t, double>>& ws,
                             size_t* pad_index)
{
  return donor_weights(make_zone(p), xyz, ws, pad_index);
}

bool build_overlap(const std::vector<OverlapPatch>& patches, std::vector<DonorTables>& out, std::string& err)
{
  const size_t np = patches.size();
  std::vector<Zone> zones(np);
  for (size_t p = 0; p < np; ++p) {
    const OverlapPatch& q = patches[p];
    for (int a = 0; a < 3; ++a) {
      if (q.n[a] < 1 || !(q.d[a] > 0)) { err = "patch " + std::to_string(p) + ": invalid size or spacing"; return false; }
      if (q.seek[2 * a] < 0 || q.seek[2 * a + 1] < 0 || q.add_protect < 0 ||
          q.seek[2 * a] + q.seek[2 * a + 1] + 2 * q.add_protect > q.n[a]) {
        err = "patch " + std::to_string(p) + ": seek/protect layers exceed the patch";
        return false;
      }
    }
    zones[p] = make_zone(q);
  }
  out.assign(np, DonorTables());
  // receiving patches are independent: spread them over the host threads
  // (the tables of each are computed by the same code, so the result does
  // not depend on the thread count)
  std::vector<std::string> errs(np);
  std::atomic<size_t> next{0};
  std::atomic<bool> failed{false};
  auto worker = [&]() {
    for (size_t r; !failed.load() && (r = next.fetch_add(1)) < np;) {
      if (!receiver_tables(r, patches, zones, out[r], errs[r])) failed.store(true);
    }
  };
  const size_t nt = std::min(np, setup_threads());
  std::vector<std::thread> pool;
  for (size_t t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (std::thread& t : pool) t.join();
  for (size_t r = 0; r < np; ++r) {
    if (!errs[r].empty()) {
      err = errs[r];
      return false;
    }
  }
  return true;
}

namespace {

// host threads of the set-up: DN_SETUP_THREADS if set, else all cores
size_t setup_threads()
{
  if (const char* e = std::getenv("DN_SETUP_THREADS")) {
    const long v = std::strtol(e, nullptr, 10);
    if (v >= 1) return (size_t)v;
  }
  const unsigned hc = std::thread::hardware_concurrency();
  return hc ? (size_t)hc : 1;
}

// Donor tables of receiving patch r against every other patch.
bool receiver_tables(size_t r, const std::vector<OverlapPatch>& patches, const std::vector<Zone>& zones,
                     DonorTables& t, std::string& err)
{
  const size_t np = patches.size();
  {
    const OverlapPatch& R = patches[r];
    const Zone& zr = zones[r];
    const size_t ni = (size_t)R.n[0], nj = (size_t)R.n[1], nk = (size_t)R.n[2];
    // receiving cells: union of the seek layers, ascending cell index
    std::vector<size_t> rec;
    for (size_t i = 0; i < ni; ++i) {
      const bool si = i < (size_t)R.seek[0] || i >= ni - (size_t)R.seek[1];
      for (size_t j = 0; j < nj; ++j) {
        const bool sj = j < (size_t)R.seek[2] || j >= nj - (size_t)R.seek[3];
        for (size_t k = 0; k < nk; ++k) {
          const bool sk = k < (size_t)R.seek[4] || k >= nk - (size_t)R.seek[5];
          if (si || sj || sk) rec.push_back((i * nj + j) * nk + k);
        }
      }
    }
    std::vector<size_t> hits(rec.size(), 0);
    std::vector<int32_t> donors;
    std::vector<std::vector<Entry>> lists;
    std::vector<Contrib> ws;
    for (size_t d = 0; d < np && !rec.empty(); ++d) {
      if (d == r || !boxes_touch(zr, zones[d])) continue;
      const Zone& zd = zones[d];
      double shift[3];
      for (int a = 0; a < 3; ++a) shift[a] = -zd.origin[a] + zr.origin[a];
      std::vector<Entry> list;
      for (size_t ll = 0; ll < rec.size(); ++ll) {
        const size_t l = rec[ll];
        const size_t i = l / (nj * nk), j = (l / nk) % nj, k = l % nk;
        double xyz[3];
        xyz[0] = (zr.cc_min[0] + (double)i * zr.d[0]) + shift[0];
        xyz[1] = (zr.cc_min[1] + (double)j * zr.d[1]) + shift[1];
        xyz[2] = (zr.cc_min[2] + (double)k * zr.d[2]) + shift[2];
        const int in = donor_weights(zd, xyz, ws);
        if (in < 0) {
          err = "receiving cell " + std::to_string(l) + " of patch " + std::to_string(r) +
                " falls into a degenerate donor zone of patch " + std::to_string(d) +
                " (donor zones must be at least two cells wide)";
          return false;
        }
        if (in == 1) {
          list.push_back(Entry{ll, l, ws});
          hits[ll]++;
        }
      }
      if (!list.empty()) {
        donors.push_back((int32_t)d);
        lists.push_back(std::move(list));
      }
    }

    for (size_t ll = 0; ll < rec.size(); ++ll) {
      if (hits[ll] > 0) t.rec_unique.push_back(rec[ll]);
      else t.no_donor++;
    }
    for (size_t q = 0; q < donors.size(); ++q) {
      std::vector<Entry>& list = lists[q];
      size_t stride = 0;
      for (Entry& e : list) {
        if (hits[e.ll] > 1) {
          const double s = 1. / (double)hits[e.ll];
          for (Contrib& c : e.ws) c.second *= s;
        }
        if (e.ws.size() > stride) stride = e.ws.size();
      }
      t.donor_patch.push_back(donors[q]);
      t.num_receivers.push_back((int64_t)list.size());
      t.stride.push_back((int32_t)stride);
      for (const Entry& e : list) {
        t.rec_concat.push_back(e.cell);
        for (size_t s = 0; s < stride; ++s) {
          if (s < e.ws.size()) {
            t.donor_idx.push_back(e.ws[s].first);
            t.weight.push_back(e.ws[s].second);
          } else {                                    // padding: first donor cell, weight 0
            t.donor_idx.push_back(e.ws[0].first);
            t.weight.push_back(0.);
          }
        }
      }
    }
  }
  return true;
}

} // namespace

void desc_spacing(const dn_patch_desc& d, double out[3])
{
  const int n[3] = {d.ni, d.nj, d.nk};
  const double h[3] = {d.dx, d.dy, d.dz};
  for (int a = 0; a < 3; ++a) out[a] = d.length[a] > 0 ? d.length[a] / n[a] : h[a];
}

OverlapPatch overlap_patch(const dn_patch_desc& d)
{
  OverlapPatch o;
  o.n[0] = d.ni; o.n[1] = d.nj; o.n[2] = d.nk;
  desc_spacing(d, o.d);
  for (int a = 0; a < 3; ++a) o.origin[a] = d.origin[a];
  for (int a = 0; a < 6; ++a) o.seek[a] = d.seek[a];
  o.add_protect = d.add_protect;
  return o;
}

} // namespace dn

// ------------------------------------------------------------ host-only C ABI


extern "C" {

int dn_overlap_build(const dn_patch_desc* patches, int np, dn_overlap** out, int64_t* no_donor)
{
  if (!out) return DN_ERR_ARG;
  *out = nullptr;
  if (!patches || np < 1) return DN_ERR_ARG;
  std::vector<dn::OverlapPatch> ops;
  for (int p = 0; p < np; ++p) ops.push_back(dn::overlap_patch(patches[p]));
  dn_overlap* ov = new dn_overlap();
  std::string err;
  if (!dn::build_overlap(ops, ov->tables, err)) {
    delete ov;
    return DN_ERR_ARG;
  }
  if (no_donor) {
    int64_t nd = 0;
    for (const auto& t : ov->tables) nd += t.no_donor;
    *no_donor = nd;
  }
  *out = ov;
  return DN_OK;
}

int dn_overlap_counts(const dn_overlap* ov, int id, int64_t counts[4])
{
  if (!ov || !counts || id < 0 || id >= (int)ov->tables.size()) return DN_ERR_ARG;
  const dn::DonorTables& t = ov->tables[id];
  counts[0] = (int64_t)t.rec_unique.size();
  counts[1] = (int64_t)t.donor_patch.size();
  counts[2] = (int64_t)t.rec_concat.size();
  counts[3] = (int64_t)t.donor_idx.size();
  return DN_OK;
}

int dn_overlap_get(const dn_overlap* ov, int id, uint64_t* rec_unique, int32_t* donor_patch, int64_t* num_receivers,
                   int32_t* stride, uint64_t* rec_concat, uint64_t* donor_idx, double* weight)
{
  if (!ov || id < 0 || id >= (int)ov->tables.size()) return DN_ERR_ARG;
  const dn::DonorTables& t = ov->tables[id];
  if ((!rec_unique && !t.rec_unique.empty()) || (!rec_concat && !t.rec_concat.empty()) ||
      (!donor_idx && !t.donor_idx.empty()) || (!weight && !t.weight.empty()) ||
      (!t.donor_patch.empty() && (!donor_patch || !num_receivers || !stride)))
    return DN_ERR_ARG;
  std::copy(t.rec_unique.begin(), t.rec_unique.end(), rec_unique);
  std::copy(t.donor_patch.begin(), t.donor_patch.end(), donor_patch);
  std::copy(t.num_receivers.begin(), t.num_receivers.end(), num_receivers);
  std::copy(t.stride.begin(), t.stride.end(), stride);
  std::copy(t.rec_concat.begin(), t.rec_concat.end(), rec_concat);
  std::copy(t.donor_idx.begin(), t.donor_idx.end(), donor_idx);
  std::copy(t.weight.begin(), t.weight.end(), weight);
  return DN_OK;
}

int dn_overlap_destroy(dn_overlap* ov)
{
  delete ov;
  return DN_OK;
}

} // extern "C"
