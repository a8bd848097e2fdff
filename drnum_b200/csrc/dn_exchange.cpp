// Exchange lists of a patch grid sharded over ranks (host code).
//
// The reference runs all patches of a grid in one process; its donor copy
// reads donor cells of other patches directly (Patch::accessDonorDataDirect,
// patch.cpp:573-653).  With patches spread over GPUs, a rank keeps a shadow
// copy of every patch it does not own and, before each donor copy, receives
// from the owners exactly the donor cells its receiving patches read: the
// donor copy then runs unchanged on local memory and gives the same bits as
// on one GPU.
#include "dn_overlap.h"

#include <algorithm>
#include <cstring>
#include <utility>

namespace dn {

namespace {

// (patch, cell) pairs of donor patches owned by `src` read by receiving
// patches owned by `dst`, unique and ascending
void needed_cells(const std::vector<DonorTables>& tables, const int32_t* owner, int src, int dst,
                  std::vector<int32_t>& patch, std::vector<uint64_t>& cell)
{
  std::vector<std::pair<int32_t, uint64_t>> items;
  for (size_t r = 0; r < tables.size(); ++r) {
    if (owner[r] != dst) continue;
    const DonorTables& t = tables[r];
    size_t pos = 0;                                   // running offset into donor_idx
    for (size_t q = 0; q < t.donor_patch.size(); ++q) {
      const size_t n = (size_t)t.num_receivers[q] * (size_t)t.stride[q];
      if (owner[t.donor_patch[q]] == src) {
        for (size_t e = 0; e < n; ++e) items.emplace_back(t.donor_patch[q], t.donor_idx[pos + e]);
      }
      pos += n;
    }
  }
  std::sort(items.begin(), items.end());
  items.erase(std::unique(items.begin(), items.end()), items.end());
  patch.resize(items.size());
  cell.resize(items.size());
  for (size_t i = 0; i < items.size(); ++i) {
    patch[i] = items[i].first;
    cell[i] = items[i].second;
  }
}

} // namespace

bool build_exchange(const std::vector<DonorTables>& tables, const int32_t* owner, int rank, int world,
                    Exchange& ex, std::string& err)
{
  if (world < 1 || rank < 0 || rank >= world) { err = "rank outside the world"; return false; }
  for (size_t p = 0; p < tables.size(); ++p) {
    if (owner[p] < 0 || owner[p] >= world) { err = "owner of patch " + std::to_string(p) + " outside the world"; return false; }
  }
  ex = Exchange();
  ex.rank = rank;
  ex.world = world;
  ex.send_patch.resize(world); ex.send_cell.resize(world);
  ex.recv_patch.resize(world); ex.recv_cell.resize(world);
  for (int q = 0; q < world; ++q) {
    if (q == rank) continue;
    needed_cells(tables, owner, rank, q, ex.send_patch[q], ex.send_cell[q]);
    needed_cells(tables, owner, q, rank, ex.recv_patch[q], ex.recv_cell[q]);
  }
  return true;
}

} // namespace dn

extern "C" {

int dn_exchange_build(const dn_overlap* ov, const int32_t* owner, int rank, int world, dn_exchange** out)
{
  if (!ov || !owner || !out) return DN_ERR_ARG;
  *out = nullptr;
  dn_exchange* e = new dn_exchange();
  std::string err;
  if (!dn::build_exchange(ov->tables, owner, rank, world, e->ex, err)) {
    delete e;
    return DN_ERR_ARG;
  }
  *out = e;
  return DN_OK;
}

int dn_exchange_counts(const dn_exchange* e, int peer, int64_t* n_send, int64_t* n_recv)
{
  if (!e || peer < 0 || peer >= e->ex.world) return DN_ERR_ARG;
  if (n_send) *n_send = (int64_t)e->ex.send_cell[peer].size();
  if (n_recv) *n_recv = (int64_t)e->ex.recv_cell[peer].size();
  return DN_OK;
}

int dn_exchange_get(const dn_exchange* e, int peer, int32_t* send_patch, uint64_t* send_cell, int32_t* recv_patch,
                    uint64_t* recv_cell)
{
  if (!e || peer < 0 || peer >= e->ex.world) return DN_ERR_ARG;
  const dn::Exchange& x = e->ex;
  if (send_patch) std::copy(x.send_patch[peer].begin(), x.send_patch[peer].end(), send_patch);
  if (send_cell) std::copy(x.send_cell[peer].begin(), x.send_cell[peer].end(), send_cell);
  if (recv_patch) std::copy(x.recv_patch[peer].begin(), x.recv_patch[peer].end(), recv_patch);
  if (recv_cell) std::copy(x.recv_cell[peer].begin(), x.recv_cell[peer].end(), recv_cell);
  return DN_OK;
}

} // extern "C"
