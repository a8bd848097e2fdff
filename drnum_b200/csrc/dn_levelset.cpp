// Level-set wall classification (see dn_levelset.h for the reference steps).
// Compiled with -ffp-contract=off: gradients, mirror points and weights must
// round exactly like the reference's.
#include "dn_levelset.h"

#include <cmath>
#include <cstdio>
#include <utility>

namespace dn {

namespace {

struct Grid {
  size_t n[3];
  size_t size() const { return n[0] * n[1] * n[2]; }
  void ijk(size_t l, size_t& i, size_t& j, size_t& k) const
  {
    i = l / (n[1] * n[2]);
    j = (l / n[2]) % n[1];
    k = l % n[2];
  }
  size_t index(size_t i, size_t j, size_t k) const { return (i * n[1] + j) * n[2] + k; }
  // face neighbours in the order k-1, k+1, j-1, j+1, i-1, i+1
  void neighbours(size_t l, std::vector<size_t>& out) const
  {
    size_t i, j, k;
    ijk(l, i, j, k);
    out.clear();
    if (k > 0) out.push_back(index(i, j, k - 1));
    if (k + 1 < n[2]) out.push_back(index(i, j, k + 1));
    if (j > 0) out.push_back(index(i, j - 1, k));
    if (j + 1 < n[1]) out.push_back(index(i, j + 1, k));
    if (i > 0) out.push_back(index(i - 1, j, k));
    if (i + 1 < n[0]) out.push_back(index(i + 1, j, k));
  }
};

LayerCell layer_cell(size_t l, double g)
{
  LayerCell c{};
  c.cell = l;
  c.g = g;
  return c;
}

// dG/dx_a by central differences, one-sided at the patch edge
double nabla(const Grid& gr, const double* G, size_t l, int axis, double d)
{
  size_t c[3];
  gr.ijk(l, c[0], c[1], c[2]);
  const bool has_plus = c[axis] + 1 < gr.n[axis];
  const bool has_minus = c[axis] > 0;
  size_t cp[3] = {c[0], c[1], c[2]}, cm[3] = {c[0], c[1], c[2]};
  cp[axis] += 1;
  cm[axis] -= 1;
  if (has_plus && has_minus) return (G[gr.index(cp[0], cp[1], cp[2])] - G[gr.index(cm[0], cm[1], cm[2])]) / (2. * d);
  if (!has_plus) return (G[l] - G[gr.index(cm[0], cm[1], cm[2])]) / d;
  return (G[gr.index(cp[0], cp[1], cp[2])] - G[l]) / d;
}

void normalised_gradient(const Grid& gr, const double* G, size_t l, const double d[3], double out[3])
{
  for (int a = 0; a < 3; ++a) out[a] = nabla(gr, G, l, a, d[a]);
  double len = 0;
  for (int a = 0; a < 3; ++a) len += out[a] * out[a];
  len = std::sqrt(len);
  for (int a = 0; a < 3; ++a) out[a] /= len;
}

} // namespace

bool classify_levelset(const OverlapPatch& patch, const double* G, int num_inner, int num_outer,
                       double min_inner_rel_dist, LevelSetLayers& out, std::string& err)
{
  if (!G) { err = "level-set field is NULL"; return false; }
  if (num_inner < 0 || num_outer < 0) { err = "negative layer count"; return false; }
  if (min_inner_rel_dist > 0 && num_inner == 0) { err = "min_inner_rel_dist needs an inner layer"; return false; }
  Grid gr;
  for (int a = 0; a < 3; ++a) {
    if (patch.n[a] < 2) { err = "level-set patches need at least 2 cells per axis"; return false; }
    gr.n[a] = (size_t)patch.n[a];
  }
  const size_t nc = gr.size();
  out = LevelSetLayers();
  out.inner.resize((size_t)num_inner);
  out.outer.resize((size_t)num_outer);

  double g_max = G[0], g_min = G[0];
  for (size_t l = 0; l < nc; ++l) {
    if (g_min > G[l]) g_min = G[l];
    if (g_max < G[l]) g_max = G[l];
  }
  const double g_eps = (g_max - g_min) * 1.e-7;

  std::vector<char> marker(nc, 0);
  std::vector<size_t> nb;
  // layer 0: a face neighbour of the other sign
  for (size_t l = 0; l < nc; ++l) {
    const double g = G[l];
    gr.neighbours(l, nb);
    bool other = false;
    for (size_t ln : nb) {
      const double t1 = (G[ln] + g_eps) * (g - g_eps);
      const double t2 = (G[ln] - g_eps) * (g + g_eps);
      if (t1 < 0. || t2 < 0.) {
        other = true;
        marker[l] = 1;
        break;
      }
    }
    if (other) {
      if (g < 0.) {
        if (num_inner > 0) out.inner[0].push_back(layer_cell(l, g));
      } else {
        if (num_outer > 0) out.outer[0].push_back(layer_cell(l, g));
      }
    }
  }

  // inner layer 0 too close to the surface: replace by deeper neighbours
  if (min_inner_rel_dist > 0.) {
    std::vector<LayerCell>& L0 = out.inner[0];
    size_t ll = 0;
    while (ll < L0.size()) {
      const size_t l = L0[ll].cell;
      gr.neighbours(l, nb);
      double min_g = G[nb[0]], max_g = G[nb[0]];
      for (size_t q = 1; q < nb.size(); ++q) {
        if (min_g > G[nb[q]]) min_g = G[nb[q]];
        if (max_g < G[nb[q]]) max_g = G[nb[q]];
      }
      const double g_difference = 0.5 * (max_g - min_g);
      const double min_distance = min_inner_rel_dist * g_difference;
      if (G[l] > -min_distance) {
        L0.erase(L0.begin() + (long)ll);
        marker[l] = 0;
        out.replaced++;
        for (size_t ln : nb) {
          if (!marker[ln] && G[ln] < G[l]) {
            L0.push_back(layer_cell(ln, G[ln]));
            marker[ln] = 1;
          }
        }
      } else {
        ++ll;
      }
    }
  }

  // further layers
  for (int layer = 1; layer < num_inner; ++layer) {
    for (size_t q = 0; q < out.inner[layer - 1].size(); ++q) {
      gr.neighbours(out.inner[layer - 1][q].cell, nb);
      for (size_t ln : nb) {
        if (!marker[ln] && G[ln] < 0.) {
          out.inner[layer].push_back(layer_cell(ln, G[ln]));
          marker[ln] = 1;
        }
      }
    }
  }
  for (int layer = 1; layer < num_outer; ++layer) {
    for (size_t q = 0; q < out.outer[layer - 1].size(); ++q) {
      gr.neighbours(out.outer[layer - 1][q].cell, nb);
      for (size_t ln : nb) {
        if (!marker[ln] && G[ln] > 0.) {
          out.outer[layer].push_back(layer_cell(ln, G[ln]));
          marker[ln] = 1;
        }
      }
    }
  }

  // gradients and mirror-point donors of the inner layers
  std::vector<std::pair<size_t, double>> ws;
  for (int layer = 0; layer < num_inner; ++layer) {
    std::vector<LayerCell> kept;
    for (LayerCell& c : out.inner[layer]) {
      normalised_gradient(gr, G, c.cell, patch.d, c.grad);
      const double shift_len = -2. * c.g;
      size_t ijk[3];
      gr.ijk(c.cell, ijk[0], ijk[1], ijk[2]);
      double xyz[3];
      for (int a = 0; a < 3; ++a) {
        const double xc = 0.5 * patch.d[a] + (double)ijk[a] * patch.d[a];
        xyz[a] = xc + shift_len * c.grad[a];
      }
      size_t pad = 0;
      const int in = cc_interpolation_weights(patch, xyz, ws, &pad);
      if (in < 0) {
        err = "mirror point of cell " + std::to_string(c.cell) + " falls into a degenerate donor zone";
        return false;
      }
      if (in == 0 || ws.empty()) continue;        // no mirror donors: dropped
      if (ws.size() > 8) { err = "more than 8 mirror donors"; return false; }
      for (size_t q = 0; q < 8; ++q) {
        if (q < ws.size()) {
          c.donor[q] = ws[q].first;
          c.weight[q] = ws[q].second;
        } else {
          c.donor[q] = pad;
          c.weight[q] = 0.;
        }
      }
      kept.push_back(c);
    }
    out.inner[layer].swap(kept);
  }
  for (int layer = 0; layer < num_outer; ++layer)
    for (LayerCell& c : out.outer[layer]) normalised_gradient(gr, G, c.cell, patch.d, c.grad);
  return true;
}

bool classify_levelset_gpu(const OverlapPatch& patch, const double* G, LevelSetGpu& out, std::string& err)
{
  if (!G) { err = "level-set field is NULL"; return false; }
  const long imax = patch.n[0], jmax = patch.n[1], kmax = patch.n[2];
  out = LevelSetGpu();
  auto idx = [&](long i, long j, long k) -> size_t { return (size_t)((i * jmax + j) * kmax + k); };
  auto g = [&](long i, long j, long k) { return G[idx(i, j, k)]; };
  // GPU_CartesianPatch::idx() etc.: 1 / spacing (CartesianPatch::computeDeltas,
  // cartesianpatch.cpp:167-174)
  const double dx = patch.d[0], dy = patch.d[1], dz = patch.d[2];
  const double idx_ = 1.0 / dx, idy = 1.0 / dy, idz = 1.0 / dz;
  for (long i = 0; i < imax; ++i) {
    for (long j = 0; j < jmax; ++j) {
      for (long k = 0; k < kmax; ++k) {
        if (!(g(i, j, k) < 0)) continue;
        out.below.push_back(idx(i, j, k));
        bool extrapolate = true;
        long i_stt = -2, i_end = 2, j_stt = -2, j_end = 2, k_stt = -2, k_end = 2;
        if (i < 2) i_stt += 2 - i;
        if (i == imax - 1) i_end = 0;
        if (i == imax - 2) i_end = 1;
        if (j < 2) j_stt += 2 - j;
        if (j == jmax - 1) j_end = 0;
        if (j == jmax - 2) j_end = 1;
        if (k < 2) k_stt += 2 - k;
        if (k == kmax - 1) k_end = 0;
        if (k == kmax - 2) k_end = 1;
        for (long di = i_stt; di <= i_end; ++di) {
          for (long dj = j_stt; dj <= j_end; ++dj) {
            for (long dk = k_stt; dk <= k_end; ++dk) {
              if (di == 0 && dj == 0 && dk == 0) continue;
              const long i2 = i + 2 * di, j2 = j + 2 * dj, k2 = k + 2 * dk;
              if (i2 < 0 || j2 < 0 || k2 < 0 || i2 >= imax || j2 >= jmax || k2 >= kmax) {
                char buf[200];
                std::snprintf(buf, sizeof buf,
                              "cell (%ld, %ld, %ld) with G < 0 lies too close to the patch edge for the GPU "
                              "level-set path (its search reaches (%ld, %ld, %ld))", i, j, k, i2, j2, k2);
                err = buf;
                return false;
              }
              if (g(i + di, j + dj, k + dk) >= 0) {
                extrapolate = false;
                break;   // the reference leaves only the innermost loop
              }
            }
          }
        }
        if (!extrapolate) continue;
        if (i < 2) i_stt = 0;
        if (i >= imax - 2) i_end = 0;
        if (j < 2) j_stt = 0;
        if (j >= jmax - 2) j_end = 0;
        if (k < 2) k_stt = 0;
        if (k >= kmax - 2) k_end = 0;
        // gradient of G (GPU_CartesianLevelSetBC::grad)
        double gx, gy, gz;
        if (i == 0) gx = idx_ * (g(i + 1, j, k) - g(i, j, k));
        else if (i == imax - 1) gx = idx_ * (g(i, j, k) - g(i - 1, j, k));
        else gx = 0.5 * idx_ * (g(i + 1, j, k) - g(i - 1, j, k));
        if (j == 0) gy = idy * (g(i, j + 1, k) - g(i, j, k));
        else if (j == jmax - 1) gy = idy * (g(i, j, k) - g(i, j - 1, k));
        else gy = 0.5 * idy * (g(i, j + 1, k) - g(i, j - 1, k));
        if (k == 0) gz = idz * (g(i, j, k + 1) - g(i, j, k));
        else if (k == kmax - 1) gz = idz * (g(i, j, k) - g(i, j, k - 1));
        else gz = 0.5 * idz * (g(i, j, k + 1) - g(i, j, k - 1));
        LsInsideCell c;
        c.cell = idx(i, j, k);
        const double g0 = g(i, j, k);
        for (long di = i_stt; di <= i_end; ++di) {
          for (long dj = j_stt; dj <= j_end; ++dj) {
            for (long dk = k_stt; dk <= k_end; ++dk) {
              if (di == 0 && dj == 0 && dk == 0) continue;
              const double gn = g(i + di, j + dj, k + dk);
              if (gn >= 0 || gn > g0) {
                const double ddx = (double)di * dx, ddy = (double)dj * dy, ddz = (double)dk * dz;
                c.nbr.push_back(idx(i + di, j + dj, k + dk));
                c.w.push_back(std::fabs(ddx * gx + ddy * gy + ddz * gz) / std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz));
              }
            }
          }
        }
        out.inside.push_back(std::move(c));
      }
    }
  }
  return true;
}

} // namespace dn

// ------------------------------------------------------------ host-only C ABI

struct dn_lslayers {
  dn::LevelSetLayers layers;
};

extern "C" {

int dn_levelset_classify(const dn_patch_desc* patch, const double* G, int num_inner_layers, int num_outer_layers,
                         double min_inner_rel_dist, dn_lslayers** out)
{
  if (!out) return DN_ERR_ARG;
  *out = nullptr;
  if (!patch || !G) return DN_ERR_ARG;
  dn_lslayers* ls = new dn_lslayers();
  std::string err;
  if (!dn::classify_levelset(dn::overlap_patch(*patch), G, num_inner_layers, num_outer_layers, min_inner_rel_dist,
                             ls->layers, err)) {
    delete ls;
    return DN_ERR_ARG;
  }
  *out = ls;
  return DN_OK;
}

int dn_lslayers_count(const dn_lslayers* ls, int inner, int layer, int64_t* n)
{
  if (!ls || !n) return DN_ERR_ARG;
  const auto& lists = inner ? ls->layers.inner : ls->layers.outer;
  if (layer < 0 || layer >= (int)lists.size()) return DN_ERR_ARG;
  *n = (int64_t)lists[layer].size();
  return DN_OK;
}

int dn_lslayers_get(const dn_lslayers* ls, int inner, int layer, uint64_t* cells, double* g, double* grad,
                    uint64_t* donors, double* weights)
{
  if (!ls) return DN_ERR_ARG;
  const auto& lists = inner ? ls->layers.inner : ls->layers.outer;
  if (layer < 0 || layer >= (int)lists.size()) return DN_ERR_ARG;
  size_t q = 0;
  for (const dn::LayerCell& lc : lists[layer]) {
    if (cells) cells[q] = lc.cell;
    if (g) g[q] = lc.g;
    for (int a = 0; a < 3; ++a) if (grad) grad[3 * q + a] = lc.grad[a];
    for (int t = 0; t < 8; ++t) {
      if (donors) donors[8 * q + t] = lc.donor[t];
      if (weights) weights[8 * q + t] = lc.weight[t];
    }
    ++q;
  }
  return DN_OK;
}

int dn_lslayers_destroy(dn_lslayers* ls)
{
  delete ls;
  return DN_OK;
}

} // extern "C"
